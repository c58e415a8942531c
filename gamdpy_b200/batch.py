"""Batched replicas: many independent Simulations advanced together on one GPU.

gamdpy runs one Simulation per process and launches one kernel grid per
system; ensembles of small systems (state-point sweeps, replicas for
averaging) leave most of a B200 idle that way.  ``SimulationBatch`` gives
every system one thread-block cluster for a whole timeblock: up to 4096
particles with positions and lists in the cluster's shared memory
(velocities in registers), larger systems with their state in global memory
and hardware cluster barriers between the phases.  Systems of one cluster
shape share one launch; systems above 131072 particles run one after another
on the persistent grid kernel.
Per system the result is that of ``Simulation.run_timeblocks``: the same
output datasets, runtime actions and state on the host after each block.
"""
import numpy as np

from . import _lib
from .integrators import NVT
from .simulation import Simulation


class SimulationBatch:
    """Advance ``simulations`` (built as usual, one ``Simulation`` each) block
    by block in one batched launch per timeblock.

    All simulations need the same device, number of particle types,
    integrator kind, ``steps_per_timeblock`` and ``dt`` (the timeblock's start
    time is shared).  ``particles_per_cta`` shapes the shared-memory clusters
    of systems up to 4096 particles (about that many particles per CTA, at
    most 256, up to 16 CTAs per system; 0 = the single-system default, so
    every system gives the same bits as alone); ``clg_particles_per_cta`` and
    ``clg_tp`` the global-memory clusters of larger systems (particles per
    1024-thread CTA, 0 = fit one wave; lanes per particle, 0 = 1).
    ``autotune`` picks all three by timing.
    """

    def __init__(self, simulations, particles_per_cta=0, clg_particles_per_cta=0, clg_tp=0):
        self.simulations = list(simulations)
        if not self.simulations:
            raise ValueError("SimulationBatch needs at least one Simulation")
        for s in self.simulations:
            if not isinstance(s, Simulation):
                raise TypeError("SimulationBatch takes gamdpy_b200.Simulation objects")
        s0 = self.simulations[0]
        for s in self.simulations[1:]:
            if s.steps_per_block != s0.steps_per_block or s.dt != s0.dt:
                raise ValueError("every Simulation of a batch needs the same steps_per_timeblock and dt")
        self.steps_per_block = s0.steps_per_block
        self.dt = s0.dt
        self.num_blocks = min(s.num_blocks for s in self.simulations)
        self.particles_per_cta = int(particles_per_cta)
        self.clg_particles_per_cta = int(clg_particles_per_cta)
        self.clg_tp = int(clg_tp)
        self._batch = self._handle()
        self.timing_blocks = None

    def _handle(self):
        return _lib.BatchHandle([s._sim for s in self.simulations], self.particles_per_cta,
                                self.clg_particles_per_cta, self.clg_tp)

    @property
    def shape(self):
        """(particles_per_cta, clg_particles_per_cta, clg_tp) of the handle."""
        return self.particles_per_cta, self.clg_particles_per_cta, self.clg_tp

    @property
    def num_particles(self):
        return int(sum(s.configuration.N for s in self.simulations))

    def paths(self):
        """Execution path each system took in the last block (1 persistent
        grid kernel, 2 cluster with the state in shared memory, 3 cluster with
        the state in global memory)."""
        return [s._sim.last_path() for s in self.simulations]

    def integrate_self(self, time_zero, steps):
        """Advance every system ``steps`` steps from ``time_zero``; returns the
        device time of the batched launch in ms.  Nothing is copied back."""
        return self._batch.run(float(np.float32(time_zero)), int(steps))

    def run_timeblocks(self, num_timeblocks=-1):
        if num_timeblocks == -1:
            num_timeblocks = self.num_blocks
        assert num_timeblocks <= self.num_blocks
        for s in self.simulations:
            s.last_num_blocks = num_timeblocks
            s.configuration.copy_to_device()
        block_times = []
        for block in range(num_timeblocks):
            for s in self.simulations:
                s.current_block = block
                for ra in s.runtime_actions:
                    ra.initialize_before_timeblock()
            ms = self.integrate_self(np.float32(block * self.steps_per_block * self.dt), self.steps_per_block)
            block_times.append(ms)
            for s in self.simulations:
                s._after_block(block)
            yield block
        self.timing_blocks = np.array(block_times)
        for s in self.simulations:
            s._finish_blocks(block_times)

    def run(self, verbose=True):
        for _ in self.run_timeblocks():
            pass
        if verbose:
            print(self.summary())

    def get_tps(self):
        """Timesteps per second of the batch (every system advanced one step)."""
        return len(self.timing_blocks) * self.steps_per_block / (np.sum(self.timing_blocks) / 1000)

    def get_atom_steps_per_second(self):
        return self.get_tps() * self.num_particles

    def summary(self):
        tps = self.get_tps()
        return (f"Systems : {len(self.simulations)}  particles : {self.num_particles}\n"
                f"Steps : {len(self.timing_blocks)} * {self.steps_per_block}  TPS: {tps:.3e}  "
                f"atom-steps/s: {tps * self.num_particles:.3e}\n")

    def autotune(self, candidates=(0, 64, 128, 192, 256), clg_candidates=(0, 2048, 4096, 8192),
                 clg_tps=(1, 2, 4), steps=None, verbose=False):
        """Pick the batch's shape by timing short batched runs, one axis at a
        time (shared-memory clusters' particles per CTA, then the
        global-memory clusters' particles per CTA, then their lanes per
        particle), each axis kept at its best before the next.  The
        configurations and thermostat states are restored afterwards.
        Returns the chosen (particles_per_cta, clg_particles_per_cta, clg_tp)."""
        steps = steps or min(self.steps_per_block, 256)
        saved = []
        for s in self.simulations:
            c = s.configuration
            # the device's xi: the host copy is behind it until a block ends
            xi = s._sim.thermostat_state() if isinstance(s.integrator, NVT) else None
            saved.append((c["r"].copy(), c["v"].copy(), c.r_im.copy(), xi))

        def restore():
            for s, (r, v, rim, xi) in zip(self.simulations, saved):
                c = s.configuration
                c["r"], c["v"] = r, v
                c.r_im[:] = rim
                if xi is not None:
                    s.integrator.thermostat_state[:] = xi
                    s._sim.set_thermostat_state(xi)
                c.copy_to_device()

        def timed(shape):
            self.particles_per_cta, self.clg_particles_per_cta, self.clg_tp = shape
            self._batch = self._handle()
            restore()
            self.integrate_self(0.0, steps)
            ms = self.integrate_self(0.0, steps)
            if verbose:
                print(f"autotune: shape={shape}: {steps / ms * 1000:.1f} TPS")
            return ms

        best = (self.particles_per_cta, self.clg_particles_per_cta, self.clg_tp)
        best_ms = timed(best)
        for axis, cands in ((0, candidates), (1, clg_candidates), (2, clg_tps)):
            for c in cands:
                shape = list(best)
                shape[axis] = int(c)
                shape = tuple(shape)
                if shape == best:
                    continue
                ms = timed(shape)
                if ms < best_ms:
                    best, best_ms = shape, ms
        self.particles_per_cta, self.clg_particles_per_cta, self.clg_tp = best
        self._batch = self._handle()
        restore()
        return best
