"""Simulation driver (gamdpy/simulation/Simulation.py, get_default_compute_plan.py,
get_default_sim.py).

Same constructor, timeblock generator, status/summary strings and output
layout as gamdpy.  Where gamdpy JIT-compiles and launches a numba kernel per
timeblock (``integrate_self``, Simulation.py:271-282), this calls
``gdb_sim_run`` once per timeblock: by default the library runs the whole
timeblock (steps, neighbour-list rebuilds, thermostat) in one persistent
cooperative kernel, or in one thread-block cluster for small systems; a
CUDA-graph replay of standalone fused force+integrate kernels is the fallback
(GDB_PERSISTENT=0).  It returns the block's device time.
"""
import math
import sys

import numpy as np

from . import _lib
from .configuration import Configuration, get_default_compute_flags, unit_cells
from .integrators import NPT_Atomic, NVE, NVT, NVT_Langevin
from .interactions import Bonds, PairPotential
from .runtime_actions import ConfigurationSaver, MomentumReset, ScalarSaver

B200_NUM_SM = 148
B200_CORES_PER_SM = 128


class Output(dict):
    """In-memory stand-in for the h5py file gamdpy writes (datasets as numpy
    arrays, ``attrs`` dict): ``output['scalars']``, ``output.attrs[...]``."""

    def __init__(self):
        super().__init__()
        self.attrs = {}

    def create_dataset(self, name, data=None, shape=None, dtype=None, **kw):
        self[name] = np.array(data, dtype=dtype) if data is not None else np.zeros(shape, dtype=dtype)
        return self[name]

    def close(self):
        pass


def get_default_compute_plan(configuration):
    """gamdpy's heuristics (get_default_compute_plan.py:8-89) with B200's
    numbers (148 SMs, 128 FP32 lanes per SM, warp 32).  ``tp`` is rounded to
    the library's 1/2/4/8 lanes per particle; ``gridsync`` and ``UtilizeNIII``
    are kept for compatibility and do not change the library's launch plan."""
    N = configuration.N
    num_SM = B200_NUM_SM
    num_cc_cores = B200_CORES_PER_SM * num_SM
    pb = 512
    # gamdpy's loop halves pb to zero (and divides by it) when N < 2 x 148;
    # it stops at one here, and the clamp below makes that 8
    while pb > 1 and N // pb < 2 * num_SM:
        pb = pb // 2
    pb = min(max(pb, 8), 256)
    tp = 1
    while N * tp < 2 * num_cc_cores:
        tp += 1
    while (pb * tp) % 32 != 0:
        tp += 1
    tp = min(tp, 16)
    skin = 0.5
    if N > 6 * 1024:
        skin = np.float32(1.0)
    UtilizeNIII = N >= 16 * 1024
    gridsync = not (N * tp > 4 * num_cc_cores)
    nblist = "N squared"
    if N > 6_000:
        nblist = "linked lists"
        skin = 0.5
    return {"pb": pb, "tp": tp, "skin": skin, "UtilizeNIII": UtilizeNIII, "gridsync": gridsync, "nblist": nblist}


def split_interactions(interactions):
    """(PairPotential, Bonds or None) of an interactions list: the library
    runs one pair potential, optionally with one set of harmonic bonds."""
    items = interactions if isinstance(interactions, list) else [interactions]
    pairs = [x for x in items if isinstance(x, PairPotential)]
    bonds = [x for x in items if isinstance(x, Bonds)]
    if len(pairs) != 1 or len(bonds) > 1 or len(pairs) + len(bonds) != len(items):
        raise NotImplementedError("gamdpy_b200 runs one PairPotential per simulation, optionally with one Bonds")
    return pairs[0], (bonds[0] if bonds else None)


def _autotune_cache_path():
    import os
    d = os.environ.get("GAMDPY_B200_CACHE") or os.path.join(os.path.expanduser("~"), ".cache", "gamdpy_b200")
    return os.path.join(d, "autotune.json")


def _autotune_cache_load():
    import json
    try:
        with open(_autotune_cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _autotune_cache_store(key, value):
    import json
    import os
    path = _autotune_cache_path()
    data = _autotune_cache_load()
    data[key] = value
    os.makedirs(os.path.dirname(path), exist_ok=True)
    tmp = path + f".{os.getpid()}"
    with open(tmp, "w") as f:
        json.dump(data, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def _lanes(tp):
    """Library lanes per particle for a gamdpy ``tp``: largest power of two
    <= tp, at most 32."""
    t = 1
    while t * 2 <= min(int(tp), 32):
        t *= 2
    return t


class Simulation:
    """Run timeblocks of a configuration under interactions, an integrator and
    runtime actions (gamdpy/simulation/Simulation.py:23-500)."""

    def __init__(self, configuration, interactions, integrator, runtime_actions, num_steps=0, num_timeblocks=0,
                 steps_per_timeblock=0, compute_plan=None, storage="output.h5", verbose=False, timing=True,
                 steps_in_kernel_test=1, device=0):
        self.configuration = configuration
        self.compute_plan = dict(compute_plan) if compute_plan is not None else get_default_compute_plan(
            configuration)
        self.interactions = interactions if isinstance(interactions, list) else [interactions]
        self._pair, self._bonds = split_interactions(self.interactions)
        self.integrator = integrator
        if not isinstance(integrator, (NVE, NVT, NVT_Langevin, NPT_Atomic)):
            raise NotImplementedError("gamdpy_b200 supports the NVE, NVT, NVT_Langevin and NPT_Atomic integrators")
        if isinstance(integrator, NPT_Atomic):
            flags = getattr(configuration, "compute_flags", None) or {}
            if not flags.get("W", True):
                raise ValueError("NPT_Atomic requires virial")  # NPT_Atomic.py:88-89
        self.dt = integrator.dt
        if num_timeblocks == 0:
            if num_steps == 0:
                raise ValueError("Either num_steps or num_timeblocks must be non-zero")
            num_timeblocks = 32
            steps_per_timeblock = 2 ** int(math.log2(math.ceil(num_steps / num_timeblocks)))
            num_timeblocks = math.ceil(num_steps / steps_per_timeblock)
        elif steps_per_timeblock == 0:
            raise ValueError("If num_timeblocks is non-zero then steps_per_timeblock must be too (num_steps is "
                             "ignored in this case)")
        self.num_blocks = num_timeblocks
        self.current_block = -1
        self.steps_per_block = steps_per_timeblock
        self.storage = storage
        self.timing = timing
        self.steps_in_kernel_test = steps_in_kernel_test
        self.memory = Output()
        self._file = storage if isinstance(storage, str) and storage.endswith(".h5") else None
        self.memory.attrs["dt"] = self.dt
        self.memory.attrs["simbox_initial"] = configuration.simbox.lengths.copy()
        self.memory.create_dataset("ptype", data=configuration.ptype, dtype=np.int32)
        self.memory.attrs["script_name"] = sys.argv[0] if sys.argv else ""

        self.runtime_actions = runtime_actions
        compute_flags = None
        for ra in runtime_actions:
            if ra.get_compute_flags() is not None:
                if compute_flags is not None:
                    raise ValueError("Can not handle more than one compute_flags in runtime_actions")
                compute_flags = ra.get_compute_flags()
        self.compute_flags = get_default_compute_flags()
        if compute_flags is not None:
            for k in compute_flags:
                if k not in self.compute_flags:
                    raise ValueError("Unknown key in compute_flags:%s" % k)
                self.compute_flags[k] = compute_flags[k]
        for k in self.compute_flags:
            if self.compute_flags[k] and not configuration.compute_flags[k]:
                raise ValueError('compute_flags["%s]" set for Simulation but not in Configuration' % k)
        for ra in runtime_actions:
            ra.setup(configuration=configuration, num_timeblocks=num_timeblocks,
                     steps_per_timeblock=steps_per_timeblock, output=self.memory)

        self._build_device(device)
        self.JIT_and_test_kernel()
        for interaction in self.interactions:
            interaction.check_datastructure_validity()

    # --- device set-up --------------------------------------------------
    def _build_device(self, device):
        conf = self.configuration
        if conf.D != 3:
            raise NotImplementedError("gamdpy_b200 simulates D = 3")
        pp = self._pair
        table, _ = pp.table()
        self._sim = _lib.Sim(conf.N, table.shape[0], device)
        conf._attach(self._sim)
        self._sim.set_box(conf.simbox.lengths)
        pp.configure_device(self._sim, conf, self.compute_plan)
        if self._bonds is not None:
            self._bonds.configure_device(self._sim, conf)
        # gamdpy's tp heuristic targets its own launch shape; the library picks
        # lanes per particle for B200 unless the plan sets "lanes"
        self._sim.set_plan(int(self.compute_plan.get("lanes", 0)))
        self.integrator.configure_device(self._sim, conf)
        scalar_every, reset_every, conf_per_block = 0, 0, 0
        self._scalar_saver = self._conf_saver = None
        for ra in self.runtime_actions:
            if isinstance(ra, ScalarSaver):
                scalar_every = ra.steps_between_output
                self._scalar_saver = ra
            elif isinstance(ra, MomentumReset):
                reset_every = ra.steps_between_reset
            elif isinstance(ra, ConfigurationSaver):
                conf_per_block = ra.conf_per_block
                self._conf_saver = ra
            else:
                raise NotImplementedError(f"runtime action {type(ra).__name__} is not supported on the B200 path")
        self._sim.set_runtime_actions(scalar_every, reset_every)
        self._sim.set_configuration_saver(conf_per_block)

    def JIT_and_test_kernel(self, adjust_compute_plan=True):
        """Upload and run ``steps_in_kernel_test`` steps as gamdpy does before
        the run (Simulation.py:200-224).  As there, the device copy is not
        brought back to the host, but the integrator state it advanced (the
        Nose-Hoover xi) is kept."""
        self.configuration.copy_to_device()
        self.integrate_self(0.0, self.steps_in_kernel_test)

    def integrate_self(self, time_zero, steps):
        return self._sim.run(float(np.float32(time_zero)), int(steps))

    @property
    def output(self):
        return self.memory

    def get_output(self, mode="r"):
        return self.memory

    # --- running -----------------------------------------------------------
    def run(self, verbose=True):
        for _ in self.run_timeblocks():
            if verbose:
                print(self.status(per_particle=True))
        if verbose:
            print(self.summary())

    def run_timeblocks(self, num_timeblocks=-1):
        """Generator over timeblocks (Simulation.py:367-451): upload once, then
        per block run on the device, copy the state to the host, check the
        neighbour list and store the runtime actions' output."""
        if num_timeblocks == -1:
            num_timeblocks = self.num_blocks
        self.last_num_blocks = num_timeblocks
        assert num_timeblocks <= self.num_blocks
        self.configuration.copy_to_device()
        block_times = []
        for block in range(num_timeblocks):
            self.current_block = block
            for ra in self.runtime_actions:
                ra.initialize_before_timeblock()
            ms = self.integrate_self(np.float32(block * self.steps_per_block * self.dt), self.steps_per_block)
            block_times.append(ms)
            self._after_block(block)
            yield block
        self._finish_blocks(block_times)

    def _after_block(self, block):
        """Host side of one finished timeblock: state back to the host, list
        validity check, runtime-action output (Simulation.py:418-447)."""
        self.configuration.copy_to_host()
        # quantities the run's compute flags leave off read zero, as in the
        # reference, whose kernels then never accumulate them
        for name in ("U", "W", "lapU", "K", "Fsq"):
            if name in self.configuration.sid and not self.compute_flags.get(name, False):
                self.configuration.scalars[:, self.configuration.sid[name]] = 0.0
        if isinstance(self.integrator, (NVT, NPT_Atomic)):
            self.integrator.sync_from_device()
        if isinstance(self.integrator, NPT_Atomic):
            # the box the run left (the reference's sim_box device array)
            self.configuration.simbox.lengths[:] = self._sim.box()
        for interaction in self.interactions:
            interaction.check_datastructure_validity()
        if self._scalar_saver is not None:
            rows = self._sim.scalar_rows(self._scalar_saver.scalar_saves_per_block)
            self._scalar_saver.update_from_rows(block, rows, self.memory, self.configuration.get_volume(),
                                                self.compute_flags)
        if self._conf_saver is not None:
            cpb = self._conf_saver.conf_per_block
            frames = self._sim.saved_configurations(cpb)
            boxes = self._sim.saved_boxes(cpb) if self._conf_saver.include_simbox else None
            self._conf_saver.update_from_frames(block, frames, self.memory, boxes)

    def _finish_blocks(self, block_times):
        if self.timing:
            self.timing_numba_blocks = np.array(block_times)
            self.timing_numba = float(np.sum(block_times))
        if self._file is not None:
            self._write_h5()

    def _write_h5(self):
        try:
            import h5py
        except ImportError:
            return
        with h5py.File(self._file, "w") as f:
            for k, v in self.memory.items():
                f.create_dataset(k, data=v)
            for k, v in self.memory.attrs.items():
                f.attrs[k] = v

    def status(self, per_particle=False):
        time = (self.current_block + 1) * self.steps_per_block * self.dt
        st = f"timeblock= {self.current_block :<6}"
        st += f"{time= :<12.3f}"
        for name in self.configuration.sid:
            if name in self.configuration.compute_flags and self.configuration.compute_flags[name]:
                data = np.sum(self.configuration[name])
                if per_particle:
                    data /= self.configuration.N
                st += f"{name}= {data:<10.3f}"
        return st

    def summary(self):
        st = f"Particles : {self.configuration.N} \n"
        st += f"Steps : {self.last_num_blocks} * {self.steps_per_block} = "
        st += f"{self.last_num_blocks * self.steps_per_block:_} \n"
        if self.timing:
            time_sim = np.sum(self.timing_numba_blocks) / 1000
            tps_sim = self.last_num_blocks * self.steps_per_block / time_sim
            st += f"Simulation time (excl. time spent between timeblocks): {time_sim:.2f} s "
            st += f"( TPS: {tps_sim:.2e} )\n"
        return st

    def get_tps(self):
        """Steps per second over the timed blocks, as benchmarks/benchmark_LJ.py:90."""
        return self.last_num_blocks * self.steps_per_block / (np.sum(self.timing_numba_blocks) / 1000)

    def autotune(self, tps_candidates=(1, 2, 4, 8, 16, 32), skins=None, nblists=None, steps=None, cache=True,
                 verbose=False):
        """Pick the neighbour-list kind, lanes per particle and skin by timing
        short runs, as Simulation.autotune (Simulation.py:636-821) searches
        nblist, tp and skin.  nblists defaults to the plan's kind plus
        'N squared' below 32 000 particles and 'linked lists' above 2000
        (gamdpy's rules); skins to the plan's skin.  The fastest plan is
        kept in ``compute_plan`` and, with ``cache``, stored per (GPU, N,
        density, type count, integrator, candidate sets) in
        ``$GAMDPY_B200_CACHE/autotune.json`` (default
        ``~/.cache/gamdpy_b200``): a later call with the same key applies it
        without timing.  The configuration, its box and the integrator state
        are restored afterwards, so the run that follows equals a run started
        with the chosen plan."""
        if isinstance(self.integrator, NVT_Langevin):
            raise NotImplementedError("autotune: the NVT_Langevin generators advance with every timed step")
        steps = steps or min(self.steps_per_block, 256)
        conf = self.configuration
        pp = self._pair
        skins = [float(x) for x in skins] if skins is not None else [float(self.compute_plan["skin"])]
        if nblists is None:
            nblists = [self.compute_plan["nblist"]]
            if nblists[0] != "N squared" and conf.N < 32000:
                nblists.append("N squared")
            if nblists[0] != "linked lists" and conf.N > 2000:
                nblists.append("linked lists")
        key = self._autotune_key(list(tps_candidates), skins, list(nblists))
        self.autotune_from_cache = False
        if cache:
            hit = _autotune_cache_load().get(key)
            if hit is not None:
                self._apply_plan(hit["nblist"], hit["lanes"], hit["skin"])
                self.autotune_from_cache = True
                return dict(self.compute_plan)
        saved = self._save_state()
        best = None
        for nblist in nblists:
            for skin in skins:
                for tp in tps_candidates:
                    self._apply_plan(nblist, tp, skin)
                    self._restore_state(saved)
                    self.integrate_self(0.0, steps)  # warm-up
                    ms = self.integrate_self(0.0, steps)
                    if verbose:
                        print(f"autotune: {nblist} tp={tp} skin={skin}: {steps / ms * 1000:.1f} TPS")
                    if best is None or ms < best[0]:
                        best = (ms, nblist, tp, skin)
        _, nblist, tp, skin = best
        self._apply_plan(nblist, tp, skin)
        self._restore_state(saved)
        if cache:
            _autotune_cache_store(key, {"nblist": nblist, "lanes": int(tp), "skin": float(skin),
                                        "tps": steps / best[0] * 1000})
        return dict(self.compute_plan)

    def _autotune_key(self, tps, skins, nblists):
        conf = self.configuration
        rho = conf.N / float(np.prod(conf.simbox.lengths.astype(np.float64)))
        return "|".join([_lib.device_name(self._sim.device), f"N={conf.N}", f"rho={rho:.4f}",
                         f"nt={int(np.max(conf.ptype)) + 1 if conf.N else 1}", type(self.integrator).__name__,
                         f"tp={tps}", f"skin={skins}", f"nblist={nblists}"])

    def _apply_plan(self, nblist, tp, skin):
        pp = self._pair
        self.compute_plan["nblist"], self.compute_plan["lanes"], self.compute_plan["skin"] = nblist, tp, skin
        kind = _lib.NBLIST_NSQ if nblist == "N squared" else _lib.NBLIST_CELLS
        pp.make_nblist(self.configuration, self.compute_plan)
        self._sim.set_nblist(kind, float(np.float32(skin)), pp.max_num_nbs)
        self._sim.set_plan(int(tp))

    def _save_state(self):
        conf = self.configuration
        st = {"r": conf["r"].copy(), "v": conf["v"].copy(), "r_im": conf.r_im.copy(),
              "box": conf.simbox.lengths.copy()}
        if isinstance(self.integrator, NVT):
            st["xi"] = self._sim.thermostat_state()
        if isinstance(self.integrator, NPT_Atomic):
            st["npt"] = self._sim.npt_state()
        return st

    def _restore_state(self, st):
        conf = self.configuration
        conf["r"], conf["v"] = st["r"], st["v"]
        conf.r_im[:] = st["r_im"]
        conf.simbox.lengths[:] = st["box"]
        if "xi" in st:
            self._sim.set_thermostat_state(st["xi"])
            self.integrator.thermostat_state[:] = st["xi"]
        if "npt" in st:
            self._sim.set_npt_state(*st["npt"])
            self.integrator.thermostat_state[:], self.integrator.barostat_state[:] = st["npt"]
        conf.copy_to_device()


def get_default_sim():
    """The single-component LJ crystal (FCC 8x8x8, rho = 0.973) in NVT at
    T = 0.7 (get_default_sim.py:3-43)."""
    from .misc import make_function_constant  # noqa: F401
    from .potential_functions import LJ_12_6_sigma_epsilon, apply_shifted_potential_cutoff

    configuration = Configuration(D=3)
    configuration.make_lattice(unit_cells.FCC, cells=[8, 8, 8], rho=0.973)
    configuration["m"] = 1.0
    temperature = 0.7
    configuration.randomize_velocities(temperature=temperature)
    pair_func = apply_shifted_potential_cutoff(LJ_12_6_sigma_epsilon)
    sig, eps, cut = 1.0, 1.0, 2.5
    pair_pot = PairPotential(pair_func, params=[sig, eps, cut], max_num_nbs=1000)
    integrator = NVT(temperature=temperature, tau=0.2, dt=0.005)
    runtime_actions = [ConfigurationSaver(), ScalarSaver(), MomentumReset(100)]
    return Simulation(configuration, pair_pot, integrator, runtime_actions, num_timeblocks=8,
                      steps_per_timeblock=1024, storage="memory")
