"""Evaluator (gamdpy/tools/Evaluator.py): interactions on a configuration
without time stepping."""
import numpy as np

from . import _lib
from .simulation import get_default_compute_plan


class Evaluator:
    """Evaluate forces, U, W and lapU of ``interactions`` on a configuration
    (tools/Evaluator.py:11-95).  ``evaluate`` uploads the configuration, runs
    the neighbour-list build and one force evaluation, and copies f and the
    per-particle scalars back."""

    def __init__(self, configuration, interactions, compute_plan=None, verbose=True, device=0):
        self.configuration = configuration
        self.compute_plan = dict(compute_plan) if compute_plan is not None else get_default_compute_plan(
            configuration)
        self.interactions = interactions if isinstance(interactions, list) else [interactions]
        from .simulation import split_interactions
        pp, bonds = split_interactions(self.interactions)
        self._pair = pp
        table, _ = pp.table()
        self._sim = _lib.Sim(configuration.N, table.shape[0], device)
        self._sim.set_box(configuration.simbox.lengths)
        pp.configure_device(self._sim, configuration, self.compute_plan)
        if bonds is not None:
            bonds.configure_device(self._sim, configuration)
        self._sim.set_plan(int(self.compute_plan.get("lanes", 0)))

    def evaluate(self, configuration=None):
        conf = configuration if configuration is not None else self.configuration
        sim = self._sim
        sim.set_box(conf.simbox.lengths)
        sim.upload(conf["r"], conf["v"], conf["m"], conf.ptype, conf.r_im)
        sim.eval_forces()
        st = sim.download(r=False, v=False, f=True, r_im=False)
        conf.vectors["f"] = st["f"]
        sc = sim.download_scalars()
        for k in ("U", "W", "lapU"):
            if k in conf.sid:
                conf.scalars[:, conf.sid[k]] = sc[k]
        self._pair.check_datastructure_validity()


def calc_dynamics(trajectory, first_block, qvalues=None):
    """Mean square displacement, non-Gaussian parameter and self-intermediate
    scattering function from ConfigurationSaver frames, as
    tools/calc_dynamics.py:23-75 (same lags, same return dictionary), with
    the sums over particles on the GPU (gdb_calc_dynamics).  ``trajectory``
    is a Simulation's output (``block`` frames, ``ptype``, attrs ``dt`` and
    ``simbox_initial``); ``qvalues`` a float or one value per type."""
    import math
    ptype = np.asarray(trajectory["ptype"][:]).copy()
    attrs = trajectory.attrs
    simbox = np.asarray(attrs["simbox_initial"]).copy()
    num_types = int(np.max(ptype)) + 1
    if isinstance(qvalues, float):
        qvalues = np.ones(num_types) * qvalues
    blocks = np.asarray(trajectory["block"])
    num_blocks, conf_per_block, _, n, d = blocks.shape
    if first_block > num_blocks - 1:
        print("Warning [calc_dynamics] first_block greater than number of blocks. Remainder will be taken")
    first_block = first_block % num_blocks
    extra_times = int(math.log2(num_blocks - first_block)) - 1
    total_times = conf_per_block - 1 + extra_times
    msd, m4d, fs, count = _lib.calc_dynamics(blocks, ptype, simbox, first_block, qvalues, total_times)
    times = attrs["dt"] * 2 ** np.arange(total_times)
    alpha2 = 3 * m4d / (5 * msd ** 2) - 1
    return {"times": times, "msd": msd, "alpha2": alpha2, "qvalues": qvalues, "Fs": fs, "count": count}
