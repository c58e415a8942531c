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
        if len(self.interactions) != 1:
            raise NotImplementedError("gamdpy_b200 evaluates one PairPotential")
        pp = self.interactions[0]
        table, _ = pp.table()
        self._sim = _lib.Sim(configuration.N, table.shape[0], device)
        self._sim.set_box(configuration.simbox.lengths)
        pp.configure_device(self._sim, configuration, self.compute_plan)
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
        self.interactions[0].check_datastructure_validity()
