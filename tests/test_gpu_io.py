"""Host <-> device copies of a Configuration attached to a Simulation.

Bars: the one-call download into the Configuration's own (page-locked)
arrays gives exactly the arrays of the per-plane downloads; arrays the user
replaced after attaching still receive the state."""
import numpy as np
import pytest

import gamdpy_b200 as gp
from gamdpy_b200 import workloads

pytestmark = pytest.mark.gpu


def _sim(n=4000, flags=None):
    conf = workloads.ka_configuration(n, seed=3, compute_flags=flags)
    plan = {"pb": 64, "tp": 1, "lanes": 0, "skin": 0.3, "UtilizeNIII": False, "gridsync": False,
            "nblist": "linked lists"}
    sim = gp.Simulation(conf, workloads.ka_pair_potential(), gp.integrators.NVT(temperature=0.45, tau=0.2, dt=0.005),
                        [gp.ScalarSaver(8, flags)], num_timeblocks=2, steps_per_timeblock=32, compute_plan=plan,
                        storage="memory")
    return conf, sim


@pytest.mark.parametrize("flags", [None, {"lapU": True, "Fsq": True}])
def test_table_download_equals_plane_downloads(flags):
    conf, sim = _sim(flags=flags)
    m0 = conf["m"].copy()
    for _ in sim.run_timeblocks():
        pass
    st = sim._sim.download()
    sc = sim._sim.download_scalars()
    for k in ("r", "v", "f"):
        assert np.array_equal(conf[k], st[k]), k
    assert np.array_equal(conf.r_im, st["r_im"])
    for k in ("U", "W", "lapU", "K", "Fsq"):
        if k in conf.sid:
            assert np.array_equal(conf[k], sc[k]), k
    assert np.array_equal(conf["m"], m0)
    assert np.abs(conf["f"]).sum() > 0 and np.abs(conf["U"]).sum() > 0


def test_replaced_host_arrays_still_receive_the_state():
    conf, sim = _sim()
    for _ in sim.run_timeblocks(1):
        pass
    ref = {k: conf[k].copy() for k in ("r", "v")}
    conf.vectors.array = np.array(conf.vectors.array[:, ::1], order="F")  # not C-contiguous: per-plane path
    conf.copy_to_host()
    for k in ("r", "v"):
        assert np.array_equal(conf[k], ref[k])
