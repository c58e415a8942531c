"""Trajectory dynamics (tools/calc_dynamics.py) with the particle sums on the GPU.

Bars: on the golden synthetic trajectory, gamdpy's own calc_dynamics output
(tests/golden/make_dynamics_golden.py) to 1e-6 relative (gamdpy averages in
float32, the library in float64); lag counts and times exact; on the frames
a Simulation's ConfigurationSaver wrote, the oracle's restatement to 1e-6;
too short a trajectory is an error.
"""
import numpy as np
import pytest

import gamdpy_b200 as gp
from conftest import golden
from gamdpy_b200 import workloads

pytestmark = pytest.mark.gpu


class Trajectory(dict):
    def __init__(self, block, ptype, dt, box):
        super().__init__(block=block, ptype=ptype)
        self.attrs = {"dt": dt, "simbox_initial": box}


@pytest.mark.parametrize("tag", ["a", "b"])
def test_dynamics_vs_gamdpy_golden(tag):
    d = golden("dynamics")
    traj = Trajectory(d["block"], d["ptype"], float(d["dt"]), d["simbox_initial"])
    q = d[f"{tag}_qvalues"]
    q = float(q[0]) if tag == "a" else q
    res = gp.tools.calc_dynamics(traj, int(d[f"{tag}_first_block"]), qvalues=q)
    assert np.array_equal(res["count"], d[f"{tag}_count"])
    np.testing.assert_allclose(res["times"], d[f"{tag}_times"], rtol=1e-12)
    for k in ("msd", "Fs"):
        np.testing.assert_allclose(res[k], d[f"{tag}_{k}"], rtol=1e-6, atol=1e-9)
    np.testing.assert_allclose(res["alpha2"], d[f"{tag}_alpha2"], rtol=1e-5, atol=1e-6)


def test_dynamics_of_a_simulation_vs_oracle(oracle):
    conf = gp.Configuration(D=3)
    conf.make_lattice(gp.unit_cells.FCC, cells=[4, 4, 4], rho=1.2)
    conf["m"] = 1.0
    conf.randomize_velocities(temperature=0.8, seed=3)
    conf.ptype[::4] = 1
    pp = workloads.ka_pair_potential(max_num_nbs=1000)
    sim = gp.Simulation(conf, pp, gp.integrators.NVE(dt=0.005), [gp.ConfigurationSaver()], num_timeblocks=8,
                        steps_per_timeblock=128, storage="memory")
    for _ in sim.run_timeblocks():
        pass
    out = sim.output
    res = gp.calc_dynamics(out, 0, qvalues=7.0)
    ref = oracle.calc_dynamics(np.asarray(out["block"]), np.asarray(out["ptype"]), out.attrs["simbox_initial"],
                               float(out.attrs["dt"]), 0, qvalues=7.0)
    assert np.array_equal(res["count"], ref["count"])
    for k in ("msd", "Fs"):
        np.testing.assert_allclose(res[k], ref[k], rtol=1e-6, atol=1e-9)
    # alpha2 = 3 m4d / (5 msd^2) - 1 is near zero: the float32 averages of the
    # restatement show as absolute differences of ~1e-7
    np.testing.assert_allclose(res["alpha2"], ref["alpha2"], rtol=1e-5, atol=1e-6)
    assert res["msd"][-1, 0] > res["msd"][0, 0] > 0


def test_dynamics_needs_two_blocks():
    d = golden("dynamics")
    traj = Trajectory(d["block"][:2], d["ptype"], float(d["dt"]), d["simbox_initial"])
    with pytest.raises(Exception):
        gp.tools.calc_dynamics(traj, 1, qvalues=7.0)
