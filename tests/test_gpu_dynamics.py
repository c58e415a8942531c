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


def _random_walk_frames(num_blocks, conf_per_block, n, seed):
    rng = np.random.default_rng(seed)
    box = np.array([5.0, 5.5, 6.0], np.float32)
    steps = num_blocks * conf_per_block
    walk = np.cumsum(rng.normal(0.0, 0.2, (steps, n, 3)), axis=0) + rng.uniform(-2, 2, (1, n, 3))
    img = np.floor(walk / box + 0.5)
    frames = np.zeros((num_blocks, conf_per_block, 2, n, 3), np.float32)
    frames[:, :, 0] = (walk - img * box).astype(np.float32).reshape(num_blocks, conf_per_block, n, 3)
    frames[:, :, 1] = img.reshape(num_blocks, conf_per_block, n, 3).astype(np.float32)
    return frames, box


def test_dynamics_more_pairs_than_one_grid_vs_oracle(oracle, monkeypatch):
    """1025 blocks of 65 frames: 65 600 lags inside blocks, more than the
    65 535 frame pairs one grid holds, plus the lags across blocks; equal to
    the oracle, and bit-identical when the pairs go in chunks of 1000 and the
    frames are staged three blocks at a time."""
    frames, box = _random_walk_frames(1025, 65, 8, seed=11)
    ptype = np.array([0, 1, 0, 0, 1, 0, 0, 0], np.int32)
    traj = Trajectory(frames, ptype, 0.005, box)
    res = gp.tools.calc_dynamics(traj, 0, qvalues=np.array([6.5, 7.5]))
    ref = oracle.calc_dynamics(frames, ptype, box, 0.005, 0, qvalues=np.array([6.5, 7.5]))
    assert np.array_equal(res["count"], ref["count"])
    for k in ("msd", "Fs"):
        np.testing.assert_allclose(res[k], ref[k], rtol=1e-6, atol=1e-9)
    monkeypatch.setenv("GDB_DYN_PAIR_CHUNK", "1000")
    monkeypatch.setenv("GDB_DYN_STAGE_BYTES", str(3 * 65 * 2 * 8 * 3 * 4))
    small = gp.tools.calc_dynamics(traj, 0, qvalues=np.array([6.5, 7.5]))
    for k in ("msd", "alpha2", "Fs"):
        assert np.array_equal(small[k], res[k])


def test_dynamics_type_without_particles_is_nan(oracle):
    """A type below max(ptype) with no particles gives NaN columns, as the
    reference's mean of an empty array; longer qvalues are cut to the types."""
    frames, box = _random_walk_frames(6, 5, 12, seed=4)
    ptype = np.zeros(12, np.int32)
    ptype[::3] = 2  # type 1 has no particles
    traj = Trajectory(frames, ptype, 0.005, box)
    q = np.array([6.0, 7.0, 8.0, 9.0])
    res = gp.tools.calc_dynamics(traj, 0, qvalues=q)
    assert res["msd"].shape == (res["count"].shape[0], 3)
    assert np.all(np.isnan(res["msd"][:, 1])) and np.all(np.isnan(res["Fs"][:, 1]))
    with np.errstate(invalid="ignore", divide="ignore"):
        import warnings
        with warnings.catch_warnings():
            warnings.simplefilter("ignore")
            ref = oracle.calc_dynamics(frames, ptype, box, 0.005, 0, qvalues=q)
    for k in ("msd", "Fs"):
        np.testing.assert_allclose(res[k], ref[k], rtol=1e-6, atol=1e-9, equal_nan=True)
