"""NVT_Langevin (integrators/NVT_Langevin.py) on the GPU.

Bars: the first step equals the oracle's (the same numba xoroshiro128+
stream per particle, float32 round-off from the fused update and the math
library's log/cos), with the generators in the same state afterwards; a
20-step trajectory stays within float32 round-off of the oracle's; the graph path and the persistent kernel agree; gamdpy's own
statistical test (tests/test_nvt_langevin.py: LJ at the T = 1.2 fcc-liquid
coexistence state point, U and K per particle within 0.05 of the published
values) passes; batches refuse Langevin systems.
"""
import numpy as np
import pytest

import gamdpy_b200 as gp

pytestmark = pytest.mark.gpu


def lj_sim(conf, temperature, alpha, dt, seed, steps, actions=(), blocks=1, plan=None):
    pp = gp.PairPotential(gp.apply_shifted_force_cutoff(gp.LJ_12_6_sigma_epsilon), params=[1.0, 1.0, 2.5],
                          max_num_nbs=1000)
    integ = gp.integrators.NVT_Langevin(temperature, alpha=alpha, dt=dt, seed=seed)
    plan = plan or {"pb": 64, "tp": 1, "skin": 0.5, "UtilizeNIII": False, "gridsync": True, "nblist": "N squared"}
    return gp.Simulation(conf, pp, integ, list(actions), num_timeblocks=blocks, steps_per_timeblock=steps,
                         compute_plan=plan, storage="memory")


def lj_conf(cells=4, rho=0.8442, temperature=1.44, seed=0):
    conf = gp.Configuration(D=3)
    conf.make_lattice(gp.unit_cells.FCC, cells=[cells] * 3, rho=rho)
    conf["m"] = 1.0
    conf.randomize_velocities(temperature=temperature, seed=seed)
    return conf


def oracle_run(oracle, conf, temperature, alpha, dt, seed, steps):
    """The oracle as the reference's Simulation runs it: the one-step kernel
    test of Simulation.__init__ (Simulation.py:209-210) leaves the
    configuration unchanged but not the integrator's device state (the
    generators have drawn one step, old_beta holds its random forces); then
    the timeblock from the original configuration."""
    table = oracle.param_table([np.float32(1.0), np.float32(1.0), np.float32(2.5)])
    run = oracle.Run(conf["r"], conf["v"], conf["m"], conf.ptype, conf.simbox.lengths, table, nblist="N squared",
                     skin=0.5, max_nbs=1000, integrator="NVT_Langevin", dt=dt, temperature=temperature,
                     alpha=alpha, seed=seed, fma=1)
    r0, v0 = run.r.copy(), run.v.copy()
    run.run_timeblock(1)
    run.r[:], run.v[:], run.img[:] = r0, v0, 0
    run.have_list.value = 0
    run.run_timeblock(steps)
    return run


@pytest.mark.parametrize("steps,rtol", [(1, 2e-6), (20, 1e-4)])
def test_langevin_trajectory_vs_oracle(oracle, steps, rtol):
    conf0 = lj_conf()
    ref = oracle_run(oracle, conf0, 1.2, 0.1, 0.005, 7, steps)
    conf = lj_conf()
    sim = lj_sim(conf, 1.2, 0.1, 0.005, 7, steps)
    for _ in sim.run_timeblocks():
        pass
    assert sim._sim.last_path() in (0, 1)
    dv = np.abs(conf["v"] - ref.v).max() / np.abs(ref.v).max()
    dr = np.abs(conf["r"] - ref.r).max()
    assert dv < rtol, dv
    assert dr < rtol * 10, dr
    assert np.array_equal(conf.r_im, ref.img)
    # the generators drew the kernel test's step and these steps, nothing else
    st, ob = sim._sim.langevin_state()
    assert np.array_equal(st, ref.rng)
    assert np.abs(ob - ref.old_beta).max() <= 1e-6


def test_langevin_graph_path_equals_persistent_kernel(monkeypatch):
    out = []
    for persistent in ("1", "0"):
        monkeypatch.setenv("GDB_PERSISTENT", persistent)
        conf = lj_conf(cells=5)
        sim = lj_sim(conf, 1.0, 0.5, 0.005, 11, 64, blocks=2)
        for _ in sim.run_timeblocks():
            pass
        out.append((conf["r"].copy(), conf["v"].copy(), sim._sim.last_path()))
    assert out[0][2] == 1 and out[1][2] == 0
    assert np.abs(out[0][0] - out[1][0]).max() < 1e-5
    assert np.abs(out[0][1] - out[1][1]).max() < 1e-4


def test_langevin_state_point_like_gamdpy():
    """tests/test_nvt_langevin.py of the reference."""
    temperature, density = 1.2, 1 / 0.9672
    expected_k = 3 / 2 * temperature
    expected_u = -4.020 - expected_k
    conf = gp.Configuration(D=3, compute_flags={"W": True, "K": True})
    conf.make_lattice(gp.unit_cells.FCC, cells=[7, 7, 7], rho=density)
    conf["m"] = 1.0
    conf.randomize_velocities(temperature=2 * temperature, seed=0)
    pp = gp.PairPotential(gp.apply_shifted_potential_cutoff(gp.LJ_12_6_sigma_epsilon), params=[1.0, 1.0, 2.5],
                          max_num_nbs=1000)
    integ = gp.integrators.NVT_Langevin(temperature, alpha=0.1, dt=0.005, seed=0)
    sim = gp.Simulation(conf, pp, integ, [gp.MomentumReset(100), gp.ScalarSaver(32, {"W": True, "K": True})],
                        num_timeblocks=32, steps_per_timeblock=512, storage="memory")
    for _ in sim.run_timeblocks():
        pass
    U, W, K = gp.extract_scalars(sim.output, ["U", "W", "K"], first_block=1)
    u, k = np.mean(U) / conf.N, np.mean(K) / conf.N
    print("U/N", u, "expected", expected_u, "K/N", k, "expected", expected_k)
    assert abs(u - expected_u) < 0.05
    assert abs(k - expected_k) < 0.05


def test_batches_refuse_langevin():
    conf = lj_conf()
    sim = lj_sim(conf, 1.0, 0.1, 0.005, 1, 32)
    with pytest.raises(Exception, match="Langevin"):
        gp.SimulationBatch([sim])
