"""NVE energy conservation and equilibrium thermodynamics on the GPU.

gamdpy's own NVE test (tests/test_LJ_nxyz.py:10-111): single-component LJ
(shifted force at 2.5) on an FCC lattice at rho 0.8442, velocities at
T 1.44, dt 0.005, two timeblocks of 4096 steps, ScalarSaver every 8 steps
with Fsq and lapU, MomentumReset every 100 steps; over the second block the
reference asserts var(E)/N < 1e-4, 0.67 < Tkin, Tconf < 0.72,
0.86 < R < 0.99 and 5.1 < Gamma < 6.6.  The same bounds here, at the
reference test's example lattices.

Long run: the 2048-particle LJ crystal of the small plain benchmark (FCC
8^3, rho 0.973, T 0.7, N^2 list with skin 0.5, dt 0.005) for 10^5 NVE steps:
the reference's bound var(E)/N < 1e-4 over the whole run, and the drift of
E/N between the first and last tenth of the run below 1e-4.
"""
import numpy as np
import pytest

import gamdpy_b200 as gp

pytestmark = pytest.mark.gpu


def lj_fcc_run(nx, ny, nz, rho, temperature, blocks, steps, every, nblist=None, skin=None, reset=100, seed=0):
    conf = gp.Configuration(D=3, compute_flags={"Fsq": True, "lapU": True})
    conf.make_lattice(gp.unit_cells.FCC, cells=[nx, ny, nz], rho=rho)
    conf["m"] = 1.0
    conf.randomize_velocities(temperature=temperature, seed=seed)
    plan = gp.get_default_compute_plan(conf)
    if nblist is not None:
        plan["nblist"] = nblist
    if skin is not None:
        plan["skin"] = np.float32(skin)
    pairfunc = gp.apply_shifted_force_cutoff(gp.LJ_12_6_sigma_epsilon)
    pp = gp.PairPotential(pairfunc, params=[1.0, 1.0, 2.5], max_num_nbs=1000)
    actions = [gp.ScalarSaver(every, {"Fsq": True, "lapU": True, "stresses": False})]
    if reset:
        actions.insert(0, gp.MomentumReset(reset))
    sim = gp.Simulation(conf, pp, gp.integrators.NVE(dt=0.005), actions, num_timeblocks=blocks,
                        steps_per_timeblock=steps, compute_plan=plan, storage="memory")
    for _ in sim.run_timeblocks():
        pass
    return sim, conf


def results(sim, n, first_block):
    """tests/test_LJ_nxyz.py:64-92."""
    U, W, lapU, Fsq, K = (np.asarray(x, np.float64)
                          for x in gp.extract_scalars(sim.output, ["U", "W", "lapU", "Fsq", "K"], first_block=first_block))
    E = U + K
    tkin = 2 * K / 3 / (n - 1)
    tconf = Fsq / lapU
    half = len(U) // 2
    dU = U[half:] - U[half:].mean()
    dW = W[half:] - W[half:].mean()
    var_e = np.var(E) / n
    R = np.dot(dW, dU) / np.sqrt(np.dot(dW, dW) * np.dot(dU, dU))
    gamma = np.dot(dW, dU) / np.dot(dU, dU)
    return var_e, tkin[half:].mean(), tconf[half:].mean(), R, gamma, E


@pytest.mark.parametrize("nx,ny,nz", [(4, 4, 4), (5, 5, 13), (16, 16, 32)])
def test_nve_like_gamdpy(nx, ny, nz):
    n = 4 * nx * ny * nz
    sim, conf = lj_fcc_run(nx, ny, nz, 0.8442, 1.44, blocks=2, steps=4096, every=8)
    var_e, tkin, tconf, R, gamma, _ = results(sim, n, first_block=1)
    print(n, var_e, tkin, tconf, R, gamma)
    assert var_e < 1e-4
    assert 0.67 < tkin < 0.72, tkin
    assert 0.67 < tconf < 0.72, tconf
    assert 0.86 < R < 0.99, R
    assert 5.1 < gamma < 6.6, gamma


def test_nve_energy_drift_over_1e5_steps():
    n = 2048
    sim, conf = lj_fcc_run(8, 8, 8, 0.973, 0.7, blocks=25, steps=4000, every=100, nblist="N squared", skin=0.5,
                           reset=0)
    var_e, _, _, _, _, E = results(sim, n, first_block=0)
    tenth = len(E) // 10
    drift = (E[-tenth:].mean() - E[:tenth].mean()) / n
    print("var(E)/N", var_e, "drift of E/N over 1e5 steps", drift)
    assert len(E) == 25 * 40
    assert var_e < 1e-4
    assert abs(drift) < 1e-4
