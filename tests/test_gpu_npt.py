"""NPT_Atomic on the GPU (integrators/NPT_Atomic.py): the trajectory, box and
thermostat/barostat states of gamdpy's own run (golden lj256_npt), the
oracle restatement on a cell-list system whose box changes, and the state
point the thermostat and barostat hold."""
import numpy as np
import pytest

import gamdpy_b200 as gp
from conftest import golden, rel_rms
from gamdpy_b200 import workloads

pytestmark = pytest.mark.gpu

FORCE_TOL = 1e-5  # relative RMS against the reference's float32 path


def npt_sim(conf, T, tau, P, tau_p, dt, nblist, skin, blocks, steps, every, lanes=0, frames=False):
    pp = gp.PairPotential(gp.apply_shifted_force_cutoff(gp.LJ_12_6_sigma_epsilon), params=[1.0, 1.0, 2.5],
                          max_num_nbs=300)
    integ = gp.integrators.NPT_Atomic(temperature=T, tau=tau, pressure=P, tau_p=tau_p, dt=dt)
    plan = {"pb": 8, "tp": 1, "lanes": lanes, "skin": skin, "nblist": nblist}
    actions = [gp.ScalarSaver(every)]
    if frames:
        actions.insert(0, gp.ConfigurationSaver(include_simbox=True))
    sim = gp.Simulation(conf, pp, integ, actions, num_timeblocks=blocks, steps_per_timeblock=steps,
                        compute_plan=plan, storage="memory")
    return sim, integ


def test_npt_trajectory_vs_gamdpy():
    d = golden("lj256_npt")
    conf = gp.Configuration(D=3, compute_flags={"Vol": True})
    conf["r"] = d["r0"].copy()
    conf["v"] = d["v0"].copy()
    conf.simbox = gp.Orthorhombic(3, d["box0"])
    conf["m"] = 1.0
    sim, integ = npt_sim(conf, float(d["temperature"]), float(d["tau"]), float(d["pressure"]), float(d["tau_p"]),
                         float(d["dt"]), str(d["nblist"]), float(d["skin"]), int(d["blocks"]), int(d["steps"]),
                         int(d["every"]), frames=True)
    ts_t, bs_t = sim._sim.npt_state()
    assert np.allclose(ts_t, d["ts_after_test"], rtol=1e-5, atol=1e-7)
    assert np.allclose(bs_t, d["bs_after_test"], rtol=1e-5, atol=1e-7)
    for _ in sim.run_timeblocks():
        pass
    assert np.allclose(conf.simbox.lengths, d["box"], rtol=1e-6, atol=0)
    assert abs(integ.thermostat_state[0] - d["thermostat_state"][0]) <= 1e-4 * abs(d["thermostat_state"][0])
    assert abs(integ.barostat_state[0] - d["barostat_state"][0]) <= 1e-4 * abs(d["barostat_state"][0])
    assert abs(integ.barostat_state[2] - d["barostat_state"][2]) <= 1e-6 * d["barostat_state"][2]
    assert np.abs(conf["r"] - d["r"]).max() < 1e-5
    assert np.array_equal(conf.r_im, d["r_im"])
    assert rel_rms(conf["v"], d["v"]) < FORCE_TOL
    out = sim.output
    assert list(out.attrs["scalar_names"]) == list(d["scalar_names"])
    ref, got = d["scalars"], out["scalars"]
    assert got.shape == ref.shape
    for c, nm in enumerate(d["scalar_names"]):
        tol = 1e-6 if str(nm) == "Vol" else 1e-5
        assert np.abs(got[:, :, c] - ref[:, :, c]).max() <= tol * np.abs(ref[:, :, c]).max(), nm
    # ConfigurationSaver(include_simbox=True): frames at steps 0, 1, 2, 4, 8
    # of each block with the box of that step
    fr, ref_fr = out["block"], d["frames"]
    assert fr.shape == ref_fr.shape
    assert np.abs(fr[:, :, 0] - ref_fr[:, :, 0]).max() < 1e-5
    assert np.array_equal(fr[:, :, 1], ref_fr[:, :, 1])
    assert np.allclose(out["sim_box"], d["frame_boxes"], rtol=1e-6, atol=0)


def test_npt_cells_vs_oracle(oracle):
    """A 4000-particle LJ liquid under cell lists, 3 timeblocks of 20 steps of
    NPT_Atomic with the box expanding: box, states and positions against the
    oracle restatement (float32 round-off grows along the chaotic
    trajectory, hence 1e-4)."""
    conf = workloads.lj_configuration([10, 10, 10], 0.973, 2.0, seed=4)
    conf.randomize_velocities(temperature=2.0, seed=4)
    r0, v0, box0 = conf["r"].copy(), conf["v"].copy(), conf.simbox.lengths.copy()
    sim, integ = npt_sim(conf, 2.0, 0.4, 4.7, 2.0, 0.004, "linked lists", 0.5, 3, 20, 4)
    ts_t, bs_t = sim._sim.npt_state()
    for _ in sim.run_timeblocks():
        pass
    table = oracle.param_table([1.0, 1.0, 2.5])
    run = oracle.Run(r0, v0, 1.0, None, box0, table, nblist="linked lists", skin=0.5, max_nbs=300,
                     integrator="NPT_Atomic", dt=0.004, temperature=2.0, tau=0.4, pressure=4.7, tau_p=2.0, fma=1)
    run.run_timeblock(1)  # Simulation's kernel test step
    assert np.allclose(run.ts, ts_t, rtol=1e-5, atol=1e-7) and np.allclose(run.bs, bs_t, rtol=1e-5, atol=1e-7)
    run.r[:], run.v[:], run.img[:], run.box[:] = r0, v0, 0, box0
    run.have_list.value = 0
    for _ in range(3):
        run.run_timeblock(20)
    assert not np.allclose(run.box, box0)  # the box moved
    assert np.allclose(conf.simbox.lengths, run.box, rtol=1e-6)
    assert abs(integ.barostat_state[0] - run.bs[0]) <= 1e-4 * abs(run.bs[0])
    assert abs(integ.thermostat_state[0] - run.ts[0]) <= 1e-4 * max(abs(run.ts[0]), 1e-2)
    L = run.box
    dr = conf["r"] - run.r
    dr -= L * np.round(dr / L)
    assert np.abs(dr).max() < 1e-4


def test_npt_state_point():
    """The reference's NPT consistency case (examples/consistency_NPT.py:15-29):
    LJ with shifted-potential cutoff, T = 2.0, P = 4.7, tau = 0.4,
    tau_p = 20, dt = 0.001, from an FCC lattice at rho = 0.754289, the
    density at which the pressure is 4.7.  After 8 timeblocks of 2048 steps,
    the next 24 give the mean density within 1.5 %, the mean kinetic
    temperature within 1 % and the mean instant pressure (N T_kin + W) / V
    (NPT_Atomic.py:152) within 3 % of those values."""
    T, P, rho = 2.0, 4.7, 0.754289412611
    conf = gp.Configuration(D=3, compute_flags={"Vol": True})
    conf.make_lattice(gp.unit_cells.FCC, cells=[8, 8, 8], rho=rho)
    conf["m"] = 1.0
    conf.randomize_velocities(temperature=T, seed=0)
    pp = gp.PairPotential(gp.apply_shifted_potential_cutoff(gp.LJ_12_6_sigma_epsilon), params=[1.0, 1.0, 2.5],
                          max_num_nbs=1000)
    integ = gp.integrators.NPT_Atomic(temperature=T, tau=0.4, pressure=P, tau_p=20, dt=0.001)
    sim = gp.Simulation(conf, pp, integ, [gp.ScalarSaver(32), gp.MomentumReset(100)], num_timeblocks=32,
                        steps_per_timeblock=2048, storage="memory")
    for _ in sim.run_timeblocks():
        pass
    U, W, K, V = gp.extract_scalars(sim.output, ["U", "W", "K", "Vol"], first_block=8)
    n = conf.N
    t_kin = 2 * K / (3 * n - 3)
    p_inst = (n * t_kin + W) / V
    print("rho", n / V.mean(), "T", t_kin.mean(), "P", p_inst.mean())
    assert abs(n / V.mean() - rho) < 0.015 * rho
    assert abs(t_kin.mean() - T) < 0.01 * T
    assert abs(p_inst.mean() - P) < 0.03 * P


def test_npt_autotune_restores_box_and_states(tmp_path, monkeypatch):
    """Simulation.autotune under NPT_Atomic: the timed trials change the box
    and the barostat; afterwards both are back, so the run that follows equals
    a run started with the chosen plan bit for bit."""
    monkeypatch.setenv("GAMDPY_B200_CACHE", str(tmp_path))

    def make(plan_lanes=0, skin=0.5, nblist="linked lists"):
        conf = workloads.lj_configuration([10, 10, 10], 0.9, 1.5, seed=9)
        pp = gp.PairPotential(gp.apply_shifted_force_cutoff(gp.LJ_12_6_sigma_epsilon), params=[1.0, 1.0, 2.5],
                              max_num_nbs=300)
        integ = gp.integrators.NPT_Atomic(temperature=1.5, tau=0.4, pressure=2.0, tau_p=2.0, dt=0.004)
        plan = {"pb": 8, "tp": 1, "lanes": plan_lanes, "skin": skin, "nblist": nblist}
        return gp.Simulation(conf, pp, integ, [gp.ScalarSaver(8)], num_timeblocks=2, steps_per_timeblock=32,
                             compute_plan=plan, storage="memory"), conf, integ

    a, ca, ia = make()
    box0 = ca.simbox.lengths.copy()
    chosen = a.autotune(tps_candidates=(1, 4), nblists=["linked lists"], steps=20)
    assert np.array_equal(ca.simbox.lengths, box0)
    for _ in a.run_timeblocks():
        pass
    b, cb, ib = make(chosen["lanes"], chosen["skin"], chosen["nblist"])
    for _ in b.run_timeblocks():
        pass
    assert np.array_equal(ca["r"], cb["r"]) and np.array_equal(ca.simbox.lengths, cb.simbox.lengths)
    assert np.array_equal(ia.barostat_state, ib.barostat_state)


def test_batches_refuse_npt():
    conf = workloads.lj_configuration([6, 6, 6], 0.9, 1.5, seed=1)
    sim, _ = npt_sim(conf, 1.5, 0.4, 2.0, 2.0, 0.004, "N squared", 0.5, 1, 16, 4)
    with pytest.raises(Exception, match="NPT"):
        gp.SimulationBatch([sim])


def test_saved_boxes_of_a_fixed_box():
    """ConfigurationSaver(include_simbox=True) under NVE: every frame's box
    row is the box."""
    conf = workloads.lj_configuration([6, 6, 6], 0.9, 1.0, seed=2)
    pp = gp.PairPotential(gp.apply_shifted_force_cutoff(gp.LJ_12_6_sigma_epsilon), params=[1.0, 1.0, 2.5],
                          max_num_nbs=300)
    sim = gp.Simulation(conf, pp, gp.integrators.NVE(dt=0.004), [gp.ConfigurationSaver(include_simbox=True)],
                        num_timeblocks=2, steps_per_timeblock=16, storage="memory")
    for _ in sim.run_timeblocks():
        pass
    boxes = sim.output["sim_box"]
    assert boxes.shape == (2, 6, 3)
    assert np.array_equal(boxes, np.broadcast_to(conf.simbox.lengths, boxes.shape))
