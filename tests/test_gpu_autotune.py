"""The autotuners (Simulation.autotune, SimulationBatch.autotune; the
reference's Simulation.autotune, simulation/Simulation.py:636-821): the
timed trials leave no trace on the state, so a tuned run equals a run
started with the chosen plan bit for bit, and the per-GPU cache replays a
choice without timing."""
import numpy as np
import pytest

import gamdpy_b200 as gp
from gamdpy_b200 import workloads

pytestmark = pytest.mark.gpu


def ka_sim(n, seed, plan, blocks=2, steps=64, rho=1.2, temperature=0.45):
    conf = workloads.ka_configuration(n, rho=rho, temperature=temperature, seed=seed)
    integ = gp.integrators.NVT(temperature=temperature, tau=0.2, dt=0.005)
    sim = gp.Simulation(conf, workloads.ka_pair_potential(max_num_nbs=300), integ,
                        [gp.ScalarSaver(8), gp.MomentumReset(100)], num_timeblocks=blocks, steps_per_timeblock=steps,
                        compute_plan=dict(plan), storage="memory")
    return sim, conf, integ


def run_all(sim):
    for _ in sim.run_timeblocks():
        pass
    return sim.configuration["r"].copy(), sim.configuration["v"].copy(), np.array(sim.output["scalars"])


def test_simulation_autotune_then_run_equals_plan_run(tmp_path, monkeypatch):
    monkeypatch.setenv("GAMDPY_B200_CACHE", str(tmp_path))
    plan = {"pb": 64, "tp": 1, "skin": 0.3, "nblist": "linked lists"}
    a, _, _ = ka_sim(6000, 3, plan)
    chosen = a.autotune(tps_candidates=(1, 2, 4), skins=(0.3, 0.4), steps=40)
    assert not a.autotune_from_cache
    assert chosen["nblist"] in ("linked lists", "N squared") and chosen["lanes"] in (1, 2, 4)
    ra, va, sa = run_all(a)
    b, _, _ = ka_sim(6000, 3, chosen)
    rb, vb, sb = run_all(b)
    assert np.array_equal(ra, rb) and np.array_equal(va, vb) and np.array_equal(sa, sb)
    # the same key again: the cached plan, no timing
    c, _, _ = ka_sim(6000, 3, plan)
    again = c.autotune(tps_candidates=(1, 2, 4), skins=(0.3, 0.4), steps=40)
    assert c.autotune_from_cache
    for k in ("nblist", "lanes", "skin"):
        assert again[k] == chosen[k]
    assert (tmp_path / "autotune.json").exists()


def test_batch_autotune_then_run_equals_shape_run():
    plan = {"pb": 64, "tp": 1, "skin": 0.3, "nblist": "linked lists"}
    sizes = [(600, 1.2, 0.5), (1500, 1.1, 0.8), (3000, 1.25, 0.6), (6000, 1.2, 0.45), (9000, 1.15, 0.9)]

    def build():
        return [ka_sim(n, k, plan, blocks=1, steps=40, rho=rho, temperature=t)[0]
                for k, (n, rho, t) in enumerate(sizes)]

    sims = build()
    batch = gp.SimulationBatch(sims)
    shape = batch.autotune(candidates=(0, 128), clg_candidates=(0, 2048, 4096), clg_tps=(1, 2), steps=20)
    assert batch.shape == shape
    for _ in batch.run_timeblocks():
        pass
    ref = build()
    batch2 = gp.SimulationBatch(ref, *shape)
    for _ in batch2.run_timeblocks():
        pass
    for x, y in zip(sims, ref):
        assert np.array_equal(x.configuration["r"], y.configuration["r"])
        assert np.array_equal(x.configuration["v"], y.configuration["v"])
        assert np.array_equal(np.array(x.output["scalars"]), np.array(y.output["scalars"]))
