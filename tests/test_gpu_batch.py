"""Thread-block-cluster path and batched replicas on the GPU.

The cluster path (systems up to 4096 particles in one thread-block cluster;
GDB_CLUSTER=1 takes it for every system that fits, as single systems with
larger lists otherwise run on the grid kernel)
must give the same neighbour sets as the global builds and forces within
float32 round-off; a system run in a batch must give bit-for-bit the result
of the same system run alone on the same path; batches are reproducible.
"""
import os

import numpy as np
import pytest

import gamdpy_b200 as gp
from conftest import rel_rms, sorted_rows
from gamdpy_b200 import _lib, workloads

pytestmark = pytest.mark.gpu


def ka_sim(n, rho=1.2, temp=0.6, seed=0, skin=0.3, max_nbs=300, block=64, saver_every=16):
    conf = workloads.ka_configuration(n, rho=rho, temperature=temp, seed=seed)
    pp = workloads.ka_pair_potential(max_num_nbs=max_nbs)
    integ = gp.integrators.NVT(temperature=temp, tau=0.2, dt=0.005)
    plan = {"pb": 64, "tp": 1, "skin": skin, "UtilizeNIII": False, "gridsync": False, "nblist": "linked lists"}
    return gp.Simulation(conf, pp, integ, [gp.ScalarSaver(saver_every), gp.MomentumReset(50)], num_timeblocks=4,
                         steps_per_timeblock=block, compute_plan=plan, storage="memory")


def state(sim):
    st = sim._sim.download(r=True, v=True, f=True, r_im=True)
    return st


@pytest.fixture(autouse=True)
def cluster_whenever_it_fits(monkeypatch):
    # a single system takes the cluster path only while its list is small;
    # these tests compare that path with the global one and with batches
    monkeypatch.setenv("GDB_CLUSTER", "1")
    yield


@pytest.fixture
def no_cluster(monkeypatch):
    monkeypatch.setenv("GDB_CLUSTER", "0")
    yield
    monkeypatch.delenv("GDB_CLUSTER", raising=False)


@pytest.mark.parametrize("n", [256, 1500, 4096])
def test_cluster_path_lists_and_forces_match_global_path(n, monkeypatch):
    a = ka_sim(n, seed=3)
    monkeypatch.setenv("GDB_CLUSTER", "0")
    b = ka_sim(n, seed=3)
    monkeypatch.delenv("GDB_CLUSTER")
    for s in (a, b):
        s.configuration.copy_to_device()
        s._sim.run(0.0, 0)  # build + force evaluation only
    assert a._sim.last_path() == 2 and b._sim.last_path() != 2
    ca, ia = sorted_rows(a._sim.nblist(300))
    cb, ib = sorted_rows(b._sim.nblist(300))
    assert np.array_equal(ca, cb) and np.array_equal(ia, ib)
    fa, fb = state(a)["f"], state(b)["f"]
    assert rel_rms(fa, fb) < 1e-6
    ua, ub = a._sim.download_scalars()["U"], b._sim.download_scalars()["U"]
    np.testing.assert_allclose(ua, ub, rtol=1e-5, atol=1e-5)


def test_cluster_path_short_trajectory_matches_global_path(monkeypatch):
    a = ka_sim(2000, seed=5)
    monkeypatch.setenv("GDB_CLUSTER", "0")
    b = ka_sim(2000, seed=5)
    monkeypatch.delenv("GDB_CLUSTER")
    for s in (a, b):
        s.configuration.copy_to_device()
        s._sim.run(0.0, 20)
    assert a._sim.last_path() == 2
    ra, rb = state(a)["r"], state(b)["r"]
    assert np.max(np.abs(ra - rb)) < 1e-4


def test_capacity_overflow_falls_back_to_global_path(monkeypatch):
    # skin 1.7: about 360 neighbours per particle, more than shared memory holds
    a = ka_sim(4096, seed=7, skin=1.7, max_nbs=700)
    monkeypatch.setenv("GDB_CLUSTER", "0")
    b = ka_sim(4096, seed=7, skin=1.7, max_nbs=700)
    monkeypatch.delenv("GDB_CLUSTER")
    for s in (a, b):
        s.configuration.copy_to_device()
        s._sim.run(0.0, 30)
    assert a._sim.last_path() != 2
    sa, sb = state(a), state(b)
    for k in ("r", "v", "r_im"):
        assert np.array_equal(sa[k], sb[k]), k


SIZES = [(256, 1.15, 0.5), (700, 1.2, 0.9), (2000, 1.25, 0.45), (4000, 1.1, 0.7), (9000, 1.3, 0.6)]


def build(sizes, seed0=10):
    return [ka_sim(n, rho=rho, temp=t, seed=seed0 + k) for k, (n, rho, t) in enumerate(sizes)]


def test_batch_equals_individual_runs():
    alone, batched = build(SIZES), build(SIZES)
    for s in alone:
        s.configuration.copy_to_device()
        for blk in range(2):
            s._sim.run(float(blk * 64 * 0.005), 64)
    batch = gp.SimulationBatch(batched)
    for s in batched:
        s.configuration.copy_to_device()
    for blk in range(2):
        batch.integrate_self(float(blk * 64 * 0.005), 64)
    paths = batch.paths()
    assert paths[:4] == [2, 2, 2, 2] and paths[4] == 3
    for k, (x, y) in enumerate(zip(alone, batched)):
        sx, sy = state(x), state(y)
        if paths[k] == 2:
            for q in ("r", "v", "r_im", "f"):
                assert np.array_equal(sx[q], sy[q]), (k, q)
            assert np.array_equal(x._sim.scalar_rows(4), y._sim.scalar_rows(4))
            assert np.array_equal(x._sim.thermostat_state(), y._sim.thermostat_state())
        else:
            # the large system ran on 16 CTAs instead of the whole grid: block
            # partial sums differ in float64 rounding only
            assert np.max(np.abs(sx["r"] - sy["r"])) < 1e-3


def test_batch_is_reproducible():
    runs = []
    for _ in range(2):
        sims = build(SIZES[:4] + [(6000, 1.2, 0.6)], seed0=40)
        batch = gp.SimulationBatch(sims)
        for s in sims:
            s.configuration.copy_to_device()
        batch.integrate_self(0.0, 100)
        runs.append([state(s)["r"] for s in sims])
    for a, b in zip(*runs):
        assert np.array_equal(a, b)


def test_simulation_batch_outputs_match_individual_simulations():
    sizes = SIZES[:3]
    alone, batched = build(sizes, seed0=70), build(sizes, seed0=70)
    for s in alone:
        for _ in s.run_timeblocks():
            pass
    batch = gp.SimulationBatch(batched)
    for _ in batch.run_timeblocks():
        pass
    for x, y in zip(alone, batched):
        assert np.array_equal(x.output["scalars"], y.output["scalars"])
        assert np.array_equal(x.configuration["r"], y.configuration["r"])
    assert batch.get_tps() > 0


def test_batch_rejects_mismatched_systems():
    a = ka_sim(256, block=64)
    b = ka_sim(256, block=32)
    with pytest.raises(ValueError):
        gp.SimulationBatch([a, b])


def test_uneven_replica_sweep_matches_individual_runs():
    # several systems per cluster shape and several global-memory clusters
    points = workloads.ka_replica_sweep(24, seed=5, n_max=12000)

    def make():
        return [ka_sim(n, rho=rho, temp=t, seed=k) for k, (n, rho, t) in enumerate(points)]

    alone, batched = make(), make()
    for s in alone:
        s.configuration.copy_to_device()
        s._sim.run(0.0, 64)
    batch = gp.SimulationBatch(batched)
    for s in batched:
        s.configuration.copy_to_device()
    batch.integrate_self(0.0, 64)
    paths = batch.paths()
    assert paths.count(2) >= 8 and paths.count(3) >= 4
    for k, (x, y) in enumerate(zip(alone, batched)):
        sx, sy = state(x), state(y)
        if paths[k] == 2:
            assert np.array_equal(sx["r"], sy["r"]) and np.array_equal(sx["v"], sy["v"]), k
        else:
            assert np.max(np.abs(sx["r"] - sy["r"])) < 1e-3, k
        assert y._sim.status() == 0


def test_cluster_lists_survive_other_work_between_blocks():
    # lists live in shared memory during a launch only; the next timeblock
    # takes them from global memory even when other systems ran in between
    a, ref = ka_sim(1800, seed=21), ka_sim(1800, seed=21)
    other = ka_sim(3000, seed=22)
    for s in (a, ref, other):
        s.configuration.copy_to_device()
    a._sim.run(0.0, 64)
    other._sim.run(0.0, 64)
    a._sim.run(0.32, 64)
    ref._sim.run(0.0, 64)
    ref._sim.run(0.32, 64)
    assert a._sim.last_path() == 2 and a._sim.status() == 0
    sa, sr = state(a), state(ref)
    for q in ("r", "v", "r_im", "f"):
        assert np.array_equal(sa[q], sr[q]), q


def test_batch_continues_individual_runs_without_upload():
    sizes = SIZES[:4]
    alone, batched = build(sizes, seed0=90), build(sizes, seed0=90)
    for s in alone + batched:
        s.configuration.copy_to_device()
        s._sim.run(0.0, 64)
    for s in alone:
        s._sim.run(0.32, 64)
    batch = gp.SimulationBatch(batched)
    batch.integrate_self(0.32, 64)
    for x, y in zip(alone, batched):
        sx, sy = state(x), state(y)
        for q in ("r", "v", "r_im"):
            assert np.array_equal(sx[q], sy[q]), q


@pytest.mark.parametrize("pb", [32, 256, 512])
def test_cluster_particles_per_cta_plan(pb, monkeypatch):
    """Any particles-per-CTA request (requests above 256 are capped) gives the
    same trajectory as the global path, to float32 round-off."""
    a = ka_sim(2048, seed=31)
    monkeypatch.setenv("GDB_CLUSTER", "0")
    b = ka_sim(2048, seed=31)
    monkeypatch.delenv("GDB_CLUSTER")
    a._sim.set_plan(0, pb)
    for s in (a, b):
        s.configuration.copy_to_device()
        s._sim.run(0.0, 20)
    assert a._sim.last_path() == 2 and a._sim.status() == 0
    assert np.max(np.abs(state(a)["r"] - state(b)["r"])) < 1e-4
