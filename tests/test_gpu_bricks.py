"""The staged-halo path of large cell-list systems on the persistent kernel
(GDB_BRICKS=1: cells numbered in bricks of 4 x 4 x 4 cells, each brick's
halo staged in shared memory by bulk copies, 16-bit neighbour lists).

Bars: neighbour sets bit-exact against the oracle's cell build, on grids
whose cell count is 8 (a halo that covers the whole grid), not a multiple of
4 (partial bricks) and with particles on the box faces; forces within 1e-5
relative RMS of the oracle on the same positions, also after particles
crossed a face since the last build; the same trajectory as the row path to
float32 round-off growth; a halo that outgrows its stage hands the run to
the row path, bit-identical to a run that never used bricks.
"""
import numpy as np
import pytest

from conftest import rel_rms, sorted_rows
from gamdpy_b200 import _lib, workloads

pytestmark = pytest.mark.gpu

FORCE_TOL = 1e-5
PATH = {"1": 4}  # gdb_get_last_path: the staged-halo path


@pytest.fixture(params=["1"], ids=["staged-halos"])
def mode(request, monkeypatch):
    monkeypatch.setenv("GDB_BRICKS", request.param)
    return request.param


def _table(oracle):
    return oracle.param_table([workloads.KA_SIGMA, workloads.KA_EPSILON, workloads.KA_CUT])


def _sim(r, L, ptype, table, v=None, integ="nve"):
    n = len(r)
    sim = _lib.Sim(n, 2)
    sim.set_box(L)
    sim.set_pair_potential(_lib.POT_LJ_SIGMA_EPSILON, _lib.CUT_SHIFTED_FORCE, table)
    sim.set_nblist(_lib.NBLIST_CELLS, 0.3, 300)
    if integ == "nvt":
        sim.set_nvt(0.005, 0.2, _lib.TFUNC_CONSTANT, [0.6])
    else:
        sim.set_nve(0.005)
    sim.upload(r, np.zeros((n, 3), np.float32) if v is None else v, np.ones(n, np.float32), ptype)
    return sim


def _small_grid(monkeypatch):
    monkeypatch.setenv("GDB_BRICK_MIN_N", "0")
    monkeypatch.setenv("GDB_NSQ_AUTO", "0")
    monkeypatch.setenv("GDB_CLUSTER", "0")


@pytest.mark.parametrize("n,rho", [
    (200000, 1.2),  # 39 cells per side: 9 bricks and one of 3 cells
    (12000, 1.0),   # 16 cells per side: whole bricks
    (5000, 1.2),    # 11 cells: bricks of 4, 4 and 3
    (2800, 1.2),    # 9 cells: a brick of one cell
    (2100, 1.2),    # 8 cells: every halo is the whole grid
])
def test_brick_lists_and_forces_vs_oracle(oracle, monkeypatch, mode, n, rho):
    _small_grid(monkeypatch)
    conf = workloads.ka_configuration(n, rho=rho, seed=n, jitter=0.25)
    L = conf.simbox.lengths
    table = _table(oracle)
    sim = _sim(conf["r"], L, conf.ptype, table)
    sim.run(0.0, 0)  # rebuild + evaluation on the persistent kernel
    assert sim.last_path() == PATH[mode]
    ref, _ = oracle.nblist_cells(conf["r"], L, 2.5, 0.3, 300, fma=1)
    c1, f1 = sorted_rows(sim.nblist(300))
    c2, f2 = sorted_rows(ref)
    assert np.array_equal(c1, c2) and np.array_equal(f1, f2)
    res = oracle.forces(conf["r"], conf.ptype, L, table, ref, fma=1)
    st = sim.download()
    assert rel_rms(st["f"], res["f"]) < FORCE_TOL
    sc = sim.download_scalars()
    for k in ("U", "W", "lapU"):
        assert rel_rms(sc[k], res[k]) < FORCE_TOL, k


def test_brick_lists_with_particles_on_the_faces(oracle, monkeypatch, mode):
    """Coordinates exactly on +-L/2 (the +L/2 face bins into cell 0): the
    build takes the full minimum-image test, the stage moves those copies
    into each brick's frame."""
    _small_grid(monkeypatch)
    conf = workloads.ka_configuration(20000, seed=3, jitter=0.25)
    r = conf["r"].copy()
    L = conf.simbox.lengths.astype(np.float32)
    for k, idx in enumerate((5, 70, 333, 1500, 4000, 9000)):
        r[idx, k % 3] = (L[k % 3] / np.float32(2.0)) * np.float32(1 if k % 2 == 0 else -1)
    table = _table(oracle)
    sim = _sim(r, L, conf.ptype, table)
    sim.run(0.0, 0)
    assert sim.last_path() == PATH[mode]
    ref, _ = oracle.nblist_cells(r, L, 2.5, 0.3, 300, fma=1)
    c1, f1 = sorted_rows(sim.nblist(300))
    c2, f2 = sorted_rows(ref)
    assert np.array_equal(c1, c2) and np.array_equal(f1, f2)
    res = oracle.forces(r, conf.ptype, L, table, ref, fma=1)
    assert rel_rms(sim.download()["f"], res["f"]) < FORCE_TOL


@pytest.mark.parametrize("n", [30000, 200000])
def test_brick_forces_after_particles_crossed_faces(oracle, monkeypatch, mode, n):
    """After 60 steps at a high temperature many particles have wrapped
    through a face since the last build; a force evaluation on the list in
    place equals the oracle's forces on the same positions."""
    _small_grid(monkeypatch)
    conf = workloads.ka_configuration(n, rho=1.2, temperature=2.0, seed=9, jitter=0.05)
    L = conf.simbox.lengths
    table = _table(oracle)
    sim = _sim(conf["r"], L, conf.ptype, table, v=conf["v"])
    sim.run(0.0, 60)
    assert sim.last_path() == PATH[mode] and sim.status() == 0
    for _ in range(100):  # a state with no rebuild pending
        if sim.nbflag()[0] == 0:
            break
        sim.run(0.0, 1)
    assert sim.nbflag()[0] == 0
    rebuilds0 = sim.nbflag()[2]
    sim.eval_forces()
    assert sim.nbflag()[2] == rebuilds0  # the list of the last build was used
    st = sim.download()
    assert np.abs(st["r_im"]).sum() > 0
    ref, _ = oracle.nblist_cells(st["r"], L, 2.5, 0.3, 300, fma=1)
    res = oracle.forces(st["r"], conf.ptype, L, table, ref, fma=1)
    assert rel_rms(st["f"], res["f"]) < FORCE_TOL


def test_brick_trajectory_equals_row_path(oracle, monkeypatch, mode):
    """200 NVT steps with rebuilds: positions equal to the row path's within
    the growth of float32 round-off (pair sums in another order)."""
    _small_grid(monkeypatch)
    conf = workloads.ka_configuration(30000, rho=1.2, temperature=0.6, seed=21, jitter=0.05)
    L = conf.simbox.lengths
    table = _table(oracle)
    out = []
    for bricks in (mode, "0"):
        monkeypatch.setenv("GDB_BRICKS", bricks)
        sim = _sim(conf["r"], L, conf.ptype, table, v=conf["v"], integ="nvt")
        sim.run(0.0, 100)
        sim.run(0.5, 100)
        out.append((sim.download(), sim.last_path(), sim.nbflag()[2]))
    (a, pa, ra), (b, pb, rb) = out
    assert pa == PATH[mode] and pb == 1 and ra > 2 and rb > 2
    assert np.array_equal(a["r_im"], b["r_im"])
    assert np.abs(a["r"] - b["r"]).max() < 2e-3
    assert rel_rms(a["v"], b["v"]) < 2e-3


def test_brick_stage_overflow_hands_the_run_to_the_row_path(oracle, monkeypatch):
    """A stage limit below the halos (GDB_BRICK_HCAP) makes the staged
    path's first build give up; the run goes on on the row path from that
    point and equals a run that never staged, bit for bit."""
    _small_grid(monkeypatch)
    conf = workloads.ka_configuration(20000, rho=1.2, temperature=0.6, seed=5, jitter=0.05)
    L = conf.simbox.lengths
    table = _table(oracle)
    out = []
    for env in ({"GDB_BRICKS": "1", "GDB_BRICK_HCAP": "1000"}, {"GDB_BRICKS": "0"}):
        for k, v in env.items():
            monkeypatch.setenv(k, v)
        sim = _sim(conf["r"], L, conf.ptype, table, v=conf["v"], integ="nvt")
        sim.run(0.0, 50)
        assert sim.status() == 0 and sim.last_path() == 1
        out.append(sim.download())
        for k in env:
            monkeypatch.delenv(k)
    assert np.array_equal(out[0]["r"], out[1]["r"]) and np.array_equal(out[0]["v"], out[1]["v"])
