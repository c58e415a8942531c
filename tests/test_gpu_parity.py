"""GPU parity: libgamdb200 (through its C ABI) against gamdpy's golden outputs
and the CPU oracle.

Bars: neighbour sets and RDF counts bit-exact; forces/energies within 1e-5
relative RMS of gamdpy's float32 path; short trajectories within float32
round-off of gamdpy's; S(q) within 1e-4 of the float64 oracle.
"""
import numpy as np
import pytest

import gamdpy_b200 as gp
from conftest import golden, rel_rms, sorted_rows
from gamdpy_b200 import _lib, workloads

pytestmark = pytest.mark.gpu

FORCE_TOL = 1e-5


def make_sim(r, box, ptype, table, kind=_lib.POT_LJ_SIGMA_EPSILON, cutmode=_lib.CUT_SHIFTED_FORCE,
             nblist=_lib.NBLIST_NSQ, skin=0.5, max_nbs=300, v=None, tp=0):
    n = len(r)
    sim = _lib.Sim(n, table.shape[0])
    sim.set_box(box)
    sim.set_pair_potential(kind, cutmode, table)
    sim.set_nblist(nblist, skin, max_nbs)
    sim.set_plan(tp)
    sim.set_nve(0.005)
    v = np.zeros((n, 3), np.float32) if v is None else v
    sim.upload(r, v, np.ones(n, np.float32), ptype if ptype is not None else np.zeros(n, np.int32))
    return sim


def table_of(d):
    from oracle import oracle as O
    return O.param_table([d["sigma"], d["epsilon"], d["cut"]])


@pytest.mark.parametrize("name,tp", [("lj256_sf", 0), ("lj256_sp", 0), ("lj256_sf", 1), ("lj256_sf", 4),
                                     ("lj256_sf", 16)])
def test_nsq_list_and_forces_vs_gamdpy(name, tp):
    d = golden(name)
    cm = _lib.CUT_SHIFTED_FORCE if str(d["cutoff"]) == "SF" else _lib.CUT_SHIFTED_POTENTIAL
    sim = make_sim(d["r"], d["box"], d["ptype"], table_of(d), cutmode=cm, skin=float(d["skin"]), tp=tp)
    sim.eval_forces()
    counts, flat = sorted_rows(sim.nblist(300))
    assert np.array_equal(counts, d["nb_counts"])
    assert np.array_equal(flat, d["nb_flat"])
    f = sim.download()["f"]
    sc = sim.download_scalars()
    assert rel_rms(f, d["f"]) < FORCE_TOL
    for k in ("U", "W", "lapU"):
        assert rel_rms(sc[k], d[k]) < FORCE_TOL, k


@pytest.mark.parametrize("tp", [0, 1, 2, 8, 32])
def test_cell_list_and_forces_vs_gamdpy(tp):
    d = golden("ka1372_cells")
    sim = make_sim(d["r"], d["box"], d["ptype"], table_of(d), nblist=_lib.NBLIST_CELLS, skin=float(d["skin"]),
                   tp=tp)
    sim.eval_forces()
    counts, flat = sorted_rows(sim.nblist(300))
    assert np.array_equal(counts, d["nb_counts"])
    assert np.array_equal(flat, d["nb_flat"])
    f = sim.download()["f"]
    sc = sim.download_scalars()
    assert rel_rms(f, d["f"]) < FORCE_TOL
    for k in ("U", "W", "lapU"):
        assert rel_rms(sc[k], d[k]) < FORCE_TOL, k


@pytest.mark.parametrize("n,nblist", [(4000, _lib.NBLIST_NSQ), (30000, _lib.NBLIST_CELLS),
                                      (8000, _lib.NBLIST_CELLS)])
def test_lists_vs_oracle_larger(oracle, n, nblist):
    """Bit-exact sets at sizes the golden runs do not reach, against the
    oracle in the same (fused) distance form."""
    conf = workloads.ka_configuration(n, seed=7, jitter=0.2)
    table = oracle.param_table([workloads.KA_SIGMA, workloads.KA_EPSILON, workloads.KA_CUT])
    sim = make_sim(conf["r"], conf.simbox.lengths, conf.ptype, table, nblist=nblist, skin=0.3)
    sim.eval_forces()
    got = sim.nblist(300)
    ref, _ = oracle.nblist_nsq(conf["r"], conf.simbox.lengths, float(np.float32(2.5) + np.float32(0.3)), 300,
                               fma=1)
    c1, f1 = sorted_rows(got)
    c2, f2 = sorted_rows(ref)
    assert np.array_equal(c1, c2) and np.array_equal(f1, f2)
    res = oracle.forces(conf["r"], conf.ptype, conf.simbox.lengths, table, ref, fma=1)
    assert rel_rms(sim.download()["f"], res["f"]) < FORCE_TOL


def test_forces_with_positions_outside_the_box(oracle):
    """Positions uploaded outside [-L/2, L/2] (some moved by a whole box
    length, up to 3L/4 out, where gamdpy's one-wrap minimum image still holds
    for every pair): every pair is taken on the minimum image.  Forces equal the oracle's on the uploaded positions, and after
    one step (every position wrapped by one box length) on the new ones."""
    conf = workloads.ka_configuration(20000, seed=23, jitter=0.2)
    L = conf.simbox.lengths
    r = conf["r"].copy()
    r -= (L * np.round(r / L)).astype(np.float32)  # the jittered lattice into the box, then some out
    rng = np.random.default_rng(5)
    pick = rng.choice(len(r), 500, replace=False)
    # components more than L/4 from the centre move to the periodic image
    # across the box, up to 3L/4 out: every pair difference stays below
    # 3L/2, where the reference's one-wrap minimum image is exact
    q = r[pick]
    q = np.where(q > L / 4, q - L, np.where(q < -L / 4, q + L, q)).astype(np.float32)
    r[pick] = q
    assert np.any(np.abs(r) > L / 2) and np.all(np.abs(r) < 0.75 * L)
    table = oracle.param_table([workloads.KA_SIGMA, workloads.KA_EPSILON, workloads.KA_CUT])
    sim = make_sim(r, L, conf.ptype, table, nblist=_lib.NBLIST_CELLS, skin=0.3)
    sim.eval_forces()
    cps = float(np.float32(2.5) + np.float32(0.3))
    ref_list, _ = oracle.nblist_nsq(r, L, cps, 300, fma=1)
    res = oracle.forces(r, conf.ptype, L, table, ref_list, fma=1)
    assert rel_rms(sim.download()["f"], res["f"]) < FORCE_TOL
    sim.run(0.0, 1)
    st = sim.download()
    assert np.all(np.abs(st["r"]) < 0.51 * L)  # wrapped by one box length
    ref_list, _ = oracle.nblist_nsq(st["r"], L, cps, 300, fma=1)
    res = oracle.forces(st["r"], conf.ptype, L, table, ref_list, fma=1)
    assert rel_rms(st["f"], res["f"]) < FORCE_TOL


@pytest.mark.parametrize("n,face", [(1372, False), (1372, True), (600, False), (900, True), (20000, True)])
def test_cell_build_paths_vs_oracle(oracle, n, face):
    """Both build paths: >= 7 cells per dimension uses per-range periodic
    shifts, smaller grids (and a particle exactly on the +L/2 face, which the
    reference's modulo bins into cell 0) use the full minimum-image test."""
    conf = workloads.ka_configuration(n, seed=11, jitter=0.25)
    r = conf["r"].copy()
    L = conf.simbox.lengths
    if face:
        r[3, 0] = np.float32(L[0]) / np.float32(2.0)
        r[17, 1] = -np.float32(L[1]) / np.float32(2.0)
        r[29, 2] = np.float32(L[2]) / np.float32(2.0)
    table = oracle.param_table([workloads.KA_SIGMA, workloads.KA_EPSILON, workloads.KA_CUT])
    sim = make_sim(r, L, conf.ptype, table, nblist=_lib.NBLIST_CELLS, skin=0.3)
    sim.eval_forces()
    got = sim.nblist(300)
    ref, _ = oracle.nblist_nsq(r, L, float(np.float32(2.5) + np.float32(0.3)), 300, fma=1)
    c1, f1 = sorted_rows(got)
    c2, f2 = sorted_rows(ref)
    assert np.array_equal(c1, c2) and np.array_equal(f1, f2)


@pytest.mark.parametrize("n", [200000])
def test_thread_per_particle_build_vs_oracle(oracle, n, monkeypatch):
    """Large systems off the brick path build a thread per particle
    (standalone chain and persistent kernel); the sets must still equal the
    oracle's cell build."""
    monkeypatch.setenv("GDB_BRICKS", "0")
    conf = workloads.ka_configuration(n, seed=13, jitter=0.2)
    L = conf.simbox.lengths
    table = oracle.param_table([workloads.KA_SIGMA, workloads.KA_EPSILON, workloads.KA_CUT])
    ref, _ = oracle.nblist_cells(conf["r"], L, 2.5, 0.3, 300, fma=1)
    c2, f2 = sorted_rows(ref)
    sim = make_sim(conf["r"], L, conf.ptype, table, nblist=_lib.NBLIST_CELLS, skin=0.3)
    sim.eval_forces()  # standalone kernels
    c1, f1 = sorted_rows(sim.nblist(300))
    assert np.array_equal(c1, c2) and np.array_equal(f1, f2)
    sim.upload(conf["r"], np.zeros((n, 3), np.float32), np.ones(n, np.float32), conf.ptype)
    sim.run(0.0, 0)  # persistent kernel: rebuild + evaluation
    c1, f1 = sorted_rows(sim.nblist(300))
    assert np.array_equal(c1, c2) and np.array_equal(f1, f2)
    res = oracle.forces(conf["r"], conf.ptype, L, table, ref, fma=1)
    assert rel_rms(sim.download()["f"], res["f"]) < FORCE_TOL


def test_force_error_against_float64(oracle):
    """The float32 forces' error against every-operation-float64 forces on the
    same list (KA, 30 000 particles, cell lists): the library's and gamdpy's
    float32 form (the oracle) are both below 2e-6 relative RMS from float64,
    and from each other."""
    conf = workloads.ka_configuration(30000, seed=7, jitter=0.2)
    L = conf.simbox.lengths
    table = oracle.param_table([workloads.KA_SIGMA, workloads.KA_EPSILON, workloads.KA_CUT])
    sim = make_sim(conf["r"], L, conf.ptype, table, nblist=_lib.NBLIST_CELLS, skin=0.3)
    sim.eval_forces()
    nbl = sim.nblist(300)
    f_gpu = sim.download()["f"]
    f_ref32 = oracle.forces(conf["r"], conf.ptype, L, table, nbl, fma=1)["f"]
    f64 = oracle.forces_fp64(conf["r"], conf.ptype, L, workloads.KA_SIGMA, workloads.KA_EPSILON,
                             workloads.KA_CUT, nbl)
    e_gpu, e_ref = rel_rms(f_gpu, f64), rel_rms(f_ref32, f64)
    print("relative RMS against float64: library", e_gpu, "gamdpy float32 form", e_ref)
    assert e_gpu < 2e-6 and e_ref < 2e-6
    assert rel_rms(f_gpu, f_ref32) < FORCE_TOL


@pytest.mark.parametrize("n", [2048, 3072])
def test_persistent_small_system_cell_request_vs_oracle(oracle, monkeypatch, n):
    """Up to 3072 particles the persistent kernel answers a cell-list request
    with the N^2 build over positions staged in shared memory (48 KiB at
    3072, beyond the default limit with the kernel's static shared memory):
    the same sets as the oracle's cell build, and the same forces to float32
    round-off."""
    monkeypatch.setenv("GDB_CLUSTER", "0")
    conf = workloads.ka_configuration(n, seed=19, jitter=0.25)
    L = conf.simbox.lengths
    table = oracle.param_table([workloads.KA_SIGMA, workloads.KA_EPSILON, workloads.KA_CUT])
    sim = make_sim(conf["r"], L, conf.ptype, table, nblist=_lib.NBLIST_CELLS, skin=0.3)
    sim.run(0.0, 0)  # persistent kernel: rebuild + evaluation
    assert sim.last_path() == 1
    ref, _ = oracle.nblist_cells(conf["r"], L, 2.5, 0.3, 300, fma=1)
    c1, f1 = sorted_rows(sim.nblist(300))
    c2, f2 = sorted_rows(ref)
    assert np.array_equal(c1, c2) and np.array_equal(f1, f2)
    res = oracle.forces(conf["r"], conf.ptype, L, table, ref, fma=1)
    assert rel_rms(sim.download()["f"], res["f"]) < FORCE_TOL


def run_api_trajectory(d):
    """Golden trajectory through the public API (Simulation + runtime actions)."""
    n = len(d["r0"])
    conf = gp.Configuration(D=3)
    conf["r"] = d["r0"].copy()
    conf["v"] = d["v0"].copy()
    conf.simbox = gp.Orthorhombic(3, d["box"])
    conf["m"] = 1.0
    conf.ptype[:] = d["ptype"]
    pp = gp.PairPotential(gp.apply_shifted_force_cutoff(gp.LJ_12_6_sigma_epsilon),
                          params=[d["sigma"], d["epsilon"], d["cut"]], max_num_nbs=300)
    if str(d["integrator"]) == "NVE":
        integ = gp.integrators.NVE(dt=float(d["dt"]))
    else:
        integ = gp.integrators.NVT(temperature=float(d["temperature"]), tau=float(d["tau"]), dt=float(d["dt"]))
    actions = [gp.ScalarSaver(int(d["every"]))]
    if int(d["reset"]):
        actions.append(gp.MomentumReset(int(d["reset"])))
    plan = {"pb": 4, "tp": 1, "skin": float(d["skin"]), "UtilizeNIII": False, "gridsync": False,
            "nblist": str(d["nblist"])}
    sim = gp.Simulation(conf, pp, integ, actions, num_timeblocks=int(d["blocks"]),
                        steps_per_timeblock=int(d["steps"]), compute_plan=plan, storage="memory")
    xi_test = integ.d_thermostat_state.copy_to_host()[0] if str(d["integrator"]) == "NVT" else 0.0
    for _ in sim.run_timeblocks():
        pass
    return sim, conf, integ, xi_test


@pytest.mark.parametrize("name", ["lj256_nve", "ka1372_nvt"])
def test_trajectory_vs_gamdpy(name):
    d = golden(name)
    sim, conf, integ, xi_test = run_api_trajectory(d)
    if str(d["integrator"]) == "NVT":
        assert abs(xi_test - d["xi_after_test"][0]) <= 1e-5 * max(1.0, abs(xi_test))
        assert abs(integ.thermostat_state[0] - d["thermostat_state"][0]) <= 1e-5 * abs(d["thermostat_state"][0])
    assert np.abs(conf["r"] - d["r"]).max() < 1e-5
    assert np.array_equal(conf.r_im, d["r_im"])
    for k in ("v", "f", "U", "W", "K"):
        assert rel_rms(conf[k], d[k]) < FORCE_TOL, k
    out = sim.output
    assert list(out.attrs["scalar_names"]) == list(d["scalar_names"])
    ref = d["scalars"]
    got = out["scalars"]
    assert got.shape == ref.shape
    assert np.abs(got - ref).max() <= 2e-6 * np.abs(ref).max()


def _rdf_conf(d, tag):
    conf = gp.Configuration(D=3)
    conf["r"] = d[f"{tag}_r"].copy()
    conf.simbox = gp.Orthorhombic(3, d[f"{tag}_box"])
    conf.ptype[:] = d[f"{tag}_ptype"]
    return conf


def test_rdf_bit_exact_vs_gamdpy(oracle, monkeypatch):
    """Unfused distance form: the counts of gamdpy itself (run on the CPU,
    where numba does not contract).  Default fused form (gamdpy's numba.cuda
    build on B200 contracts, tests/golden/numba_contraction.json): the oracle's
    fused counts."""
    d = golden("rdf")
    for tag in ("lj256", "ka1372"):
        calc = gp.CalculatorRadialDistribution(_rdf_conf(d, tag), bins=100)
        calc.update()
        fused = oracle.rdf(d[f"{tag}_r"], d[f"{tag}_ptype"], d[f"{tag}_box"], 100, fma=1)
        assert np.array_equal(calc.rdf_list[0], fused.astype(np.float64)), tag
    monkeypatch.setenv("GDB_NBLIST_FMA", "0")
    for tag in ("lj256", "ka1372"):
        calc = gp.CalculatorRadialDistribution(_rdf_conf(d, tag), bins=100)
        calc.update()
        assert np.array_equal(calc.rdf_list[0], d[f"{tag}_bins_numba"]), tag
    # the normalised reading agrees with gamdpy's read()
    calc = gp.CalculatorRadialDistribution(_rdf_conf(d, "lj256"), bins=100)
    calc.update()
    assert np.allclose(calc.read()["rdf"], d["lj256_read_rdf"], rtol=1e-12)


def test_rdf_short_range_cells_vs_oracle(oracle):
    """r_max < L/3 takes the cell path: the same counts as the oracle's all
    pairs; r_max = L/2 takes the all-pairs path."""
    conf = workloads.ka_configuration(20000, seed=3, jitter=0.3)
    L = conf.simbox.lengths
    got = _lib.rdf_compute(conf["r"], conf.ptype, L, 2, 500, r_max=5.0)
    ref = oracle.rdf(conf["r"], conf.ptype, L, 500, fma=1, r_max=5.0)
    assert got.sum() > 0 and np.array_equal(got, ref)
    allpairs = _lib.rdf_compute(conf["r"], conf.ptype, L, 2, 500)
    assert np.array_equal(allpairs, oracle.rdf(conf["r"], conf.ptype, L, 500, fma=1))


def _random_types(n, nt, seed):
    return np.random.default_rng(seed).integers(0, nt, n).astype(np.int32)


@pytest.mark.parametrize("case", [
    # (n, types, bins, r_max as a fraction of L, fused distance form)
    (3000, 3, 200, 0.333, 1),  # three cells per side: the half shell wraps onto itself
    (3000, 2, 7000, 0.25, 1),  # 28 000 bins: histogram in global memory (cell path)
    (2501, 2, 7000, 0.0, 1),  # 28 000 bins, all pairs
    (1000, 1, 64, 0.2, 0),  # unfused distance form, cell path
    (777, 3, 50, 0.0, 0),  # unfused, all pairs, odd tile count
    (2, 1, 10, 0.0, 1),  # one pair
])
def test_rdf_paths_and_edges_vs_oracle(oracle, case, monkeypatch):
    """Cell and all-pairs searches, shared and global histograms, both
    distance forms: bit-exact counts against the oracle's all pairs."""
    n, nt, bins, frac, fma = case
    conf = workloads.ka_configuration(max(n, 4), rho=1.1, seed=n, jitter=0.3)
    r = conf["r"][:n].copy()
    L = conf.simbox.lengths
    pt = _random_types(n, nt, n)
    r_max = frac * float(np.min(L))
    monkeypatch.setenv("GDB_NBLIST_FMA", str(fma))
    got = _lib.rdf_compute(r, pt, L, nt, bins, r_max=r_max)
    ref = oracle.rdf(r, pt, L, bins, fma=fma, r_max=r_max)
    if ref.shape[0] < nt:  # the oracle sizes its histogram by the largest type present
        ref = np.pad(ref, ((0, nt - ref.shape[0]), (0, nt - ref.shape[1]), (0, 0)))
    assert got.sum() == ref.sum() and np.array_equal(got, ref)
    if n > 2:
        assert got.sum() > 0


@pytest.mark.parametrize("outside", [False, True])
@pytest.mark.parametrize("frac", [0.1, 0.2, 0.333])
def test_rdf_cells_faces_and_outside_positions_vs_oracle(oracle, frac, outside):
    """Particles exactly on the +-L/2 faces (the +L/2 face bins into cell 0)
    and, in the second form, particles one box length outside: the cell
    search must count what the minimum image gives, bit for bit."""
    conf = workloads.ka_configuration(4000, rho=1.1, seed=17, jitter=0.3)
    r = conf["r"].copy()
    L = conf.simbox.lengths.astype(np.float32)
    for k, idx in enumerate((3, 40, 77, 150, 600, 901)):
        r[idx, k % 3] = (L[k % 3] / np.float32(2.0)) * np.float32(1 if k % 2 == 0 else -1)
    if outside:
        r[1000:1040, 0] += L[0]
        r[2000:2010, 2] -= L[2]
    pt = conf.ptype
    r_max = frac * float(np.min(L))
    got = _lib.rdf_compute(r, pt, L, 2, 300, r_max=r_max)
    ref = oracle.rdf(r, pt, L, 300, fma=1, r_max=r_max)
    assert got.sum() > 0 and np.array_equal(got, ref)


def test_rdf_device_path_matches_host_path(oracle):
    d = golden("ka1372_cells")
    conf = gp.Configuration(D=3)
    conf["r"] = d["r"].copy()
    conf.simbox = gp.Orthorhombic(3, d["box"])
    conf.ptype[:] = d["ptype"]
    conf["m"] = 1.0
    sim = make_sim(d["r"], d["box"], d["ptype"], table_of(d), nblist=_lib.NBLIST_CELLS, skin=0.3)
    sim.eval_forces()  # reorders particles by cell on the device
    out = np.zeros((2, 2, 100), np.uint64)
    sim.rdf_update(100, 0.0, out)
    assert np.array_equal(out, oracle.rdf(d["r"], d["ptype"], d["box"], 100, fma=1))
    assert sim.last_analysis_ms() > 0.0


def test_sq_vs_gamdpy_and_oracle(oracle):
    d = golden("sq")
    rho = _lib.sq_compute(d["r"], d["box"], d["n_vectors"])
    ref64 = oracle.sq(d["r"], d["q"])
    assert np.abs(rho - ref64).max() < 1e-4 * max(1.0, np.abs(ref64).max())
    assert np.abs(rho - d["multi_rho_q"]).max() < 2e-3 * max(1.0, np.abs(ref64).max())
    # form factors, through the calculator API
    conf = gp.Configuration(D=3)
    conf["r"] = d["r"].copy()
    conf.simbox = gp.Orthorhombic(3, d["box"])
    calc = gp.CalculatorStructureFactor(conf, atomic_form_factors=d["ff"])
    calc.generate_q_vectors(q_max=6.0)
    calc.update()
    raw = calc.read(None)
    assert np.allclose(raw["q"], d["ff_q"])
    assert np.abs(raw["rho_q"][0] - d["ff_rho_q"]).max() < 2e-3 * max(1.0, np.abs(d["ff_rho_q"]).max())


def test_rdf_and_sq_at_the_large_lj_geometry(oracle):
    """The structure analysis of the large LJ workload (rho 0.84, r < 5 with
    1000 bins, S(q) on the first 200 |n|^2 shells of the reference's
    non-negative generator) on a box of its kind: 186 624 particles (FCC
    36^3, +-0.1 jitter, 20 NVE steps) in L = 60.6, a grid of 12^3 cells of
    edge >= 5 of which 1000 lie off the box faces (the plain-difference
    shortcut).  Through the device-resident path of a running Simulation
    (particles in cell order): counts bit-exact against the oracle's all
    pairs; S(q) within 1e-4 of the float64 oracle."""
    conf = workloads.lj_configuration([36, 36, 36], 0.84, 1.0, seed=5)
    L = conf.simbox.lengths.astype(np.float32)
    rng = np.random.default_rng(8)
    r = conf["r"].astype(np.float64) + rng.uniform(-0.1, 0.1, (conf.N, 3))
    r -= L * np.round(r / L)
    conf["r"] = r.astype(np.float32)
    plan = {"pb": 256, "tp": 1, "lanes": 0, "skin": 0.5, "UtilizeNIII": False, "gridsync": False,
            "nblist": "linked lists"}
    sim = gp.Simulation(conf, workloads.lj_pair_potential(max_num_nbs=200), gp.integrators.NVE(dt=0.004), [],
                        num_timeblocks=1, steps_per_timeblock=20, compute_plan=plan, storage="memory")
    for _ in sim.run_timeblocks():
        pass
    rdf = gp.CalculatorRadialDistribution(conf, bins=1000, r_max=5.0)
    rdf.update()
    got = rdf.rdf_list[-1]
    ref = oracle.rdf(conf["r"], conf.ptype, L, 1000, fma=1, r_max=5.0)
    assert ref.sum() > 5e7 and np.array_equal(got, ref.astype(np.float64))
    sq = gp.CalculatorStructureFactor(conf)
    sq.generate_q_vectors(2 * np.pi * np.sqrt(237.5) / float(L[0]))
    assert len(sq.q_vectors) == 2219
    sq.update()
    ref64 = oracle.sq(conf["r"], sq.q_vectors)
    assert np.abs(sq.list_of_rho_q[-1] - ref64).max() < 1e-4 * max(1.0, np.abs(ref64).max())


def test_sq_negative_and_large_n_vectors(oracle):
    conf = workloads.ka_configuration(5000, seed=2)
    L = conf.simbox.lengths
    rng = np.random.default_rng(0)
    nv = rng.integers(-12, 13, size=(300, 3))
    rho = _lib.sq_compute(conf["r"], L, nv)
    q = (2 * np.pi * nv / L).astype(np.float32)
    ref = oracle.sq(conf["r"], q)
    assert np.abs(rho - ref).max() < 1e-4 * max(1.0, np.abs(ref).max())


def test_overflow_raises_like_gamdpy():
    d = golden("lj256_sf")
    conf = gp.Configuration(D=3)
    conf["r"] = d["r"].copy()
    conf.simbox = gp.Orthorhombic(3, d["box"])
    conf["m"] = 1.0
    pp = gp.PairPotential(gp.apply_shifted_force_cutoff(gp.LJ_12_6_sigma_epsilon), params=[1.0, 1.0, 2.5],
                          max_num_nbs=40)
    ev = gp.Evaluator(conf, pp, compute_plan={"pb": 8, "tp": 1, "skin": 0.5, "nblist": "N squared"})
    with pytest.raises(Exception, match="Neighbor-list is invalid"):
        ev.evaluate()


def test_nan_position_reports_error_not_fault():
    d = golden("ka1372_cells")
    r = d["r"].copy()
    r[5] = np.nan
    sim = make_sim(r, d["box"], d["ptype"], table_of(d), nblist=_lib.NBLIST_CELLS, skin=0.3)
    with pytest.raises(_lib.GdbError):
        sim.run(0.0, 3)
    assert sim.status() & _lib.STATUS_NAN


def test_runs_are_bitwise_reproducible():
    conf = workloads.ka_configuration(4000, seed=5)
    outs = []
    for _ in range(2):
        c = workloads.ka_configuration(4000, seed=5)
        sim = gp.Simulation(c, workloads.ka_pair_potential(), gp.integrators.NVT(0.45, 0.2, 0.005),
                            [gp.ScalarSaver(10), gp.MomentumReset(50)], num_timeblocks=2, steps_per_timeblock=200,
                            compute_plan={"pb": 64, "tp": 4, "skin": 0.3, "nblist": "linked lists"},
                            storage="memory")
        for _ in sim.run_timeblocks():
            pass
        outs.append((c["r"].copy(), c["v"].copy(), sim.output["scalars"].copy()))
    for a, b in zip(outs[0], outs[1]):
        assert np.array_equal(a, b)
    assert conf.N == 4000


@pytest.mark.parametrize("n, lanes, cap", [(2048, 0, 0), (65536, 1, 100), (20000, 4, 0)])
def test_step_barrier_forms_agree_bit_for_bit(monkeypatch, n, lanes, cap):
    """The persistent grid's step barrier in its two forms -- every block
    keeping the step's books from rows double-buffered by step parity (the
    default for grids of up to 320 blocks) and the last block to arrive
    keeping them (GDB_STEP_BARRIER=0) -- give the same trajectory, scalars
    and thermostat state bit for bit: the same rows summed in the same order.
    NVT with a ScalarSaver and MomentumReset, so the full rows, the momentum
    shift and the friction all pass through the books; with a grid of 100
    blocks for 256 rounds, the rounds are handed out by the counter."""
    monkeypatch.setenv("GDB_CLUSTER", "0")
    monkeypatch.setenv("GDB_GRID_CAP", str(cap))
    outs = []
    for mode in ("1", "0"):
        monkeypatch.setenv("GDB_STEP_BARRIER", mode)
        c = workloads.ka_configuration(n, seed=7)
        integ = gp.integrators.NVT(0.45, 0.2, 0.005)
        sim = gp.Simulation(c, workloads.ka_pair_potential(max_num_nbs=300), integ,
                            [gp.ScalarSaver(10), gp.MomentumReset(30)], num_timeblocks=2, steps_per_timeblock=150,
                            compute_plan={"pb": 64, "tp": 1, "lanes": lanes, "skin": 0.3, "nblist": "linked lists"},
                            storage="memory")
        for _ in sim.run_timeblocks():
            pass
        assert sim._sim.last_path() == 1
        outs.append((c["r"].copy(), c["v"].copy(), np.array(sim.output["scalars"]), integ.thermostat_state.copy()))
    for a, b in zip(*outs):
        assert np.array_equal(a, b)


def test_nve_energy_conservation():
    """tests/test_LJ_nxyz.py:10-111 of the reference: LJ rho 0.8442, T0 1.44,
    shifted force, dt 0.005, 2 x 4096 steps: var(E)/N < 1e-4 and
    Tkin, Tconf in (0.67, 0.72)."""
    conf = gp.Configuration(D=3, compute_flags={"Fsq": True, "lapU": True})
    conf.make_lattice(gp.unit_cells.FCC, cells=[8, 8, 8], rho=0.8442)
    conf["m"] = 1.0
    conf.randomize_velocities(temperature=1.44, seed=0)
    pp = gp.PairPotential(gp.apply_shifted_force_cutoff(gp.LJ_12_6_sigma_epsilon), params=[1.0, 1.0, 2.5],
                          max_num_nbs=1000)
    sim = gp.Simulation(conf, pp, gp.integrators.NVE(dt=0.005),
                        [gp.MomentumReset(100), gp.ConfigurationSaver(),
                         gp.ScalarSaver(8, {"Fsq": True, "lapU": True, "stresses": False})],
                        num_timeblocks=2, steps_per_timeblock=4096, storage="memory")
    for _ in sim.run_timeblocks():
        pass
    U, W, lapU, Fsq, K = gp.extract_scalars(sim.output, ["U", "W", "lapU", "Fsq", "K"], first_block=1)
    N = conf.N
    E = U + K
    var_e = np.var(E) / N
    half = len(U) // 2
    Tkin = np.mean(2 * K[half:] / 3 / (N - 1))
    Tconf = np.mean(Fsq[half:] / lapU[half:])
    assert var_e < 1e-4
    assert 0.67 < Tkin < 0.72
    assert 0.67 < Tconf < 0.72
    frames = sim.output["block"]
    assert frames.shape == (2, 14, 2, N, 3)
    assert np.abs(frames[1, -1, 0] - conf["r"]).max() < 1e-6  # step 4096 frame = final positions


def test_kob_andersen_reference_state_point():
    """examples/kablj.py of the reference: KA (shifted potential) at rho 1.2,
    N 2000, melted at T 2 and ramped to 0.8, then 32 x 2048 production steps;
    asserts |u - (-6.346)| < 0.01 and |w - 5.534| < 0.03 per particle (RUMD3,
    examples/kablj.py:120-131)."""
    N, rho, T, dt = 2000, 1.2, 0.8, 0.004
    conf = gp.Configuration(D=3, compute_flags={"Fsq": True, "lapU": True, "Vol": True})
    conf.make_positions(N=N, rho=rho)
    conf["m"] = 1.0
    conf.randomize_velocities(temperature=2.0)
    conf.ptype[::5] = 1
    pp = gp.PairPotential(gp.apply_shifted_potential_cutoff(gp.LJ_12_6_sigma_epsilon),
                          params=[workloads.KA_SIGMA, workloads.KA_EPSILON, workloads.KA_CUT], max_num_nbs=1000)
    blocks, steps = 32, 2048
    run_time = dt * blocks * steps
    ramp = gp.make_function_ramp(value0=2.0, x0=run_time / 8, value1=T, x1=run_time / 4)
    sim = gp.Simulation(conf, pp, gp.integrators.NVT(temperature=ramp, tau=0.2, dt=dt), [gp.MomentumReset(100)],
                        num_timeblocks=blocks, steps_per_timeblock=steps, storage="memory")
    for _ in sim.run_timeblocks():
        pass
    sim = gp.Simulation(conf, pp, gp.integrators.NVT(temperature=T, tau=0.2, dt=dt),
                        [gp.MomentumReset(100), gp.ScalarSaver(16, {"Fsq": True, "lapU": True})],
                        num_timeblocks=blocks, steps_per_timeblock=steps, storage="memory")
    for _ in sim.run_timeblocks():
        pass
    U, W = gp.extract_scalars(sim.output, ["U", "W"], first_block=0)
    mu, mw = np.mean(U) / N, np.mean(W) / N
    assert abs(mu - (-6.346)) < 0.01, mu
    assert abs(mw - 5.534) < 0.03, mw


def test_barrier_wait_runs_out_and_reports(oracle):
    """The bounded grid-barrier wait gives up (a block that never arrives),
    sets the status bit, and the device stays usable."""
    import ctypes
    st = ctypes.c_uint(0)
    rc = _lib.lib().gdb_selftest_barrier_timeout(0, 2_000_000, ctypes.byref(st))
    assert rc == _lib.GDB_OK
    assert st.value & 0x2  # GDB_STATUS_BARRIER_TIMEOUT
    conf = workloads.ka_configuration(500, seed=2)
    table = oracle.param_table([workloads.KA_SIGMA, workloads.KA_EPSILON, workloads.KA_CUT])
    sim = make_sim(conf["r"], conf.simbox.lengths, conf.ptype, table, nblist=_lib.NBLIST_CELLS, skin=0.3)
    sim.run(0.0, 10)
    assert sim.status() == 0
