"""The CPU oracle against gamdpy's own outputs (tests/golden, produced by
tests/golden/make_golden.py from the reference run on the CPU) and against the
known answers of gamdpy's tests.  This pins the oracle the GPU parity tests
then use."""
import numpy as np
import pytest

from conftest import golden, rel_rms, sorted_rows


def test_known_answers(oracle):
    """tests/test_potential_functions.py:9-10 and the cutoff wrappers on a grid."""
    d = golden("known_answers")
    got = oracle.pair_potential(1, [2, 3, 100], kind=oracle.POT_LJ_12_6, cutmode=oracle.CUT_NONE)
    assert tuple(got) == (5.0, 42.0, 438.0) == tuple(d["lj_12_6_1_23"])
    got = oracle.pair_potential(1, [2, 3, 100], kind=oracle.POT_LJ_SIGMA_EPSILON, cutmode=oracle.CUT_NONE)
    assert tuple(got) == (48384.0, 585216.0, 7635456.0) == tuple(d["lj_se_1_23"])
    for tag, cm in (("sf", oracle.CUT_SF), ("sp", oracle.CUT_SP)):
        for key, prm in (("lj", [1.0, 1.0, 2.5]), ("ka", [0.8, 1.5, 2.0])):
            got = np.array([oracle.pair_potential(x, prm, cutmode=cm) for x in d[f"{tag}_r"]])
            # bit-identical to numba's float32 evaluation
            assert np.array_equal(got.astype(np.float64), d[f"{tag}_{key}"])


def test_minimum_image_known_answer(oracle):
    """tests/test_simbox.py:10-19: dist_sq 5.5, dr (-1, -1.5, -1.5)."""
    d2, dr = oracle.dist_sq([2.5, 3, 4], [0.5, 0.5, 0.5], [3, 4, 5])
    assert d2 == 5.5 == float(golden("known_answers")["mic_dist_sq"])
    assert np.array_equal(dr, [-1, -1.5, -1.5])


def test_pbc_known_answer(oracle):
    """tests/test_simbox.py:21-33."""
    r, img = oracle.apply_pbc([4, 5, 6], [0, 1, 2], [3, 4, 5])
    assert np.array_equal(r, [1, 1, 1]) and np.array_equal(img, [1, 2, 3])
    r, img = oracle.apply_pbc([-4, -5, -6], [0, 1, 2], [3, 4, 5])
    assert np.array_equal(r, [-1, -1, -1]) and np.array_equal(img, [-1, 0, 1])


@pytest.mark.parametrize("name", ["lj256_sf", "lj256_sp"])
def test_nsq_list_and_forces(oracle, name):
    d = golden(name)
    nbl, mx = oracle.nblist_nsq(d["r"], d["box"], float(np.float32(d["cut"].max()) + np.float32(d["skin"])), 300)
    counts, flat = sorted_rows(nbl)
    assert np.array_equal(counts, d["nb_counts"])
    assert np.array_equal(flat, d["nb_flat"])
    cm = oracle.CUT_SF if str(d["cutoff"]) == "SF" else oracle.CUT_SP
    res = oracle.forces(d["r"], d["ptype"], d["box"], oracle.param_table([d["sigma"], d["epsilon"], d["cut"]]),
                        nbl, cutmode=cm)
    for k in ("f", "U", "W", "lapU"):
        assert rel_rms(res[k], d[k]) < 2e-6, k


def test_cell_list_and_forces(oracle):
    d = golden("ka1372_cells")
    nbl, mx = oracle.nblist_cells(d["r"], d["box"], float(d["cut"].max()), float(d["skin"]), 300)
    counts, flat = sorted_rows(nbl)
    assert np.array_equal(counts, d["nb_counts"])
    assert np.array_equal(flat, d["nb_flat"])
    # the N^2 build gives the same sets (tests/test_linked_lists_nblist.py:104-106)
    nbl2, _ = oracle.nblist_nsq(d["r"], d["box"], float(np.float32(d["cut"].max()) + np.float32(d["skin"])), 300)
    c2, f2 = sorted_rows(nbl2)
    assert np.array_equal(c2, counts) and np.array_equal(f2, flat)
    res = oracle.forces(d["r"], d["ptype"], d["box"], oracle.param_table([d["sigma"], d["epsilon"], d["cut"]]), nbl)
    for k in ("f", "U", "W", "lapU"):
        assert rel_rms(res[k], d[k]) < 3e-6, k


def test_fma_variant_changes_nothing_here(oracle):
    """The fused distance form (libNVVM's default contraction) gives the same
    sets on these fixtures; it only matters within one ulp of (rc+skin)^2."""
    d = golden("ka1372_cells")
    a, _ = oracle.nblist_cells(d["r"], d["box"], float(d["cut"].max()), float(d["skin"]), 300, fma=0)
    b, _ = oracle.nblist_cells(d["r"], d["box"], float(d["cut"].max()), float(d["skin"]), 300, fma=1)
    assert np.array_equal(sorted_rows(a)[1], sorted_rows(b)[1])


def run_golden_trajectory(oracle, d):
    tab = oracle.param_table([d["sigma"], d["epsilon"], d["cut"]])
    nvt = str(d["integrator"]) == "NVT"
    run = oracle.Run(d["r0"], d["v0"], 1.0, d["ptype"], d["box"], tab, nblist=str(d["nblist"]),
                     skin=float(d["skin"]), max_nbs=300, integrator=str(d["integrator"]), dt=float(d["dt"]),
                     temperature=float(d["temperature"]) if nvt else None, tau=float(d["tau"]) if nvt else None,
                     every=int(d["every"]), reset_every=int(d["reset"]))
    # Simulation.__init__ runs one test step on the device copy
    # (gamdpy/simulation/Simulation.py:200-211); the thermostat keeps its update
    run.run_timeblock(1)
    xi_test = float(run.state[0])
    run.r[:] = d["r0"]
    run.v[:] = d["v0"]
    run.img[:] = 0
    run.have_list.value = 0
    rows = np.array([run.run_timeblock(int(d["steps"])) for _ in range(int(d["blocks"]))])
    return run, rows, xi_test


@pytest.mark.parametrize("name", ["lj256_nve", "ka1372_nvt"])
def test_trajectory(oracle, name):
    d = golden(name)
    run, rows, xi_test = run_golden_trajectory(oracle, d)
    assert abs(xi_test - float(d["xi_after_test"][0])) <= 1e-5 * max(1.0, abs(xi_test))
    assert abs(run.state[0] - d["thermostat_state"][0]) <= 1e-5 * max(1.0, abs(run.state[0]))
    assert np.abs(run.r - d["r"]).max() < 1e-5
    assert np.array_equal(run.img, d["r_im"])
    for k, got in (("v", run.v), ("f", run.f), ("U", run.U), ("W", run.W), ("K", run.K)):
        assert rel_rms(got, d[k]) < 1e-5, k
    cols = {"U": 0, "W": 1, "K": 2}
    for c, nm in enumerate(d["scalar_names"]):
        ref = d["scalars"][:, :, c]
        assert np.abs(rows[:, :, cols[str(nm)]] - ref).max() <= 2e-6 * np.abs(ref).max(), nm


def test_rdf_bit_exact(oracle):
    """Integer counts equal gamdpy's (numba-typed evaluation and the
    simulator run of the kernel itself)."""
    d = golden("rdf")
    for tag in ("lj256", "ka1372"):
        got = oracle.rdf(d[f"{tag}_r"], d[f"{tag}_ptype"], d[f"{tag}_box"], 100)
        assert np.array_equal(got.astype(np.float64), d[f"{tag}_bins_numba"]), tag
    assert np.array_equal(d["lj256_bins_simulator"], d["lj256_bins_numba"])


def test_sq_against_reference_backends(oracle):
    d = golden("sq")
    q = d["q"]
    got = oracle.sq(d["r"], q)
    for key in ("multi", "single"):
        ref = d[f"{key}_rho_q"]
        # gamdpy evaluates in complex64 (float32 q.r): agreement to ~1e-4
        assert np.abs(got - ref).max() < 2e-3 * max(1.0, np.abs(ref).max()), key
        assert rel_rms(np.abs(got) ** 2, d[f"{key}_S"]) < 1e-3, key
    got = oracle.sq(d["r"], d["ff_q"], d["ff"])
    assert np.abs(got - d["ff_rho_q"]).max() < 2e-3 * max(1.0, np.abs(d["ff_rho_q"]).max())


def test_float64_forces_pin_to_gamdpy(oracle):
    """The every-operation-float64 force restatement against gamdpy's own
    float32 forces on its golden list (LJ 256, shifted force): they differ by
    float32 round-off only."""
    d = golden("lj256_sf")
    counts = np.asarray(d["nb_counts"])
    n, width = len(counts), int(counts.max()) + 1
    nbl = np.zeros((n, width), np.int32)
    starts = np.concatenate([[0], np.cumsum(counts)[:-1]])
    for i in range(n):
        nbl[i, :counts[i]] = d["nb_flat"][starts[i]:starts[i] + counts[i]]
        nbl[i, -1] = counts[i]
    one = np.ones((1, 1))
    f64 = oracle.forces_fp64(d["r"], d["ptype"], d["box"], one * float(d["sigma"]), one * float(d["epsilon"]),
                             one * float(d["cut"]), nbl)
    assert rel_rms(d["f"], f64) < 2e-6


def test_langevin_random_numbers_pin_to_numba(oracle):
    """The oracle's restatement of numba.cuda.random (the generator of
    integrators/NVT_Langevin.py:48, :105) against numba's own CPU output:
    states, raw 64-bit outputs and float32 normals, all bit-exact."""
    d = golden("langevin_rng")
    n = len(d["states_s0"])
    st = oracle.xoro_states(n, int(d["seed"]))
    assert np.array_equal(st[:, 0], d["states_s0"]) and np.array_equal(st[:, 1], d["states_s1"])
    raw = st.copy()
    for row, i in enumerate(d["next_index"]):
        got = [oracle.xoro_next(raw, int(i)) for _ in range(d["next_u64"].shape[1])]
        assert np.array_equal(np.array(got, np.uint64), d["next_u64"][row])
    normals = np.array([[oracle.xoro_normal_f32(st, i) for _ in range(d["normals"].shape[1])] for i in range(n)],
                       np.float32)
    assert np.array_equal(normals.view(np.int32), d["normals"].view(np.int32))


@pytest.mark.parametrize("tag", ["a", "b"])
def test_calc_dynamics_restatement_vs_gamdpy(oracle, tag):
    """The oracle's restatement of tools/calc_dynamics.py against the output
    of gamdpy's own function on the same synthetic trajectory."""
    d = golden("dynamics")
    q = d[f"{tag}_qvalues"]
    q = float(q[0]) if tag == "a" else q
    res = oracle.calc_dynamics(d["block"], d["ptype"], d["simbox_initial"], float(d["dt"]),
                               int(d[f"{tag}_first_block"]), qvalues=q)
    assert np.array_equal(res["count"], d[f"{tag}_count"])
    np.testing.assert_allclose(res["times"], d[f"{tag}_times"], rtol=1e-12)
    for k in ("msd", "alpha2", "Fs"):
        np.testing.assert_allclose(res[k], d[f"{tag}_{k}"], rtol=1e-12, atol=1e-12)


def test_oracle_molecules_vs_gamdpy(oracle):
    """The oracle's exclusion filter and bond terms against gamdpy's chain
    fixture: the N^2 list without the bonded pairs equals gamdpy's list, and
    pair forces on it plus the bond terms equal gamdpy's forces and energies."""
    d = golden("chain200_bonds")
    r, box = d["r"], d["box"]
    full, _ = oracle.nblist_nsq(r, box, float(np.float32(2.5) + np.float32(0.5)), 300, fma=0)
    nbl = oracle.exclude(full, d["exclusions"])
    counts = nbl[:, -1]
    flat = np.concatenate([np.sort(nbl[i, : counts[i]]) for i in range(len(nbl))])
    assert np.array_equal(counts, d["nb_counts"]) and np.array_equal(flat, d["nb_flat"])
    table = oracle.param_table([np.float32(1.0), np.float32(1.0), np.float32(2.5)])
    pair = oracle.forces(r, np.zeros(len(r), np.int32), box, table, nbl, fma=0)
    bond = oracle.bond_terms(r, box, d["bond_indices"], d["bond_params"])
    for k in ("f", "U", "W", "lapU"):
        got = np.asarray(pair[k], np.float64) + bond[k]
        ref = d[k].astype(np.float64)
        assert np.sqrt(np.mean((got - ref) ** 2) / np.mean(ref ** 2)) < 1e-5, k


def run_npt_golden(oracle, d):
    """The oracle through gamdpy's sequence for lj256_npt: Simulation's one
    test step on the device copy (Simulation.py:200-211; the configuration
    and the box are uploaded again afterwards, the thermostat and barostat
    states keep the step), then the timeblocks."""
    tab = oracle.param_table([d["sigma"], d["epsilon"], d["cut"]])
    run = oracle.Run(d["r0"], d["v0"], 1.0, None, d["box0"], tab, nblist=str(d["nblist"]), skin=float(d["skin"]),
                     max_nbs=300, integrator="NPT_Atomic", dt=float(d["dt"]), temperature=float(d["temperature"]),
                     tau=float(d["tau"]), pressure=float(d["pressure"]), tau_p=float(d["tau_p"]),
                     every=int(d["every"]))
    run.run_timeblock(1)
    states_test = (run.ts.copy(), run.bs.copy())
    run.r[:] = d["r0"]
    run.v[:] = d["v0"]
    run.img[:] = 0
    run.box[:] = d["box0"]
    run.have_list.value = 0
    rows = np.array([run.run_timeblock(int(d["steps"])) for _ in range(int(d["blocks"]))])
    return run, rows, states_test


def test_npt_atomic_trajectory_vs_gamdpy(oracle):
    """NPT_Atomic restated in the oracle against gamdpy's own run: states
    after the test step and after two timeblocks, the box, positions,
    velocities and the saved U, W, K to float32 round-off (the reference sums
    K and W with float32 atomics in an undefined order)."""
    d = golden("lj256_npt")
    run, rows, (ts_t, bs_t) = run_npt_golden(oracle, d)
    assert np.allclose(ts_t, d["ts_after_test"], rtol=1e-5, atol=1e-7)
    assert np.allclose(bs_t, d["bs_after_test"], rtol=1e-5, atol=1e-7)
    assert np.allclose(run.box, d["box"], rtol=2e-7, atol=0)
    assert abs(run.ts[0] - d["thermostat_state"][0]) <= 1e-5 * abs(d["thermostat_state"][0])
    assert abs(run.bs[0] - d["barostat_state"][0]) <= 1e-5 * abs(d["barostat_state"][0])
    assert abs(run.bs[2] - d["barostat_state"][2]) <= 1e-6 * d["barostat_state"][2]
    assert np.abs(run.r - d["r"]).max() < 1e-5
    assert np.array_equal(run.img, d["r_im"])
    assert rel_rms(run.v, d["v"]) < 1e-5
    cols = {"U": 0, "W": 1, "K": 2}
    for c, nm in enumerate(d["scalar_names"]):
        if str(nm) in cols:
            # 1e-5: the virial sum cancels (pairs of both signs), and the box
            # feeds every float32 rounding of the run back into the forces
            ref = d["scalars"][:, :, c]
            assert np.abs(rows[:, :, cols[str(nm)]] - ref).max() <= 1e-5 * np.abs(ref).max(), nm
