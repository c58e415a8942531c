"""Host-side API: gamdpy's names, shapes and known answers, without a GPU."""
import numpy as np
import pytest

import gamdpy_b200 as gp
from conftest import golden


def test_potential_function_known_answers():
    """tests/test_potential_functions.py:9-10 of the reference."""
    assert gp.LJ_12_6(1, [2, 3]) == (5.0, 42.0, 438.0)
    assert gp.LJ_12_6_sigma_epsilon(1, [2, 3]) == (48384.0, 585216.0, 7635456.0)


@pytest.mark.parametrize("tag,wrap", [("sf", gp.apply_shifted_force_cutoff),
                                      ("sp", gp.apply_shifted_potential_cutoff)])
def test_cutoff_wrappers_match_reference(tag, wrap):
    d = golden("known_answers")
    pot = wrap(gp.LJ_12_6_sigma_epsilon)
    got = np.array([pot(np.float32(x), np.array([1.0, 1.0, 2.5], np.float32)) for x in d[f"{tag}_r"]])
    assert np.array_equal(got.astype(np.float64), d[f"{tag}_lj"])
    assert pot._gdb_cutmode == (0 if tag == "sf" else 1)


def test_simbox_known_answers():
    """tests/test_simbox.py:5-50 of the reference."""
    box = gp.Orthorhombic(D=3, lengths=np.array([3, 4, 5]))
    ri, rj = np.array([2.5, 3, 4]), np.array([0.5, 0.5, 0.5])
    dr = 0 * ri
    assert box.get_dist_sq_dr_function()(ri, rj, box.lengths, dr) == 5.5
    assert np.all(dr == np.array([-1, -1.5, -1.5]))
    assert box.get_dist_sq_function()(ri, rj, box.lengths) == 5.5
    r, img = np.array([4, 5, 6]), np.array([0, 1, 2])
    box.get_apply_PBC()(r, img, box.lengths)
    assert np.all(r == 1) and np.all(img == np.array([1, 2, 3]))
    assert box.get_volume_function()(box.lengths) == 60
    r_current = np.array([1, 1, 1])
    assert box.get_dist_moved_sq_function()(r_current, r_current + 0.75 * box.lengths, box.lengths,
                                            box.lengths) == 3.125
    f = box.get_dist_moved_exceeds_limit_function()
    assert not f(r_current, r_current + 0.5, box.lengths, box.lengths, 2.0, 1.0)
    assert f(r_current, r_current + 0.75, box.lengths, box.lengths, 2.0, 1.0)


def test_velocities_reproduce_reference_rng():
    """Configuration.randomize_velocities uses gamdpy's RNG call order: the
    golden run's initial velocities came from gamdpy with the same seed."""
    d = golden("lj256_nve")
    c = gp.Configuration(D=3)
    c["r"] = np.zeros((256, 3), np.float32)
    c["m"] = 1.0
    c.randomize_velocities(temperature=0.7, seed=0)
    assert np.array_equal(c["v"], d["v0"])


def test_lattice_matches_reference_layout():
    pos, box = gp.configuration.make_lattice(gp.unit_cells.FCC, cells=[2, 3, 4], rho=0.973)
    assert pos.shape == (96, 3)
    assert np.allclose(np.prod(box) * 0.973, 96)
    assert np.all(pos >= -box / 2) and np.all(pos < box / 2)
    # first cell = unit-cell fractional coordinates (C-order cell enumeration)
    a = box[0] / 2
    assert np.allclose(pos[1] - pos[0], [0.5 * a, 0.5 * a, 0.0])


def test_configuration_columns():
    c = gp.Configuration(D=3, N=10, compute_flags={"lapU": True, "Fsq": True})
    assert c.vector_columns == ["r", "v", "f"]
    assert c.scalar_columns == ["U", "W", "lapU", "K", "Fsq", "m"]
    assert c["r"].shape == (10, 3) and c["m"].shape == (10,)
    with pytest.raises(ValueError):
        c["q"] = 1


def test_default_compute_plan_for_b200():
    c = gp.Configuration(D=3)
    c.make_lattice(gp.unit_cells.FCC, cells=[8, 8, 8], rho=0.973)
    plan = gp.get_default_compute_plan(c)
    assert plan["nblist"] == "N squared" and plan["gridsync"]
    big = gp.Configuration(D=3, N=65536)
    assert gp.get_default_compute_plan(big)["nblist"] == "linked lists"
    # below 2 x 148 particles gamdpy's pb loop would reach zero; here pb stays 8
    for n in (1, 100, 256, 295):
        small = gp.Configuration(D=3, N=n)
        assert gp.get_default_compute_plan(small)["pb"] == 8


def test_param_table_and_untagged_potential_rejected():
    pp = gp.PairPotential(gp.apply_shifted_force_cutoff(gp.LJ_12_6_sigma_epsilon),
                          params=[[[1.0, 0.8], [0.8, 0.88]], [[1.0, 1.5], [1.5, 0.5]], [[2.5, 2.0], [2.0, 2.2]]],
                          max_num_nbs=100)
    table, max_cut = pp.table()
    assert table.shape == (2, 2, 3) and max_cut == np.float32(2.5)
    rec, mc = pp.convert_user_params()
    assert rec[0, 1][1] == np.float32(1.5)
    bad = gp.PairPotential(lambda r, p: (0, 0, 0), params=[1.0, 1.0, 2.5], max_num_nbs=10)
    with pytest.raises(NotImplementedError):
        bad.kernel_kind()


def test_runtime_action_validation():
    with pytest.raises(ValueError):
        gp.ScalarSaver(-1)
    with pytest.raises(ValueError):
        gp.MomentumReset(1.5)
    out = gp.simulation.Output()
    conf = gp.Configuration(D=3, N=4)
    ss = gp.ScalarSaver(4)
    with pytest.raises(ValueError):
        ss.setup(conf, 2, 4, out)
    ss.setup(conf, 2, 16, out)
    assert out["scalars"].shape == (2, 4, 3) and out.attrs["scalar_names"] == ["U", "W", "K"]
    rows = np.arange(24, dtype=np.float64).reshape(4, 6)
    rows[:, 5] = 0.0  # no per-step volume: a fixed box
    ss.update_from_rows(1, rows, out, 1.0)
    U, K = gp.extract_scalars(out, ["U", "K"], first_block=1)
    assert np.array_equal(U, rows[:, 0]) and np.array_equal(K, rows[:, 3])


def test_workload_builders():
    from gamdpy_b200 import workloads
    c = workloads.ka_configuration(2048, seed=1)
    assert c.N == 2048 and abs(c.N / c.get_volume() - 1.2) < 1e-4
    assert (c.ptype == 1).sum() == 2048 // 5
    assert np.all(np.abs(c["r"]) <= c.simbox.lengths / 2 + 1e-6)
    assert abs(np.sum(c["v"] ** 2) / (3 * (c.N - 1)) - 0.45) < 1e-4


def test_make_positions_equals_gamdpy():
    """Configuration.make_positions reproduces gamdpy's positions (the chain
    fixture was made with them) bit for bit."""
    d = golden("chain200_bonds")
    c = gp.Configuration(D=3)
    c.make_positions(N=200, rho=1.0)
    assert np.array_equal(c["r"], d["r"])
    assert np.array_equal(c.simbox.lengths, d["box"])


def test_bond_exclusions_equal_gamdpy():
    """Bonds.get_exclusions builds gamdpy's (N, 21) table (bonds.py:137-150)."""
    d = golden("chain200_bonds")
    c = gp.Configuration(D=3)
    c.make_positions(N=200, rho=1.0)
    bonds = gp.Bonds(gp.harmonic_bond_function, d["bond_params"].tolist(), d["bond_indices"].tolist())
    assert np.array_equal(bonds.get_exclusions(c), d["exclusions"])
    u, s, umm = gp.harmonic_bond_function(np.float32(1.2), [1.0, 3000.0])
    assert np.isclose(u, 0.5 * 3000 * 0.2 ** 2, rtol=1e-6) and np.isclose(s, -3000 * 0.2 / 1.2, rtol=1e-6)
    assert umm == 3000.0


def test_autotune_cache_round_trip(tmp_path, monkeypatch):
    """The autotuner's per-GPU cache: a stored plan is read back by key, and
    entries under other keys stay (host logic only)."""
    from gamdpy_b200 import simulation as S
    monkeypatch.setenv("GAMDPY_B200_CACHE", str(tmp_path))
    assert S._autotune_cache_load() == {}
    S._autotune_cache_store("gpu|N=10", {"nblist": "N squared", "lanes": 4, "skin": 0.3})
    S._autotune_cache_store("gpu|N=20", {"nblist": "linked lists", "lanes": 1, "skin": 0.5})
    d = S._autotune_cache_load()
    assert d["gpu|N=10"]["lanes"] == 4 and d["gpu|N=20"]["nblist"] == "linked lists"
    assert (tmp_path / "autotune.json").exists()


def test_trace_summary_splits_the_step_barrier():
    """bench.trace_summary: block 0's marks give the step, phase and barrier
    times; the last block's arrival and release marks (tags 7, 8, written
    from another block, so possibly out of order) split the barrier."""
    import bench
    tags = [5, 6, 8, 7, 1, 6, 7, 8, 1]
    ns = [0, 100, 300, 200, 400, 500, 650, 700, 800]
    t = bench.trace_summary(tags, ns)
    assert t["steps"] == 1 and abs(t["step_barrier_us_median"] - 0.3) < 1e-9
    split = t["barrier_split_us_median"]
    assert abs(split["to_last_arrival"] - 0.125) < 1e-9
    assert abs(split["bookkeeping"] - 0.075) < 1e-9 and abs(split["release_to_block0"] - 0.1) < 1e-9
