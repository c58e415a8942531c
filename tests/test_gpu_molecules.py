"""Molecules: harmonic bonds (interactions/bonds.py) with the bonded pairs
excluded from the pair potential's neighbour list (nblist.py:120-123,
nblist_linked_lists.py:174-178), against gamdpy's own output on chains of
10 beads (tests/golden/make_golden.py: chain200_bonds, chain200_nve,
chain1200_cells) and, at a size the goldens do not reach, against the
oracle's list with the excluded pairs removed and its bond terms.

Bars: neighbour sets bit-exact; forces, U, W and lapU within 1e-5 relative
RMS of gamdpy's float32 path; an 8-step NVE trajectory within float32
round-off growth (1e-4 relative)."""
import numpy as np
import pytest

import gamdpy_b200 as gp
from conftest import golden, rel_rms, sorted_rows
from gamdpy_b200 import _lib

pytestmark = pytest.mark.gpu

FORCE_TOL = 1e-5


def chain_objects(d, max_nbs=300):
    conf = gp.Configuration(D=3, compute_flags={"lapU": True, "Fsq": True})
    conf["r"] = d["r"].copy() if "r" in d.files and "r0" not in d.files else d["r0"].copy()
    conf.simbox = gp.Orthorhombic(3, d["box"])
    conf["m"] = 1.0
    conf["v"] = (d["v"] if "v0" not in d.files else d["v0"]).copy()
    bonds = gp.Bonds(gp.harmonic_bond_function, d["bond_params"].tolist(), d["bond_indices"].tolist())
    excl = bonds.get_exclusions(conf)
    assert np.array_equal(excl, d["exclusions"])
    pp = gp.PairPotential(gp.apply_shifted_force_cutoff(gp.LJ_12_6_sigma_epsilon), params=[1.0, 1.0, 2.5],
                          exclusions=excl, max_num_nbs=max_nbs)
    return conf, bonds, pp


def plan(nblist):
    return {"pb": 8, "tp": 1, "skin": 0.5, "UtilizeNIII": False, "gridsync": False, "nblist": nblist}


@pytest.mark.parametrize("name,nblist", [("chain200_bonds", "N squared"), ("chain1200_cells", "linked lists")])
def test_bonds_and_exclusions_vs_gamdpy(name, nblist):
    d = golden(name)
    conf, bonds, pp = chain_objects(d)
    ev = gp.Evaluator(conf, [pp, bonds], compute_plan=plan(nblist))
    ev.evaluate()
    counts, flat = sorted_rows(pp.get_nblist())
    assert np.array_equal(counts, d["nb_counts"]) and np.array_equal(flat, d["nb_flat"])
    assert rel_rms(conf["f"], d["f"]) < FORCE_TOL
    for k in ("U", "W", "lapU"):
        assert rel_rms(conf[k], d[k]) < FORCE_TOL, k


def test_bonded_nve_trajectory_vs_gamdpy():
    d = golden("chain200_nve")
    conf, bonds, pp = chain_objects(d)
    sim = gp.Simulation(conf, [pp, bonds], gp.integrators.NVE(dt=float(d["dt"])), [gp.ScalarSaver(int(d["every"]))],
                        num_timeblocks=1, steps_per_timeblock=int(d["steps"]), compute_plan=plan("N squared"),
                        storage="memory")
    for _ in sim.run_timeblocks():
        pass
    assert np.abs(conf["r"] - d["r"]).max() < 1e-4
    assert rel_rms(conf["v"], d["v"]) < 1e-4
    assert rel_rms(conf["f"], d["f"]) < 1e-4
    assert np.array_equal(conf.r_im, d["r_im"])
    # U, W, K saved; lapU and Fsq off in the run's compute flags read zero in both
    assert list(sim.output.attrs["scalar_names"]) == list(d["scalar_names"])
    np.testing.assert_allclose(sim.output["scalars"][0], d["scalars"][0], rtol=1e-4, atol=1e-3)
    assert np.all(conf["lapU"] == 0) and np.all(d["scalars"][0][:, 2] == 0)


@pytest.mark.parametrize("persistent", ["1", "0"])
def test_bonded_chains_large_vs_oracle(oracle, monkeypatch, persistent):
    """30 000 particles in 3 000 chains of 10 beads, cell lists, on the
    persistent kernel and on the standalone kernels: the list equals the
    oracle's cell list with the bonded pairs taken out, and the forces equal
    the oracle's pair forces on that list plus the bond forces."""
    monkeypatch.setenv("GDB_PERSISTENT", persistent)
    n = 30000
    conf = gp.Configuration(D=3, compute_flags={"lapU": True})
    conf.make_positions(N=n, rho=1.0)
    conf["m"] = 1.0
    conf.ptype[:] = 0
    indices = np.array([[i, i + 1, i % 2] for i in range(n - 1) if i % 10 != 9], np.int32)
    params = np.array([[1.0, 3000.0], [1.1, 2000.0]], np.float32)
    bonds = gp.Bonds(gp.harmonic_bond_function, params.tolist(), indices.tolist())
    excl = bonds.get_exclusions(conf)
    pp = gp.PairPotential(gp.apply_shifted_force_cutoff(gp.LJ_12_6_sigma_epsilon), params=[1.0, 1.0, 2.5],
                          exclusions=excl, max_num_nbs=300)
    ev = gp.Evaluator(conf, [pp, bonds], compute_plan=plan("linked lists"))
    ev.evaluate()
    L = conf.simbox.lengths
    r = conf["r"]
    full, _ = oracle.nblist_cells(r, L, 2.5, 0.5, 300, fma=1)
    want = oracle.exclude(full, excl)
    c1, f1 = sorted_rows(pp.get_nblist())
    c2, f2 = sorted_rows(want)
    assert np.array_equal(c1, c2) and np.array_equal(f1, f2)
    table = oracle.param_table([np.float32(1.0), np.float32(1.0), np.float32(2.5)])
    pair = oracle.forces(r, conf.ptype, L, table, want, fma=1)
    bond = oracle.bond_terms(r, L, indices, params)
    for k in ("f", "U", "W", "lapU"):
        assert rel_rms(conf[k], np.asarray(pair[k], np.float64) + bond[k]) < FORCE_TOL, k


def test_bonds_energy_conservation():
    """LJ chains (examples/LJchain.py's system at 2 000 particles), NVE dt
    0.002 for 4 096 steps after a thermalising NVT run: var(E)/N < 1e-4 as the
    reference's energy-conservation bound (tests/test_LJ_nxyz.py:87)."""
    conf = gp.Configuration(D=3, compute_flags={"lapU": True})
    conf.make_positions(N=2000, rho=1.0)
    conf["m"] = 1.0
    conf.randomize_velocities(temperature=1.44, seed=0)
    indices = [[i, i + 1, 0] for i in range(conf.N - 1) if i % 10 != 9]
    bonds = gp.Bonds(gp.harmonic_bond_function, [[1.0, 3000.0]], indices)
    pp = gp.PairPotential(gp.apply_shifted_force_cutoff(gp.LJ_12_6_sigma_epsilon), params=[1.0, 1.0, 2.5],
                          exclusions=bonds.get_exclusions(conf), max_num_nbs=1000)
    cp = gp.get_default_compute_plan(conf)
    warm = gp.Simulation(conf, [pp, bonds], gp.integrators.NVT(0.7, tau=0.2, dt=0.002), [], num_timeblocks=4,
                         steps_per_timeblock=1024, compute_plan=cp, storage="memory")
    for _ in warm.run_timeblocks():
        pass
    sim = gp.Simulation(conf, [pp, bonds], gp.integrators.NVE(dt=0.002), [gp.ScalarSaver(16)], num_timeblocks=4,
                        steps_per_timeblock=1024, compute_plan=cp, storage="memory")
    for _ in sim.run_timeblocks():
        pass
    U, K = gp.extract_scalars(sim.output, ["U", "K"], first_block=1)
    E = (U + K) / conf.N
    assert np.var(E) < 1e-4, np.var(E)
    assert np.all(np.isfinite(conf["r"]))
