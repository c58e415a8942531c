"""Seeded synthetic systems of the benchmark configurations.

The reference benchmarks on synthetic lattices too (benchmarks/benchmark_LJ.py:
28-47); these builders produce the Kob-Andersen and single-component LJ systems
used by bench.py and the tests, through the public API only.
"""
import numpy as np

from .configuration import Configuration, make_lattice, unit_cells
from .interactions import PairPotential
from .potential_functions import LJ_12_6_sigma_epsilon, apply_shifted_force_cutoff, apply_shifted_potential_cutoff
from .simulation_boxes import Orthorhombic

# Kob-Andersen 80:20 (sigma, epsilon) per type pair, cut at 2.5 sigma
KA_SIGMA = np.array([[1.0, 0.8], [0.8, 0.88]], np.float32)
KA_EPSILON = np.array([[1.0, 1.5], [1.5, 0.5]], np.float32)
KA_CUT = (2.5 * KA_SIGMA).astype(np.float32)


def ka_configuration(N, rho=1.2, temperature=0.45, seed=0, jitter=0.05, compute_flags=None):
    """KA mixture: FCC sites of ceil((N/4)^(1/3))^3 cells trimmed to N, box from
    the density, 20 % B chosen by a seeded permutation, uniform jitter of
    +-``jitter`` sigma, unit masses, Maxwell-Boltzmann velocities at T."""
    nc = int(np.ceil((N / 4) ** (1.0 / 3.0) - 1e-9))
    sites, _ = make_lattice(unit_cells.FCC, cells=[nc, nc, nc], rho=None)
    L = (N / rho) ** (1.0 / 3.0)
    a = L / nc
    sites = (sites + nc / 2.0) * a  # lattice made centred on [-nc/2, nc/2)
    pos = sites[:N] - L / 2.0
    rng = np.random.default_rng(seed)
    pos = pos + rng.uniform(-jitter, jitter, pos.shape)
    pos -= L * np.round(pos / L)
    conf = Configuration(D=3, compute_flags=compute_flags)
    conf["r"] = pos.astype(np.float32)
    conf.simbox = Orthorhombic(3, [L, L, L])
    conf.ptype[rng.permutation(N)[: N // 5]] = 1
    conf["m"] = 1.0
    conf.randomize_velocities(temperature=temperature, seed=seed)
    return conf


def ka_pair_potential(max_num_nbs=300):
    """Shifted-force KA potential (LJ_12_6_sigma_epsilon, cut 2.5 sigma_ab)."""
    return PairPotential(apply_shifted_force_cutoff(LJ_12_6_sigma_epsilon),
                         params=[KA_SIGMA, KA_EPSILON, KA_CUT], max_num_nbs=max_num_nbs)


def lj_configuration(cells, rho, temperature, seed=0, compute_flags=None):
    """Single-component LJ on an FCC lattice (gamdpy's get_default_sim recipe)."""
    conf = Configuration(D=3, compute_flags=compute_flags)
    conf.make_lattice(unit_cells.FCC, cells=cells, rho=rho)
    conf["m"] = 1.0
    conf.randomize_velocities(temperature=temperature, seed=seed)
    return conf


def lj_pair_potential(cut=2.5, shifted_force=True, max_num_nbs=300):
    wrap = apply_shifted_force_cutoff if shifted_force else apply_shifted_potential_cutoff
    return PairPotential(wrap(LJ_12_6_sigma_epsilon), params=[1.0, 1.0, cut], max_num_nbs=max_num_nbs)


def ka_replica_sweep(count=128, seed=0, n_min=256, n_max=32768):
    """State points of the batched-replica workload: ``count`` KA systems with
    N log-uniform in [n_min, n_max] (rounded to a multiple of 4, FCC sites
    trimmed to N), density uniform in [1.1, 1.3] and temperature uniform in
    [0.4, 1.0], all drawn from ``seed``.  Returns a list of (N, rho, T)."""
    rng = np.random.default_rng(seed)
    ns = np.exp(rng.uniform(np.log(n_min), np.log(n_max), count))
    ns = np.clip((np.round(ns / 4) * 4).astype(int), n_min, n_max)
    rhos = rng.uniform(1.1, 1.3, count)
    temps = rng.uniform(0.4, 1.0, count)
    return [(int(n), float(r), float(t)) for n, r, t in zip(ns, rhos, temps)]
