"""Pair-potential functions (gamdpy/interactions/potential_functions/).

In gamdpy a potential is an arbitrary numba-compilable Python function that
the pair kernel inlines.  Here the pair kernel is hand-written CUDA, so the
potentials it supports are *tagged* callables: calling one evaluates it on the
host in float32 with the reference's formula (so gamdpy's own known-answer
tests hold), and the tag ``_gdb_kind`` / ``_gdb_cutmode`` tells PairPotential
which device kernel variant to use.  An untagged function is rejected by
PairPotential with NotImplementedError: there is no fallback path.
"""
import numpy as np

from . import _lib

f32 = np.float32


def _powi(a, k):
    """Binary exponentiation in the operand's type (numba's lowering of
    ``x ** k`` for an integer literal k)."""
    result = f32(1.0) if not isinstance(a, np.ndarray) else np.ones_like(a)
    while k:
        if k & 1:
            result = result * a
        a = a * a
        k >>= 1
    return result


def LJ_12_6_sigma_epsilon(dist, params):
    """u = 4 eps ((sigma/r)^12 - (sigma/r)^6); returns (u, s = -u'/r, u'')
    (potential_functions/LJ_12_6_sigma_epsilon.py:6-36)."""
    sigma, epsilon = f32(params[0]), f32(params[1])
    OneOdist = f32(1.0) / (dist if isinstance(dist, np.ndarray) else f32(dist))
    sigmaOdist = sigma * OneOdist
    x12, x6, o2 = _powi(sigmaOdist, 12), _powi(sigmaOdist, 6), _powi(OneOdist, 2)
    u = f32(4.0) * epsilon * (x12 - x6)
    s = f32(24.0) * epsilon * (f32(2.0) * x12 - x6) * o2
    umm = f32(24.0) * epsilon * (f32(26.0) * x12 - f32(7.0) * x6) * o2
    return u, s, umm


LJ_12_6_sigma_epsilon._gdb_kind = _lib.POT_LJ_SIGMA_EPSILON


def LJ_12_6(dist, params):
    """u = A12 r^-12 + A6 r^-6; returns (u, s = -u'/r, u'')
    (potential_functions/LJ_12_6.py:3-41)."""
    A12, A6 = f32(params[0]), f32(params[1])
    inv = f32(1.0) / (dist if isinstance(dist, np.ndarray) else f32(dist))
    u = A12 * _powi(inv, 12) + A6 * _powi(inv, 6)
    s = f32(12.0) * A12 * _powi(inv, 14) + f32(6.0) * A6 * _powi(inv, 8)
    umm = f32(156.0) * A12 * _powi(inv, 14) + f32(42.0) * A6 * _powi(inv, 8)
    return u, s, umm


LJ_12_6._gdb_kind = _lib.POT_LJ_12_6


def apply_shifted_force_cutoff(pair_potential):
    """u(r) - u(rc) + s(rc) rc (r - rc), s(r) - s(rc); rc = params[-1]
    (potential_functions/apply_shifted_force_cutoff.py:3-39)."""

    def potential(dist, params):
        cut = f32(params[-1])
        u, s, umm = pair_potential(dist, params)
        u_cut, s_cut, umm_cut = pair_potential(cut, params)
        u = u - (u_cut - s_cut * cut * (dist - cut))
        s = s - s_cut
        return u, s, umm

    potential._gdb_kind = getattr(pair_potential, "_gdb_kind", None)
    potential._gdb_cutmode = _lib.CUT_SHIFTED_FORCE
    potential.__name__ = f"shifted_force({getattr(pair_potential, '__name__', 'potential')})"
    return potential


def apply_shifted_potential_cutoff(pair_potential):
    """u(r) - u(rc); rc = params[-1]
    (potential_functions/apply_shifted_potential_cutoff.py:6-49)."""

    def potential(dist, params):
        cut = f32(params[-1])
        u, s, umm = pair_potential(dist, params)
        u_cut, s_cut, umm_cut = pair_potential(cut, params)
        u = u - u_cut
        return u, s, umm

    potential._gdb_kind = getattr(pair_potential, "_gdb_kind", None)
    potential._gdb_cutmode = _lib.CUT_SHIFTED_POTENTIAL
    potential.__name__ = f"shifted_potential({getattr(pair_potential, '__name__', 'potential')})"
    return potential


def harmonic_bond_function(dist, params):
    """u = k (r - r0)^2 / 2; returns (u, s = -u'/r, u'') with params (r0, k)
    (potential_functions/harmonic_bond_function.py:6-43)."""
    length, strength = f32(params[0]), f32(params[1])
    d = dist if isinstance(dist, np.ndarray) else f32(dist)
    u = f32(0.5) * strength * (d - length) ** 2
    s = -strength * (d - length) / d
    umm = strength
    return u, s, umm


harmonic_bond_function._gdb_bond = "harmonic"
