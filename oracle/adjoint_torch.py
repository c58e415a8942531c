"""Float64 torch restatement of the adjoint workload's forward, for tests.

TEST INFRASTRUCTURE ONLY: the checker of gamdpy_b200.adjoint, never called
by the product path.  The reference has no differentiation, so there is no
golden vector for the gradients; parity is pinned instead by two independent
float64 routes that this module provides:
  * torch.autograd through this forward, and
  * central finite differences of this forward.
The forward restates, in float64 over all pairs (the NbList2 pair set):
  integrators/NVE.py:78-97          v += f/m dt; r += v dt; K from mean half-step v
  LJ_12_6_sigma_epsilon.py:26-36    u = 4 eps ((s/r)^12 - (s/r)^6), s = -u'/r
  apply_shifted_force_cutoff.py:30-37  s -= s(rc); u += s(rc) rc (r - rc) - u(rc)
  orthorhombic.py:50-53, 75-86      minimum image and periodic wrap
plus the Gaussian-kernel type-0 radial distribution of the library's adjoint
module (same bin truncation: bins floor((r -/+ 8w - r_lo)/dr), r inside
(r_lo - 8w, r_hi + 8w)).
"""
import math

import numpy as np
import torch

KW = 8.0  # kernel support in widths, as the library


def _tables(theta, nt):
    pairs = [(a, b) for a in range(nt) for b in range(a, nt)]
    m = len(pairs)
    eps = [[None] * nt for _ in range(nt)]
    sig = [[None] * nt for _ in range(nt)]
    for k, (a, b) in enumerate(pairs):
        eps[a][b] = eps[b][a] = theta[k]
        sig[a][b] = sig[b][a] = theta[m + k]
    return torch.stack([torch.stack(r) for r in sig]), torch.stack([torch.stack(r) for r in eps])


def _pair_terms(r, types, box, sig_t, eps_t, cut_t):
    """Per-pair quantities for all ordered pairs i != j (float64)."""
    d = r[:, None, :] - r[None, :, :]  # r_i - r_j
    d = d - box * torch.round(d / box)
    r2 = (d * d).sum(-1)
    n = r.shape[0]
    eye = torch.eye(n, dtype=torch.bool)
    r2s = torch.where(eye, torch.ones_like(r2), r2)
    ti, tj = types[:, None], types[None, :]
    sig = sig_t[ti, tj]
    eps = eps_t[ti, tj]
    cut = cut_t[ti, tj]
    inside = (~eye) & (r2s < cut * cut)
    sr6 = (sig * sig / r2s) ** 3
    s0 = eps * (48.0 * sr6 * sr6 - 24.0 * sr6) / r2s
    src6 = (sig / cut) ** 6
    s_c = eps * (48.0 * src6 * src6 - 24.0 * src6) / (cut * cut)
    u0 = 4.0 * eps * (sr6 * sr6 - sr6)
    u_c = 4.0 * eps * (src6 * src6 - src6)
    rr = torch.sqrt(r2s)
    s = torch.where(inside, s0 - s_c, torch.zeros_like(s0))
    u = torch.where(inside, u0 - u_c + s_c * cut * (rr - cut), torch.zeros_like(u0))
    return d, r2s, rr, s, u, eye


def _soft_rdf_sum(rr, eye, types, rdf):
    bins, lo, hi, w = rdf["bins"], rdf["r_lo"], rdf["r_hi"], rdf["width"]
    dr = (hi - lo) / bins
    aa = (types[:, None] == 0) & (types[None, :] == 0) & (~eye)
    inr = aa & (rr > lo - KW * w) & (rr < lo + bins * dr + KW * w)
    centres = lo + (torch.arange(bins, dtype=torch.float64) + 0.5) * dr
    rsel = rr[inr]
    b0 = torch.clamp(torch.floor((rsel - KW * w - lo) / dr), min=0)
    b1 = torch.clamp(torch.floor((rsel + KW * w - lo) / dr), max=bins - 1)
    bidx = torch.arange(bins, dtype=torch.float64)
    mask = (bidx[None, :] >= b0[:, None]) & (bidx[None, :] <= b1[:, None])
    x = rsel[:, None] - centres[None, :]
    k = torch.exp(-x * x / (2.0 * w * w)) / (math.sqrt(2.0 * math.pi) * w)
    return torch.where(mask, k, torch.zeros_like(k)).sum(0)


def observables(theta, r0, v0, types, mass, box, cut, dt, steps, rdf=None, window=0):
    """Time averages [<U>, <W>, <K>, <g_b>...] of the float64 trajectory.

    theta: torch float64 (eps of the unordered pairs, then sigma); the rest
    numpy.  Differentiable in theta.  window W > 0 detaches the state at every
    multiple of W steps (the truncated adjoint's gradient)."""
    nt = int(np.max(types)) + 1
    sig_t, eps_t = _tables(theta, nt)
    cut_t = torch.as_tensor(np.broadcast_to(np.asarray(cut, np.float64), (nt, nt)).copy())
    r = torch.as_tensor(np.asarray(r0, np.float64))
    v = torch.as_tensor(np.asarray(v0, np.float64))
    ty = torch.as_tensor(np.asarray(types, np.int64))
    m = torch.as_tensor(np.asarray(mass, np.float64))[:, None]
    L = torch.as_tensor(np.asarray(box, np.float64))
    accU = accW = accK = torch.zeros((), dtype=torch.float64)
    accG = None
    nsamp = 0
    for n in range(steps):
        if window > 0 and n % window == 0:
            r, v = r.detach(), v.detach()
        d, r2, rr, s, u, eye = _pair_terms(r, ty, L, sig_t, eps_t, cut_t)
        f = (s[:, :, None] * d).sum(1)
        accU = accU + 0.5 * u.sum()
        accW = accW + (r2 * s).sum() / 6.0
        if rdf and rdf.get("every", 0) > 0 and n % rdf["every"] == 0:
            g = _soft_rdf_sum(rr, eye, ty, rdf)
            accG = g if accG is None else accG + g
            nsamp += 1
        v1 = v + f / m * dt
        vm = 0.5 * (v + v1)
        accK = accK + (0.5 * m * vm * vm).sum()
        r = r + v1 * dt
        r = torch.where(r * 2.0 > L, r - L, r)
        r = torch.where(r * 2.0 < -L, r + L, r)
        v = v1
    out = [accU / steps, accW / steps, accK / steps]
    if rdf:
        bins, lo, hi = rdf["bins"], rdf["r_lo"], rdf["r_hi"]
        dr = (hi - lo) / bins
        na = float(np.sum(np.asarray(types) == 0))
        vol = float(np.prod(box))
        centres = lo + (np.arange(bins) + 0.5) * dr
        norm = torch.as_tensor(1.0 / (nsamp * na * (na / vol) * 4.0 * math.pi * centres ** 2))
        out = torch.stack(out)
        return torch.cat([out, accG * norm])
    return torch.stack(out)


def central_differences(fun, theta, h=1e-4, richardson=False):
    """dfun/dtheta by central differences (float64), fun: numpy -> float.

    The O(h^2) truncation error of a central difference is, for losses built
    from squared deviations of trajectory averages, about 1e-4 of the
    gradient at h = 1e-4; richardson=True combines steps h and h/2 as
    (4 D(h/2) - D(h)) / 3, which cancels it (O(h^4))."""
    theta = np.asarray(theta, np.float64)

    def diff(step):
        g = np.zeros_like(theta)
        for k in range(len(theta)):
            tp, tm = theta.copy(), theta.copy()
            tp[k] += step
            tm[k] -= step
            g[k] = (fun(tp) - fun(tm)) / (2.0 * step)
        return g

    if not richardson:
        return diff(h)
    return (4.0 * diff(0.5 * h) - diff(h)) / 3.0
