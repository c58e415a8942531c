"""ctypes front end of the CPU oracle (md_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, by ``__graft_entry__.smoke()``
and by ``bench.py``'s CPU-baseline leg, always as the checker or the timed CPU
reference, never as part of the product path (gamdpy_b200 does not import it).

Arrays follow gamdpy's host layout: positions (N, 3) float32, types (N,)
int32, parameter tables (ntypes, ntypes, nparams) float32 with the cut last
(gamdpy/interactions/pair_potential.py:40-47), neighbour lists (N, max_nbs+1)
int32 with the count in the last column (gamdpy/interactions/nblist.py:8).
"""
import ctypes
import math
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

POT_LJ_SIGMA_EPSILON = 0
POT_LJ_12_6 = 1
CUT_SF = 0
CUT_SP = 1
CUT_NONE = 2

_lib = None


def build():
    """Compile md_oracle.c into liboracle.so (make, in this directory)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        P = ctypes.c_void_p
        i, f, d = ctypes.c_int, ctypes.c_float, ctypes.c_double
        L.orc_num_threads.restype = i
        L.orc_set_num_threads.argtypes = [i]
        L.orc_pair_potential.argtypes = [i, i, f, P, i, P]
        L.orc_dist_sq.argtypes = [P, P, P, P, i]
        L.orc_dist_sq.restype = f
        L.orc_apply_pbc.argtypes = [P, P, P]
        L.orc_nblist_nsq.argtypes = [i, P, P, f, i, P, i]
        L.orc_nblist_nsq.restype = i
        L.orc_cells_per_dimension.argtypes = [P, f, f, P]
        L.orc_cells_per_dimension.restype = i
        L.orc_cell_coords.argtypes = [i, P, P, P, P]
        L.orc_nblist_cells.argtypes = [i, P, P, f, f, i, P, i]
        L.orc_nblist_cells.restype = i
        L.orc_forces.argtypes = [i, P, P, P, P, i, i, i, i, P, i, P, P, P, P, P, i]
        L.orc_nve_step.argtypes = [i, P, P, P, P, P, P, f, P, P]
        L.orc_nvt_step.argtypes = [i, P, P, P, P, P, P, f, f, P, P]
        L.orc_nvt_step.restype = d
        L.orc_nvt_thermostat_update.argtypes = [f, d, f, f, ctypes.c_longlong, f]
        L.orc_nvt_thermostat_update.restype = f
        L.orc_momentum_reset.argtypes = [i, P, P]
        L.orc_run_timeblock.argtypes = [i, P, P, P, P, P, P, P, P, i, i, i, i, i, f, i, P, P, P, i, f,
                                        P, f, f, i, i, i, P, P, P, P, i]
        L.orc_run_timeblock.restype = i
        L.orc_rdf.argtypes = [i, P, P, P, i, i, P, i, d]
        L.orc_sq.argtypes = [i, P, P, i, P, P, P]
        u64 = ctypes.c_uint64
        L.orc_xoro_init.argtypes = [i, u64, P]
        L.orc_xoro_next.argtypes = [P]
        L.orc_xoro_next.restype = u64
        L.orc_xoro_uniform_f32.argtypes = [P]
        L.orc_xoro_uniform_f32.restype = f
        L.orc_xoro_normal_f32.argtypes = [P]
        L.orc_xoro_normal_f32.restype = f
        L.orc_langevin_step.argtypes = [i, P, P, P, P, P, P, f, f, f, P, P, P]
        L.orc_set_langevin.argtypes = [P, P, f]
        L.orc_set_npt.argtypes = [P, P, f, f, f]
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def num_threads():
    return lib().orc_num_threads()


def set_num_threads(n):
    lib().orc_set_num_threads(int(n))


def param_table(params):
    """gamdpy's user params [p0, p1, ..., cut] (scalars or ntypes x ntypes)
    -> (nt, nt, np) float32 table (pair_potential.py:23-51)."""
    mats = [np.atleast_2d(np.asarray(p, dtype=np.float32)) for p in params]
    nt = max(m.shape[0] for m in mats)
    mats = [np.broadcast_to(m, (nt, nt)) for m in mats]
    return np.ascontiguousarray(np.stack(mats, axis=-1), dtype=np.float32)


def pair_potential(dist, p, kind=POT_LJ_SIGMA_EPSILON, cutmode=CUT_SF):
    p = _f32(p)
    out = np.zeros(3, np.float32)
    lib().orc_pair_potential(kind, cutmode, float(dist), _p(p), len(p), _p(out))
    return out


def dist_sq(ri, rj, box, fma=0):
    ri, rj, box = _f32(ri), _f32(rj), _f32(box)
    dr = np.zeros(3, np.float32)
    d2 = lib().orc_dist_sq(_p(ri), _p(rj), _p(box), _p(dr), fma)
    return np.float32(d2), dr


def apply_pbc(r, img, box):
    r, img, box = _f32(r).copy(), _i32(img).copy(), _f32(box)
    lib().orc_apply_pbc(_p(r), _p(img), _p(box))
    return r, img


def nblist_nsq(r, box, cut_plus_skin, max_nbs, fma=0):
    r, box = _f32(r), _f32(box)
    nbl = np.zeros((len(r), max_nbs + 1), np.int32)
    mx = lib().orc_nblist_nsq(len(r), _p(r), _p(box), float(cut_plus_skin), max_nbs, _p(nbl), fma)
    return nbl, mx


def cells_per_dimension(box, max_cut, skin):
    nc = np.zeros(3, np.int32)
    ok = lib().orc_cells_per_dimension(_p(_f32(box)), float(max_cut), float(skin), _p(nc))
    return nc if ok == 0 else None


def cell_coords(r, box, nc):
    r, box, nc = _f32(r), _f32(box), _i32(nc)
    out = np.zeros((len(r), 3), np.int32)
    lib().orc_cell_coords(len(r), _p(r), _p(box), _p(nc), _p(out))
    return out


def nblist_cells(r, box, max_cut, skin, max_nbs, fma=0):
    r, box = _f32(r), _f32(box)
    nbl = np.zeros((len(r), max_nbs + 1), np.int32)
    mx = lib().orc_nblist_cells(len(r), _p(r), _p(box), float(max_cut), float(skin), max_nbs, _p(nbl), fma)
    if mx == -1:
        raise ValueError("cell grid too small (gamdpy asserts > 4 cells per dimension, > 6 in x)")
    return nbl, mx


def forces(r, ptype, box, table, nbl, kind=POT_LJ_SIGMA_EPSILON, cutmode=CUT_SF, fma=0):
    r, box, table, nbl = _f32(r), _f32(box), _f32(table), _i32(nbl)
    n = len(r)
    nt, _, npar = table.shape
    pt = _i32(ptype) if ptype is not None else np.zeros(n, np.int32)
    f = np.zeros((n, 3), np.float32)
    U, W, lap, fsq = (np.zeros(n, np.float32) for _ in range(4))
    lib().orc_forces(n, _p(r), _p(pt), _p(box), _p(table), npar, nt, kind, cutmode, _p(nbl),
                     nbl.shape[1] - 1, _p(f), _p(U), _p(W), _p(lap), _p(fsq), fma)
    return {"f": f, "U": U, "W": W, "lapU": lap, "Fsq": fsq}


def exclude(nbl, exclusions):
    """A neighbour list without the excluded pairs, as the builds' exclusion
    test (interactions/nblist.py:120-123, nblist_linked_lists.py:174-178)
    leaves it: a candidate is dropped when it appears among the first
    exclusions[i, -1] entries of particle i's row; the order of the rest is
    kept."""
    nbl = np.asarray(nbl)
    ex = np.asarray(exclusions)
    out = np.zeros_like(nbl)
    for i in range(len(nbl)):
        drop = set(ex[i, : ex[i, -1]].tolist())
        row = [j for j in nbl[i, : nbl[i, -1]].tolist() if j not in drop]
        out[i, : len(row)] = row
        out[i, -1] = len(row)
    return out


def bond_terms(r, box, indices, params):
    """Harmonic bond contributions per particle (interactions/bonds.py:102-135
    with potential_functions/harmonic_bond_function.py:37-43), each bond in
    float32 as the reference computes it: dr = r_j - r_i by the minimum image,
    dist = sqrt(dist_sq), u = k (dist - r0)^2 / 2, s = -k (dist - r0) / dist;
    f_i -= dr s, f_j += dr s, u / 2 and dr^2 s / (2 D) to both ends, and
    (1 - D) s + k to both lapU entries; per-particle sums in float64.
    Returns dict f (N, 3), U, W, lapU (N,)."""
    r, box = _f32(r), _f32(box)
    n = len(r)
    f = np.zeros((n, 3)); U = np.zeros(n); W = np.zeros(n); lap = np.zeros(n)
    half, vf = np.float32(0.5), np.float32(0.5 / 3)
    for i, j, t in np.asarray(indices):
        r0, k = np.float32(params[t][0]), np.float32(params[t][1])
        dr = np.zeros(3, np.float32)
        for c in range(3):
            d = r[j, c] - r[i, c]
            d = d - box[c] if np.float32(2.0) * d > box[c] else (d + box[c] if np.float32(2.0) * d < -box[c] else d)
            dr[c] = d
        dist = np.float32(math.sqrt(np.float32(dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2])))
        u = half * k * (dist - r0) ** 2
        s = -k * (dist - r0) / dist
        f[i] -= dr * s
        f[j] += dr * s
        w = np.float32(np.sum(dr * dr * s * vf))
        U[i] += u * half; U[j] += u * half
        W[i] += w; W[j] += w
        lp = np.float32(-2.0) * s + k
        lap[i] += lp; lap[j] += lp
    return {"f": f, "U": U, "W": W, "lapU": lap}


def forces_fp64(r, ptype, box, sigma, epsilon, cut, nbl):
    """Forces of the shifted-force LJ_12_6_sigma_epsilon pair potential over
    a neighbour list, every operation in float64 (the float32 positions taken
    exactly): the formula of LJ_12_6_sigma_epsilon.py:26-36 with
    apply_shifted_force_cutoff.py:30-37 (s -= s(cut)) and the minimum image
    of orthorhombic.py:50-53.  The yardstick for the float32 paths' error."""
    r = np.asarray(r, np.float64)
    box = np.asarray(box, np.float64)
    n = len(r)
    pt = np.zeros(n, np.int64) if ptype is None else np.asarray(ptype, np.int64)
    nbl = np.asarray(nbl)
    cnt = np.minimum(nbl[:, -1], nbl.shape[1] - 1)
    rows = np.repeat(np.arange(n), cnt)
    cols = nbl[:, :-1][np.arange(nbl.shape[1] - 1)[None, :] < cnt[:, None]]
    dr = r[cols] - r[rows]
    dr -= box * np.where(2 * dr > box, 1.0, np.where(2 * dr < -box, -1.0, 0.0))
    d2 = np.einsum("ij,ij->i", dr, dr)
    sg = np.asarray(sigma, np.float64)[pt[rows], pt[cols]]
    ep = np.asarray(epsilon, np.float64)[pt[rows], pt[cols]]
    rc = np.asarray(cut, np.float64)[pt[rows], pt[cols]]

    def s_of(x2):
        x6 = (sg * sg / x2) ** 3
        return 24.0 * ep * (2.0 * x6 * x6 - x6) / x2

    inside = d2 < rc * rc
    s = np.where(inside, s_of(d2) - s_of(rc * rc), 0.0)
    f = np.zeros((n, 3))
    np.add.at(f, rows, -dr * s[:, None])
    return f


def rdf(r, ptype, box, bins, fma=0, r_max=0.0):
    r, box = _f32(r), _f32(box)
    n = len(r)
    pt = _i32(ptype) if ptype is not None else np.zeros(n, np.int32)
    nt = int(pt.max()) + 1
    out = np.zeros((nt, nt, bins), np.uint64)
    lib().orc_rdf(n, _p(r), _p(pt), _p(box), nt, bins, _p(out), fma, float(r_max))
    return out


def sq(r, q, ff=None):
    r, q = _f32(r), _f32(q)
    ffa = _f32(ff) if ff is not None else None
    re = np.zeros(len(q), np.float64)
    im = np.zeros(len(q), np.float64)
    lib().orc_sq(len(r), _p(r), _p(ffa), len(q), _p(q), _p(re), _p(im))
    return re + 1j * im


def calc_dynamics(block, ptype, box, dt, first_block, qvalues=None):
    """tools/calc_dynamics.py:6-75 restated: per time lag and type, the mean
    square displacement, the mean fourth power, and the self-intermediate
    scattering function (the mean of cos(q dr) over particles and
    components); lags inside a block (frame i+1 against frame 0) and across
    blocks (first frames 2^(i+1) blocks apart); displacements unwrapped with
    the image counts; alpha2 = 3 m4d / (5 msd^2) - 1."""
    block = np.asarray(block)
    ptype = np.asarray(ptype)
    box = np.asarray(box, np.float32)
    num_types = int(ptype.max()) + 1
    if isinstance(qvalues, float):
        qvalues = np.ones(num_types) * qvalues
    num_blocks, conf_per_block, _, n, d = block.shape
    first_block = first_block % num_blocks
    extra = int(math.log2(num_blocks - first_block)) - 1
    total = conf_per_block - 1 + extra
    count = np.zeros((total, 1), np.int32)
    msd, m4d, fs = (np.zeros((total, num_types)) for _ in range(3))

    def add(b0, c0, b1, c1, ti):
        dr = block[b1, c1, 0] - block[b0, c0, 0]
        dr += (block[b1, c1, 1] - block[b0, c0, 1]) * box
        for t in range(num_types):
            dt_ = dr[ptype == t]
            sq = np.sum(dt_ ** 2, axis=1)
            msd[ti, t] += np.mean(sq)
            m4d[ti, t] += np.mean(sq ** 2)
            fs[ti, t] += np.mean(np.cos(dt_ * qvalues[t]))

    for b in range(first_block, num_blocks):
        for i in range(conf_per_block - 1):
            count[i] += 1
            add(b, i + 1, b, 0, i)
    for b in range(first_block, num_blocks):
        for i in range(extra):
            other = b + 2 ** (i + 1)
            if other < num_blocks:
                count[conf_per_block - 1 + i] += 1
                add(other, 0, b, 0, conf_per_block - 1 + i)
    msd /= count
    m4d /= count
    fs /= count
    return {"times": dt * 2 ** np.arange(total), "msd": msd, "alpha2": 3 * m4d / (5 * msd ** 2) - 1,
            "qvalues": qvalues, "Fs": fs, "count": count}


def xoro_states(n, seed):
    """numba.cuda.random.create_xoroshiro128p_states(n, seed) restated:
    (n, 2) uint64 (s0, s1)."""
    st = np.zeros((n, 2), np.uint64)
    lib().orc_xoro_init(int(n), int(seed) & 0xFFFFFFFFFFFFFFFF, _p(st))
    return st


def xoro_next(states, index):
    """xoroshiro128p_next on states[index] (advances it)."""
    row = states[index]
    out = lib().orc_xoro_next(row.ctypes.data_as(ctypes.c_void_p))
    return np.uint64(out)


def xoro_normal_f32(states, index):
    """xoroshiro128p_normal_float32 on states[index] (advances it twice)."""
    row = states[index]
    return np.float32(lib().orc_xoro_normal_f32(row.ctypes.data_as(ctypes.c_void_p)))


def npt_masses(n, D, tau, tau_p):
    """Thermostat and barostat masses without the temperature factor, as
    integrators/NPT_Atomic.py:44-48 computes them (numpy float32)."""
    degrees = n * D - D
    factor = np.float32(1. / (4 * np.pi * np.pi))
    mass_t = np.float32((degrees - 1) * D * factor * tau * tau)
    mass_p = np.float32((degrees - 1) * D * factor * tau_p * tau_p)
    return mass_t, mass_p


class Run:
    """State of one oracle simulation, advanced one timeblock at a time with
    the reference's composed loop (gamdpy/simulation/Simulation.py:330-346).
    integrator "NVT_Langevin" takes temperature, alpha and seed
    (integrators/NVT_Langevin.py:44-53); "NPT_Atomic" takes temperature,
    tau, pressure and tau_p, with the state arrays ``ts`` (2) and ``bs`` (3)
    and the masses of integrators/NPT_Atomic.py:38-50; its box changes in
    place."""

    def __init__(self, r, v, m, ptype, box, table, kind=POT_LJ_SIGMA_EPSILON, cutmode=CUT_SF,
                 nblist="N squared", skin=0.5, max_nbs=300, integrator="NVE", dt=0.005,
                 temperature=None, tau=None, every=0, reset_every=0, fma=0, alpha=None, seed=0, pressure=None,
                 tau_p=None):
        n = len(r)
        self.n = n
        self.r = _f32(r).copy()
        self.v = _f32(v).copy()
        self.m = np.broadcast_to(np.asarray(m, np.float32), (n,)).copy()
        self.ptype = _i32(ptype).copy() if ptype is not None else np.zeros(n, np.int32)
        self.box = _f32(box).copy()
        self.table = _f32(table)
        self.kind, self.cutmode = kind, cutmode
        self.nblist_kind = 0 if nblist == "N squared" else 1
        self.skin, self.max_nbs = float(skin), int(max_nbs)
        self.integrator = {"NVE": 0, "NVT": 1, "NVT_Langevin": 2, "NPT_Atomic": 3}[integrator]
        if self.integrator == 3:
            self.ts = np.zeros(2, np.float32)
            self.bs = np.zeros(3, np.float32)
            self.bs[2] = np.float32(np.prod(self.box.astype(np.float32)))
            self.mass_t, self.mass_p = npt_masses(n, 3, tau, tau_p)
            self.P = np.float32(pressure)
        if self.integrator == 2:
            self.alpha = np.float32(alpha)
            self.rng = xoro_states(n, seed)
            self.old_beta = np.zeros((n, 3), np.float32)
        self.dt = np.float32(dt)
        self.T = np.float32(temperature or 0.0)
        self.omega2 = np.float32(4.0 * np.pi * np.pi / tau / tau) if tau else np.float32(0)
        self.every, self.reset_every, self.fma = int(every), int(reset_every), int(fma)
        self.f = np.zeros((n, 3), np.float32)
        self.img = np.zeros((n, 3), np.int32)
        self.U, self.W, self.K = (np.zeros(n, np.float32) for _ in range(3))
        self.nbl = np.zeros((n, self.max_nbs + 1), np.int32)
        self.r_ref = np.zeros((n, 3), np.float32)
        self.have_list = ctypes.c_int(0)
        self.state = np.zeros(2, np.float32)
        self.rebuilds = 0

    def run_timeblock(self, steps):
        nsave = steps // self.every if self.every else 0
        scal = np.zeros((max(nsave, 1), 4), np.float64)
        nt, _, npar = self.table.shape
        if self.integrator == 2:
            lib().orc_set_langevin(_p(self.rng), _p(self.old_beta), float(self.alpha))
        if self.integrator == 3:
            lib().orc_set_npt(_p(self.ts), _p(self.bs), float(self.mass_t), float(self.mass_p), float(self.P))
        rc = lib().orc_run_timeblock(
            self.n, _p(self.r), _p(self.v), _p(self.f), _p(self.m), _p(self.img), _p(self.ptype),
            _p(self.box), _p(self.table), npar, nt, self.kind, self.cutmode, self.nblist_kind,
            self.skin, self.max_nbs, _p(self.nbl), _p(self.r_ref), ctypes.byref(self.have_list),
            self.integrator, float(self.dt), _p(self.state), float(self.omega2), float(self.T),
            int(steps), self.every, self.reset_every, _p(self.U), _p(self.W), _p(self.K),
            _p(scal), self.fma)
        if rc == -1:
            raise ValueError("cell grid too small")
        if rc == -2:
            raise RuntimeError("neighbour list overflow")
        self.rebuilds += rc
        return scal[:nsave]
