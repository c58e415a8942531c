"""Gradients of trajectory averages with respect to the pair parameters.

gamdpy has no differentiation; this module adds it beside the plain path.
``AdjointNVE`` runs an NVE leapfrog trajectory of a Configuration under the
shifted-force Lennard-Jones pair potential (the forward of
integrators/NVE.py:78-97 with LJ_12_6_sigma_epsilon and
apply_shifted_force_cutoff) on the GPU and returns time-averaged
observables; ``TrajectoryObservables`` is the ``torch.autograd.Function``
whose backward is the library's hand-written discrete adjoint (reverse
leapfrog sweep with Hessian-vector products of the pair forces, recomputed
from checkpoints kept every ``checkpoint_every`` steps).

Parameters are the unordered type pairs' (epsilon, sigma), ``theta =
[eps_00, eps_01, ..., eps_(nt-1)(nt-1), sig_00, sig_01, ...]`` (upper
triangle, row major); the cutoffs stay fixed.  Observables are
``[<U>, <W>, <K>, <g_AA(r_b)>...]``: sums over particles averaged over the
steps, and a Gaussian-kernel radial distribution of type-0 pairs.  torch is
only the autograd bridge: every number comes from libgamdb200.
"""
import ctypes

import numpy as np

from . import _lib

OBS_U, OBS_W, OBS_K, OBS_G0 = 0, 1, 2, 3


def _pairs(nt):
    return [(a, b) for a in range(nt) for b in range(a, nt)]


def theta_from_tables(sigma, epsilon):
    """theta vector (eps of the unordered pairs, then sigma) from symmetric tables."""
    sigma, epsilon = np.asarray(sigma, np.float64), np.asarray(epsilon, np.float64)
    pairs = _pairs(sigma.shape[0])
    return np.array([epsilon[a, b] for a, b in pairs] + [sigma[a, b] for a, b in pairs], np.float64)


def tables_from_theta(theta, nt):
    theta = np.asarray(theta, np.float64)
    pairs = _pairs(nt)
    m = len(pairs)
    sig, eps = np.zeros((nt, nt)), np.zeros((nt, nt))
    for k, (a, b) in enumerate(pairs):
        eps[a, b] = eps[b, a] = theta[k]
        sig[a, b] = sig[b, a] = theta[m + k]
    return sig, eps


class AdjointNVE:
    """Differentiable NVE trajectory of ``configuration`` (positions,
    velocities, types, masses and box are taken at construction).

    cut: (nt, nt) cutoffs (fixed).  rdf: None or dict(bins, r_lo, r_hi,
    width, every) for the type-0 soft radial distribution."""

    def __init__(self, configuration, cut, dt, steps, checkpoint_every=50, rdf=None, window=0, device=0):
        conf = configuration
        self.n = conf.N
        self.nt = int(np.max(conf.ptype)) + 1
        self.cut = np.broadcast_to(np.asarray(cut, np.float64), (self.nt, self.nt)).copy()
        self.dt, self.steps, self.checkpoint_every = float(dt), int(steps), int(checkpoint_every)
        self.rdf = dict(rdf) if rdf else None
        self.nbins = int(self.rdf["bins"]) if self.rdf else 0
        self.volume = float(np.prod(conf.simbox.lengths))
        self.r0 = np.ascontiguousarray(conf["r"], np.float32)
        self.v0 = np.ascontiguousarray(conf["v"], np.float32)
        self.ptype = np.ascontiguousarray(conf.ptype, np.int32)
        self.mass = np.ascontiguousarray(conf["m"], np.float32)
        self.box = np.ascontiguousarray(conf.simbox.lengths, np.float32)
        self.h = ctypes.c_void_p()
        self._call_create(device)
        r = self.rdf or {"bins": 0, "r_lo": 0.0, "r_hi": 1.0, "width": 1.0, "every": 0}
        self._check(_lib.lib().gdb_adj_setup(self.h, _lib.ptr(self.box), _lib.ptr(self.ptype),
                                             _lib.ptr(self.mass), float(self.dt), self.steps,
                                             self.checkpoint_every, int(r["bins"]), float(r["r_lo"]),
                                             float(r["r_hi"]), float(r["width"]), int(r["every"])),
                    "gdb_adj_setup")
        self.forward_count = 0
        self._last_theta = None
        self.set_window(window)

    def set_window(self, window):
        """0: the exact adjoint.  W > 0: the truncated adjoint that treats the
        state at every multiple of W steps as a constant (a trajectory of a
        chaotic system has an exact gradient growing like exp(lambda t))."""
        self.window = int(window)
        self._check(_lib.lib().gdb_adj_set_window(self.h, self.window), "gdb_adj_set_window")

    @property
    def n_obs(self):
        return 3 + self.nbins

    def bin_centres(self):
        r = self.rdf
        dr = (r["r_hi"] - r["r_lo"]) / r["bins"]
        return r["r_lo"] + (np.arange(r["bins"]) + 0.5) * dr

    def _call_create(self, device):
        rc = _lib.lib().gdb_adj_create(self.n, self.nt, int(device), ctypes.byref(self.h))
        if rc != _lib.GDB_OK:
            self._check(rc, "gdb_adj_create", handle=False)

    def _check(self, rc, name, handle=True):
        if rc != _lib.GDB_OK:
            buf = ctypes.create_string_buffer(512)
            _lib.lib().gdb_adj_get_last_error(self.h if handle else None, buf, 512)
            raise _lib.GdbError(rc, f"{name}: {buf.value.decode(errors='replace')}")

    def _params(self, theta):
        sig, eps = tables_from_theta(theta, self.nt)
        p = np.zeros((self.nt, self.nt, 3), np.float64)
        p[..., 0], p[..., 1], p[..., 2] = sig, eps, self.cut
        return np.ascontiguousarray(p)

    def forward(self, theta):
        """Observables (numpy float64) of the trajectory at parameters theta."""
        obs = np.zeros(self.n_obs, np.float64)
        p = self._params(theta)
        self._check(_lib.lib().gdb_adj_forward(self.h, _lib.ptr(p), _lib.ptr(self.r0), _lib.ptr(self.v0),
                                               _lib.ptr(obs)), "gdb_adj_forward")
        self.forward_count += 1
        self._last_theta = np.array(theta, np.float64)
        return obs

    def backward(self, grad_obs):
        """dL/dtheta for the last forward, given dL/dobs."""
        g = np.ascontiguousarray(grad_obs, np.float64)
        out = np.zeros((self.nt, self.nt, 3), np.float64)
        self._check(_lib.lib().gdb_adj_backward(self.h, _lib.ptr(g), _lib.ptr(out)), "gdb_adj_backward")
        pairs = _pairs(self.nt)
        return np.array([out[a, b, 1] for a, b in pairs] + [out[a, b, 0] for a, b in pairs], np.float64)

    def final_state(self):
        r = np.zeros((self.n, 3), np.float32)
        v = np.zeros((self.n, 3), np.float32)
        self._check(_lib.lib().gdb_adj_final_state(self.h, _lib.ptr(r), _lib.ptr(v)), "gdb_adj_final_state")
        return r, v

    def observables(self, theta):
        """torch entry point: observables as a differentiable function of theta."""
        return TrajectoryObservables.apply(theta, self)

    def __del__(self):
        try:
            if self.h:
                _lib.lib().gdb_adj_destroy(self.h)
                self.h = ctypes.c_void_p()
        except Exception:
            pass


def _torch():
    import torch
    return torch


def _make_function():
    torch = _torch()

    class TrajectoryObservablesFn(torch.autograd.Function):
        """obs = TrajectoryObservables.apply(theta, engine); backward runs the
        library's adjoint sweep.  If the engine ran another forward in
        between, the forward at this theta is repeated first (the adjoint
        needs its checkpoints)."""

        @staticmethod
        def forward(ctx, theta, engine):
            th = theta.detach().to("cpu", torch.float64).numpy()
            obs = engine.forward(th)
            ctx.engine, ctx.theta, ctx.token = engine, th.copy(), engine.forward_count
            ctx.dtype, ctx.device = theta.dtype, theta.device
            return torch.as_tensor(obs, dtype=torch.float64, device=theta.device)

        @staticmethod
        def backward(ctx, grad_obs):
            eng = ctx.engine
            if eng.forward_count != ctx.token:
                eng.forward(ctx.theta)
            g = eng.backward(grad_obs.detach().to("cpu", torch.float64).numpy())
            return torch.as_tensor(g, dtype=ctx.dtype, device=ctx.device), None

    return TrajectoryObservablesFn


class _Lazy:
    """Defers the torch import until the Function is first used."""

    _fn = None

    def apply(self, theta, engine):
        if _Lazy._fn is None:
            _Lazy._fn = _make_function()
        return _Lazy._fn.apply(theta, engine)


TrajectoryObservables = _Lazy()


def pressure(obs, volume):
    """P = (2 <K> / 3 + <W>) / V, the pressure of the averaged sums (D = 3)."""
    return (2.0 / 3.0 * obs[OBS_K] + obs[OBS_W]) / volume


def matching_loss(obs, target, n, volume, dr):
    """Squared deviations of <U>/N and P from the target's, plus the L2
    distance of the A-A radial distributions: the loss of the parameter-fitting
    workload.  Works on numpy arrays and torch tensors alike."""
    du = obs[OBS_U] / n - target[OBS_U] / n
    dp = pressure(obs, volume) - pressure(target, volume)
    dg = obs[OBS_G0:] - target[OBS_G0:]
    return du * du + dp * dp + (dg * dg).sum() * dr
