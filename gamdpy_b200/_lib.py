"""ctypes bindings of libgamdb200.so (declared in include/gamdb200.h).

The library is the only compute path of this package: there is no CPU
fallback.  ``lib()`` raises ``RuntimeError`` when the shared library is
missing or cannot be loaded, and every wrapper raises when a call returns a
non-zero status, with the library's own error message.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("GAMDB200_LIB", os.path.join(HERE, "libgamdb200.so"))

GDB_OK = 0
GDB_ERR_ARG = 1
GDB_ERR_CUDA = 2
GDB_ERR_STATE = 3
GDB_ERR_NBLIST = 4
GDB_ERR_NUMERIC = 5
GDB_ERR_UNSUPPORTED = 6

STATUS_NBLIST_OVERFLOW = 0x1
STATUS_BARRIER_TIMEOUT = 0x2
STATUS_NAN = 0x4
STATUS_BAD_ARG = 0x8

POT_LJ_SIGMA_EPSILON = 0
POT_LJ_12_6 = 1
CUT_SHIFTED_FORCE = 0
CUT_SHIFTED_POTENTIAL = 1
NBLIST_NSQ = 0
NBLIST_CELLS = 1
INTEGRATOR_NVE = 0
INTEGRATOR_NVT = 1
TFUNC_CONSTANT = 0
TFUNC_RAMP = 1
NUM_SCALARS = 6  # U, W, lapU, K, Fsq, Vol (NPT_Atomic runs)

# every exported entry point with its argument types (order as in gamdb200.h)
_P = ctypes.c_void_p
_i = ctypes.c_int
_f = ctypes.c_float
_d = ctypes.c_double
SIGNATURES = {
    "gdb_version": ([], _i),
    "gdb_device_count": ([_P], _i),
    "gdb_device_name": ([_i, ctypes.c_char_p, _i], _i),
    "gdb_sim_create": ([_i, _i, _i, _P], _i),
    "gdb_sim_destroy": ([_P], _i),
    "gdb_set_box": ([_P, _P], _i),
    "gdb_upload_state": ([_P, _P, _P, _P, _P, _P], _i),
    "gdb_download_state": ([_P, _P, _P, _P, _P], _i),
    "gdb_download_scalars": ([_P, _P, _P, _P, _P, _P], _i),
    "gdb_download_table": ([_P, _P, _P, _P, _i, _P], _i),
    "gdb_host_alloc": ([ctypes.c_size_t, _P], _i),
    "gdb_host_free": ([_P], _i),
    "gdb_set_pair_potential": ([_P, _i, _i, _i, _P, _i], _i),
    "gdb_set_nblist": ([_P, _i, _f, _i], _i),
    "gdb_set_exclusions": ([_P, _P, _i], _i),
    "gdb_set_bonds": ([_P, _i, _P, _i, _P], _i),
    "gdb_set_plan": ([_P, _i, _i], _i),
    "gdb_set_integrator_nve": ([_P, _f], _i),
    "gdb_set_integrator_nvt": ([_P, _f, _f, _i, _P], _i),
    "gdb_get_thermostat_state": ([_P, _P], _i),
    "gdb_set_thermostat_state": ([_P, _P], _i),
    "gdb_set_runtime_actions": ([_P, _i, _i], _i),
    "gdb_set_configuration_saver": ([_P, _i], _i),
    "gdb_get_saved_configurations": ([_P, _P, _i], _i),
    "gdb_get_saved_boxes": ([_P, _P, _i], _i),
    "gdb_eval_forces": ([_P], _i),
    "gdb_sim_run": ([_P, _d, _i, _P], _i),
    "gdb_set_trace": ([_P, _i], _i),
    "gdb_get_trace": ([_P, _P, _i, _P], _i),
    "gdb_time_step_kernel": ([_P, _i, _P], _i),
    "gdb_nblist_stats": ([_P, _P, _P], _i),
    "gdb_get_scalar_rows": ([_P, _P, _i], _i),
    "gdb_get_nblist": ([_P, _P, _i], _i),
    "gdb_get_nbflag": ([_P, _P], _i),
    "gdb_status_word": ([_P], ctypes.c_uint32),
    "gdb_clear_status": ([_P], _i),
    "gdb_get_last_path": ([_P], _i),
    "gdb_get_last_error": ([_P, ctypes.c_char_p, _i], _i),
    "gdb_rdf_update": ([_P, _i, _d, _P], _i),
    "gdb_sq_update": ([_P, _i, _P, _P, _P, _P], _i),
    "gdb_set_integrator_langevin": ([_P, _f, _f, ctypes.c_uint64, _i, _P], _i),
    "gdb_get_langevin_state": ([_P, _P, _P], _i),
    "gdb_set_integrator_npt": ([_P, _f, _f, _f, _i, _P, _i, _P], _i),
    "gdb_get_npt_state": ([_P, _P, _P], _i),
    "gdb_set_npt_state": ([_P, _P, _P], _i),
    "gdb_get_box": ([_P, _P], _i),
    "gdb_calc_dynamics": ([_i, _i, _i, _P, _P, _i, _P, _i, _P, _i, _P, _P, _P, _P], _i),
    "gdb_last_analysis_ms": ([_P, _P], _i),
    "gdb_rdf_compute": ([_i, _P, _P, _P, _i, _i, _d, _P], _i),
    "gdb_sq_compute": ([_i, _P, _P, _P, _i, _P, _P, _P], _i),
    "gdb_sq_compute_noalloc": ([_i, _P, _P, _P, _i, _P, _i, _P, _P, _P], _i),
    "gdb_batch_create": ([_P, _i, _i, _P], _i),
    "gdb_batch_create_ex": ([_P, _i, _i, _i, _i, _P], _i),
    "gdb_batch_run": ([_P, _d, _i, _P], _i),
    "gdb_batch_destroy": ([_P], _i),
    "gdb_batch_get_last_error": ([_P, ctypes.c_char_p, _i], _i),
    "gdb_selftest_barrier_timeout": ([_i, ctypes.c_longlong, _P], _i),
    "gdb_adj_create": ([_i, _i, _i, _P], _i),
    "gdb_adj_destroy": ([_P], _i),
    "gdb_adj_setup": ([_P, _P, _P, _P, _f, _i, _i, _i, _f, _f, _f, _i], _i),
    "gdb_adj_forward": ([_P, _P, _P, _P, _P], _i),
    "gdb_adj_backward": ([_P, _P, _P], _i),
    "gdb_adj_final_state": ([_P, _P, _P], _i),
    "gdb_adj_set_window": ([_P, _i], _i),
    "gdb_adj_get_last_error": ([_P, ctypes.c_char_p, _i], _i),
}

_lib = None


def lib():
    """Load the shared library (once).  Raises RuntimeError if it is absent."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"libgamdb200.so not found at {LIB_PATH}; build it with `python -m gamdpy_b200.build` "
                "(gamdpy_b200 has no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (args, res) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _lib = L
    return _lib


def ptr(a):
    """Pointer to a numpy array's data (None passes NULL)."""
    if a is None:
        return None
    return ctypes.c_void_p(a.ctypes.data)


def last_error(h=None):
    buf = ctypes.create_string_buffer(512)
    lib().gdb_get_last_error(h, buf, 512)
    return buf.value.decode(errors="replace")


class GdbError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(msg)
        self.code = code


def check(rc, h=None, what=""):
    if rc != GDB_OK:
        msg = last_error(h)
        if rc == GDB_ERR_ARG:
            raise ValueError(f"{what}: {msg}")
        if rc == GDB_ERR_UNSUPPORTED:
            raise NotImplementedError(f"{what}: {msg}")
        raise GdbError(rc, f"{what}: {msg}" if what else msg)
    return rc


def f32(a, shape=None):
    a = np.ascontiguousarray(a, dtype=np.float32)
    if shape is not None and a.shape != shape:
        raise ValueError(f"expected shape {shape}, got {a.shape}")
    return a


def i32(a, shape=None):
    a = np.ascontiguousarray(a, dtype=np.int32)
    if shape is not None and a.shape != shape:
        raise ValueError(f"expected shape {shape}, got {a.shape}")
    return a


def pinned_empty(shape, dtype):
    """A numpy array in page-locked host memory from gdb_host_alloc, freed
    when the last view of it is gone; None when no GPU is available (the
    caller then keeps ordinary numpy memory)."""
    dtype = np.dtype(dtype)
    nbytes = int(np.prod(shape)) * dtype.itemsize
    p = ctypes.c_void_p()
    try:
        if lib().gdb_host_alloc(ctypes.c_size_t(max(nbytes, 1)), ctypes.byref(p)) != GDB_OK or not p.value:
            return None
    except (RuntimeError, OSError):
        return None
    addr = p.value

    def _free(_self, addr=addr):
        try:
            lib().gdb_host_free(ctypes.c_void_p(addr))
        except Exception:
            pass

    owner_t = type("PinnedBytes", (ctypes.c_char * max(nbytes, 1),), {"__del__": _free})
    owner = owner_t.from_address(addr)
    return np.frombuffer(owner, dtype=dtype, count=int(np.prod(shape))).reshape(shape)


def device_name(device=0):
    buf = ctypes.create_string_buffer(256)
    check(lib().gdb_device_name(int(device), buf, 256), None, "gdb_device_name")
    return buf.value.decode()


class Sim:
    """Owner of one gdb_sim handle (device state of one configuration)."""

    def __init__(self, n, ntypes, device=0):
        self.h = ctypes.c_void_p()
        check(lib().gdb_sim_create(int(n), int(ntypes), int(device), ctypes.byref(self.h)), None,
              "gdb_sim_create")
        self.n, self.ntypes = int(n), int(ntypes)
        self.device = int(device)

    def __del__(self):
        try:
            if self.h:
                lib().gdb_sim_destroy(self.h)
                self.h = ctypes.c_void_p()
        except Exception:
            pass

    def call(self, name, *args):
        return check(getattr(lib(), name)(self.h, *args), self.h, name)

    # --- state --------------------------------------------------------
    def set_box(self, lengths):
        L = f32(lengths, (3,))
        self.call("gdb_set_box", ptr(L))

    def upload(self, r, v, m, ptype, r_im=None):
        n = self.n
        r, v = f32(r, (n, 3)), f32(v, (n, 3))
        m, pt = f32(m, (n,)), i32(ptype, (n,))
        im = i32(r_im, (n, 3)) if r_im is not None else None
        self.call("gdb_upload_state", ptr(r), ptr(v), ptr(m), ptr(pt), ptr(im))

    def download(self, r=True, v=True, f=True, r_im=True):
        n = self.n
        out = {k: (np.empty((n, 3), np.int32 if k == "r_im" else np.float32) if want else None)
               for k, want in (("r", r), ("v", v), ("f", f), ("r_im", r_im))}
        self.call("gdb_download_state", ptr(out["r"]), ptr(out["v"]), ptr(out["f"]), ptr(out["r_im"]))
        return out

    def download_scalars(self, out=None):
        """Per-particle U, W, lapU, K, Fsq; `out` (a dict of (n,) float32
        arrays) is filled in place when given."""
        n = self.n
        if out is None:
            out = {k: np.empty(n, np.float32) for k in ("U", "W", "lapU", "K", "Fsq")}
        for k in ("U", "W", "lapU", "K", "Fsq"):
            a = out[k]
            assert a.dtype == np.float32 and a.shape == (n,) and a.flags.c_contiguous
        self.call("gdb_download_scalars", *(ptr(out[k]) for k in ("U", "W", "lapU", "K", "Fsq")))
        return out

    def download_into(self, r=None, v=None, f=None, r_im=None):
        """Fill caller-owned (n, 3) arrays in place (float32; int32 for r_im):
        no fresh host pages per call, which dominate large copies otherwise."""
        n = self.n
        for a, dt in ((r, np.float32), (v, np.float32), (f, np.float32), (r_im, np.int32)):
            if a is not None:
                assert a.dtype == dt and a.shape == (n, 3) and a.flags.c_contiguous
        self.call("gdb_download_state", ptr(r), ptr(v), ptr(f), ptr(r_im))

    def download_table(self, vectors, r_im, scalars, cols):
        """Fill a Configuration's own arrays in place in one call: vectors
        (3, n, 3) float32 r, v, f; r_im (n, 3) int32; scalars (n, nscal)
        float32 with cols = the columns of U, W, lapU, K, Fsq, m (-1 absent).
        Any array may be None."""
        n = self.n
        if vectors is not None:
            assert vectors.dtype == np.float32 and vectors.shape == (3, n, 3) and vectors.flags.c_contiguous
        if r_im is not None:
            assert r_im.dtype == np.int32 and r_im.shape == (n, 3) and r_im.flags.c_contiguous
        nscal = 0
        c = None
        if scalars is not None:
            assert scalars.dtype == np.float32 and scalars.ndim == 2 and scalars.shape[0] == n
            assert scalars.flags.c_contiguous
            nscal = scalars.shape[1]
            c = np.ascontiguousarray(cols, np.int32)
            assert c.shape == (6,)
        self.call("gdb_download_table", ptr(vectors), ptr(r_im), ptr(scalars), int(nscal), ptr(c))

    # --- configuration of the step ------------------------------------
    def set_pair_potential(self, kind, cutmode, table):
        t = f32(table)
        nt, _, npar = t.shape
        self.call("gdb_set_pair_potential", int(kind), int(cutmode), int(nt), ptr(t), int(npar))

    def set_nblist(self, kind, skin, max_nbs):
        self.call("gdb_set_nblist", int(kind), float(skin), int(max_nbs))

    def set_exclusions(self, excl):
        """(n, max + 1) int32 exclusion table with the count last, or None."""
        if excl is None:
            self.call("gdb_set_exclusions", None, 0)
            return
        ex = i32(excl)
        if ex.ndim != 2 or ex.shape[0] != self.n:
            raise ValueError(f"exclusions must be ({self.n}, max + 1)")
        self.call("gdb_set_exclusions", ptr(ex), int(ex.shape[1] - 1))

    def set_bonds(self, indices, params):
        """indices (nbonds, 3) int32 (i, j, type); params (ntypes, 2) (r0, k)."""
        ind = i32(indices).reshape(-1, 3)
        prm = f32(params).reshape(-1, 2)
        self.call("gdb_set_bonds", int(len(ind)), ptr(ind), int(len(prm)), ptr(prm))

    def set_plan(self, tp=0, pb=0):
        self.call("gdb_set_plan", int(tp), int(pb))

    def set_nve(self, dt):
        self.call("gdb_set_integrator_nve", float(dt))

    def set_nvt(self, dt, tau, tfunc, tparams):
        tp = f32(np.resize(np.asarray(tparams, np.float32), 4))
        self.call("gdb_set_integrator_nvt", float(dt), float(tau), int(tfunc), ptr(tp))

    def set_langevin(self, dt, alpha, seed, tfunc, tparams):
        tp = f32(np.resize(np.asarray(tparams, np.float32), 4))
        self.call("gdb_set_integrator_langevin", float(dt), float(alpha), int(seed) & 0xFFFFFFFFFFFFFFFF, int(tfunc),
                  ptr(tp))

    def set_npt(self, dt, mass_t, mass_p, tfunc, tparams, pfunc, pparams):
        tp = f32(np.resize(np.asarray(tparams, np.float32), 4))
        pp = f32(np.resize(np.asarray(pparams, np.float32), 4))
        self.call("gdb_set_integrator_npt", float(dt), float(mass_t), float(mass_p), int(tfunc), ptr(tp), int(pfunc),
                  ptr(pp))

    def npt_state(self):
        """(thermostat_state (2,), barostat_state (3,)) float32."""
        ts = np.zeros(2, np.float32)
        bs = np.zeros(3, np.float32)
        self.call("gdb_get_npt_state", ptr(ts), ptr(bs))
        return ts, bs

    def set_npt_state(self, ts, bs):
        ts = f32(ts, (2,))
        bs = f32(bs, (3,))
        self.call("gdb_set_npt_state", ptr(ts), ptr(bs))

    def box(self):
        b = np.zeros(3, np.float32)
        self.call("gdb_get_box", ptr(b))
        return b

    def langevin_state(self):
        """(states (n, 2) uint64, old_beta (n, 3) float32) in user order."""
        st = np.zeros((self.n, 2), np.uint64)
        ob = np.zeros((self.n, 3), np.float32)
        self.call("gdb_get_langevin_state", ptr(st), ptr(ob))
        return st, ob

    def thermostat_state(self):
        s = np.zeros(2, np.float32)
        self.call("gdb_get_thermostat_state", ptr(s))
        return s

    def set_thermostat_state(self, s):
        s = f32(s, (2,))
        self.call("gdb_set_thermostat_state", ptr(s))

    def set_runtime_actions(self, scalar_every, momentum_every):
        self.call("gdb_set_runtime_actions", int(scalar_every), int(momentum_every))

    def set_configuration_saver(self, conf_per_block):
        self.call("gdb_set_configuration_saver", int(conf_per_block))

    def saved_boxes(self, conf_per_block):
        out = np.zeros((conf_per_block, 3), np.float32)
        self.call("gdb_get_saved_boxes", ptr(out), int(conf_per_block))
        return out

    def saved_configurations(self, conf_per_block):
        out = np.zeros((conf_per_block, 2, self.n, 3), np.float32)
        self.call("gdb_get_saved_configurations", ptr(out), int(conf_per_block))
        return out

    # --- execution ----------------------------------------------------
    def eval_forces(self):
        self.call("gdb_eval_forces")

    def run(self, time_zero, steps):
        ms = ctypes.c_float(0.0)
        self.call("gdb_sim_run", float(time_zero), int(steps), ctypes.byref(ms))
        return ms.value

    def set_trace(self, capacity):
        self.call("gdb_set_trace", int(capacity))

    def trace(self, capacity=1 << 16):
        """Phase trace entries as (tag, ns) arrays; restarts the trace."""
        buf = np.zeros(capacity, np.uint64)
        cnt = ctypes.c_int(0)
        self.call("gdb_get_trace", ptr(buf), int(capacity), ctypes.byref(cnt))
        buf = buf[: cnt.value]
        return (buf >> np.uint64(56)).astype(np.int64), (buf & np.uint64((1 << 56) - 1)).astype(np.int64)

    def time_step_kernel(self, reps):
        ms = ctypes.c_float(0.0)
        self.call("gdb_time_step_kernel", int(reps), ctypes.byref(ms))
        return ms.value

    def nblist_stats(self):
        mean, mx = ctypes.c_double(0.0), ctypes.c_int(0)
        self.call("gdb_nblist_stats", ctypes.byref(mean), ctypes.byref(mx))
        return mean.value, mx.value

    def scalar_rows(self, rows):
        out = np.zeros((rows, NUM_SCALARS), np.float64)
        if rows:
            self.call("gdb_get_scalar_rows", ptr(out), int(rows))
        return out

    def nblist(self, max_nbs):
        out = np.zeros((self.n, max_nbs + 1), np.int32)
        self.call("gdb_get_nblist", ptr(out), int(max_nbs))
        return out

    def nbflag(self):
        out = np.zeros(3, np.int32)
        self.call("gdb_get_nbflag", ptr(out))
        return out

    def last_path(self):
        """0 graph launches, 1 persistent grid kernel, 2 thread-block cluster with the
        state in shared memory, 3 thread-block cluster with the state in global
        memory (batched systems)."""
        return int(lib().gdb_get_last_path(self.h))

    def status(self):
        return int(lib().gdb_status_word(self.h))

    def clear_status(self):
        self.call("gdb_clear_status")

    # --- calculators --------------------------------------------------
    def rdf_update(self, bins, r_max, out):
        assert out.dtype == np.uint64 and out.flags.c_contiguous
        self.call("gdb_rdf_update", int(bins), float(r_max), ptr(out))

    def last_analysis_ms(self):
        """Device time of the last rdf_update / sq_update (CUDA events)."""
        ms = ctypes.c_float()
        self.call("gdb_last_analysis_ms", ctypes.byref(ms))
        return float(ms.value)

    def sq_update(self, n_vectors, ff=None):
        nv = i32(n_vectors)
        nq = nv.shape[0]
        re, im = np.zeros(nq), np.zeros(nq)
        ffa = f32(ff, (self.n,)) if ff is not None else None
        self.call("gdb_sq_update", int(nq), ptr(nv), ptr(ffa), ptr(re), ptr(im))
        return re + 1j * im


def rdf_compute(r, ptype, box, ntypes, bins, r_max=0.0):
    r = f32(r)
    n = r.shape[0]
    pt = i32(ptype, (n,)) if ptype is not None else None
    L = f32(box, (3,))
    out = np.zeros((ntypes, ntypes, bins), np.uint64)
    check(lib().gdb_rdf_compute(int(n), ptr(r), ptr(pt), ptr(L), int(ntypes), int(bins), float(r_max), ptr(out)),
          None, "gdb_rdf_compute")
    return out


def calc_dynamics(frames, ptype, box, first_block, qvalues, total_times):
    """gdb_calc_dynamics: (msd, m4d, fs, count) for ConfigurationSaver frames."""
    frames = f32(frames)
    nb, cpb, two, n, d = frames.shape
    if two != 2 or d != 3:
        raise ValueError("frames must be (num_blocks, conf_per_block, 2, N, 3)")
    pt = i32(ptype, (n,))
    # one column per type 0 ... max(ptype), as tools/calc_dynamics.py:30
    nt = int(pt.max()) + 1
    qv = np.asarray(qvalues, np.float64).reshape(-1)
    if qv.shape[0] < nt:
        raise ValueError(f"calc_dynamics: {qv.shape[0]} q-values for {nt} particle types")
    q = np.ascontiguousarray(qv[:nt])
    L = f32(box, (3,))
    msd, m4d, fs = (np.zeros((total_times, nt)) for _ in range(3))
    count = np.zeros((total_times, 1), np.int32)
    check(lib().gdb_calc_dynamics(int(nb), int(cpb), int(n), ptr(frames), ptr(pt), nt, ptr(L), int(first_block),
                                  ptr(q), int(total_times), ptr(msd), ptr(m4d), ptr(fs), ptr(count)), None,
          "gdb_calc_dynamics")
    return msd, m4d, fs, count


def sq_compute(r, box, n_vectors, ff=None):
    r = f32(r)
    n = r.shape[0]
    nv = i32(n_vectors)
    L = f32(box, (3,))
    re, im = np.zeros(len(nv)), np.zeros(len(nv))
    ffa = f32(ff, (n,)) if ff is not None else None
    check(lib().gdb_sq_compute(int(n), ptr(r), ptr(ffa), ptr(L), int(len(nv)), ptr(nv), ptr(re), ptr(im)), None,
          "gdb_sq_compute")
    return re + 1j * im


class BatchHandle:
    """Owner of one gdb_batch handle: several Sim handles advanced together."""

    def __init__(self, sims, particles_per_cta=0, clg_particles_per_cta=0, clg_tp=0):
        self.sims = list(sims)
        arr = (ctypes.c_void_p * len(self.sims))(*[s.h.value for s in self.sims])
        self.h = ctypes.c_void_p()
        rc = lib().gdb_batch_create_ex(arr, len(self.sims), int(particles_per_cta), int(clg_particles_per_cta),
                                       int(clg_tp), ctypes.byref(self.h))
        if rc != GDB_OK:
            buf = ctypes.create_string_buffer(512)
            lib().gdb_batch_get_last_error(None, buf, 512)
            raise GdbError(rc, f"gdb_batch_create: {buf.value.decode(errors='replace')}")

    def run(self, time_zero, steps):
        ms = ctypes.c_float(0.0)
        rc = lib().gdb_batch_run(self.h, float(time_zero), int(steps), ctypes.byref(ms))
        if rc != GDB_OK:
            buf = ctypes.create_string_buffer(512)
            lib().gdb_batch_get_last_error(self.h, buf, 512)
            raise GdbError(rc, f"gdb_batch_run: {buf.value.decode(errors='replace')}")
        return ms.value

    def __del__(self):
        try:
            if self.h:
                lib().gdb_batch_destroy(self.h)
                self.h = ctypes.c_void_p()
        except Exception:
            pass
