"""gdb_sq_compute_noalloc: S(q) for callers that cannot let the library
allocate device memory (their own allocator or pool owns the GPU, or they run
under a hard memory budget).  Checked against the allocating entry point
gdb_sq_compute on the same inputs, on two calls in a row (the shared scratch
array must be cleared between calls).  Collected last on purpose."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_noalloc_sq_matches_allocating_entry_point():
    import torch

    from gamdpy_b200 import _lib

    L = _lib.lib()
    rng = np.random.default_rng(42)
    n, nq, n_max = 3000, 700, 10
    box = np.array([14.0, 14.0, 15.5], np.float32)
    r = ((rng.random((n, 3)) - 0.5) * box).astype(np.float32)
    ff = rng.uniform(0.5, 1.5, n).astype(np.float32)
    nv = rng.integers(-n_max, n_max + 1, size=(nq, 3)).astype(np.int32)
    ref = _lib.sq_compute(r, box, nv, ff)

    dev = torch.device("cuda", 0)
    r_d = torch.from_numpy(r).to(dev)
    ff_d = torch.from_numpy(ff).to(dev)
    nv_d = torch.from_numpy(nv).to(dev)
    re_d = torch.empty(nq, dtype=torch.float64, device=dev)
    im_d = torch.empty(nq, dtype=torch.float64, device=dev)
    scale = np.abs(ref).max()
    for _ in range(2):
        re_d.fill_(float("nan"))
        im_d.fill_(float("nan"))
        torch.cuda.synchronize()
        rc = L.gdb_sq_compute_noalloc(n, ctypes.c_void_p(r_d.data_ptr()), ctypes.c_void_p(ff_d.data_ptr()),
                                      box.ctypes.data_as(ctypes.c_void_p), nq, ctypes.c_void_p(nv_d.data_ptr()),
                                      n_max, ctypes.c_void_p(re_d.data_ptr()), ctypes.c_void_p(im_d.data_ptr()),
                                      None)
        assert rc == 0, _lib.last_error()
        got = re_d.cpu().numpy() + 1j * im_d.cpu().numpy()
        assert np.abs(got - ref).max() <= 1e-9 * scale

    # limits are rejected with an error, not run
    rc = L.gdb_sq_compute_noalloc(n, ctypes.c_void_p(r_d.data_ptr()), None, box.ctypes.data_as(ctypes.c_void_p),
                                  70000, ctypes.c_void_p(nv_d.data_ptr()), n_max, ctypes.c_void_p(re_d.data_ptr()),
                                  ctypes.c_void_p(im_d.data_ptr()), None)
    assert rc == _lib.GDB_ERR_ARG and "65536" in _lib.last_error()
