"""Generator of the fixture numba_contraction.json: does numba.cuda (the
compiler gamdpy's kernels go through) fuse ``dist_sq = dist_sq + dr_k * dr_k``
into a multiply-add on this GPU?  The library's default distance form
(fused accumulation, GDB_NBLIST_FMA=1) rests on the answer recorded there.

gamdpy computes neighbour distances with that accumulation
(gamdpy/simulation_boxes/orthorhombic.py:59-73) and numba passes no ``fma``
option to libNVVM unless fastmath is requested, so libNVVM's default decides.
This script compiles an independent numba.cuda kernel with the same
expression on random inputs and counts how often its results equal the
unfused and the fused float32 evaluation.  It runs on a GPU machine; the
result it prints is recorded in numba_contraction.json beside it.

    python tests/golden/make_numba_contraction.py [out.json]
"""
import json
import sys

import numba
import numpy as np
from numba import cuda


@cuda.jit
def dist_kernel(a, b, L, out):
    i = cuda.grid(1)
    if i < a.shape[0]:
        dist_sq = numba.float32(0.0)
        for k in range(3):
            d = a[i, k] - b[i, k]
            box_k = L[k]
            d += (-box_k if numba.float32(2.0) * d > +box_k else
                  (+box_k if numba.float32(2.0) * d < -box_k else numba.float32(0.0)))
            dist_sq = dist_sq + d * d
        out[i] = dist_sq


def host_forms(a, b, L):
    d = (a - b).astype(np.float32)
    d = np.where(2 * d > L, d - L, np.where(2 * d < -L, d + L, d)).astype(np.float32)
    unfused = np.float32(0)
    unfused = (d[:, 0] * d[:, 0]).astype(np.float32)
    unfused = (unfused + (d[:, 1] * d[:, 1]).astype(np.float32)).astype(np.float32)
    unfused = (unfused + (d[:, 2] * d[:, 2]).astype(np.float32)).astype(np.float32)
    # fused: round(d*d + acc) once; float32 products are exact in float128/long double
    ld = np.longdouble
    fused = (d[:, 0] * d[:, 0]).astype(np.float32)
    fused = (d[:, 1].astype(ld) * d[:, 1].astype(ld) + fused.astype(ld)).astype(np.float32)
    fused = (d[:, 2].astype(ld) * d[:, 2].astype(ld) + fused.astype(ld)).astype(np.float32)
    return unfused, fused


def main():
    rng = np.random.default_rng(0)
    n = 1 << 20
    L = np.array([12.8156, 12.8156, 12.8156], np.float32)
    a = rng.uniform(-L / 2, L / 2, (n, 3)).astype(np.float32)
    b = (a + rng.uniform(-3, 3, (n, 3))).astype(np.float32)
    out = np.zeros(n, np.float32)
    dist_kernel[(n + 255) // 256, 256](cuda.to_device(a), cuda.to_device(b), cuda.to_device(L), out)
    unfused, fused = host_forms(a, b, L)
    res = {
        "numba": numba.__version__,
        "device": cuda.get_current_device().name.decode() if isinstance(cuda.get_current_device().name, bytes)
        else str(cuda.get_current_device().name),
        "cc": list(cuda.get_current_device().compute_capability),
        "samples": n,
        "equal_unfused": int(np.sum(out == unfused)),
        "equal_fused": int(np.sum(out == fused)),
        "forms_differ": int(np.sum(unfused != fused)),
    }
    res["verdict"] = "fused" if res["equal_fused"] > res["equal_unfused"] else "unfused"
    print(json.dumps(res))
    if len(sys.argv) > 1:
        with open(sys.argv[1], "w") as f:
            json.dump(res, f, indent=1)


if __name__ == "__main__":
    main()
