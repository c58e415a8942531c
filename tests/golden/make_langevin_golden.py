"""Golden vectors of the random numbers of gamdpy's NVT_Langevin integrator.

integrators/NVT_Langevin.py:48 creates its per-particle generators with
numba.cuda.random.create_xoroshiro128p_states(N, seed) and :105 draws
xoroshiro128p_normal_float32.  Both come from numba (0.65.0 here), which
initialises the states on the CPU (init_xoroshiro128p_states_cpu) and whose
generator functions also run on the CPU; this script records them:

  states_s0, states_s1   the 64 initial states for seed 2024
  next_u64               the first 8 raw outputs of states 0, 1 and 63
  normals                the first 12 normal float32 draws of every state

Run from the repository root:  python tests/golden/make_langevin_golden.py
"""
import os

import numpy as np
import numba.cuda.random as R

N, SEED = 64, 2024


def main():
    st = np.empty(N, dtype=R.xoroshiro128p_dtype)
    R.init_xoroshiro128p_states_cpu(st, SEED, 0)
    s0, s1 = st["s0"].copy(), st["s1"].copy()
    raw = np.empty(N, dtype=R.xoroshiro128p_dtype)
    raw[:] = st
    nxt = np.array([[R.xoroshiro128p_next(raw, i) for _ in range(8)] for i in (0, 1, N - 1)], np.uint64)
    normals = np.array([[R.xoroshiro128p_normal_float32(st, i) for _ in range(12)] for i in range(N)], np.float32)
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "langevin_rng.npz")
    np.savez(out, seed=np.uint64(SEED), states_s0=s0, states_s1=s1, next_u64=nxt, next_index=np.array([0, 1, N - 1]),
             normals=normals)
    print("wrote", out)


if __name__ == "__main__":
    main()
