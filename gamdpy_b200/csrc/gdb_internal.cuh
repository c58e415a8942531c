// gdb_internal.cuh -- device data layout and helpers shared by the kernels of
// libgamdb200.so (sm_100a).
//
// Device layout of one simulation (all arrays in internal particle order,
// which is cell order after a cell-list rebuild, user order in N^2 mode):
//   pos[2]  float4 (x, y, z, type bits)   ping-pong: a step reads pos[cur] and
//                                          writes pos[cur^1]
//   vel     float4 (vx, vy, vz, mass)
//   img     int4   (image counters, w unused)
//   frc     float4 (fx, fy, fz, 0)         written by force-only evaluations
//   rref    float4 positions at the last neighbour-list build
//   orig    int    user index of each slot
//   nbl     int    neighbour list in chunks of four: entry k of particle i lives
//                  at (k / 4) * (stride * 4) + i * 4 + (k % 4); one int4 load
//                  gives four neighbours, a warp reads 512 contiguous bytes
//   nbc     int    neighbour counts
//   pscal   float  per-particle U, W, lapU, K, Fsq (5 planes of n)
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#define GDB_MAX_TYPES 8
#define GDB_BLOCK 256

namespace gdb {

// Pair potential of one type pair in a form shared by both LJ flavours:
//   x6 = (c / r^2)^3, x12 = x6^2
//   u   = cu12 x12 + cu6 x6                 (- uc [+ sc*cut*(r-cut)] by cutoff)
//   s   = (cs12 x12 + cs6 x6) / r^2         (- sc for shifted force)
//   umm = (cm12 x12 + cm6 x6) / r^2
// LJ_12_6_sigma_epsilon (potential_functions/LJ_12_6_sigma_epsilon.py:26-36):
//   c = sigma^2, cu = 4eps(1, -1), cs = 24eps(2, -1), cm = 24eps(26, -7)
// LJ_12_6 (potential_functions/LJ_12_6.py:34-41):
//   c = 1, cu = (A12, A6), cs = (12 A12, 6 A6), cm = (156 A12, 42 A6)
struct PairEntry {
    float c, cu12, cu6, cs12, cs6, cm12, cm6;
    float cut, cut2;
    float uc;   // u(cut)
    float sc;   // s(cut), subtracted from s for shifted force (else 0)
    float sccut;  // s(cut)*cut for the shifted-force energy term (else 0)
};

struct PairTable {
    int nt;
    int cutmode;  // 0 shifted force, 1 shifted potential
    PairEntry e[GDB_MAX_TYPES * GDB_MAX_TYPES];
};

// Device control block (one per simulation).
struct DevCtrl {
    int rebuild;       // 1 = neighbour list must be rebuilt before the next force evaluation
    int rebuild_next;  // set during a persistent step, promoted to `rebuild` at the barrier
    int cell_wrap;     // a coordinate sat exactly on +L/2 (binned to cell 0 by the modulo)
    int maxcount;      // largest neighbour count of the last build
    int nrebuild;      // number of builds (gamdpy nbflag[2])
    unsigned status;   // GDB_STATUS_* bits
    int step;          // step index within the running timeblock
    unsigned ticket;   // last-block counter of the step kernel
    unsigned ticket2;  // last-block counter of rebuild kernels
    int pending[2];    // momentum shift pending, by step parity
    float shift[2][4]; // momentum shift vector, by step parity
    float xi;          // Nose-Hoover friction (NVT.thermostat_state[0])
    float npt_ts0;     // NPT_Atomic: thermostat state p_xi/Q
    float npt_bs0;     // NPT_Atomic: barostat state p_eps/W
    float npt_vol;     // NPT_Atomic: volume (barostat_state[2])
    float box[3];      // current box lengths (changed by NPT_Atomic steps)
    float sumK;        // last kinetic-energy sum (float copy, NVT.thermostat_state[1] analogue)
    double time_zero;  // simulated time at the start of the timeblock
    double evalU, evalW;  // sums of the last force-only evaluation
    unsigned bar_count;   // grid barrier of the persistent kernel: top-level arrivals
    unsigned bar_gen;
    unsigned bar_group[64];  // arrivals per group of 16 blocks (grids up to 1024 blocks)
    unsigned bar_all[3];  // step barrier where every block keeps the books: arrivals, by barrier index mod 3
    int abort;            // set when a barrier wait timed out
    unsigned work[2];     // persistent step: next round to hand out, by step parity
    long long bar_timeout;  // grid-barrier wait limit in SM clock cycles (0: the default, ~1 s)
    unsigned long long *trace;  // optional phase trace: (tag << 56) | globaltimer ns
    int trace_cap;
    int trace_len;
};

// Phase trace (block 0, thread 0 of the persistent kernel): one entry per
// barrier with a tag naming the phase that just finished.
enum TraceTag {
    TR_STEP = 1,
    TR_EVAL = 2,
    TR_REBUILD_PHASE = 3,
    TR_REBUILD_DONE = 4,
    TR_START = 5,
    TR_STEP_PHASE = 6,
    TR_BAR_LAST_IN = 7,  // the last block to arrive at a grid barrier, before its bookkeeping
    TR_BAR_RELEASE = 8   // the same block, releasing the others
};

// Entry by the last block of a grid barrier (any block index): the slot is
// taken atomically, as block 0 writes its own entries meanwhile.
__device__ __forceinline__ void trace_mark_last(DevCtrl *c, int tag) {
    if (c->trace && threadIdx.x == 0) {
        unsigned long long t;
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
        const int k = atomicAdd(&c->trace_len, 1);
        if (k < c->trace_cap) c->trace[k] = ((unsigned long long)tag << 56) | (t & 0x00ffffffffffffffULL);
    }
}

__device__ __forceinline__ void trace_mark(DevCtrl *c, int tag) {
    if (c->trace && blockIdx.x == 0 && threadIdx.x == 0) {
        unsigned long long t;
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
        const int k = atomicAdd(&c->trace_len, 1);
        if (k < c->trace_cap) c->trace[k] = ((unsigned long long)tag << 56) | (t & 0x00ffffffffffffffULL);
    }
}

// Minimum-image displacement of one component exactly as
// simulation_boxes/orthorhombic.py:50-53 (float32: 2*dr compared with +-L).
__device__ __forceinline__ float mic(float d, float L) {
    float t = __fmul_rn(2.0f, d);
    return (t > L) ? __fsub_rn(d, L) : ((t < -L) ? __fadd_rn(d, L) : d);
}

// Squared distance for neighbour-list decisions, IEEE-exact in a fixed
// evaluation order (orthorhombic.py:59-73, ri = other, rj = self).  FMA selects
// the fused accumulation dist_sq = fma(dr, dr, dist_sq) that libNVVM's default
// contraction gives the reference's numba.cuda build; otherwise the product
// is rounded first (the reference's CPU build).
template <bool FMA>
__device__ __forceinline__ float dist_sq_exact(float4 a, float4 b, float Lx, float Ly, float Lz) {
    float dx = mic(__fsub_rn(a.x, b.x), Lx);
    float dy = mic(__fsub_rn(a.y, b.y), Ly);
    float dz = mic(__fsub_rn(a.z, b.z), Lz);
    float s;
    if (FMA) {
        s = __fmul_rn(dx, dx);
        s = __fmaf_rn(dy, dy, s);
        s = __fmaf_rn(dz, dz, s);
    } else {
        s = __fmul_rn(dx, dx);
        s = __fadd_rn(s, __fmul_rn(dy, dy));
        s = __fadd_rn(s, __fmul_rn(dz, dz));
    }
    return s;
}

__device__ __forceinline__ int ptype_of(float4 p) { return __float_as_int(p.w); }

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Sum of NQ doubles over the block (blockDim.x == GDB_BLOCK); result valid
// in thread 0.  Fixed reduction tree: deterministic.
template <int NQ>
__device__ __forceinline__ void block_sum(double (&v)[NQ], double *smem /* NQ * 32 */) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < NQ; q++) v[q] = warp_sum(v[q]);
    if (lane == 0) {
#pragma unroll
        for (int q = 0; q < NQ; q++) smem[q * 32 + warp] = v[q];
    }
    __syncthreads();
    if (warp == 0) {
        const int nw = blockDim.x >> 5;
#pragma unroll
        for (int q = 0; q < NQ; q++) {
            double x = lane < nw ? smem[q * 32 + lane] : 0.0;
            v[q] = warp_sum(x);
        }
    }
    __syncthreads();
}

// Temporaries of the library's calls (staging copies, cell-sort scratch,
// result buffers) come from a stream-ordered pool per device that the library
// owns and that keeps up to 1 GiB mapped between calls; the default pool
// hands its memory back to the driver at every synchronisation, and mapping a
// few hundred MB again costs tens of ms per call.  Free with cudaFreeAsync.
cudaError_t pool_alloc_raw(void **p, size_t bytes, cudaStream_t st);
template <class T>
inline cudaError_t pool_alloc(T **p, size_t bytes, cudaStream_t st) {
    return pool_alloc_raw((void **)p, bytes, st);
}

}  // namespace gdb

// Host-side helpers shared by the translation units.
struct gdb_error_sink {
    char msg[512];
};
