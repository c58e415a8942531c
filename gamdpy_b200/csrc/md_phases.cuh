// md_phases.cuh -- device phases of one MD time step, and the kernels that
// run them.
//
// Every phase is a grid-stride device function over its items (particles,
// cells, chunks), so the same code runs
//   * as one standalone kernel per phase, launched in a CUDA graph (large N), and
//   * inside k_run, a persistent cooperative kernel that advances a whole
//     chunk of steps, rebuilds included, with a bounded grid barrier between
//     phases (gamdpy's gridsync mode, simulation/Simulation.py:306-328).
//
// Data written inside k_run by one block and read by another (positions,
// neighbour lists, cell tables) is read with ordinary coherent loads; the
// non-coherent read-only path (__ldg) is used only by the standalone kernels,
// where kernel boundaries order the accesses.
#pragma once

#include "../../include/gamdb200.h"
#include "gdb_internal.cuh"

namespace gdb {

constexpr int NQ = 9;  // block reductions: K, U, W, lapU, Fsq, px, py, pz, m
constexpr int SCAN_CHUNK = 2048;
constexpr int MODE_STEP = 0;
constexpr int MODE_EVAL = 1;
constexpr int NB_CHUNK = 4;  // neighbour indices stored and loaded 4 at a time (int4)

// Neighbour list layout: entry k of particle i at
//   (k / 4) * (stride * 4) + i * 4 + (k % 4)
// so one int4 load gives four consecutive neighbours of a particle and a warp
// of consecutive particles reads 512 contiguous bytes.
__device__ __forceinline__ size_t nbl_index(int i, int k, int stride) {
    return (size_t)(k >> 2) * ((size_t)stride * NB_CHUNK) + (size_t)i * NB_CHUNK + (k & 3);
}

struct SimArgs {
    float4 *pos0, *pos1;  // ping-pong position buffers
    float4 *vel;
    int4 *img;
    float4 *rref;
    float4 *frc;
    float4 *pos_tmp, *vel_tmp;
    int4 *img_tmp;
    int *orig, *orig_tmp;
    int *nbl, *nbc;
    float *pscal, *pscal_tmp;  // 5 planes of n: U, W, lapU, K, Fsq
    int *cell_count, *cell_start, *pcell, *prank, *perm, *scell, *bsum;
    double *partials, *rows;
    float *conf;
    float *conf_box;  // ConfigurationSaver: the box of each frame (4 floats a frame)
    DevCtrl *ctrl;
    int n, stride, max_nbs;
    int ncell, nchunks, ncx, ncy, ncz;
    int nbx, nby, nbz;  // bricks per dimension (staged-halo path, md_bricks.cuh), 0: cells x fastest
    int brick_hcap;     // staged positions a brick's halo may hold (<= BRICK_HCAP)
    int nb_kind, fma;
    int nsq_smem;  // persistent N^2 build stages all positions in dynamic shared memory
    int bar_all;   // persistent grid: every block keeps the step's books (grids of <= BAR_FLAT_MAX blocks)
    float Lx, Ly, Lz;
    float cps2;    // (max_cut + skin)^2, nblist.py:152
    float skin2q;  // skin*skin*0.25, orthorhombic.py:131
    float dt, omega2;
    long long dof;  // N*D - D (NVT.py:35)
    int tfunc;
    float tp0, tp1, tp2, tp3;
    // NPT_Atomic: masses without the temperature factor, target pressure
    // function, and the cell grid the box may use (recomputed per build)
    float npt_mass_t, npt_mass_p;
    int pfunc;
    float pp0, pp1, pp2, pp3;
    float min_cell;
    int ncx_max, ncy_max, ncz_max;
    int every, reset_every, nrows, conf_per_block;
    // NVT_Langevin: generator (s0, s1) and previous random force per user index
    ulonglong2 *rng;
    float4 *lbeta;
    float alpha;
    // molecules: pair exclusions and harmonic bonds, by user index
    const int *excl;          // (n, max_excl + 1), count last; NULL: no exclusions
    int max_excl;
    const int *bond_cnt;      // bonds of each particle; NULL: no bonds
    const int *bond_j;        // partner (user index), (n, bond_max)
    const int *bond_t;        // bond type, (n, bond_max)
    const float2 *bond_prm;   // (r0, k) per bond type
    int bond_max;
    int *slot_of;             // slot of each user index, kept by the cell sort (bonds)
};

// The pair (ui, uj) of user indices is in ui's exclusion row
// (interactions/nblist.py:120-123, nblist_linked_lists.py:174-178).
__device__ __forceinline__ bool excluded(const SimArgs &a, int ui, int uj) {
    const int *row = a.excl + (size_t)ui * (a.max_excl + 1);
    const int cnt = min(row[a.max_excl], a.max_excl);
    for (int k = 0; k < cnt; k++)
        if (row[k] == uj) return true;
    return false;
}

__device__ __forceinline__ float4 *cur_pos(const SimArgs &a, int cur) { return cur ? a.pos1 : a.pos0; }

// The blocks that share one system's work: the whole grid (standalone and
// persistent kernels) or the CTAs of one thread-block cluster (batched
// systems).  b is this block's index among them, nb their number.
struct Span {
    int b, nb;
};
__device__ __forceinline__ Span grid_span() { return Span{(int)blockIdx.x, (int)gridDim.x}; }

template <bool NC, typename T>
__device__ __forceinline__ T load(const T *p) {
    if (NC) return __ldg(p);
    return *p;
}

// ---------------------------------------------------------------------------
// bounded grid barrier (k_run only; the launch is cooperative, so every block
// is resident).  The last block to arrive runs `last` with the whole block
// before releasing the others.  A wait that exceeds ~1 s of SM clock sets
// GDB_STATUS_BARRIER_TIMEOUT and ctrl->abort; callers return when it fails.
// ---------------------------------------------------------------------------
constexpr long long BARRIER_TIMEOUT_CYCLES = 2000000000LL;

__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned *p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ unsigned atom_add_acq_rel_gpu(unsigned *p, unsigned v) {
    unsigned old;
    asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}
__device__ __forceinline__ void st_release_gpu(unsigned *p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Arrival is an acq_rel add (after a CTA barrier, so the block's writes are
// ordered before it): on one counter for grids of up to BAR_FLAT_MAX blocks,
// hierarchical above (the counter of the block's group of 16, and the last
// of a group adds to the top counter).  The last block to arrive has seen
// every block's writes.  It runs `last`, resets the counters and publishes the
// next generation with a release store; waiters poll it with acquire loads.
constexpr int BAR_GROUP = 16;
constexpr int BAR_FLAT_MAX = 320;

// A block may arrive with a flag (a particle of it moved more than skin/2):
// the arrival adds FLAG_ONE as well, so the last block learns from the
// counter whether any block raised it (*any) without another read.
constexpr unsigned BAR_FLAG_ONE = 1u << 20;  // counts live in the low 20 bits
constexpr unsigned BAR_COUNT_MASK = BAR_FLAG_ONE - 1u;

template <typename F>
__device__ __forceinline__ bool grid_barrier(DevCtrl *c, F last, bool flag = false, int *any = nullptr) {
    __shared__ int s_last, s_ok;
    __syncthreads();
    if (threadIdx.x == 0 && *(volatile int *)&c->abort) {
        // another block gave up: arrive nowhere, leave with the others
        s_last = 0;
        s_ok = 0;
    } else if (threadIdx.x == 0) {
        const unsigned gen = ld_acquire_gpu(&c->bar_gen);
        const unsigned grp = blockIdx.x / BAR_GROUP;
        const unsigned gsize = min((unsigned)BAR_GROUP, gridDim.x - grp * BAR_GROUP);
        const unsigned ngroups = (gridDim.x + BAR_GROUP - 1) / BAR_GROUP;
        bool top = false, raised = false;
        const unsigned inc = 1u | (flag ? BAR_FLAG_ONE : 0u);
        if (gridDim.x <= BAR_FLAT_MAX) {
            const unsigned old = atom_add_acq_rel_gpu(&c->bar_count, inc);
            top = (old & BAR_COUNT_MASK) == gridDim.x - 1;
            raised = ((old + inc) >> 20) != 0u;
        } else {
            const unsigned oldg = atom_add_acq_rel_gpu(&c->bar_group[grp], inc);
            if ((oldg & BAR_COUNT_MASK) == gsize - 1) {
                c->bar_group[grp] = 0;  // no block of this group arrives again before the release
                const unsigned ginc = 1u | (((oldg + inc) >> 20) != 0u ? BAR_FLAG_ONE : 0u);
                const unsigned oldt = atom_add_acq_rel_gpu(&c->bar_count, ginc);
                top = (oldt & BAR_COUNT_MASK) == ngroups - 1;
                raised = ((oldt + ginc) >> 20) != 0u;
            }
        }
        if (top && any) *any = raised;
        s_last = top;
        s_ok = 1;
        if (!s_last) {
            const long long t0 = clock64();
            const long long limit = c->bar_timeout > 0 ? c->bar_timeout : BARRIER_TIMEOUT_CYCLES;
            int polls = 0;
            while (ld_acquire_gpu(&c->bar_gen) == gen) {
                if (*(volatile int *)&c->abort) {
                    s_ok = 0;
                    break;
                }
                if ((++polls & 63) == 0 && clock64() - t0 > limit) {
                    atomicOr(&c->status, GDB_STATUS_BARRIER_TIMEOUT);
                    c->abort = 1;
                    s_ok = 0;
                    break;
                }
                if (polls > 64) __nanosleep(32);
            }
        }
    }
    __syncthreads();
    if (!s_ok) return false;
    if (s_last) {
        trace_mark_last(c, TR_BAR_LAST_IN);
        last();
        __syncthreads();
        if (threadIdx.x == 0) {
            c->bar_count = 0;
            trace_mark_last(c, TR_BAR_RELEASE);
            st_release_gpu(&c->bar_gen, *(volatile unsigned *)&c->bar_gen + 1u);
        }
        __syncthreads();
    }
    return s_ok != 0;
}

// Step barrier of a persistent grid of at most BAR_FLAT_MAX blocks in which
// every block does the step's bookkeeping itself (finalize_step_all): no
// block runs a phase between arrival and departure, so there is no release
// to wait for.  Barrier `seq` (counted from 0 in each launch) counts arrivals
// on bar_all[seq % 3], with the moved flag in the high bits as above; every
// block leaves when the count reaches the grid and reads the same final word.
// Block 0 clears bar_all[(seq + 2) % 3] on its way out: every block has
// arrived here, so none still polls barrier seq - 1, and block 0's arrival at
// barrier seq + 1 orders the clear before any arrival at barrier seq + 2.
// The launch starts with all three words zero.  Same abort and wait limit as
// grid_barrier.
__device__ __forceinline__ bool step_barrier_all(DevCtrl *c, unsigned seq, bool flag, int *any) {
    __shared__ int s_ok2;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1, raised = 0;
        if (*(volatile int *)&c->abort) {
            ok = 0;
        } else {
            unsigned *cnt = &c->bar_all[seq % 3u];
            const unsigned inc = 1u | (flag ? BAR_FLAG_ONE : 0u);
            unsigned v = atom_add_acq_rel_gpu(cnt, inc) + inc;
            const long long t0 = clock64();
            const long long limit = c->bar_timeout > 0 ? c->bar_timeout : BARRIER_TIMEOUT_CYCLES;
            int polls = 0;
            while ((v & BAR_COUNT_MASK) != gridDim.x) {
                if (*(volatile int *)&c->abort) {
                    ok = 0;
                    break;
                }
                if ((++polls & 63) == 0 && clock64() - t0 > limit) {
                    atomicOr(&c->status, GDB_STATUS_BARRIER_TIMEOUT);
                    c->abort = 1;
                    ok = 0;
                    break;
                }
                if (polls > 64) __nanosleep(32);
                v = ld_acquire_gpu(cnt);
            }
            raised = (v >> 20) != 0u;
            if (ok && blockIdx.x == 0) c->bar_all[(seq + 2u) % 3u] = 0u;
        }
        *any = raised;
        s_ok2 = ok;
    }
    __syncthreads();
    return s_ok2 != 0;
}

// ---------------------------------------------------------------------------
// neighbour-list phases
// ---------------------------------------------------------------------------

// One pass of the N^2 candidate walk of a warp: lanes test candidates
// j0 + 32u + lane (u < 4, loaded before they are tested) against particle i0
// and, with TWO, i1; hits are appended in ascending j by ballot + popc.  CHECK
// (the last, partial pass only) masks candidates j >= n.  The tests are
// combined without short-circuit branches: the distance is cheap and pure.
template <bool B>
struct BoolTag {
    static constexpr bool value = B;
};

struct NsqWalk {
    const float4 *pos, *src;
    int n, max_nbs;
    size_t cstride;  // stride * NB_CHUNK: entries k and k + 4 of a particle
    float Lx, Ly, Lz, cps2;
    const int *excl, *orig;
    int *nbl;
    int lane;
    unsigned below;
};
template <bool FMA, bool NC, bool TWO, bool CHECK>
__device__ __forceinline__ void nsq_pass(const SimArgs &a, const NsqWalk &w, int j0, int i0, int i1, float4 p0,
                                         float4 p1, int u0, int u1, int &c0, int &c1) {
    float4 q[4];
#pragma unroll
    for (int u = 0; u < 4; u++) {
        const int j = j0 + 32 * u + w.lane;
        // one load kind per instantiation: the read-only path for the
        // standalone kernel (never staged), plain loads from the staged copy
        // or the coherent buffer otherwise
        q[u] = (!CHECK || j < w.n) ? (NC ? load<true>(w.pos + j) : w.src[j]) : p0;
    }
#pragma unroll
    for (int u = 0; u < 4; u++) {
        const int j = j0 + 32 * u + w.lane;
        const bool in = !CHECK || j < w.n;
        bool h0 = in & (j != i0) & (dist_sq_exact<FMA>(q[u], p0, w.Lx, w.Ly, w.Lz) < w.cps2);
        bool h1 = false;
        if (TWO) h1 = in & (j != i1) & (dist_sq_exact<FMA>(q[u], p1, w.Lx, w.Ly, w.Lz) < w.cps2);
        if (w.excl) {
            if (h0) h0 = !excluded(a, u0, w.orig[j]);
            if (TWO && h1) h1 = !excluded(a, u1, w.orig[j]);
        }
        const unsigned m0 = __ballot_sync(0xffffffffu, h0);
        if (h0) {
            const int k = c0 + __popc(m0 & w.below);
            if (k < w.max_nbs) w.nbl[(size_t)(k >> 2) * w.cstride + (size_t)i0 * NB_CHUNK + (k & 3)] = j;
        }
        c0 += __popc(m0);
        if (TWO) {
            const unsigned m1 = __ballot_sync(0xffffffffu, h1);
            if (h1) {
                const int k = c1 + __popc(m1 & w.below);
                if (k < w.max_nbs) w.nbl[(size_t)(k >> 2) * w.cstride + (size_t)i1 * NB_CHUNK + (k & 3)] = j;
            }
            c1 += __popc(m1);
        }
    }
}

// N^2 build (interactions/nblist.py:88-143): a warp per particle, lanes
// stride over j, ballot + popc append hits in ascending j (deterministic).
// A warp takes its particles two at a time (i and i + the number of warps):
// every candidate is loaded once for both, and the two append chains are
// independent.  Whether a warp has a second particle is uniform over the
// warp, so the walk is instantiated for one and for two particles, and the
// full passes skip the j < n test of the last one.  With `spos` (shared
// memory for all n positions) the block first copies the positions there,
// so the candidate loads are shared-memory loads.
template <bool FMA, bool NC>
__device__ inline void phase_nbl_nsq(const SimArgs &a, int cur, Span g = grid_span(), float4 *spos = nullptr) {
    const float4 *pos = cur_pos(a, cur);
    const float4 *src = pos;
    if (spos) {
        // eight loads in flight per thread before they are stored
        const int bd = blockDim.x;
        for (int k0 = threadIdx.x; k0 < a.n; k0 += 8 * bd) {
            float4 t[8];
#pragma unroll
            for (int u = 0; u < 8; u++)
                if (k0 + u * bd < a.n) t[u] = pos[k0 + u * bd];
#pragma unroll
            for (int u = 0; u < 8; u++)
                if (k0 + u * bd < a.n) spos[k0 + u * bd] = t[u];
        }
        __syncthreads();
        src = spos;
        trace_mark(a.ctrl, TR_REBUILD_PHASE);
    }
    // the arguments the loop reads, in registers: the list stores could
    // otherwise force them to be reloaded after every store
    NsqWalk w;
    w.pos = pos;
    w.src = src;
    w.n = a.n;
    w.max_nbs = a.max_nbs;
    w.cstride = (size_t)a.stride * NB_CHUNK;
    w.Lx = a.Lx;
    w.Ly = a.Ly;
    w.Lz = a.Lz;
    w.cps2 = a.cps2;
    w.excl = a.excl;
    w.orig = a.orig;
    w.nbl = a.nbl;
    w.lane = threadIdx.x & 31;
    w.below = (1u << w.lane) - 1u;
    const int n = w.n;
    const int nfull = n & ~127;  // candidates covered by full passes
    const int warps = (g.nb * (int)blockDim.x) >> 5;
    for (int i0 = (g.b * (int)blockDim.x + (int)threadIdx.x) >> 5; i0 < n; i0 += 2 * warps) {
        const int i1 = i0 + warps;
        const bool has1 = i1 < n;  // the same for every lane of the warp
        const float4 p0 = NC ? load<true>(pos + i0) : src[i0];
        const float4 p1 = has1 ? (NC ? load<true>(pos + i1) : src[i1]) : p0;
        const int u0 = w.excl ? w.orig[i0] : 0, u1 = (w.excl && has1) ? w.orig[i1] : 0;
        int c0 = 0, c1 = 0;
        if (has1) {
            int j0 = 0;
            for (; j0 < nfull; j0 += 128) nsq_pass<FMA, NC, true, false>(a, w, j0, i0, i1, p0, p1, u0, u1, c0, c1);
            if (j0 < n) nsq_pass<FMA, NC, true, true>(a, w, j0, i0, i1, p0, p1, u0, u1, c0, c1);
        } else {
            int j0 = 0;
            for (; j0 < nfull; j0 += 128) nsq_pass<FMA, NC, false, false>(a, w, j0, i0, i1, p0, p1, u0, u1, c0, c1);
            if (j0 < n) nsq_pass<FMA, NC, false, true>(a, w, j0, i0, i1, p0, p1, u0, u1, c0, c1);
        }
        if (w.lane == 0) {
            a.nbc[i0] = c0;
            a.rref[i0] = p0;
            atomicMax(&a.ctrl->maxcount, c0);
            if (has1) {
                a.nbc[i1] = c1;
                a.rref[i1] = p1;
                atomicMax(&a.ctrl->maxcount, c1);
            }
        }
    }
}

// Cell coordinate as nblist_linked_lists.py:127 (float64, Python modulo);
// non-finite coordinates map to cell 0 and raise the NAN bit.
__device__ __forceinline__ int cell_coord(float x, float L, int nc, DevCtrl *ctrl) {
    const double v = ((double)x + 0.5 * (double)L) * (double)nc / (double)L;
    if (!(v > -1e9 && v < 1e9)) {
        atomicOr(&ctrl->status, GDB_STATUS_NAN);
        return 0;
    }
    const long long c = (long long)floor(v);
    long long m = c % nc;
    if (m < 0) m += nc;
    // outside [0, nc) only for a coordinate on the box face (or beyond it):
    // the build then uses the general minimum-image test
    if (c != m) ctrl->cell_wrap = 1;
    return (int)m;
}

template <bool NC>
__device__ inline void phase_cell_assign(const SimArgs &a, int cur, Span g = grid_span()) {
    const float4 *pos = cur_pos(a, cur);
    for (int i = g.b * (int)blockDim.x + (int)threadIdx.x; i < a.n; i += g.nb * (int)blockDim.x) {
        const float4 p = load<NC>(pos + i);
        const int cx = cell_coord(p.x, a.Lx, a.ncx, a.ctrl);
        const int cy = cell_coord(p.y, a.Ly, a.ncy, a.ctrl);
        const int cz = cell_coord(p.z, a.Lz, a.ncz, a.ctrl);
        // x fastest over the grid, or brick by brick (bricks of 4 x 4 x 4 cells)
        const int c = a.nbx ? ((((cz >> 2) * a.nby + (cy >> 2)) * a.nbx + (cx >> 2)) << 6) |
                                  ((((cz & 3) << 2) | (cy & 3)) << 2) | (cx & 3)
                            : (cz * a.ncy + cy) * a.ncx + cx;
        a.pcell[i] = c;
        a.prank[i] = atomicAdd(&a.cell_count[c], 1);
    }
}

// Block-wide exclusive scan of SCAN_CHUNK ints (ceil(SCAN_CHUNK / blockDim)
// per thread: 8 for 256 or 288 threads, 2 for 1024; threads past the chunk
// hold nothing).
__device__ __forceinline__ void chunk_scan(const int *in, int len, int base, int *out_excl, int add, int *total,
                                           int *sm /* 32 */) {
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int ept = (SCAN_CHUNK + (int)blockDim.x - 1) / (int)blockDim.x;
    int v[8];
    int s = 0;
#pragma unroll
    for (int q = 0; q < 8; q++) {
        const int idx = base + t * ept + q;
        v[q] = (q < ept && t * ept + q < SCAN_CHUNK && idx < len) ? in[idx] : 0;
        s += v[q];
    }
    int incl = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) sm[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        const int w = lane < (int)(blockDim.x >> 5) ? sm[lane] : 0;
        int wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += y;
        }
        sm[lane] = wi - w;
        if (lane == 31 && total) *total = wi;
    }
    __syncthreads();
    if (out_excl) {
        int run = add + sm[warp] + incl - s;
#pragma unroll
        for (int q = 0; q < 8; q++) {
            const int idx = base + t * ept + q;
            if (q < ept && t * ept + q < SCAN_CHUNK && idx < len) out_excl[idx] = run;
            run += v[q];
        }
    }
    __syncthreads();
}

__device__ inline void phase_scan_partial(const SimArgs &a, Span g = grid_span()) {
    __shared__ int sm[32];
    __shared__ int tot;
    for (int c = g.b; c < a.nchunks; c += g.nb) {
        chunk_scan(a.cell_count, a.ncell, c * SCAN_CHUNK, nullptr, 0, &tot, sm);
        if (threadIdx.x == 0) a.bsum[c] = tot;
        __syncthreads();
    }
}

// exclusive scan of the chunk sums, by one block
__device__ inline void block_scan_chunks(const SimArgs &a) {
    __shared__ int sm[32];
    __shared__ int tot;
    int carry = 0;
    for (int base = 0; base < a.nchunks; base += SCAN_CHUNK) {
        chunk_scan(a.bsum, a.nchunks, base, a.bsum, carry, &tot, sm);
        carry += tot;
        __syncthreads();
    }
}

__device__ inline void phase_scan_final(const SimArgs &a, Span g = grid_span()) {
    __shared__ int sm[32];
    for (int c = g.b; c < a.nchunks; c += g.nb)
        chunk_scan(a.cell_count, a.ncell, c * SCAN_CHUNK, a.cell_start, a.bsum[c], nullptr, sm);
    if (g.b == 0 && threadIdx.x == 0) a.cell_start[a.ncell] = a.n;
}

__device__ inline void phase_scatter(const SimArgs &a, Span g = grid_span()) {
    for (int i = g.b * (int)blockDim.x + (int)threadIdx.x; i < a.n; i += g.nb * (int)blockDim.x) {
        const int slot = a.cell_start[a.pcell[i]] + a.prank[i];
        if ((unsigned)slot < (unsigned)a.n)
            a.perm[slot] = i;
        else
            atomicOr(&a.ctrl->status, GDB_STATUS_BAD_INDEX);
    }
}

// Order every cell's particles by user index: the atomics of the assignment
// rank them arbitrarily; this makes the layout and every sum deterministic.
__device__ inline void phase_sort_cells(const SimArgs &a, Span g = grid_span()) {
    for (int c = g.b * (int)blockDim.x + (int)threadIdx.x; c < a.ncell; c += g.nb * (int)blockDim.x) {
        const int lo = a.cell_start[c], hi = a.cell_start[c + 1];
        for (int x = lo + 1; x < hi; x++) {
            const int v = a.perm[x];
            const int key = a.orig[v];
            int y = x - 1;
            while (y >= lo && a.orig[a.perm[y]] > key) {
                a.perm[y + 1] = a.perm[y];
                y--;
            }
            a.perm[y + 1] = v;
        }
    }
}

__device__ inline void phase_gather(const SimArgs &a, int cur, Span g = grid_span()) {
    const float4 *pos = cur_pos(a, cur);
    const size_t n = a.n;
    for (int s = g.b * (int)blockDim.x + (int)threadIdx.x; s < a.n; s += g.nb * (int)blockDim.x) {
        int i = a.perm[s];
        if ((unsigned)i >= (unsigned)a.n) {
            atomicOr(&a.ctrl->status, GDB_STATUS_BAD_INDEX);
            i = s;
        }
        a.pos_tmp[s] = pos[i];
        a.vel_tmp[s] = a.vel[i];
        a.img_tmp[s] = a.img[i];
        a.orig_tmp[s] = a.orig[i];
        a.scell[s] = a.pcell[i];
        // K and Fsq travel with the particle; U, W, lapU are rewritten by the
        // next force evaluation
        a.pscal_tmp[3 * n + s] = a.pscal[3 * n + i];
        a.pscal_tmp[4 * n + s] = a.pscal[4 * n + i];
    }
}

// Exact squared distance with a known periodic shift per component: the
// reference computes d = rj - ri, then d += -L / +L / 0 from 2d vs L
// (orthorhombic.py:59-73).  When the shift is known in advance the result is
// __fadd_rn(__fsub_rn(rj, ri), shift), bit for bit.
template <bool FMA>
__device__ __forceinline__ float dist_sq_shifted(float4 pj, float4 pi, float sx, float sy, float sz) {
    const float dx = __fadd_rn(__fsub_rn(pj.x, pi.x), sx);
    const float dy = __fadd_rn(__fsub_rn(pj.y, pi.y), sy);
    const float dz = __fadd_rn(__fsub_rn(pj.z, pi.z), sz);
    float s = __fmul_rn(dx, dx);
    if (FMA) {
        s = __fmaf_rn(dy, dy, s);
        s = __fmaf_rn(dz, dz, s);
    } else {
        s = __fadd_rn(s, __fmul_rn(dy, dy));
        s = __fadd_rn(s, __fmul_rn(dz, dz));
    }
    return s;
}

// Cell-list build (nblist_linked_lists.py:133-183 semantics: all particles of
// the 5x5x5 stencil with dist_sq < (max_cut+skin)^2, j != i).  One warp per
// cell: the cell's particles share the stencil.  Slots are sorted by cell
// with x fastest, so the five x-cells of one (dy, dz) row are one contiguous
// slot range (two at the x wrap); the warp lists the <= 50 ranges with their
// prefix sums in shared memory and walks the packed candidate sequence 64 at
// a time, testing each candidate against up to NBW particles of the cell held
// in registers.  Ballot + popc append in candidate order: deterministic.
//
// SHIFTED (every dimension >= 7 cells, no coordinate on a box face): a pair
// in cells at most two apart is closer than 3 cell edges < L/2 without a
// wrap and farther than L/2 with one, so the minimum-image decision of the
// reference is fixed per range and the distance needs no comparisons.
// Otherwise (small grids) every candidate takes the reference's full test,
// and grids with fewer than five cells in a dimension visit each cell once.
constexpr int NBW = 4;         // particles of a cell handled per pass
constexpr int NB_SEG_MAX = 64; // 25 rows x at most 2 ranges

__device__ __forceinline__ int wrapi(int x, int n) { return ((x % n) + n) % n; }
// x within two cells of [0, n), n >= 5: one compare each way, no division
__device__ __forceinline__ int wrap_near(int x, int n) { return x < 0 ? x + n : (x >= n ? x - n : x); }

// s_lo, s_pre, s_sh: per-warp segment tables in shared memory (block warp w
// uses entries [w * NB_SEG_MAX, ...), s_pre one more).
template <bool FMA, bool SHIFTED>
__device__ inline void phase_nbl_cells_t(const SimArgs &a, Span g, int *s_lo, int *s_pre, float3 *s_sh) {
    const float4 *pos = a.pos_tmp;
    const int ncx = a.ncx, ncy = a.ncy, ncz = a.ncz;
    const float Lx = a.Lx, Ly = a.Ly, Lz = a.Lz;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    int *lo_s = s_lo + wib * NB_SEG_MAX, *pre_s = s_pre + wib * (NB_SEG_MAX + 1);
    float3 *sh_s = s_sh + wib * NB_SEG_MAX;
    const int nwarps = (g.nb * (int)blockDim.x) >> 5;
    const int ry = ncy < 5 ? ncy : 5, rz = ncz < 5 ? ncz : 5;
    const int nrows = ry * rz;
    for (int c = (g.b * (int)blockDim.x + (int)threadIdx.x) >> 5; c < a.ncell; c += nwarps) {
        const int cs = a.cell_start[c], ce = a.cell_start[c + 1];
        if (cs == ce) continue;
        const int cx = c % ncx, cy = (c / ncx) % ncy, cz = c / (ncx * ncy);
        // lane r < nrows builds the x-range(s) of stencil row r
        int len0 = 0, len1 = 0, lo0 = 0, lo1 = 0;
        float sy = 0.f, sz = 0.f, sx0 = 0.f, sx1 = 0.f;
        if (lane < nrows) {
            const int za = lane / ry, yb = lane % ry;
            const int zu = cz - 2 + za, yu = cy - 2 + yb;  // unwrapped (SHIFTED: grid >= 7 cells)
            const int z = ncz < 5 ? za : wrapi(zu, ncz);
            const int y = ncy < 5 ? yb : wrapi(yu, ncy);
            if (SHIFTED) {  // cells past the low face hold coordinates near +L/2: shift -L
                sz = zu < 0 ? -Lz : (zu >= ncz ? Lz : 0.f);
                sy = yu < 0 ? -Ly : (yu >= ncy ? Ly : 0.f);
            }
            const int rowbase = (z * ncy + y) * ncx;
            int l0, h0, l1 = 0, h1 = 0;
            if (ncx <= 5) {
                l0 = rowbase;
                h0 = rowbase + ncx;
            } else {
                const int x0 = cx - 2, x1 = cx + 2;
                if (x0 >= 0 && x1 < ncx) {
                    l0 = rowbase + x0;
                    h0 = rowbase + x1 + 1;
                } else if (x0 < 0) {
                    l0 = rowbase + x0 + ncx;
                    h0 = rowbase + ncx;
                    l1 = rowbase;
                    h1 = rowbase + x1 + 1;
                    sx0 = -Lx;
                } else {
                    l0 = rowbase + x0;
                    h0 = rowbase + ncx;
                    l1 = rowbase;
                    h1 = rowbase + x1 - ncx + 1;
                    sx1 = Lx;
                }
            }
            lo0 = a.cell_start[l0];
            len0 = a.cell_start[h0] - lo0;
            if (h1 > l1) {
                lo1 = a.cell_start[l1];
                len1 = a.cell_start[h1] - lo1;
            }
        }
        // segments in row order: row r gives entries 2r, 2r+1 (second may be empty)
        const int tot = len0 + len1;
        int incl = tot;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        const int excl = incl - tot;
        if (lane < nrows) {
            lo_s[2 * lane] = lo0;
            pre_s[2 * lane] = excl;
            lo_s[2 * lane + 1] = lo1;
            pre_s[2 * lane + 1] = excl + len0;
            if (SHIFTED) {
                sh_s[2 * lane] = make_float3(sx0, sy, sz);
                sh_s[2 * lane + 1] = make_float3(sx1, sy, sz);
            }
        }
        const int T = __shfl_sync(0xffffffffu, incl, 31);
        if (lane == 0) pre_s[2 * nrows] = T;
        __syncwarp();
        const int nseg = 2 * nrows;
        for (int g0 = cs; g0 < ce; g0 += NBW) {
            const int gn = min(NBW, ce - g0);
            float4 pi[NBW];
            int cnt[NBW];
#pragma unroll
            for (int p = 0; p < NBW; p++) {
                pi[p] = p < gn ? pos[g0 + p] : make_float4(0.f, 0.f, 0.f, 0.f);
                cnt[p] = 0;
            }
            // each lane walks the segments forward as its candidate index grows
            // (64 candidates per iteration: two independent position loads)
            int seg = 0;
            for (int v0 = 0; v0 < T; v0 += 64) {
                const int va = v0 + lane, vb = va + 32;
                const bool oka = va < T, okb = vb < T;
                int ja = 0, jb = 0;
                float4 pa = make_float4(0.f, 0.f, 0.f, 0.f), pb = pa;
                float3 sha = make_float3(0.f, 0.f, 0.f), shb = sha;
                if (oka) {
                    while (seg + 1 < nseg && pre_s[seg + 1] <= va) seg++;
                    ja = lo_s[seg] + (va - pre_s[seg]);
                    pa = pos[ja];
                    if (SHIFTED) sha = sh_s[seg];
                }
                if (okb) {
                    while (seg + 1 < nseg && pre_s[seg + 1] <= vb) seg++;
                    jb = lo_s[seg] + (vb - pre_s[seg]);
                    pb = pos[jb];
                    if (SHIFTED) shb = sh_s[seg];
                }
#pragma unroll
                for (int half = 0; half < 2; half++) {
                    const bool ok = half ? okb : oka;
                    const int j = half ? jb : ja;
                    const float4 pj = half ? pb : pa;
                    const float3 sh = half ? shb : sha;
#pragma unroll
                    for (int p = 0; p < NBW; p++) {
                        if (p >= gn) break;
                        const float d2 = SHIFTED ? dist_sq_shifted<FMA>(pj, pi[p], sh.x, sh.y, sh.z)
                                                 : dist_sq_exact<FMA>(pj, pi[p], Lx, Ly, Lz);
                        bool hit = ok && j != g0 + p && d2 < a.cps2;
                        if (hit && a.excl) hit = !excluded(a, a.orig_tmp[g0 + p], a.orig_tmp[j]);
                        const unsigned m = __ballot_sync(0xffffffffu, hit);
                        if (hit) {
                            const int k = cnt[p] + __popc(m & ((1u << lane) - 1u));
                            if (k < a.max_nbs) a.nbl[nbl_index(g0 + p, k, a.stride)] = j;
                        }
                        cnt[p] += __popc(m);
                    }
                }
            }
#pragma unroll
            for (int p = 0; p < NBW; p++) {
                if (p < gn && lane == p) {
                    a.nbc[g0 + p] = cnt[p];
                    atomicMax(&a.ctrl->maxcount, cnt[p]);
                }
            }
        }
        __syncwarp();
    }
}

// Cell-list build, one thread per particle slot: the thread walks the
// stencil rows in the same order as phase_nbl_cells_t's packed candidate
// sequence and appends hits in that order, so both builds give identical
// lists.  No ballots and no segment search: about half the instructions per
// candidate, at one lane per particle; used when the grid has at least one
// thread per particle.
template <bool FMA, bool SHIFTED>
__device__ inline void phase_nbl_cells_tpp(const SimArgs &a, Span g) {
    const float4 *pos = a.pos_tmp;
    const int ncx = a.ncx, ncy = a.ncy, ncz = a.ncz;
    const float Lx = a.Lx, Ly = a.Ly, Lz = a.Lz;
    const float cps2 = a.cps2;
    const int maxn = a.max_nbs;
    const size_t cs = (size_t)a.stride * NB_CHUNK;
    const int ry = ncy < 5 ? ncy : 5, rz = ncz < 5 ? ncz : 5;
    // the arguments the walk reads, in registers: the list stores could
    // otherwise force them to be reloaded after every store
    const int n = a.n;
    const int *excl = a.excl;
    const int *orig_tmp = a.orig_tmp;
    const int *cstart = a.cell_start;
    const int *scell = a.scell;
    int *nbl = a.nbl;
    // the walk instantiated with and without pair exclusions (uniform)
    auto walk = [&](auto ex_tag) {
        constexpr bool EX = decltype(ex_tag)::value;
        for (int s = g.b * (int)blockDim.x + (int)threadIdx.x; s < n; s += g.nb * (int)blockDim.x) {
            const float4 pi = pos[s];
            const int c = scell[s];
            const int cxy = ncx * ncy;
            const int cz = c / cxy, rem = c - cz * cxy;
            const int cy = rem / ncx, cx = rem - cy * ncx;
            // entry k of slot s at chunk k/4 (cs apart), position k%4
            int *chunk = nbl + (size_t)s * NB_CHUNK;
            int cnt = 0;
            const int ui = EX ? orig_tmp[s] : 0;
            // the append without a branch: the store (predicated), the count and
            // the step to the next chunk when one fills
            auto test = [&](float4 pj, int j, float sx, float sy, float sz) {
                const float d2 =
                    SHIFTED ? dist_sq_shifted<FMA>(pj, pi, sx, sy, sz) : dist_sq_exact<FMA>(pj, pi, Lx, Ly, Lz);
                bool hit = (d2 < cps2) & (j != s);
                if (EX && hit) hit = !excluded(a, ui, orig_tmp[j]);
                if (hit & (cnt < maxn)) chunk[cnt & 3] = j;
                cnt += hit ? 1 : 0;
                chunk += (hit & ((cnt & 3) == 0)) ? cs : (size_t)0;
            };
            for (int za = 0; za < rz; za++) {
                const int zu = cz - 2 + za;
                const int z = ncz < 5 ? za : wrap_near(zu, ncz);
                const float sz = SHIFTED ? (zu < 0 ? -Lz : (zu >= ncz ? Lz : 0.f)) : 0.f;
                for (int yb = 0; yb < ry; yb++) {
                    const int yu = cy - 2 + yb;
                    const int y = ncy < 5 ? yb : wrap_near(yu, ncy);
                    const float sy = SHIFTED ? (yu < 0 ? -Ly : (yu >= ncy ? Ly : 0.f)) : 0.f;
                    const int rowbase = (z * ncy + y) * ncx;
                    int l0, h0, l1 = 0, h1 = 0;
                    float sx0 = 0.f, sx1 = 0.f;
                    if (ncx <= 5) {
                        l0 = rowbase;
                        h0 = rowbase + ncx;
                    } else {
                        const int x0 = cx - 2, x1 = cx + 2;
                        if (x0 >= 0 && x1 < ncx) {
                            l0 = rowbase + x0;
                            h0 = rowbase + x1 + 1;
                        } else if (x0 < 0) {
                            l0 = rowbase + x0 + ncx;
                            h0 = rowbase + ncx;
                            l1 = rowbase;
                            h1 = rowbase + x1 + 1;
                            sx0 = -Lx;
                        } else {
                            l0 = rowbase + x0;
                            h0 = rowbase + ncx;
                            l1 = rowbase;
                            h1 = rowbase + x1 - ncx + 1;
                            sx1 = Lx;
                        }
                    }
    #pragma unroll
                    for (int r = 0; r < 2; r++) {
                        const int lc = r ? l1 : l0, hc = r ? h1 : h0;
                        if (hc <= lc) continue;
                        const float sx = r ? sx1 : sx0;
                        const int lo = cstart[lc], hi = cstart[hc];
                        int j = lo;
                        for (; j + 4 <= hi; j += 4) {  // four independent loads in flight
                            const float4 q0 = pos[j], q1 = pos[j + 1], q2 = pos[j + 2], q3 = pos[j + 3];
                            test(q0, j, sx, sy, sz);
                            test(q1, j + 1, sx, sy, sz);
                            test(q2, j + 2, sx, sy, sz);
                            test(q3, j + 3, sx, sy, sz);
                        }
                        for (; j < hi; j++) test(pos[j], j, sx, sy, sz);
                    }
                }
            }
            a.nbc[s] = cnt;
            atomicMax(&a.ctrl->maxcount, cnt);
        }
    };
    if (excl)
        walk(BoolTag<true>{});
    else
        walk(BoolTag<false>{});
}

// Per-warp segment tables of the cell build, in shared memory, for blocks of
// up to WPB warps.  Declared once per kernel and handed down.
template <int WPB>
struct NbScratch {
    int lo[WPB * NB_SEG_MAX];
    int pre[WPB * (NB_SEG_MAX + 1)];
    float3 sh[WPB * NB_SEG_MAX];
};

template <bool FMA, int WPB>
__device__ inline void phase_nbl_cells(const SimArgs &a, Span g, NbScratch<WPB> &scr) {
    const bool shifted = a.ncx >= 7 && a.ncy >= 7 && a.ncz >= 7 && !*(volatile int *)&a.ctrl->cell_wrap;
    // a warp per cell while threads outnumber particles, a thread per
    // particle beyond (measured on B200: 1.7x faster at 1M particles, 1.6x
    // slower at 32k on the whole GPU)
    const bool tpp = a.n >= g.nb * (int)blockDim.x;
    if (tpp) {
        if (shifted)
            phase_nbl_cells_tpp<FMA, true>(a, g);
        else
            phase_nbl_cells_tpp<FMA, false>(a, g);
    } else if (shifted) {
        phase_nbl_cells_t<FMA, true>(a, g, scr.lo, scr.pre, scr.sh);
    } else {
        phase_nbl_cells_t<FMA, false>(a, g, scr.lo, scr.pre, scr.sh);
    }
}

// Move the reordered state into place, record r_ref, clear the cell counters.
__device__ inline void phase_finish_cells(const SimArgs &a, int cur, Span g = grid_span()) {
    float4 *pos = cur_pos(a, cur);
    const size_t n = a.n;
    for (int s = g.b * (int)blockDim.x + (int)threadIdx.x; s < a.n; s += g.nb * (int)blockDim.x) {
        const float4 p = a.pos_tmp[s];
        pos[s] = p;
        a.rref[s] = p;
        a.vel[s] = a.vel_tmp[s];
        a.img[s] = a.img_tmp[s];
        a.orig[s] = a.orig_tmp[s];
        if (a.slot_of) a.slot_of[a.orig_tmp[s]] = s;
        a.pscal[3 * n + s] = a.pscal_tmp[3 * n + s];
        a.pscal[4 * n + s] = a.pscal_tmp[4 * n + s];
    }
    for (int c = g.b * (int)blockDim.x + (int)threadIdx.x; c < a.ncell; c += g.nb * (int)blockDim.x) a.cell_count[c] = 0;
}

__device__ __forceinline__ void rebuild_done(DevCtrl *c) {
    c->rebuild = 0;
    c->nrebuild += 1;
    c->cell_wrap = 0;
}

// ---------------------------------------------------------------------------
// force + integrate phase
// ---------------------------------------------------------------------------
__device__ __forceinline__ double target_temperature(const SimArgs &a, double t) {
    if (a.tfunc == GDB_TFUNC_RAMP) {  // misc/make_function.py:27-32
        if (t < a.tp1) return a.tp0;
        if (t < a.tp3) return a.tp0 + (t - a.tp1) * ((double)(a.tp2 - a.tp0) / (double)(a.tp3 - a.tp1));
        return a.tp2;
    }
    return a.tp0;
}

// Target pressure of NPT_Atomic: the same constant / ramp forms.
__device__ __forceinline__ double target_pressure(const SimArgs &a, double t) {
    if (a.pfunc == GDB_TFUNC_RAMP) {
        if (t < a.pp1) return a.pp0;
        if (t < a.pp3) return a.pp0 + (t - a.pp1) * ((double)(a.pp2 - a.pp0) / (double)(a.pp3 - a.pp1));
        return a.pp2;
    }
    return a.pp0;
}

// Per-step constants of NPT_Atomic's particle update (integrators/
// NPT_Atomic.py:108-113, with numba's typing: factor in float64, plus, minus
// and rfactor in float32) and the box scaling of scale_box (:168-181): every
// coordinate times sf = (1 + dt D bs0)^(1/3), the box lengths too.
struct NptStep {
    float plus, minus, rfactor;
    double sf;
    float Lx, Ly, Lz;  // box after the scaling
};
__device__ __forceinline__ NptStep npt_step_consts(const SimArgs &a, const DevCtrl *ctrl) {
    NptStep ns;
    const float ts0 = ctrl->npt_ts0, bs0 = ctrl->npt_bs0;
    const double factor = (double)(0.5f * a.dt) * ((1.0 + 3.0 / (double)a.dof) * (double)bs0 + (double)ts0);
    ns.plus = 1.0f / (float)(1.0 + factor);
    ns.minus = (float)(1.0 - factor);
    ns.rfactor = bs0 * a.dt;
    ns.sf = pow(1.0 + (double)a.dt * 3.0 * (double)bs0, 1.0 / 3.0);
    ns.Lx = (float)((double)a.Lx * ns.sf);
    ns.Ly = (float)((double)a.Ly * ns.sf);
    ns.Lz = (float)((double)a.Lz * ns.sf);
    return ns;
}

// numba.cuda.random's generator, the one of integrators/NVT_Langevin.py:105:
// xoroshiro128+ with the (55, 14, 36) update, uniform float32 =
// float32((x >> 11) 2^-53), normal = first Box-Muller value of two draws.
__device__ __forceinline__ unsigned long long xoro_next(ulonglong2 &s) {
    const unsigned long long s0 = s.x;
    unsigned long long s1 = s.y;
    const unsigned long long result = s0 + s1;
    s1 ^= s0;
    s.x = ((s0 << 55) | (s0 >> 9)) ^ s1 ^ (s1 << 14);
    s.y = (s1 << 36) | (s1 >> 28);
    return result;
}
__device__ __forceinline__ float xoro_uniform(ulonglong2 &s) {
    return (float)((double)(xoro_next(s) >> 11) * (1.0 / 9007199254740992.0));
}
__device__ __forceinline__ float xoro_normal(ulonglong2 &s) {
    const float u1 = xoro_uniform(s);
    const float u2 = xoro_uniform(s);
    return sqrtf(-2.0f * logf(u1)) * cosf(6.28318530717958647692f * u2);
}

// ConfigurationSaver slot of a step (runtime_actions/configuration_saver.py:
// 115-141): step 0 -> 0, step 2^b -> b + 1, others -> -1.
__device__ __forceinline__ int conf_save_index(int step) {
    if (step == 0) return 0;
    if (step & (step - 1)) return -1;
    return 32 - __clz(step);
}

// Pair parameters a particle of type ti needs for its neighbours.  NT is the
// number of particle types when it is 1 or 2: the five force parameters of
// each neighbour type (c, cs12, cs6, sc, cut^2) sit in registers and a
// neighbour's type selects them; NT = 0 reads a general table in shared
// memory.  Energy and virial terms (saved steps only) always come from the
// shared-memory row.
template <int NT>
struct PairRow {
    const PairEntry *row;
    float c0, a0, b0, s0, k0, c1, a1, b1, s1, k1;
    __device__ __forceinline__ PairRow(const PairEntry *tab, int nt, int ti) : row(tab + ti * nt) {
        if (NT >= 1) {
            c0 = row[0].c, a0 = row[0].cs12, b0 = row[0].cs6, s0 = row[0].sc, k0 = row[0].cut2;
        }
        if (NT == 2) {
            c1 = row[1].c, a1 = row[1].cs12, b1 = row[1].cs6, s1 = row[1].sc, k1 = row[1].cut2;
        }
    }
    __device__ __forceinline__ void force(int tj, float &c, float &cs12, float &cs6, float &sc, float &cut2) const {
        if (NT == 1) {
            c = c0, cs12 = a0, cs6 = b0, sc = s0, cut2 = k0;
        } else if (NT == 2) {
            const bool t = tj != 0;
            c = t ? c1 : c0, cs12 = t ? a1 : a0, cs6 = t ? b1 : b0, sc = t ? s1 : s0, cut2 = t ? k1 : k0;
        } else {
            const PairEntry &e = row[tj];
            c = e.c, cs12 = e.cs12, cs6 = e.cs6, sc = e.sc, cut2 = e.cut2;
        }
    }
};

// Minimum image for list pairs (|d| < L): d - L*rint(d/L) equals the
// reference's 2d-vs-L selection for every pair closer than L/2.
template <bool REC, int NT>
__device__ __forceinline__ void pair_force(const PairRow<NT> &pr, float4 pi, float4 pj, bool valid, float Lx, float Ly,
                                           float Lz, float ilx, float ily, float ilz, float &fx, float &fy, float &fz,
                                           float &u, float &w, float &l) {
    float dx = pj.x - pi.x, dy = pj.y - pi.y, dz = pj.z - pi.z;
    dx -= Lx * rintf(dx * ilx);
    dy -= Ly * rintf(dy * ily);
    dz -= Lz * rintf(dz * ilz);
    const float d2 = dx * dx + dy * dy + dz * dz;
    const int tj = NT == 1 ? 0 : ptype_of(pj);
    float c, cs12, cs6, sc, cut2;
    pr.force(tj, c, cs12, cs6, sc, cut2);
    if (valid && d2 < cut2) {
        const float inv2 = __fdividef(1.0f, d2);
        const float x2 = c * inv2;
        const float x6 = x2 * x2 * x2;
        const float x12 = x6 * x6;
        const float s = (cs12 * x12 + cs6 * x6) * inv2 - sc;
        fx -= dx * s;
        fy -= dy * s;
        fz -= dz * s;
        if (REC) {
            const PairEntry &e = pr.row[tj];
            const float r = sqrtf(d2);
            const float uu = e.cu12 * x12 + e.cu6 * x6 - e.uc + e.sccut * (r - e.cut);
            u += 0.5f * uu;
            w += d2 * s * (1.0f / 6.0f);
            l += -2.0f * s + (e.cm12 * x12 + e.cm6 * x6) * inv2;
        }
    }
}

// Neighbours of particle i handled by lane `sub` of TP: chunks of four
// indices (one int4 load), four independent position gathers per chunk.
// pair_potential.py:223-231 with the full-list calculator :164-178.
template <int TP, int NT, bool REC, bool NC>
__device__ __forceinline__ void neighbour_loop(const SimArgs &a, const float4 *pos, const PairEntry *tab, int nt,
                                               int i, int sub, float4 pi, float &fx, float &fy, float &fz, float &u,
                                               float &w, float &l) {
    const PairRow<NT> pr(tab, nt, NT == 1 ? 0 : ptype_of(pi));
    const int cnt = min(a.nbc[i], a.max_nbs);
    const int nch = (cnt + 3) >> 2;
    const float Lx = a.Lx, Ly = a.Ly, Lz = a.Lz;
    const float ilx = 1.0f / Lx, ily = 1.0f / Ly, ilz = 1.0f / Lz;
    const int4 *base = reinterpret_cast<const int4 *>(a.nbl) + i;
    const size_t cstride = (size_t)a.stride;  // int4 units between chunks
    // the index chunks of the next two iterations are loaded before this
    // one's positions: the list streams from HBM, so its latency overlaps the
    // work (measured on B200: two ahead beats one and three).  The first two
    // are loaded without waiting for the count: every slot has max_nbs + 4
    // entries, so their guard is a constant and the count's latency overlaps
    // theirs (entries past the count are never used).
    const int chunks_alloc = (a.max_nbs + NB_CHUNK) / NB_CHUNK;
    int4 jn = sub < chunks_alloc ? load<NC>(base + sub * cstride) : make_int4(i, i, i, i);
    int4 jn2 = sub + TP < chunks_alloc ? load<NC>(base + (sub + TP) * cstride) : make_int4(i, i, i, i);
    for (int ch = sub; ch < nch; ch += TP) {
        const int4 jj = jn;
        jn = jn2;
        if (ch + 2 * TP < nch) jn2 = load<NC>(base + (ch + 2 * TP) * cstride);
        const int k0 = ch * 4;
        const bool v1 = k0 + 1 < cnt, v2 = k0 + 2 < cnt, v3 = k0 + 3 < cnt;
        const int j0 = jj.x, j1 = v1 ? jj.y : i, j2 = v2 ? jj.z : i, j3 = v3 ? jj.w : i;
        const float4 p0 = load<NC>(pos + j0);
        const float4 p1 = load<NC>(pos + j1);
        const float4 p2 = load<NC>(pos + j2);
        const float4 p3 = load<NC>(pos + j3);
        pair_force<REC, NT>(pr, pi, p0, true, Lx, Ly, Lz, ilx, ily, ilz, fx, fy, fz, u, w, l);
        pair_force<REC, NT>(pr, pi, p1, v1, Lx, Ly, Lz, ilx, ily, ilz, fx, fy, fz, u, w, l);
        pair_force<REC, NT>(pr, pi, p2, v2, Lx, Ly, Lz, ilx, ily, ilz, fx, fy, fz, u, w, l);
        pair_force<REC, NT>(pr, pi, p3, v3, Lx, Ly, Lz, ilx, ily, ilz, fx, fy, fz, u, w, l);
    }
}

// Harmonic bonds of the particle in slot i, its own side of each
// (interactions/bonds.py:102-135 with potential_functions/
// harmonic_bond_function.py:37-43): dr = r_partner - r_i by the minimum
// image, u = k (r - r0)^2 / 2 and s = -k (r - r0) / r; the particle takes
// f -= dr s, half of u, its half of the virial dr^2 s / (2 D), and the whole
// (1 - D) s + k into lapU, as the reference adds to both ends of a bond.
__device__ __forceinline__ void bond_forces(const SimArgs &a, int i, float4 pi, const float4 *pos, bool rec, float &fx,
                                            float &fy, float &fz, float &u, float &w, float &l) {
    const int ui = a.orig[i];
    const int cnt = a.bond_cnt[ui];
    for (int b = 0; b < cnt; b++) {
        const size_t e = (size_t)ui * a.bond_max + b;
        const int j = a.slot_of[a.bond_j[e]];
        const float2 prm = a.bond_prm[a.bond_t[e]];
        const float4 pj = pos[j];
        const float dx = mic(__fsub_rn(pj.x, pi.x), a.Lx), dy = mic(__fsub_rn(pj.y, pi.y), a.Ly),
                    dz = mic(__fsub_rn(pj.z, pi.z), a.Lz);
        const float d2 = dx * dx + dy * dy + dz * dz;
        const float d = sqrtf(d2);
        const float s = -prm.y * (d - prm.x) / d;
        fx -= dx * s;
        fy -= dy * s;
        fz -= dz * s;
        if (rec) {
            u += 0.5f * (0.5f * prm.y * (d - prm.x) * (d - prm.x));
            w += d2 * s * (1.0f / 6.0f);
            l += -2.0f * s + prm.y;
        }
    }
}

// Everything a step does for particle i once its force is summed (shared by
// the row and brick force phases): ConfigurationSaver frame, pending
// momentum shift, per-particle scalars, the integrator update
// (MODE_STEP) or the force store (MODE_EVAL), periodic wrap with images, the
// skin check for the next step and this particle's share of the block sums.
template <int INTEG, int MODE>
__device__ __forceinline__ void finish_particle(const SimArgs &a, int i, float4 pi, float4 v, float4 rr, float fx,
                                                float fy, float fz, float u, float w, float l, bool rec, bool reset,
                                                int step, bool shift_pending, float shx, float shy, float shz,
                                                float xi, float4 *pos_next, double (&red)[NQ], bool &moved,
                                                const NptStep *ns = nullptr) {
    DevCtrl *ctrl = a.ctrl;
    const size_t n = a.n;
    // ConfigurationSaver: frame taken before this step's integration
    if (a.conf) {
        const int si = conf_save_index(step);
        if (si >= 0 && si < a.conf_per_block) {
            const int4 im = a.img[i];
            const size_t uidx = (size_t)a.orig[i];
            float *fr = a.conf + (size_t)si * 2 * n * 3;
            fr[3 * uidx] = pi.x;
            fr[3 * uidx + 1] = pi.y;
            fr[3 * uidx + 2] = pi.z;
            fr += n * 3;
            fr[3 * uidx] = (float)im.x;
            fr[3 * uidx + 1] = (float)im.y;
            fr[3 * uidx + 2] = (float)im.z;
            if (uidx == 0 && a.conf_box) {  // include_simbox (configuration_saver.py:137-139)
                a.conf_box[4 * si] = a.Lx;
                a.conf_box[4 * si + 1] = a.Ly;
                a.conf_box[4 * si + 2] = a.Lz;
            }
        }
    }
    if (shift_pending) {
        v.x -= shx;
        v.y -= shy;
        v.z -= shz;
    }
    const float fsq = fx * fx + fy * fy + fz * fz;
    if (rec) {
        a.pscal[i] = u;
        a.pscal[n + i] = w;
        a.pscal[2 * n + i] = l;
    }
    red[1] += u;
    red[2] += w;
    red[3] += l;
    red[4] += fsq;
    if (MODE == MODE_EVAL) {
        a.frc[i] = make_float4(fx, fy, fz, 0.f);
        if (shift_pending) a.vel[i] = v;
    } else {
        const float m = v.w;
        float kin = 0.f;
        float r[3] = {pi.x, pi.y, pi.z};
        float vv[3] = {v.x, v.y, v.z};
        const float ff[3] = {fx, fy, fz};
        if (INTEG == GDB_INTEGRATOR_NVE) {  // integrators/NVE.py:78-97
#pragma unroll
            for (int k = 0; k < 3; k++) {
                float v_mean = vv[k];
                vv[k] += ff[k] / m * a.dt;
                v_mean += vv[k];
                v_mean *= 0.5f;
                kin += 0.5f * m * v_mean * v_mean;
                r[k] += vv[k] * a.dt;
            }
        } else if (INTEG == GDB_INTEGRATOR_LANGEVIN) {  // integrators/NVT_Langevin.py:98-122
            const size_t uidx = (size_t)a.orig[i];
            ulonglong2 st = a.rng[uidx];
            float4 ob = a.lbeta[uidx];
            float obk[3] = {ob.x, ob.y, ob.z};
            const float T = (float)target_temperature(a, ctrl->time_zero + (double)step * (double)a.dt);
            const float numerator = 2.0f * m - a.alpha * a.dt;
            const float denominator = 2.0f * m + a.alpha * a.dt;
            const float fa = numerator / denominator;
            const float b_over_m = 2.0f / denominator;
            const float bscale = sqrtf(2.0f * a.alpha * T * a.dt);
#pragma unroll
            for (int k = 0; k < 3; k++) {
                const float beta = bscale * xoro_normal(st);
                kin += 0.5f * m * vv[k] * vv[k];  // the velocity before the update
                vv[k] = fa * vv[k] + b_over_m * ff[k] * a.dt + b_over_m * 0.5f * (beta + obk[k]);
                obk[k] = beta;
                r[k] += vv[k] * a.dt;
            }
            a.rng[uidx] = st;
            a.lbeta[uidx] = make_float4(obk[0], obk[1], obk[2], 0.f);
        } else if (INTEG == GDB_INTEGRATOR_NPT) {  // integrators/NPT_Atomic.py:118-127
#pragma unroll
            for (int k = 0; k < 3; k++) {
                vv[k] = ns->plus * (ns->minus * vv[k] + ff[k] / m * a.dt);
                kin += 0.5f * m * vv[k] * vv[k];
                r[k] += vv[k] * a.dt + ns->rfactor * r[k];
            }
        } else {  // integrators/NVT.py:83-102
            const float factor = 0.5f * xi * a.dt;
            const float plus = 1.0f / (1.0f + factor);
            const float minus = 1.0f - factor;
#pragma unroll
            for (int k = 0; k < 3; k++) {
                vv[k] = plus * (minus * vv[k] + ff[k] / m * a.dt);
                kin += 0.5f * m * vv[k] * vv[k];
                r[k] += vv[k] * a.dt;
            }
        }
        // periodic boundaries with image counters (orthorhombic.py:75-86)
        const float L[3] = {a.Lx, a.Ly, a.Lz};
        int dimg[3] = {0, 0, 0};
        bool wrapped = false;
#pragma unroll
        for (int k = 0; k < 3; k++) {
            if (r[k] * 2.0f > L[k]) {
                r[k] -= L[k];
                dimg[k] += 1;
                wrapped = true;
            }
            if (r[k] * 2.0f < -L[k]) {
                r[k] += L[k];
                dimg[k] -= 1;
                wrapped = true;
            }
        }
        if (wrapped) {
            int4 im = a.img[i];
            im.x += dimg[0];
            im.y += dimg[1];
            im.z += dimg[2];
            a.img[i] = im;
        }
        if (INTEG == GDB_INTEGRATOR_NPT) {  // scale_box, after the wrap in the step's box
#pragma unroll
            for (int k = 0; k < 3; k++) r[k] = (float)(ns->sf * (double)r[k]);
        }
        if (!(fabsf(r[0]) <= L[0] && fabsf(r[1]) <= L[1] && fabsf(r[2]) <= L[2]))
            atomicOr(&ctrl->status, GDB_STATUS_NAN);
        const float4 pn = make_float4(r[0], r[1], r[2], pi.w);
        pos_next[i] = pn;
        a.vel[i] = make_float4(vv[0], vv[1], vv[2], m);
        a.pscal[3 * n + i] = kin;
        a.pscal[4 * n + i] = fsq;
        // skin check for the next step (nblist.py:57-86), in the next step's box
        if (INTEG == GDB_INTEGRATOR_NPT)
            moved |= dist_sq_exact<false>(pn, rr, ns->Lx, ns->Ly, ns->Lz) > a.skin2q;
        else
            moved |= dist_sq_exact<false>(pn, rr, a.Lx, a.Ly, a.Lz) > a.skin2q;
        red[0] += kin;
        if (reset) {
            red[5] += (double)m * vv[0];
            red[6] += (double)m * vv[1];
            red[7] += (double)m * vv[2];
            red[8] += m;
        }
    }  // MODE_STEP
}

// Control state a step reads after the barrier, loaded at once by one thread
// of the persistent kernels (StepCtl; NULL: read from ctrl here).
struct StepCtl {
    int rebuild, step, pending[2];
    float shift[2][3];
    float xi;
    double time_zero;
};
__device__ __forceinline__ void load_step_ctl(const DevCtrl *c, StepCtl *sc) {
    const int rb = *(volatile const int *)&c->rebuild;
    const int st = *(volatile const int *)&c->step;
    const int p0 = *(volatile const int *)&c->pending[0], p1 = *(volatile const int *)&c->pending[1];
    float sh[2][3];
#pragma unroll
    for (int q = 0; q < 2; q++)
#pragma unroll
        for (int k = 0; k < 3; k++) sh[q][k] = *(volatile const float *)&c->shift[q][k];
    const float xi = *(volatile const float *)&c->xi;
    const double tz = *(volatile const double *)&c->time_zero;
    sc->rebuild = rb;
    sc->step = st;
    sc->pending[0] = p0;
    sc->pending[1] = p1;
#pragma unroll
    for (int q = 0; q < 2; q++)
#pragma unroll
        for (int k = 0; k < 3; k++) sc->shift[q][k] = sh[q][k];
    sc->xi = xi;
    sc->time_zero = tz;
}

// Forces from pos[cur], integration into pos[cur^1] (MODE_STEP) or forces
// only (MODE_EVAL).  A round is blockDim/TP consecutive particles.
// Standalone launches (PERSIST false) take rounds g.b, g.b + g.nb, ... and
// write one float64 partial row per block to partials[g.b].  The persistent
// kernels (PERSIST true) hand rounds out through an atomic counter (blocks on
// faster SMs take more) and write one row per round to partials[round], so
// the fixed-order sum does not depend on which block ran which round.  Only
// the sums the step needs are reduced: all of them on saved and reset steps,
// the kinetic energy (NVT) otherwise.  Returns (persistent kernels) or sets
// (standalone) the rebuild flag when a particle has moved more than skin/2
// since the build.  `part` (persistent kernels) replaces partials as the
// rows' base.
template <int TP, int NT, int INTEG, int MODE, bool NC, bool PERSIST>
__device__ inline bool phase_step(const SimArgs &a, const PairEntry *tab, int nt, int cur, int step, double *s_red,
                                  Span g = grid_span(), const StepCtl *sc = nullptr, double *part = nullptr) {
    DevCtrl *ctrl = a.ctrl;
    double *prow = part ? part : a.partials;  // the rows this step writes
    const float4 *pos = cur_pos(a, cur);
    float4 *pos_next = cur_pos(a, cur ^ 1);
    // NPT_Atomic reads every particle's virial every step (NPT_Atomic.py:115)
    const bool rec = MODE == MODE_EVAL || INTEG == GDB_INTEGRATOR_NPT || (a.every > 0 && step % a.every == 0);
    const bool reset = MODE == MODE_STEP && a.reset_every > 0 && step % a.reset_every == 0;
    const int ppar = (step & 1) ^ 1;
    // independent loads, issued together (one latency after the barrier), or
    // the copy the persistent kernels loaded with the step index
    const bool shift_pending = (sc ? sc->pending[ppar] : ctrl->pending[ppar]) != 0;
    const float shx0 = sc ? sc->shift[ppar][0] : ctrl->shift[ppar][0];
    const float shy0 = sc ? sc->shift[ppar][1] : ctrl->shift[ppar][1];
    const float shz0 = sc ? sc->shift[ppar][2] : ctrl->shift[ppar][2];
    const float shx = shift_pending ? shx0 : 0.f, shy = shift_pending ? shy0 : 0.f, shz = shift_pending ? shz0 : 0.f;
    const float xi = sc ? sc->xi : ctrl->xi;
    NptStep ns;
    if (INTEG == GDB_INTEGRATOR_NPT && MODE == MODE_STEP) ns = npt_step_consts(a, ctrl);
    const int per_block = blockDim.x / TP;
    const int rounds_total = (a.n + per_block - 1) / per_block;
    const bool full = rec || reset;
    const bool needk = full || INTEG == GDB_INTEGRATOR_NVT;
    double red[NQ];
#pragma unroll
    for (int q = 0; q < NQ; q++) red[q] = 0.0;
    bool moved = false;
    __shared__ int s_round;
    int round = g.b;
    // the persistent kernels hand out rounds through a counter unless every
    // block has at most one (small systems: two atomics less per step)
    const bool dynamic = PERSIST && rounds_total > g.nb;
    if (dynamic) {
        if (threadIdx.x == 0) s_round = (int)atomicAdd(&ctrl->work[step & 1], 1u);
        __syncthreads();
        round = s_round;
    }
    while (round < rounds_total) {
        const int i = round * per_block + threadIdx.x / TP;
        const int sub = threadIdx.x % TP;
        const bool active = i < a.n;
        float fx = 0.f, fy = 0.f, fz = 0.f, u = 0.f, w = 0.f, l = 0.f;
        float4 pi = make_float4(0.f, 0.f, 0.f, 0.f);
        // the integrating lane's own state, loaded before the neighbour loop so
        // its latency overlaps the gathers
        float4 v = make_float4(0.f, 0.f, 0.f, 1.f), rr = v;
        if (active && sub == 0) {
            v = a.vel[i];
            if (MODE == MODE_STEP) rr = a.rref[i];
        }
        if (active) {
            pi = pos[i];
            if (rec)
                neighbour_loop<TP, NT, true, NC>(a, pos, tab, nt, i, sub, pi, fx, fy, fz, u, w, l);
            else
                neighbour_loop<TP, NT, false, NC>(a, pos, tab, nt, i, sub, pi, fx, fy, fz, u, w, l);
        }
        if (TP > 1) {
#pragma unroll
            for (int o = TP / 2; o > 0; o >>= 1) {
                fx += __shfl_xor_sync(0xffffffffu, fx, o);
                fy += __shfl_xor_sync(0xffffffffu, fy, o);
                fz += __shfl_xor_sync(0xffffffffu, fz, o);
                if (rec) {
                    u += __shfl_xor_sync(0xffffffffu, u, o);
                    w += __shfl_xor_sync(0xffffffffu, w, o);
                    l += __shfl_xor_sync(0xffffffffu, l, o);
                }
            }
        }
        if (active && sub == 0 && a.bond_cnt) bond_forces(a, i, pi, pos, rec, fx, fy, fz, u, w, l);
        if (active && sub == 0)
            finish_particle<INTEG, MODE>(a, i, pi, v, rr, fx, fy, fz, u, w, l, rec, reset, step, shift_pending, shx,
                                         shy, shz, xi, pos_next, red, moved, &ns);
        if (PERSIST) {
            // this round's sums to partials[round]; the next round
            if (full) {
                block_sum<NQ>(red, s_red);
                if (threadIdx.x == 0) {
#pragma unroll
                    for (int q = 0; q < NQ; q++) prow[(size_t)round * NQ + q] = red[q];
                }
            } else if (needk) {
                double rk[1] = {red[0]};
                block_sum<1>(rk, s_red);
                if (threadIdx.x == 0) prow[(size_t)round * NQ] = rk[0];
            }
#pragma unroll
            for (int q = 0; q < NQ; q++) red[q] = 0.0;
            if (dynamic) {
                __syncthreads();  // every thread has read s_round
                if (threadIdx.x == 0) s_round = (int)atomicAdd(&ctrl->work[step & 1], 1u);
                __syncthreads();
                round = s_round;
            } else {
                __syncthreads();  // s_red is free again
                round = rounds_total;
            }
        } else {
            round += g.nb;
        }
    }
    bool block_moved = false;
    if (MODE == MODE_STEP) {
        // inside the persistent kernels other blocks may still be reading
        // ctrl->rebuild for this step: the flag goes to the barrier, which
        // raises it for the next step (the caller)
        block_moved = __syncthreads_or(moved) != 0;
        if (!PERSIST && block_moved && threadIdx.x == 0) ctrl->rebuild = 1;
    }
    if (!PERSIST) {
        block_sum<NQ>(red, s_red);
        if (threadIdx.x == 0) {
#pragma unroll
            for (int q = 0; q < NQ; q++) a.partials[(size_t)g.b * NQ + q] = red[q];
        }
    }
    return block_moved;
}

// Fixed-order float64 sums of `nrows` partial rows (blocks or rounds): every
// column (full) or the kinetic energy alone (needk); the result is valid in
// thread 0.  Each thread sums rows threadIdx.x, + blockDim.x, ... in that
// order; the rows of a batch are loaded before they are added, so several
// loads are in flight (the same sums as one row at a time, bit for bit).
__device__ inline void sum_partial_rows(const double *part, int nrows, bool full, bool needk, double *s_red,
                                        double (&tot)[NQ]) {
#pragma unroll
    for (int q = 0; q < NQ; q++) tot[q] = 0.0;
    const int bs = blockDim.x;
    if (full) {
        int b = threadIdx.x;
        for (; b + 3 * bs < nrows; b += 4 * bs) {
            double v[4][NQ];
#pragma unroll
            for (int u = 0; u < 4; u++)
#pragma unroll
                for (int q = 0; q < NQ; q++) v[u][q] = __ldcg(part + (size_t)(b + u * bs) * NQ + q);
#pragma unroll
            for (int u = 0; u < 4; u++)
#pragma unroll
                for (int q = 0; q < NQ; q++) tot[q] += v[u][q];
        }
        for (; b < nrows; b += bs) {
#pragma unroll
            for (int q = 0; q < NQ; q++) tot[q] += __ldcg(part + (size_t)b * NQ + q);
        }
        block_sum<NQ>(tot, s_red);
    } else if (needk) {
        double t1[1] = {0.0};
        int b = threadIdx.x;
        for (; b + 7 * bs < nrows; b += 8 * bs) {
            double v[8];
#pragma unroll
            for (int u = 0; u < 8; u++) v[u] = __ldcg(part + (size_t)(b + u * bs) * NQ);
#pragma unroll
            for (int u = 0; u < 8; u++) t1[0] += v[u];
        }
        for (; b < nrows; b += bs) t1[0] += __ldcg(part + (size_t)b * NQ);
        block_sum<1>(t1, s_red);
        tot[0] = t1[0];
    }
}

// Nose-Hoover friction after a step with kinetic-energy sum `sumk`
// (NVT.py:113-124).
__device__ __forceinline__ float nose_hoover_next(const SimArgs &a, float xi, double sumk, double time) {
    const double T = target_temperature(a, time);
    const double dev = 2.0 * sumk / ((double)a.dof * T) - 1.0;
    return (float)((double)xi + (double)(a.dt * a.omega2) * dev);
}

// The ScalarSaver row of a recorded step (scalar_saver.py:165-179).
__device__ __forceinline__ void write_scalar_row(const SimArgs &a, int step, const double tot[NQ]) {
    if (step / a.every >= a.nrows) return;
    double *row = a.rows + (size_t)(step / a.every) * GDB_NUM_SCALARS;
    row[GDB_SCALAR_U] = tot[1];
    row[GDB_SCALAR_W] = tot[2];
    row[GDB_SCALAR_LAPU] = tot[3];
    row[GDB_SCALAR_K] = tot[0];
    row[GDB_SCALAR_FSQ] = tot[4];
}

// Fixed-order float64 sum of `nblocks` partial rows (blocks or rounds) and the
// bookkeeping of a finished step (NVT.py:113-124, scalar_saver.py:165-179,
// momentum_reset.py:64-78).  Run by one whole block.
template <int MODE, int INTEG = GDB_INTEGRATOR_NVE>
__device__ inline void finalize_step(const SimArgs &a, int step, int nblocks, double *s_red) {
    DevCtrl *ctrl = a.ctrl;
    const bool rec = MODE == MODE_EVAL || (a.every > 0 && step % a.every == 0);
    const bool reset = MODE == MODE_STEP && a.reset_every > 0 && step % a.reset_every == 0;
    const int par = step & 1, ppar = par ^ 1;
    const bool npt = INTEG == GDB_INTEGRATOR_NPT && MODE == MODE_STEP;
    const bool full = rec || reset || npt;
    const bool needk = full || a.omega2 > 0.f;
    double tot[NQ];
    sum_partial_rows(a.partials, nblocks, full, needk, s_red, tot);
    if (threadIdx.x == 0) {
        if (MODE == MODE_STEP) {
            const double time = ctrl->time_zero + (double)step * (double)a.dt;
            if (npt) {
                // update_thermostat_barostat_state (integrators/NPT_Atomic.py:
                // 138-166) with numba's typing; the float32 accumulators
                // thermostat_state[1] and barostat_state[1] are the float64
                // sums of K and W rounded to float32
                const float ts1 = (float)tot[0], bs1 = (float)tot[2];
                const float bs0 = ctrl->npt_bs0;
                const long long deg = a.dof;
                const double temperature = 2.0 * (double)ts1 / (double)deg;
                const double sf3 = 1.0 + (double)a.dt * 3.0 * (double)bs0;
                const double mass_t = (double)a.npt_mass_t * temperature;
                const double mass_p = (double)a.npt_mass_p * temperature;
                const float vol = (float)((double)ctrl->npt_vol * sf3);
                ctrl->npt_vol = vol;
                const double sf = pow(sf3, 1.0 / 3.0);
                ctrl->box[0] = (float)((double)ctrl->box[0] * sf);
                ctrl->box[1] = (float)((double)ctrl->box[1] * sf);
                ctrl->box[2] = (float)((double)ctrl->box[2] * sf);
                const double T_target = target_temperature(a, time);
                const double P_target = target_pressure(a, time);
                const double p_inst = (temperature * (double)a.n + (double)bs1) / (double)vol;
                const double ke_dev =
                    ((double)(2.0f * ts1) + (double)(bs0 * bs0) * mass_p) / ((double)(deg + 1) * T_target) - 1.0;
                const double p_dev = 3.0 * ((double)vol * (p_inst - P_target) + (double)(0.5f * ts1) / (double)deg);
                const float ts0 = (float)((double)ctrl->npt_ts0 +
                                          (double)a.dt * ke_dev * (double)(deg + 1) * T_target / mass_t);
                ctrl->npt_ts0 = ts0;
                ctrl->npt_bs0 = (float)((double)bs0 + (double)a.dt * (p_dev / mass_p + (double)(ts0 * bs0)));
            } else if (a.omega2 > 0.f) {
                ctrl->xi = nose_hoover_next(a, ctrl->xi, tot[0], time);
            }
            ctrl->sumK = (float)tot[0];
            if (rec) {
                write_scalar_row(a, step, tot);
                if (npt && step / a.every < a.nrows) {  // the saver reads the box the step left (scalar_saver.py:195)
                    float vol = ctrl->box[0];
                    vol *= ctrl->box[1];
                    vol *= ctrl->box[2];
                    a.rows[(size_t)(step / a.every) * GDB_NUM_SCALARS + GDB_SCALAR_VOL] = vol;
                }
            }
            if (reset) {
                ctrl->shift[par][0] = (float)(tot[5] / tot[8]);
                ctrl->shift[par][1] = (float)(tot[6] / tot[8]);
                ctrl->shift[par][2] = (float)(tot[7] / tot[8]);
                ctrl->pending[par] = 1;
            }
            ctrl->step = step + 1;
            ctrl->work[(step + 1) & 1] = 0;  // round counter of the next step (persistent kernels)
        } else {
            ctrl->evalU = tot[1];
            ctrl->evalW = tot[2];
        }
        ctrl->pending[ppar] = 0;
    }
}

// The bookkeeping of finalize_step for a step (not NPT_Atomic) by every block
// of the persistent grid after step_barrier_all: each block sums the same
// rows (part, this step's half of the double-buffered rows) in the same
// order, so each computes the same next control state, into its StepCtl.
// Block 0 also writes that state to ctrl (for the host and the next launch)
// with the scalar row, and clears the round counter of step + 2: every block
// took its last round of this step before it arrived at the barrier.
template <int INTEG>
__device__ inline void finalize_step_all(const SimArgs &a, int step, int nrows, const double *part, double *s_red,
                                         StepCtl *sc, int any) {
    DevCtrl *ctrl = a.ctrl;
    const bool rec = a.every > 0 && step % a.every == 0;
    const bool reset = a.reset_every > 0 && step % a.reset_every == 0;
    const int par = step & 1, ppar = par ^ 1;
    const bool full = rec || reset;
    const bool needk = full || a.omega2 > 0.f;
    double tot[NQ];
    sum_partial_rows(part, nrows, full, needk, s_red, tot);
    if (threadIdx.x == 0) {
        const bool writer = blockIdx.x == 0;
        if (a.omega2 > 0.f) {
            sc->xi = nose_hoover_next(a, sc->xi, tot[0], sc->time_zero + (double)step * (double)a.dt);
            if (writer) ctrl->xi = sc->xi;
        }
        if (reset) {
            sc->shift[par][0] = (float)(tot[5] / tot[8]);
            sc->shift[par][1] = (float)(tot[6] / tot[8]);
            sc->shift[par][2] = (float)(tot[7] / tot[8]);
            sc->pending[par] = 1;
        }
        sc->pending[ppar] = 0;
        sc->step = step + 1;
        sc->rebuild = any;
        if (writer) {
            ctrl->sumK = (float)tot[0];
            if (rec) write_scalar_row(a, step, tot);
            if (reset) {
#pragma unroll
                for (int k = 0; k < 3; k++) ctrl->shift[par][k] = sc->shift[par][k];
                ctrl->pending[par] = 1;
            }
            ctrl->pending[ppar] = 0;
            ctrl->step = step + 1;
            if (any) ctrl->rebuild = 1;
            ctrl->work[step & 1] = 0;
        }
    }
}

}  // namespace gdb
