// md_core.cu -- simulation handle, neighbour lists, fused force+integrate step.
//
// Replaces, B200-native, the numba.cuda kernels of gamdpy's hot path:
//   interactions/pair_potential.py:141-246   (forces, U, W, lapU)
//   interactions/nblist.py:57-143            (N^2 list: check + build)
//   interactions/nblist_linked_lists.py:84-218 (cell list: check, cells, build, clear)
//   integrators/NVE.py:59-105, integrators/NVT.py:188-237
//   runtime_actions/scalar_saver.py:270-304, runtime_actions/momentum_reset.py:372-408
//   simulation/Simulation.py:306-346          (composed step loop)
//
// Design (see the layout notes in gdb_internal.cuh):
//  * One fused kernel per time step: forces of particle i from pos[cur],
//    immediately integrated (leapfrog NVE or Nose-Hoover NVT) and written to
//    pos[cur^1].  Forces never round-trip through HBM.  tp lanes share one
//    particle's neighbour list and combine with warp shuffles.
//  * Reductions (K for the thermostat, ScalarSaver sums, momentum) are float64:
//    per-block partials, then the last block to finish (ticket counter) sums
//    them in a fixed order, updates xi / the saved row / the momentum shift and
//    advances the device step counter.  Runs are bitwise reproducible.
//  * The neighbour-list rebuild is a chain of kernels that return at once
//    unless the step kernel flagged a particle beyond skin/2.  Cell lists use a
//    counting sort (histogram, scan, scatter, in-cell sort by user index) and
//    physically reorder the particles by cell, so neighbour gathers hit L1/L2.
//  * The launch sequence of a chunk of steps is captured once in a CUDA graph
//    and replayed.
#include <cuda_runtime.h>
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <vector>

#include "../../include/gamdb200.h"
#include "gdb_internal.cuh"

using namespace gdb;

namespace {

constexpr int NQ = 9;  // K, U, W, lapU, Fsq, px, py, pz, m
constexpr int SCAN_CHUNK = 2048;
constexpr int MODE_STEP = 0;
constexpr int MODE_EVAL = 1;

char g_lib_error[512] = "";

}  // namespace

struct gdb_sim {
    int n = 0, ntypes = 1, dev = 0;
    cudaStream_t st = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    float box[3] = {1, 1, 1};
    // potential
    int pot_kind = 0, cutmode = 0, nparams = 0;
    std::vector<float> params;
    PairTable table{};
    float max_cut = 0;
    bool have_pot = false;
    // neighbour list
    int nb_kind = GDB_NBLIST_NSQ;
    float skin = 0.5f;
    int max_nbs = 0;
    int tp = 0, tp_req = 0, pb_req = 0;
    int stride = 0;
    int nc[3] = {0, 0, 0};
    int ncell = 0;
    int fma = 1;
    // integrator + actions
    int integ = GDB_INTEGRATOR_NVE;
    float dt = 0.005f, tau = 0.2f, omega2 = 0;
    int tfunc = 0;
    float tparams[4] = {0, 0, 0, 0};
    int scalar_every = 0, momentum_every = 0;
    // device buffers
    float4 *pos[2] = {nullptr, nullptr}, *vel = nullptr, *frc = nullptr, *rref = nullptr;
    float4 *pos_tmp = nullptr, *vel_tmp = nullptr;
    int4 *img = nullptr, *img_tmp = nullptr;
    int *orig = nullptr, *orig_tmp = nullptr;
    int *nbl = nullptr, *nbc = nullptr;
    size_t nbl_elems = 0;
    float *pscal = nullptr, *pscal_tmp = nullptr;  // 5 planes
    int *cell_count = nullptr, *cell_start = nullptr, *pcell = nullptr, *prank = nullptr, *perm = nullptr,
        *scell = nullptr, *bsum = nullptr;
    int cell_cap = 0;
    DevCtrl *ctrl = nullptr;
    DevCtrl *h_ctrl = nullptr;  // pinned mirror
    double *partials = nullptr;
    int partial_cap = 0;
    double *rows = nullptr;
    int rows_cap = 0;
    float *conf = nullptr;  // ConfigurationSaver frames
    int conf_per_block = 0;
    int cur = 0;
    bool uploaded = false;
    // graphs: [parity] for chunks of GRAPH_STEPS steps
    cudaGraphExec_t gexec[2] = {nullptr, nullptr};
    int graph_steps = 0;
    bool use_graphs = true;
    char err[512] = "";
};

// ---------------------------------------------------------------------------
// error helpers
// ---------------------------------------------------------------------------
static int set_err(gdb_sim *h, int code, const char *fmt, ...) {
    char *dst = h ? h->err : g_lib_error;
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(dst, 512, fmt, ap);
    va_end(ap);
    return code;
}

#define CK(call)                                                                              \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess)                                                                \
            return set_err(h, GDB_ERR_CUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                           __FILE__, __LINE__);                                               \
    } while (0)

#define CKL()                                                                                  \
    do {                                                                                       \
        cudaError_t e_ = cudaGetLastError();                                                   \
        if (e_ != cudaSuccess)                                                                 \
            return set_err(h, GDB_ERR_CUDA, "kernel launch failed: %s (%s:%d)", cudaGetErrorString(e_), \
                           __FILE__, __LINE__);                                                \
    } while (0)

// ---------------------------------------------------------------------------
// kernels: neighbour list
// ---------------------------------------------------------------------------

// N^2 build (interactions/nblist.py:88-143): one warp per particle, lanes
// stride over j; ballot + popc append the hits in ascending j, so the list is
// deterministic.  Full list, no exclusions.
template <bool FMA>
__global__ void __launch_bounds__(GDB_BLOCK) k_nbl_nsq(const float4 *__restrict__ pos, int n, float Lx, float Ly,
                                                       float Lz, float cps2, int *__restrict__ nbl,
                                                       int *__restrict__ nbc, int stride, int tp, int max_nbs,
                                                       DevCtrl *ctrl) {
    if (!ctrl->rebuild) return;
    const int lane = threadIdx.x & 31;
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (i >= n) return;
    const float4 pi = pos[i];
    int count = 0;
    for (int j0 = 0; j0 < n; j0 += 32) {
        const int j = j0 + lane;
        bool hit = false;
        if (j < n && j != i) {
            const float4 pj = pos[j];
            hit = dist_sq_exact<FMA>(pj, pi, Lx, Ly, Lz) < cps2;
        }
        const unsigned m = __ballot_sync(0xffffffffu, hit);
        if (hit) {
            const int k = count + __popc(m & ((1u << lane) - 1u));
            if (k < max_nbs) nbl[nb_index(i, k, tp, stride)] = j;
        }
        count += __popc(m);
    }
    if (lane == 0) {
        nbc[i] = count;
        atomicMax(&ctrl->maxcount, count);
    }
}

// Cell coordinate as nblist_linked_lists.py:127 (float64 arithmetic, Python
// modulo).  Non-finite coordinates map to cell 0 and raise the NAN bit.
__device__ __forceinline__ int cell_coord(float x, float L, int nc, DevCtrl *ctrl) {
    double v = ((double)x + 0.5 * (double)L) * (double)nc / (double)L;
    if (!(v > -1e9 && v < 1e9)) {
        atomicOr(&ctrl->status, GDB_STATUS_NAN);
        return 0;
    }
    long long c = (long long)floor(v);
    long long m = c % nc;
    if (m < 0) m += nc;
    return (int)m;
}

__global__ void k_cell_assign(const float4 *__restrict__ pos, int n, float Lx, float Ly, float Lz, int ncx,
                              int ncy, int ncz, int *__restrict__ pcell, int *__restrict__ prank,
                              int *__restrict__ cell_count, DevCtrl *ctrl) {
    if (!ctrl->rebuild) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 p = pos[i];
    const int cx = cell_coord(p.x, Lx, ncx, ctrl);
    const int cy = cell_coord(p.y, Ly, ncy, ctrl);
    const int cz = cell_coord(p.z, Lz, ncz, ctrl);
    // linear index with x fastest: the x-neighbours of a cell are contiguous
    const int c = (cz * ncy + cy) * ncx + cx;
    pcell[i] = c;
    prank[i] = atomicAdd(&cell_count[c], 1);
}

// Block-wide exclusive scan of SCAN_CHUNK ints (8 per thread).
__device__ __forceinline__ void chunk_scan(const int *in, int len, int base, int *out_excl, int add, int *total,
                                           int *sm /* 32 */) {
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    int v[8];
    int s = 0;
#pragma unroll
    for (int q = 0; q < 8; q++) {
        const int idx = base + t * 8 + q;
        v[q] = idx < len ? in[idx] : 0;
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
        int w = lane < (int)(blockDim.x >> 5) ? sm[lane] : 0;
        int wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += y;
        }
        sm[lane] = wi - w;  // exclusive prefix of warp totals
        if (lane == 31 && total) *total = wi;
    }
    __syncthreads();
    if (out_excl) {
        int run = add + sm[warp] + incl - s;
#pragma unroll
        for (int q = 0; q < 8; q++) {
            const int idx = base + t * 8 + q;
            if (idx < len) out_excl[idx] = run;
            run += v[q];
        }
    }
    __syncthreads();
}

__global__ void __launch_bounds__(GDB_BLOCK) k_scan_partial(const int *__restrict__ in, int len, int *__restrict__ bsum,
                                                            DevCtrl *ctrl) {
    if (!ctrl->rebuild) return;
    __shared__ int sm[32];
    __shared__ int tot;
    chunk_scan(in, len, blockIdx.x * SCAN_CHUNK, nullptr, 0, &tot, sm);
    if (threadIdx.x == 0) bsum[blockIdx.x] = tot;
}

// Exclusive scan of the block sums in one block (nb <= 8 * 1024 * ... handled
// by looping over chunks serially).
__global__ void __launch_bounds__(GDB_BLOCK) k_scan_top(int *__restrict__ bsum, int nb, DevCtrl *ctrl) {
    if (!ctrl->rebuild) return;
    __shared__ int sm[32];
    __shared__ int tot;
    int carry = 0;
    for (int base = 0; base < nb; base += SCAN_CHUNK) {
        chunk_scan(bsum, nb, base, bsum, carry, &tot, sm);
        carry += tot;
        __syncthreads();
    }
}

__global__ void __launch_bounds__(GDB_BLOCK) k_scan_final(const int *__restrict__ in, int len,
                                                          const int *__restrict__ bsum, int *__restrict__ out,
                                                          int n, DevCtrl *ctrl) {
    if (!ctrl->rebuild) return;
    __shared__ int sm[32];
    chunk_scan(in, len, blockIdx.x * SCAN_CHUNK, out, bsum[blockIdx.x], nullptr, sm);
    if (blockIdx.x == 0 && threadIdx.x == 0) out[len] = n;
}

__global__ void k_scatter(const int *__restrict__ pcell, const int *__restrict__ prank,
                          const int *__restrict__ cell_start, int *__restrict__ perm, int n, DevCtrl *ctrl) {
    if (!ctrl->rebuild) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    perm[cell_start[pcell[i]] + prank[i]] = i;
}

// Order every cell's particles by user index: the atomics of k_cell_assign
// rank them arbitrarily, this makes the layout (and every sum) deterministic.
__global__ void k_sort_cells(const int *__restrict__ cell_start, int ncell, int *__restrict__ perm,
                             const int *__restrict__ orig, DevCtrl *ctrl) {
    if (!ctrl->rebuild) return;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncell) return;
    const int a = cell_start[c], b = cell_start[c + 1];
    for (int x = a + 1; x < b; x++) {
        const int v = perm[x];
        const int key = orig[v];
        int y = x - 1;
        while (y >= a && orig[perm[y]] > key) {
            perm[y + 1] = perm[y];
            y--;
        }
        perm[y + 1] = v;
    }
}

__global__ void k_gather(const int *__restrict__ perm, int n, const float4 *__restrict__ pos,
                         const float4 *__restrict__ vel, const int4 *__restrict__ img, const int *__restrict__ orig,
                         const float *__restrict__ pscal, const int *__restrict__ pcell, float4 *__restrict__ pos_t,
                         float4 *__restrict__ vel_t, int4 *__restrict__ img_t, int *__restrict__ orig_t,
                         float *__restrict__ pscal_t, int *__restrict__ scell, DevCtrl *ctrl) {
    if (!ctrl->rebuild) return;
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const int i = perm[s];
    pos_t[s] = pos[i];
    vel_t[s] = vel[i];
    img_t[s] = img[i];
    orig_t[s] = orig[i];
    scell[s] = pcell[i];
    // K and Fsq planes (3, 4) travel with the particle; U, W, lapU are rewritten
    // by the next force evaluation
    pscal_t[3 * (size_t)n + s] = pscal[3 * (size_t)n + i];
    pscal_t[4 * (size_t)n + s] = pscal[4 * (size_t)n + i];
}

// Cell-list build (nblist_linked_lists.py:133-183 semantics: every particle
// of the 5x5x5 stencil of cells with dist_sq < (max_cut+skin)^2, j != i).
// Particles are sorted by cell with x fastest, so the five x-cells of one
// (dy, dz) row are one contiguous slot range (two at the x wrap).  Grids with
// fewer than five cells in a dimension visit each cell once.
template <bool FMA>
__global__ void __launch_bounds__(GDB_BLOCK) k_nbl_cells(const float4 *__restrict__ pos, const int *__restrict__ scell,
                                                         const int *__restrict__ cell_start, int n, float Lx, float Ly,
                                                         float Lz, int ncx, int ncy, int ncz, float cps2,
                                                         int *__restrict__ nbl, int *__restrict__ nbc, int stride,
                                                         int tp, int max_nbs, DevCtrl *ctrl) {
    if (!ctrl->rebuild) return;
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const float4 pi = pos[s];
    const int c = scell[s];
    const int cx = c % ncx, cy = (c / ncx) % ncy, cz = c / (ncx * ncy);
    const int ry = ncy < 5 ? ncy : 5, rz = ncz < 5 ? ncz : 5;
    const int oy = ncy < 5 ? 0 : cy - 2, oz = ncz < 5 ? 0 : cz - 2;
    int count = 0;
    for (int a = 0; a < rz; a++) {
        int z = oz + a;
        z = (z % ncz + ncz) % ncz;
        for (int b = 0; b < ry; b++) {
            int y = oy + b;
            y = (y % ncy + ncy) % ncy;
            const int rowbase = (z * ncy + y) * ncx;
            // x segments
            int seg_lo[2], seg_hi[2], nseg;
            if (ncx <= 5) {
                seg_lo[0] = rowbase;
                seg_hi[0] = rowbase + ncx;
                nseg = 1;
            } else {
                const int x0 = cx - 2, x1 = cx + 2;
                if (x0 >= 0 && x1 < ncx) {
                    seg_lo[0] = rowbase + x0;
                    seg_hi[0] = rowbase + x1 + 1;
                    nseg = 1;
                } else if (x0 < 0) {
                    seg_lo[0] = rowbase + x0 + ncx;
                    seg_hi[0] = rowbase + ncx;
                    seg_lo[1] = rowbase;
                    seg_hi[1] = rowbase + x1 + 1;
                    nseg = 2;
                } else {
                    seg_lo[0] = rowbase + x0;
                    seg_hi[0] = rowbase + ncx;
                    seg_lo[1] = rowbase;
                    seg_hi[1] = rowbase + x1 - ncx + 1;
                    nseg = 2;
                }
            }
            for (int q = 0; q < nseg; q++) {
                const int j0 = cell_start[seg_lo[q]], j1 = cell_start[seg_hi[q]];
                for (int j = j0; j < j1; j++) {
                    if (j == s) continue;
                    const float4 pj = pos[j];
                    if (dist_sq_exact<FMA>(pj, pi, Lx, Ly, Lz) < cps2) {
                        if (count < max_nbs) nbl[nb_index(s, count, tp, stride)] = j;
                        count++;
                    }
                }
            }
        }
    }
    nbc[s] = count;
    atomicMax(&ctrl->maxcount, count);
}

// Last kernel of a rebuild: move the reordered state into place (cell mode),
// record r_ref, clear the cell counters for the next build, and (last block)
// clear the rebuild flag and count the build (gamdpy nbflag[0], nbflag[2]).
template <bool CELLS>
__global__ void k_rebuild_finish(int n, float4 *__restrict__ pos, float4 *__restrict__ vel, int4 *__restrict__ img,
                                 int *__restrict__ orig, float *__restrict__ pscal, const float4 *__restrict__ pos_t,
                                 const float4 *__restrict__ vel_t, const int4 *__restrict__ img_t,
                                 const int *__restrict__ orig_t, const float *__restrict__ pscal_t,
                                 float4 *__restrict__ rref, int *__restrict__ cell_count, int ncell,
                                 DevCtrl *ctrl) {
    __shared__ bool last;
    if (!ctrl->rebuild) return;
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < n) {
        if (CELLS) {
            const float4 p = pos_t[s];
            pos[s] = p;
            rref[s] = p;
            vel[s] = vel_t[s];
            img[s] = img_t[s];
            orig[s] = orig_t[s];
            pscal[3 * (size_t)n + s] = pscal_t[3 * (size_t)n + s];
            pscal[4 * (size_t)n + s] = pscal_t[4 * (size_t)n + s];
        } else {
            rref[s] = pos[s];
        }
    }
    if (CELLS)
        for (int c = s; c < ncell; c += gridDim.x * blockDim.x) cell_count[c] = 0;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(&ctrl->ticket2, 1u) == gridDim.x - 1;
    __syncthreads();
    if (last && threadIdx.x == 0) {
        ctrl->rebuild = 0;
        ctrl->nrebuild += 1;
        ctrl->ticket2 = 0;
    }
}

// ---------------------------------------------------------------------------
// kernels: fused force + integrate step
// ---------------------------------------------------------------------------
struct StepArgs {
    const float4 *pos;
    float4 *pos_next;
    float4 *vel;
    int4 *img;
    const float4 *rref;
    float4 *frc;
    const int *nbl;
    const int *nbc;
    float *pscal;
    double *partials;
    double *rows;
    DevCtrl *ctrl;
    int n, stride, max_nbs;
    float Lx, Ly, Lz;
    float skin2q;  // skin*skin*0.25 (nblist.py / orthorhombic.py:131)
    float dt;
    float omega2;
    long long dof;  // N*D - D (NVT.py:35)
    int tfunc;
    float tp0, tp1, tp2, tp3;
    int every, reset_every;
    int nrows;            // ScalarSaver rows allocated (writes beyond are dropped)
    float *conf;          // ConfigurationSaver frames (conf_per_block, 2, n, 3) or null
    int conf_per_block;
    const int *orig;      // user index of each slot
};

// ConfigurationSaver save slot of a step (runtime_actions/configuration_saver.py:
// 115-141): step 0 -> 0, step 2^b -> b + 1, others -> -1.
__device__ __forceinline__ int conf_save_index(int step) {
    if (step == 0) return 0;
    if (step & (step - 1)) return -1;
    return 32 - __clz(step);
}

__device__ __forceinline__ double target_temperature(const StepArgs &a, double t) {
    if (a.tfunc == GDB_TFUNC_RAMP) {  // misc/make_function.py:27-32
        if (t < a.tp1) return a.tp0;
        if (t < a.tp3) return a.tp0 + (t - a.tp1) * ((double)(a.tp2 - a.tp0) / (double)(a.tp3 - a.tp1));
        return a.tp2;
    }
    return a.tp0;
}

// Loop over particle i's neighbours (lane `sub` of TP): pair_potential.py:223-231
// with the full-list calculator :164-178.
template <int TP, bool NT1, bool REC>
__device__ __forceinline__ void neighbour_loop(const StepArgs &a, const PairEntry *tab, int nt, int i, int sub,
                                               float4 pi, float &fx, float &fy, float &fz, float &u, float &w,
                                               float &l) {
    const int ti = NT1 ? 0 : ptype_of(pi);
    const int cnt = min(a.nbc[i], a.max_nbs);
    const int *row = a.nbl + (size_t)i * TP + sub;
    const size_t slice = (size_t)a.stride * TP;
    const PairEntry *trow = tab + ti * nt;
    const float Lx = a.Lx, Ly = a.Ly, Lz = a.Lz;
    const float hLx = 0.5f * Lx, hLy = 0.5f * Ly, hLz = 0.5f * Lz;
    int kk = 0;
#pragma unroll 2
    for (int k = sub; k < cnt; k += TP, kk++) {
        const int j = __ldg(row + kk * slice);
        const float4 pj = __ldg(a.pos + j);
        float dx = pj.x - pi.x, dy = pj.y - pi.y, dz = pj.z - pi.z;
        dx = dx > hLx ? dx - Lx : (dx < -hLx ? dx + Lx : dx);
        dy = dy > hLy ? dy - Ly : (dy < -hLy ? dy + Ly : dy);
        dz = dz > hLz ? dz - Lz : (dz < -hLz ? dz + Lz : dz);
        const float d2 = dx * dx + dy * dy + dz * dz;
        const PairEntry &e = NT1 ? tab[0] : trow[ptype_of(pj)];
        if (d2 < e.cut2) {
            const float inv2 = __fdividef(1.0f, d2);
            const float x2 = e.c * inv2;
            const float x6 = x2 * x2 * x2;
            const float x12 = x6 * x6;
            const float s = (e.cs12 * x12 + e.cs6 * x6) * inv2 - e.sc;
            fx -= dx * s;
            fy -= dy * s;
            fz -= dz * s;
            if (REC) {
                const float r = sqrtf(d2);
                const float uu = e.cu12 * x12 + e.cu6 * x6 - e.uc + e.sccut * (r - e.cut);
                u += 0.5f * uu;
                w += d2 * s * (1.0f / 6.0f);
                l += -2.0f * s + (e.cm12 * x12 + e.cm6 * x6) * inv2;
            }
        }
    }
}

template <int TP, bool NT1, int INTEG, int MODE>
__global__ void __launch_bounds__(GDB_BLOCK) k_step(StepArgs a, PairTable tab) {
    __shared__ PairEntry s_tab[NT1 ? 1 : GDB_MAX_TYPES * GDB_MAX_TYPES];
    __shared__ double s_red[NQ * 32];
    __shared__ bool s_last;
    const int nt = tab.nt;
    if (NT1) {
        if (threadIdx.x == 0) s_tab[0] = tab.e[0];
    } else {
        for (int t = threadIdx.x; t < nt * nt; t += blockDim.x) s_tab[t] = tab.e[t];
    }
    __syncthreads();

    DevCtrl *ctrl = a.ctrl;
    const int step = ctrl->step;
    const bool rec = MODE == MODE_EVAL || (a.every > 0 && step % a.every == 0);
    const bool reset = MODE == MODE_STEP && a.reset_every > 0 && step % a.reset_every == 0;
    const int par = step & 1, ppar = par ^ 1;
    const bool shift_pending = ctrl->pending[ppar] != 0;

    const int gt = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = gt / TP, sub = gt % TP;
    const bool active = i < a.n;
    const size_t n = a.n;
    float fx = 0.f, fy = 0.f, fz = 0.f, u = 0.f, w = 0.f, l = 0.f;
    float4 pi = make_float4(0.f, 0.f, 0.f, 0.f);
    if (active) {
        pi = a.pos[i];
        if (rec)
            neighbour_loop<TP, NT1, true>(a, s_tab, nt, i, sub, pi, fx, fy, fz, u, w, l);
        else
            neighbour_loop<TP, NT1, false>(a, s_tab, nt, i, sub, pi, fx, fy, fz, u, w, l);
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

    double red[NQ];
#pragma unroll
    for (int q = 0; q < NQ; q++) red[q] = 0.0;
    bool moved = false;
    if (active && sub == 0 && a.conf) {
        const int si = conf_save_index(step);
        if (si >= 0 && si < a.conf_per_block) {
            const int4 im = a.img[i];
            const int u = a.orig[i];
            float *fr = a.conf + ((size_t)si * 2) * n * 3;
            fr[3 * (size_t)u] = pi.x;
            fr[3 * (size_t)u + 1] = pi.y;
            fr[3 * (size_t)u + 2] = pi.z;
            fr += n * 3;
            fr[3 * (size_t)u] = (float)im.x;
            fr[3 * (size_t)u + 1] = (float)im.y;
            fr[3 * (size_t)u + 2] = (float)im.z;
        }
    }
    if (active && sub == 0) {
        float4 v = a.vel[i];
        if (shift_pending) {
            const float *sh = ctrl->shift[ppar];
            v.x -= sh[0];
            v.y -= sh[1];
            v.z -= sh[2];
        }
        const float fsq = fx * fx + fy * fy + fz * fz;
        if (rec) {
            a.pscal[i] = u;
            a.pscal[n + i] = w;
            a.pscal[2 * n + i] = l;
        }
        if (MODE == MODE_EVAL) {
            a.frc[i] = make_float4(fx, fy, fz, 0.f);
            if (shift_pending) a.vel[i] = v;
        } else {
            const float m = v.w;
            float kin;
            float r[3] = {pi.x, pi.y, pi.z};
            float vv[3] = {v.x, v.y, v.z};
            const float ff[3] = {fx, fy, fz};
            if (INTEG == GDB_INTEGRATOR_NVE) {  // integrators/NVE.py:78-97
                kin = 0.f;
#pragma unroll
                for (int k = 0; k < 3; k++) {
                    float v_mean = vv[k];
                    vv[k] += ff[k] / m * a.dt;
                    v_mean += vv[k];
                    v_mean *= 0.5f;
                    kin += 0.5f * m * v_mean * v_mean;
                    r[k] += vv[k] * a.dt;
                }
            } else {  // integrators/NVT.py:196-215
                const float factor = 0.5f * ctrl->xi * a.dt;
                const float plus = 1.0f / (1.0f + factor);
                const float minus = 1.0f - factor;
                kin = 0.f;
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
            if (!(fabsf(r[0]) <= L[0] && fabsf(r[1]) <= L[1] && fabsf(r[2]) <= L[2]))
                atomicOr(&ctrl->status, GDB_STATUS_NAN);
            const float4 pn = make_float4(r[0], r[1], r[2], pi.w);
            a.pos_next[i] = pn;
            a.vel[i] = make_float4(vv[0], vv[1], vv[2], m);
            a.pscal[3 * n + i] = kin;
            a.pscal[4 * n + i] = fsq;
            // skin check for the next step (nblist.py:57-86)
            const float4 rr = a.rref[i];
            moved = dist_sq_exact<false>(pn, rr, a.Lx, a.Ly, a.Lz) > a.skin2q;
            red[0] = kin;
            red[5] = (double)m * vv[0];
            red[6] = (double)m * vv[1];
            red[7] = (double)m * vv[2];
            red[8] = m;
        }
        red[1] = u;
        red[2] = w;
        red[3] = l;
        red[4] = fsq;
    }
    if (MODE == MODE_STEP) {
        if (__syncthreads_or(moved) && threadIdx.x == 0) ctrl->rebuild = 1;
    }
    const bool need_red = MODE == MODE_STEP && (INTEG == GDB_INTEGRATOR_NVT || rec || reset);
    if (need_red) {
        block_sum<NQ>(red, s_red);
        if (threadIdx.x == 0) {
#pragma unroll
            for (int q = 0; q < NQ; q++) a.partials[(size_t)blockIdx.x * NQ + q] = red[q];
        }
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) s_last = atomicAdd(&ctrl->ticket, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!s_last) return;

    // last block: fixed-order float64 reduction of the partials
    double tot[NQ];
#pragma unroll
    for (int q = 0; q < NQ; q++) tot[q] = 0.0;
    if (need_red) {
        for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) {
#pragma unroll
            for (int q = 0; q < NQ; q++) tot[q] += __ldcg(a.partials + (size_t)b * NQ + q);
        }
        block_sum<NQ>(tot, s_red);
    }
    if (threadIdx.x == 0) {
        if (MODE == MODE_STEP) {
            const double time = ctrl->time_zero + (double)step * (double)a.dt;
            if (INTEG == GDB_INTEGRATOR_NVT) {  // NVT.py:226-237
                const double T = target_temperature(a, time);
                const double dev = 2.0 * tot[0] / ((double)a.dof * T) - 1.0;
                ctrl->xi = (float)((double)ctrl->xi + (double)(a.dt * a.omega2) * dev);
                ctrl->sumK = (float)tot[0];
            }
            if (rec && step / a.every < a.nrows) {  // scalar_saver.py:274-288
                double *row = a.rows + (size_t)(step / a.every) * GDB_NUM_SCALARS;
                row[GDB_SCALAR_U] = tot[1];
                row[GDB_SCALAR_W] = tot[2];
                row[GDB_SCALAR_LAPU] = tot[3];
                row[GDB_SCALAR_K] = tot[0];
                row[GDB_SCALAR_FSQ] = tot[4];
            }
            if (reset) {  // momentum_reset.py:379-393
                ctrl->shift[par][0] = (float)(tot[5] / tot[8]);
                ctrl->shift[par][1] = (float)(tot[6] / tot[8]);
                ctrl->shift[par][2] = (float)(tot[7] / tot[8]);
                ctrl->pending[par] = 1;
            }
            ctrl->step = step + 1;
        }
        ctrl->pending[ppar] = 0;
        ctrl->ticket = 0;
    }
}

__global__ void k_block_begin(DevCtrl *ctrl, double time_zero) {
    ctrl->step = 0;
    ctrl->time_zero = time_zero;
}

// upload helpers: gamdpy layout -> float4 / int4
__global__ void k_pack(int n, const float *r, const float *v, const float *m, const int *pt, const int *im,
                       float4 *pos, float4 *vel, int4 *img, int *orig) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    pos[i] = make_float4(r[3 * i], r[3 * i + 1], r[3 * i + 2], __int_as_float(pt[i]));
    vel[i] = make_float4(v[3 * i], v[3 * i + 1], v[3 * i + 2], m[i]);
    img[i] = im ? make_int4(im[3 * i], im[3 * i + 1], im[3 * i + 2], 0) : make_int4(0, 0, 0, 0);
    orig[i] = i;
}

// download helper: internal order float4 -> user order (N,3)
__global__ void k_unpack3(int n, const float4 *src, const int *orig, float *dst) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const float4 p = src[s];
    const int i = orig[s];
    dst[3 * i] = p.x;
    dst[3 * i + 1] = p.y;
    dst[3 * i + 2] = p.z;
}
__global__ void k_unpack3i(int n, const int4 *src, const int *orig, int *dst) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const int4 p = src[s];
    const int i = orig[s];
    dst[3 * i] = p.x;
    dst[3 * i + 1] = p.y;
    dst[3 * i + 2] = p.z;
}
__global__ void k_unpack1(int n, const float *src, const int *orig, float *dst) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    dst[orig[s]] = src[s];
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
static int grid_for(long long threads, int block = GDB_BLOCK) { return (int)((threads + block - 1) / block); }

static void build_table(gdb_sim *h) {
    PairTable &T = h->table;
    T.nt = h->ntypes;
    T.cutmode = h->cutmode;
    h->max_cut = 0;
    for (int a = 0; a < h->ntypes * h->ntypes; a++) {
        const float *p = &h->params[(size_t)a * h->nparams];
        PairEntry &e = T.e[a];
        const double p0 = p[0], p1 = p[1], cut = p[h->nparams - 1];
        if (h->pot_kind == GDB_POT_LJ_12_6) {
            e.c = 1.0f;
            e.cu12 = (float)p0;
            e.cu6 = (float)p1;
            e.cs12 = (float)(12.0 * p0);
            e.cs6 = (float)(6.0 * p1);
            e.cm12 = (float)(156.0 * p0);
            e.cm6 = (float)(42.0 * p1);
        } else {
            e.c = (float)(p0 * p0);
            e.cu12 = (float)(4.0 * p1);
            e.cu6 = (float)(-4.0 * p1);
            e.cs12 = (float)(48.0 * p1);
            e.cs6 = (float)(-24.0 * p1);
            e.cm12 = (float)(624.0 * p1);
            e.cm6 = (float)(-168.0 * p1);
        }
        e.cut = (float)cut;
        e.cut2 = p[h->nparams - 1] * p[h->nparams - 1];
        // potential and s at the cut (float64, then rounded)
        const double i2 = 1.0 / (cut * cut);
        const double x2 = (h->pot_kind == GDB_POT_LJ_12_6 ? 1.0 : p0 * p0) * i2;
        const double x6 = x2 * x2 * x2, x12 = x6 * x6;
        double uc, sc;
        if (h->pot_kind == GDB_POT_LJ_12_6) {
            uc = p0 * x12 + p1 * x6;
            sc = (12.0 * p0 * x12 + 6.0 * p1 * x6) * i2;
        } else {
            uc = 4.0 * p1 * (x12 - x6);
            sc = 24.0 * p1 * (2.0 * x12 - x6) * i2;
        }
        e.uc = (float)uc;
        if (h->cutmode == GDB_CUT_SHIFTED_FORCE) {
            e.sc = (float)sc;
            e.sccut = (float)(sc * cut);
        } else {
            e.sc = 0.f;
            e.sccut = 0.f;
        }
        if ((float)cut > h->max_cut) h->max_cut = (float)cut;
    }
}

static void free_graphs(gdb_sim *h) {
    for (int p = 0; p < 2; p++)
        if (h->gexec[p]) {
            cudaGraphExecDestroy(h->gexec[p]);
            h->gexec[p] = nullptr;
        }
}

static int choose_tp(const gdb_sim *h) {
    if (h->tp_req > 0) return h->tp_req;
    // enough lanes for ~1.5 waves of 148 SMs x 2048 threads
    const long long want = 148LL * 2048;
    int tp = 1;
    while (tp < 8 && (long long)h->n * tp < want) tp *= 2;
    return tp;
}

static int ensure_nblist(gdb_sim *h) {
    const int tp = choose_tp(h);
    const int stride = (h->n + 31) / 32 * 32;
    const size_t need = (size_t)(h->max_nbs + tp) * stride;
    if (tp != h->tp || need > h->nbl_elems) {
        if (h->nbl) cudaFree(h->nbl);
        h->nbl = nullptr;
        CK(cudaMalloc(&h->nbl, need * sizeof(int)));
        h->nbl_elems = need;
        h->tp = tp;
        h->stride = stride;
        free_graphs(h);
        if (h->uploaded) CK(cudaMemsetAsync(&h->ctrl->rebuild, 0xff, sizeof(int), h->st));  // nonzero
    }
    h->stride = stride;
    if (h->nb_kind == GDB_NBLIST_CELLS) {
        // cells per dimension as nblist_linked_lists.py:36-39
        const float min_cell = (h->max_cut + h->skin) / 2.0f;
        int nc[3];
        for (int k = 0; k < 3; k++) {
            nc[k] = (int)(h->box[k] / min_cell);
            if (nc[k] < 1) nc[k] = 1;
        }
        const int ncell = nc[0] * nc[1] * nc[2];
        if (ncell > h->cell_cap) {
            if (h->cell_count) cudaFree(h->cell_count);
            if (h->cell_start) cudaFree(h->cell_start);
            if (h->bsum) cudaFree(h->bsum);
            h->cell_count = h->cell_start = h->bsum = nullptr;
            CK(cudaMalloc(&h->cell_count, (size_t)ncell * sizeof(int)));
            CK(cudaMalloc(&h->cell_start, ((size_t)ncell + 1) * sizeof(int)));
            CK(cudaMalloc(&h->bsum, ((size_t)ncell / SCAN_CHUNK + 2) * sizeof(int)));
            CK(cudaMemsetAsync(h->cell_count, 0, (size_t)ncell * sizeof(int), h->st));
            h->cell_cap = ncell;
        }
        if (nc[0] != h->nc[0] || nc[1] != h->nc[1] || nc[2] != h->nc[2]) free_graphs(h);
        memcpy(h->nc, nc, sizeof(nc));
        h->ncell = ncell;
    }
    return GDB_OK;
}

static int ensure_partials(gdb_sim *h, int nblocks) {
    if (nblocks > h->partial_cap) {
        if (h->partials) cudaFree(h->partials);
        h->partials = nullptr;
        CK(cudaMalloc(&h->partials, (size_t)nblocks * NQ * sizeof(double)));
        h->partial_cap = nblocks;
        free_graphs(h);
    }
    return GDB_OK;
}

// Enqueue the (flag-gated) rebuild chain for the current buffer.
static int enqueue_rebuild(gdb_sim *h) {
    const int n = h->n;
    const float cps = h->max_cut + h->skin;  // nblist.py:152 (max_cut+skin, float32)
    const float cps2 = cps * cps;
    const float4 *pos = h->pos[h->cur];
    if (h->nb_kind == GDB_NBLIST_NSQ) {
        if (h->fma)
            k_nbl_nsq<true><<<grid_for((long long)n * 32), GDB_BLOCK, 0, h->st>>>(
                pos, n, h->box[0], h->box[1], h->box[2], cps2, h->nbl, h->nbc, h->stride, h->tp, h->max_nbs, h->ctrl);
        else
            k_nbl_nsq<false><<<grid_for((long long)n * 32), GDB_BLOCK, 0, h->st>>>(
                pos, n, h->box[0], h->box[1], h->box[2], cps2, h->nbl, h->nbc, h->stride, h->tp, h->max_nbs, h->ctrl);
        CKL();
        k_rebuild_finish<false><<<grid_for(n), GDB_BLOCK, 0, h->st>>>(
            n, h->pos[h->cur], h->vel, h->img, h->orig, h->pscal, nullptr, nullptr, nullptr, nullptr, nullptr, h->rref,
            nullptr, 0, h->ctrl);
        CKL();
        return GDB_OK;
    }
    const int ncell = h->ncell;
    const int nchunks = (ncell + SCAN_CHUNK - 1) / SCAN_CHUNK;
    k_cell_assign<<<grid_for(n), GDB_BLOCK, 0, h->st>>>(pos, n, h->box[0], h->box[1], h->box[2], h->nc[0], h->nc[1],
                                                        h->nc[2], h->pcell, h->prank, h->cell_count, h->ctrl);
    CKL();
    k_scan_partial<<<nchunks, GDB_BLOCK, 0, h->st>>>(h->cell_count, ncell, h->bsum, h->ctrl);
    CKL();
    k_scan_top<<<1, GDB_BLOCK, 0, h->st>>>(h->bsum, nchunks, h->ctrl);
    CKL();
    k_scan_final<<<nchunks, GDB_BLOCK, 0, h->st>>>(h->cell_count, ncell, h->bsum, h->cell_start, n, h->ctrl);
    CKL();
    k_scatter<<<grid_for(n), GDB_BLOCK, 0, h->st>>>(h->pcell, h->prank, h->cell_start, h->perm, n, h->ctrl);
    CKL();
    k_sort_cells<<<grid_for(ncell), GDB_BLOCK, 0, h->st>>>(h->cell_start, ncell, h->perm, h->orig, h->ctrl);
    CKL();
    k_gather<<<grid_for(n), GDB_BLOCK, 0, h->st>>>(h->perm, n, pos, h->vel, h->img, h->orig, h->pscal, h->pcell,
                                                   h->pos_tmp, h->vel_tmp, h->img_tmp, h->orig_tmp, h->pscal_tmp,
                                                   h->scell, h->ctrl);
    CKL();
    if (h->fma)
        k_nbl_cells<true><<<grid_for(n), GDB_BLOCK, 0, h->st>>>(
            h->pos_tmp, h->scell, h->cell_start, n, h->box[0], h->box[1], h->box[2], h->nc[0], h->nc[1], h->nc[2], cps2,
            h->nbl, h->nbc, h->stride, h->tp, h->max_nbs, h->ctrl);
    else
        k_nbl_cells<false><<<grid_for(n), GDB_BLOCK, 0, h->st>>>(
            h->pos_tmp, h->scell, h->cell_start, n, h->box[0], h->box[1], h->box[2], h->nc[0], h->nc[1], h->nc[2], cps2,
            h->nbl, h->nbc, h->stride, h->tp, h->max_nbs, h->ctrl);
    CKL();
    k_rebuild_finish<true><<<grid_for(n), GDB_BLOCK, 0, h->st>>>(
        n, h->pos[h->cur], h->vel, h->img, h->orig, h->pscal, h->pos_tmp, h->vel_tmp, h->img_tmp, h->orig_tmp,
        h->pscal_tmp, h->rref, h->cell_count, ncell, h->ctrl);
    CKL();
    return GDB_OK;
}

static StepArgs make_args(gdb_sim *h, int mode) {
    StepArgs a;
    a.pos = h->pos[h->cur];
    a.pos_next = h->pos[h->cur ^ 1];
    a.vel = h->vel;
    a.img = h->img;
    a.rref = h->rref;
    a.frc = h->frc;
    a.nbl = h->nbl;
    a.nbc = h->nbc;
    a.pscal = h->pscal;
    a.partials = h->partials;
    a.rows = h->rows;
    a.ctrl = h->ctrl;
    a.n = h->n;
    a.stride = h->stride;
    a.max_nbs = h->max_nbs;
    a.Lx = h->box[0];
    a.Ly = h->box[1];
    a.Lz = h->box[2];
    a.skin2q = h->skin * h->skin * 0.25f;
    a.dt = h->dt;
    a.omega2 = h->omega2;
    a.dof = 3LL * h->n - 3;
    a.tfunc = h->tfunc;
    a.tp0 = h->tparams[0];
    a.tp1 = h->tparams[1];
    a.tp2 = h->tparams[2];
    a.tp3 = h->tparams[3];
    a.every = h->scalar_every;
    a.reset_every = h->momentum_every;
    a.nrows = h->rows ? h->rows_cap : 0;
    a.conf = h->conf;
    a.conf_per_block = h->conf_per_block;
    a.orig = h->orig;
    (void)mode;
    return a;
}

template <int TP, bool NT1>
static void launch_step_tp(gdb_sim *h, const StepArgs &a, int mode, int grid) {
    if (mode == MODE_EVAL)
        k_step<TP, NT1, 0, MODE_EVAL><<<grid, GDB_BLOCK, 0, h->st>>>(a, h->table);
    else if (h->integ == GDB_INTEGRATOR_NVT)
        k_step<TP, NT1, GDB_INTEGRATOR_NVT, MODE_STEP><<<grid, GDB_BLOCK, 0, h->st>>>(a, h->table);
    else
        k_step<TP, NT1, GDB_INTEGRATOR_NVE, MODE_STEP><<<grid, GDB_BLOCK, 0, h->st>>>(a, h->table);
}

template <bool NT1>
static void launch_step_nt(gdb_sim *h, const StepArgs &a, int mode, int grid) {
    switch (h->tp) {
        case 1: launch_step_tp<1, NT1>(h, a, mode, grid); break;
        case 2: launch_step_tp<2, NT1>(h, a, mode, grid); break;
        case 4: launch_step_tp<4, NT1>(h, a, mode, grid); break;
        default: launch_step_tp<8, NT1>(h, a, mode, grid); break;
    }
}

static int enqueue_step(gdb_sim *h, int mode) {
    const int grid = grid_for((long long)h->n * h->tp);
    int rc = ensure_partials(h, grid);
    if (rc) return rc;
    StepArgs a = make_args(h, mode);
    if (h->ntypes == 1)
        launch_step_nt<true>(h, a, mode, grid);
    else
        launch_step_nt<false>(h, a, mode, grid);
    CKL();
    if (mode == MODE_STEP) h->cur ^= 1;
    return GDB_OK;
}

static int check_ready(gdb_sim *h) {
    if (!h) return set_err(nullptr, GDB_ERR_ARG, "NULL handle");
    if (!h->uploaded) return set_err(h, GDB_ERR_STATE, "state not uploaded");
    if (!h->have_pot) return set_err(h, GDB_ERR_STATE, "pair potential not set");
    if (h->max_nbs <= 0) return set_err(h, GDB_ERR_STATE, "neighbour list not configured");
    CK(cudaSetDevice(h->dev));
    return ensure_nblist(h);
}

static int read_ctrl(gdb_sim *h) {
    CK(cudaMemcpyAsync(h->h_ctrl, h->ctrl, sizeof(DevCtrl), cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    return GDB_OK;
}

static int status_to_rc(gdb_sim *h) {
    if (h->h_ctrl->maxcount >= h->max_nbs) {
        h->h_ctrl->status |= GDB_STATUS_NBLIST_OVERFLOW;
        return set_err(h, GDB_ERR_NBLIST,
                       "Neighbor-list is invalid. Try allocating space for more neighbors (max_num_nbs in PairPot "
                       "object). Allocated size: %d, but %d neighbours found.",
                       h->max_nbs, h->h_ctrl->maxcount + 1);
    }
    if (h->h_ctrl->status & GDB_STATUS_NAN)
        return set_err(h, GDB_ERR_NUMERIC, "non-finite or runaway particle position");
    return GDB_OK;
}

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

int gdb_version(void) { return 100; }

int gdb_device_count(int *count) {
    gdb_sim *h = nullptr;
    if (!count) return set_err(h, GDB_ERR_ARG, "NULL count");
    CK(cudaGetDeviceCount(count));
    return GDB_OK;
}

int gdb_sim_create(int n, int ntypes, int device, gdb_sim **out) {
    gdb_sim *h = nullptr;
    if (!out || n < 1 || ntypes < 1 || ntypes > GDB_MAX_TYPES)
        return set_err(h, GDB_ERR_ARG, "gdb_sim_create: bad arguments (n=%d, ntypes=%d, max types %d)", n, ntypes,
                       GDB_MAX_TYPES);
    CK(cudaSetDevice(device));
    h = new gdb_sim();
    h->n = n;
    h->ntypes = ntypes;
    h->dev = device;
    const char *g = getenv("GDB_GRAPHS");
    if (g && g[0] == '0') h->use_graphs = false;
    const char *fm = getenv("GDB_NBLIST_FMA");
    if (fm && fm[0] == '0') h->fma = 0;
    auto fail = [&](cudaError_t e) {
        snprintf(g_lib_error, sizeof(g_lib_error), "gdb_sim_create: %s", cudaGetErrorString(e));
        gdb_sim_destroy(h);
        return GDB_ERR_CUDA;
    };
    cudaError_t e;
#define AL(ptr, bytes)                                   \
    if ((e = cudaMalloc(&(ptr), (bytes))) != cudaSuccess) \
        return fail(e);
    const size_t N = n;
    if ((e = cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking)) != cudaSuccess) return fail(e);
    if ((e = cudaEventCreate(&h->ev0)) != cudaSuccess) return fail(e);
    if ((e = cudaEventCreate(&h->ev1)) != cudaSuccess) return fail(e);
    AL(h->pos[0], N * sizeof(float4));
    AL(h->pos[1], N * sizeof(float4));
    AL(h->vel, N * sizeof(float4));
    AL(h->frc, N * sizeof(float4));
    AL(h->rref, N * sizeof(float4));
    AL(h->pos_tmp, N * sizeof(float4));
    AL(h->vel_tmp, N * sizeof(float4));
    AL(h->img, N * sizeof(int4));
    AL(h->img_tmp, N * sizeof(int4));
    AL(h->orig, N * sizeof(int));
    AL(h->orig_tmp, N * sizeof(int));
    AL(h->nbc, N * sizeof(int));
    AL(h->pscal, 5 * N * sizeof(float));
    AL(h->pscal_tmp, 5 * N * sizeof(float));
    AL(h->pcell, N * sizeof(int));
    AL(h->prank, N * sizeof(int));
    AL(h->perm, N * sizeof(int));
    AL(h->scell, N * sizeof(int));
    AL(h->ctrl, sizeof(DevCtrl));
#undef AL
    if ((e = cudaMallocHost(&h->h_ctrl, sizeof(DevCtrl))) != cudaSuccess) return fail(e);
    if ((e = cudaMemset(h->ctrl, 0, sizeof(DevCtrl))) != cudaSuccess) return fail(e);
    if ((e = cudaMemset(h->pscal, 0, 5 * N * sizeof(float))) != cudaSuccess) return fail(e);
    if ((e = cudaMemset(h->frc, 0, N * sizeof(float4))) != cudaSuccess) return fail(e);
    if ((e = cudaMemset(h->nbc, 0, N * sizeof(int))) != cudaSuccess) return fail(e);
    memset(h->h_ctrl, 0, sizeof(DevCtrl));
    *out = h;
    return GDB_OK;
}

int gdb_sim_destroy(gdb_sim *h) {
    if (!h) return GDB_OK;
    cudaSetDevice(h->dev);
    if (h->st) cudaStreamSynchronize(h->st);
    free_graphs(h);
    void *bufs[] = {h->pos[0], h->pos[1], h->vel,        h->frc,       h->rref,  h->pos_tmp, h->vel_tmp,
                    h->img,    h->img_tmp, h->orig,      h->orig_tmp,  h->nbl,   h->nbc,     h->pscal,
                    h->pscal_tmp, h->cell_count, h->cell_start, h->pcell, h->prank, h->perm, h->scell,
                    h->bsum,   h->ctrl,   h->partials,   h->rows,  h->conf};
    for (void *p : bufs)
        if (p) cudaFree(p);
    if (h->h_ctrl) cudaFreeHost(h->h_ctrl);
    if (h->ev0) cudaEventDestroy(h->ev0);
    if (h->ev1) cudaEventDestroy(h->ev1);
    if (h->st) cudaStreamDestroy(h->st);
    delete h;
    return GDB_OK;
}

int gdb_set_box(gdb_sim *h, const float lengths[3]) {
    if (!h || !lengths) return set_err(h, GDB_ERR_ARG, "gdb_set_box: NULL argument");
    for (int k = 0; k < 3; k++)
        if (!(lengths[k] > 0.f)) return set_err(h, GDB_ERR_ARG, "gdb_set_box: non-positive length");
    memcpy(h->box, lengths, sizeof(h->box));
    free_graphs(h);
    if (h->uploaded) {
        CK(cudaSetDevice(h->dev));
        int one = 1;
        CK(cudaMemcpyAsync(&h->ctrl->rebuild, &one, sizeof(int), cudaMemcpyHostToDevice, h->st));
        CK(cudaStreamSynchronize(h->st));
    }
    return GDB_OK;
}

int gdb_upload_state(gdb_sim *h, const float *r, const float *v, const float *m, const int32_t *ptype,
                     const int32_t *r_im) {
    if (!h || !r || !v || !m || !ptype) return set_err(h, GDB_ERR_ARG, "gdb_upload_state: NULL argument");
    for (int i = 0; i < h->n; i++)
        if (ptype[i] < 0 || ptype[i] >= h->ntypes)
            return set_err(h, GDB_ERR_ARG, "gdb_upload_state: particle %d has type %d outside [0, %d)", i, ptype[i],
                           h->ntypes);
    CK(cudaSetDevice(h->dev));
    const size_t N = h->n;
    // staging: one device buffer for the raw host arrays
    char *stage = nullptr;
    const size_t bytes = N * (3 + 3 + 1) * sizeof(float) + N * sizeof(int) + N * 3 * sizeof(int);
    CK(cudaMallocAsync((void **)&stage, bytes, h->st));
    float *dr = (float *)stage, *dv = dr + 3 * N, *dm = dv + 3 * N;
    int *dpt = (int *)(dm + N), *dim = dpt + N;
    CK(cudaMemcpyAsync(dr, r, 3 * N * sizeof(float), cudaMemcpyHostToDevice, h->st));
    CK(cudaMemcpyAsync(dv, v, 3 * N * sizeof(float), cudaMemcpyHostToDevice, h->st));
    CK(cudaMemcpyAsync(dm, m, N * sizeof(float), cudaMemcpyHostToDevice, h->st));
    CK(cudaMemcpyAsync(dpt, ptype, N * sizeof(int), cudaMemcpyHostToDevice, h->st));
    if (r_im) CK(cudaMemcpyAsync(dim, r_im, 3 * N * sizeof(int), cudaMemcpyHostToDevice, h->st));
    h->cur = 0;
    k_pack<<<grid_for(h->n), GDB_BLOCK, 0, h->st>>>(h->n, dr, dv, dm, dpt, r_im ? dim : nullptr, h->pos[0], h->vel,
                                                   h->img, h->orig);
    CKL();
    CK(cudaFreeAsync(stage, h->st));
    int one = 1;
    CK(cudaMemcpyAsync(&h->ctrl->rebuild, &one, sizeof(int), cudaMemcpyHostToDevice, h->st));
    CK(cudaStreamSynchronize(h->st));
    h->uploaded = true;
    return GDB_OK;
}

static int download_planes(gdb_sim *h, const void *src, int kind, void *dst) {
    // kind 0: float4 -> (N,3) float, 1: int4 -> (N,3) int, 2: float plane -> (N,) float
    const size_t N = h->n;
    const size_t bytes = (kind == 2 ? 1 : 3) * N * 4;
    void *tmp = nullptr;
    CK(cudaMallocAsync(&tmp, bytes, h->st));
    if (kind == 0)
        k_unpack3<<<grid_for(h->n), GDB_BLOCK, 0, h->st>>>(h->n, (const float4 *)src, h->orig, (float *)tmp);
    else if (kind == 1)
        k_unpack3i<<<grid_for(h->n), GDB_BLOCK, 0, h->st>>>(h->n, (const int4 *)src, h->orig, (int *)tmp);
    else
        k_unpack1<<<grid_for(h->n), GDB_BLOCK, 0, h->st>>>(h->n, (const float *)src, h->orig, (float *)tmp);
    CKL();
    CK(cudaMemcpyAsync(dst, tmp, bytes, cudaMemcpyDeviceToHost, h->st));
    CK(cudaFreeAsync(tmp, h->st));
    return GDB_OK;
}

int gdb_download_state(gdb_sim *h, float *r, float *v, float *f, int32_t *r_im) {
    if (!h) return set_err(h, GDB_ERR_ARG, "NULL handle");
    if (!h->uploaded) return set_err(h, GDB_ERR_STATE, "state not uploaded");
    CK(cudaSetDevice(h->dev));
    int rc;
    if (r && (rc = download_planes(h, h->pos[h->cur], 0, r))) return rc;
    if (v && (rc = download_planes(h, h->vel, 0, v))) return rc;
    if (f && (rc = download_planes(h, h->frc, 0, f))) return rc;
    if (r_im && (rc = download_planes(h, h->img, 1, r_im))) return rc;
    CK(cudaStreamSynchronize(h->st));
    return GDB_OK;
}

int gdb_download_scalars(gdb_sim *h, float *U, float *W, float *lapU, float *K, float *Fsq) {
    if (!h) return set_err(h, GDB_ERR_ARG, "NULL handle");
    if (!h->uploaded) return set_err(h, GDB_ERR_STATE, "state not uploaded");
    CK(cudaSetDevice(h->dev));
    float *outs[5] = {U, W, lapU, K, Fsq};
    for (int q = 0; q < 5; q++) {
        if (!outs[q]) continue;
        int rc = download_planes(h, h->pscal + (size_t)q * h->n, 2, outs[q]);
        if (rc) return rc;
    }
    CK(cudaStreamSynchronize(h->st));
    return GDB_OK;
}

int gdb_set_pair_potential(gdb_sim *h, int kind, int cutmode, int ntypes, const float *params, int nparams) {
    if (!h || !params) return set_err(h, GDB_ERR_ARG, "gdb_set_pair_potential: NULL argument");
    if (kind != GDB_POT_LJ_SIGMA_EPSILON && kind != GDB_POT_LJ_12_6)
        return set_err(h, GDB_ERR_UNSUPPORTED, "unsupported potential kind %d", kind);
    if (cutmode != GDB_CUT_SHIFTED_FORCE && cutmode != GDB_CUT_SHIFTED_POTENTIAL)
        return set_err(h, GDB_ERR_UNSUPPORTED, "unsupported cutoff mode %d", cutmode);
    if (ntypes != h->ntypes) return set_err(h, GDB_ERR_ARG, "parameter table has %d types, sim has %d", ntypes, h->ntypes);
    if (nparams < 3) return set_err(h, GDB_ERR_ARG, "need at least 3 parameters (p0, p1, cut)");
    for (int a = 0; a < ntypes * ntypes; a++) {
        const float cut = params[(size_t)a * nparams + nparams - 1];
        if (!(cut > 0.f)) return set_err(h, GDB_ERR_ARG, "non-positive cut for pair %d", a);
        if (kind == GDB_POT_LJ_SIGMA_EPSILON && !(params[(size_t)a * nparams] > 0.f))
            return set_err(h, GDB_ERR_ARG, "non-positive sigma for pair %d", a);
    }
    h->pot_kind = kind;
    h->cutmode = cutmode;
    h->nparams = nparams;
    h->params.assign(params, params + (size_t)ntypes * ntypes * nparams);
    build_table(h);
    h->have_pot = true;
    free_graphs(h);
    return GDB_OK;
}

int gdb_set_nblist(gdb_sim *h, int kind, float skin, int max_nbs) {
    if (!h) return set_err(h, GDB_ERR_ARG, "NULL handle");
    if (kind != GDB_NBLIST_NSQ && kind != GDB_NBLIST_CELLS) return set_err(h, GDB_ERR_ARG, "bad nblist kind %d", kind);
    if (!(skin >= 0.f) || max_nbs < 1) return set_err(h, GDB_ERR_ARG, "bad skin / max_nbs");
    if (kind != h->nb_kind || skin != h->skin || max_nbs != h->max_nbs) free_graphs(h);
    h->nb_kind = kind;
    h->skin = skin;
    h->max_nbs = max_nbs;
    if (h->uploaded) {
        CK(cudaSetDevice(h->dev));
        int one = 1;
        CK(cudaMemcpyAsync(&h->ctrl->rebuild, &one, sizeof(int), cudaMemcpyHostToDevice, h->st));
        CK(cudaStreamSynchronize(h->st));
    }
    return GDB_OK;
}

int gdb_set_plan(gdb_sim *h, int tp, int pb) {
    if (!h) return set_err(h, GDB_ERR_ARG, "NULL handle");
    if (tp != 0 && tp != 1 && tp != 2 && tp != 4 && tp != 8)
        return set_err(h, GDB_ERR_ARG, "tp must be 0 (auto), 1, 2, 4 or 8");
    h->tp_req = tp;
    h->pb_req = pb;
    return GDB_OK;
}

int gdb_set_integrator_nve(gdb_sim *h, float dt) {
    if (!h || !(dt > 0.f)) return set_err(h, GDB_ERR_ARG, "gdb_set_integrator_nve: bad arguments");
    h->integ = GDB_INTEGRATOR_NVE;
    h->dt = dt;
    free_graphs(h);
    return GDB_OK;
}

int gdb_set_integrator_nvt(gdb_sim *h, float dt, float tau, int tfunc, const float *tparams) {
    if (!h || !(dt > 0.f) || !(tau > 0.f) || !tparams)
        return set_err(h, GDB_ERR_ARG, "gdb_set_integrator_nvt: bad arguments");
    if (tfunc != GDB_TFUNC_CONSTANT && tfunc != GDB_TFUNC_RAMP)
        return set_err(h, GDB_ERR_UNSUPPORTED, "unsupported temperature function %d", tfunc);
    h->integ = GDB_INTEGRATOR_NVT;
    h->dt = dt;
    h->tau = tau;
    // omega2 = np.float32(4 pi^2 / tau / tau) (NVT.py:34)
    h->omega2 = (float)(4.0 * M_PI * M_PI / (double)tau / (double)tau);
    h->tfunc = tfunc;
    const int np_ = tfunc == GDB_TFUNC_RAMP ? 4 : 1;
    for (int k = 0; k < 4; k++) h->tparams[k] = k < np_ ? tparams[k] : 0.f;
    free_graphs(h);
    return GDB_OK;
}

int gdb_get_thermostat_state(gdb_sim *h, float state[2]) {
    if (!h || !state) return set_err(h, GDB_ERR_ARG, "NULL argument");
    CK(cudaSetDevice(h->dev));
    int rc = read_ctrl(h);
    if (rc) return rc;
    state[0] = h->h_ctrl->xi;
    state[1] = 0.0f;  // the sum is consumed by every update, as NVT.py:236
    return GDB_OK;
}

int gdb_set_thermostat_state(gdb_sim *h, const float state[2]) {
    if (!h || !state) return set_err(h, GDB_ERR_ARG, "NULL argument");
    CK(cudaSetDevice(h->dev));
    CK(cudaMemcpyAsync(&h->ctrl->xi, &state[0], sizeof(float), cudaMemcpyHostToDevice, h->st));
    CK(cudaStreamSynchronize(h->st));
    return GDB_OK;
}

int gdb_set_runtime_actions(gdb_sim *h, int scalar_every, int momentum_every) {
    if (!h || scalar_every < 0 || momentum_every < 0) return set_err(h, GDB_ERR_ARG, "bad runtime actions");
    h->scalar_every = scalar_every;
    h->momentum_every = momentum_every;
    free_graphs(h);
    return GDB_OK;
}

int gdb_set_configuration_saver(gdb_sim *h, int conf_per_block) {
    if (!h || conf_per_block < 0 || conf_per_block > 40) return set_err(h, GDB_ERR_ARG, "bad conf_per_block");
    CK(cudaSetDevice(h->dev));
    if (h->conf) cudaFree(h->conf);
    h->conf = nullptr;
    h->conf_per_block = 0;
    if (conf_per_block > 0) {
        const size_t bytes = (size_t)conf_per_block * 2 * h->n * 3 * sizeof(float);
        CK(cudaMalloc(&h->conf, bytes));
        CK(cudaMemset(h->conf, 0, bytes));
        h->conf_per_block = conf_per_block;
    }
    free_graphs(h);
    return GDB_OK;
}

int gdb_get_saved_configurations(gdb_sim *h, float *out, int conf_per_block) {
    if (!h || !out) return set_err(h, GDB_ERR_ARG, "NULL argument");
    if (conf_per_block != h->conf_per_block || !h->conf)
        return set_err(h, GDB_ERR_STATE, "configuration saver holds %d frames", h->conf_per_block);
    CK(cudaSetDevice(h->dev));
    const size_t bytes = (size_t)conf_per_block * 2 * h->n * 3 * sizeof(float);
    CK(cudaMemcpyAsync(out, h->conf, bytes, cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    return GDB_OK;
}

int gdb_eval_forces(gdb_sim *h) {
    int rc = check_ready(h);
    if (rc) return rc;
    CK(cudaMemsetAsync(&h->ctrl->maxcount, 0, sizeof(int), h->st));
    if ((rc = enqueue_rebuild(h))) return rc;
    if ((rc = enqueue_step(h, MODE_EVAL))) return rc;
    if ((rc = read_ctrl(h))) return rc;
    return status_to_rc(h);
}

// Capture GRAPH chunk: for s in 0..G-1: rebuild chain, step.
static int build_graph(gdb_sim *h, int parity, int G) {
    const int saved = h->cur;
    h->cur = parity;
    cudaGraph_t g;
    CK(cudaStreamBeginCapture(h->st, cudaStreamCaptureModeThreadLocal));
    int rc = GDB_OK;
    for (int s = 0; s < G && rc == GDB_OK; s++) {
        rc = enqueue_rebuild(h);
        if (rc == GDB_OK) rc = enqueue_step(h, MODE_STEP);
    }
    cudaError_t e = cudaStreamEndCapture(h->st, &g);
    h->cur = saved;
    if (rc) return rc;
    if (e != cudaSuccess) return set_err(h, GDB_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
    e = cudaGraphInstantiate(&h->gexec[parity], g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return set_err(h, GDB_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
    return GDB_OK;
}

int gdb_sim_run(gdb_sim *h, double time_zero, int steps, float *ms) {
    int rc = check_ready(h);
    if (rc) return rc;
    if (steps < 0) return set_err(h, GDB_ERR_ARG, "negative steps");
    const int rows = h->scalar_every > 0 ? steps / h->scalar_every : 0;
    if (rows > h->rows_cap) {
        if (h->rows) cudaFree(h->rows);
        h->rows = nullptr;
        CK(cudaMalloc(&h->rows, (size_t)rows * GDB_NUM_SCALARS * sizeof(double)));
        h->rows_cap = rows;
        free_graphs(h);
    }
    if (rows > 0) CK(cudaMemsetAsync(h->rows, 0, (size_t)rows * GDB_NUM_SCALARS * sizeof(double), h->st));
    {
        const int grid = grid_for((long long)h->n * h->tp);
        if ((rc = ensure_partials(h, grid))) return rc;
    }
    CK(cudaMemsetAsync(&h->ctrl->maxcount, 0, sizeof(int), h->st));
    CK(cudaEventRecord(h->ev0, h->st));
    k_block_begin<<<1, 1, 0, h->st>>>(h->ctrl, time_zero);
    CKL();
    const int G = 16;
    int s = 0;
    if (h->use_graphs && steps >= G) {
        h->graph_steps = G;
        while (s + G <= steps) {
            if (!h->gexec[h->cur] && (rc = build_graph(h, h->cur, G))) return rc;
            CK(cudaGraphLaunch(h->gexec[h->cur], h->st));
            // G is even: the current buffer is unchanged after a chunk
            s += G;
        }
    }
    for (; s < steps; s++) {
        if ((rc = enqueue_rebuild(h))) return rc;
        if ((rc = enqueue_step(h, MODE_STEP))) return rc;
    }
    if ((rc = enqueue_rebuild(h))) return rc;
    if ((rc = enqueue_step(h, MODE_EVAL))) return rc;
    CK(cudaEventRecord(h->ev1, h->st));
    if ((rc = read_ctrl(h))) return rc;
    if (ms) CK(cudaEventElapsedTime(ms, h->ev0, h->ev1));
    return status_to_rc(h);
}

int gdb_time_step_kernel(gdb_sim *h, int reps, float *ms_per_launch) {
    int rc = check_ready(h);
    if (rc) return rc;
    if (reps < 1 || !ms_per_launch) return set_err(h, GDB_ERR_ARG, "bad arguments");
    const int grid = grid_for((long long)h->n * h->tp);
    if ((rc = ensure_partials(h, grid))) return rc;
    // a list for the current positions, then `reps` step kernels alone
    if ((rc = enqueue_rebuild(h))) return rc;
    k_block_begin<<<1, 1, 0, h->st>>>(h->ctrl, 0.0);
    CKL();
    const int saved_every = h->scalar_every, saved_reset = h->momentum_every;
    h->scalar_every = 0;
    h->momentum_every = 0;
    CK(cudaEventRecord(h->ev0, h->st));
    for (int r = 0; r < reps && rc == GDB_OK; r++) rc = enqueue_step(h, MODE_STEP);
    h->scalar_every = saved_every;
    h->momentum_every = saved_reset;
    if (rc) return rc;
    CK(cudaEventRecord(h->ev1, h->st));
    CK(cudaEventSynchronize(h->ev1));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
    *ms_per_launch = ms / reps;
    return GDB_OK;
}

int gdb_nblist_stats(gdb_sim *h, double *mean_count, int *max_count) {
    if (!h || !mean_count || !max_count) return set_err(h, GDB_ERR_ARG, "bad arguments");
    if (!h->nbl) return set_err(h, GDB_ERR_STATE, "no neighbour list built yet");
    CK(cudaSetDevice(h->dev));
    std::vector<int> nbc(h->n);
    CK(cudaMemcpyAsync(nbc.data(), h->nbc, (size_t)h->n * sizeof(int), cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    double s = 0;
    int mx = 0;
    for (int c : nbc) {
        s += c;
        mx = c > mx ? c : mx;
    }
    *mean_count = s / h->n;
    *max_count = mx;
    return GDB_OK;
}

int gdb_get_scalar_rows(gdb_sim *h, double *out, int rows) {
    if (!h || !out || rows < 0) return set_err(h, GDB_ERR_ARG, "bad arguments");
    if (rows > h->rows_cap) return set_err(h, GDB_ERR_ARG, "only %d rows available", h->rows_cap);
    if (rows == 0) return GDB_OK;
    CK(cudaSetDevice(h->dev));
    CK(cudaMemcpyAsync(out, h->rows, (size_t)rows * GDB_NUM_SCALARS * sizeof(double), cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    return GDB_OK;
}

int gdb_get_nblist(gdb_sim *h, int32_t *out, int max_nbs) {
    if (!h || !out || max_nbs < 1) return set_err(h, GDB_ERR_ARG, "bad arguments");
    if (!h->nbl) return set_err(h, GDB_ERR_STATE, "no neighbour list built yet");
    CK(cudaSetDevice(h->dev));
    const size_t N = h->n;
    std::vector<int> nbl(h->nbl_elems), nbc(N), orig(N);
    CK(cudaMemcpyAsync(nbl.data(), h->nbl, h->nbl_elems * sizeof(int), cudaMemcpyDeviceToHost, h->st));
    CK(cudaMemcpyAsync(nbc.data(), h->nbc, N * sizeof(int), cudaMemcpyDeviceToHost, h->st));
    CK(cudaMemcpyAsync(orig.data(), h->orig, N * sizeof(int), cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    const int tp = h->tp, stride = h->stride;
    for (size_t s = 0; s < N; s++) {
        const int i = orig[s];
        int32_t *row = out + (size_t)i * (max_nbs + 1);
        const int cnt = nbc[s];
        const int lim = std::min(std::min(cnt, h->max_nbs), max_nbs);
        for (int k = 0; k < lim; k++) row[k] = orig[nbl[(size_t)(k / tp) * stride * tp + s * tp + (k % tp)]];
        row[max_nbs] = cnt;
    }
    return GDB_OK;
}

int gdb_get_nbflag(gdb_sim *h, int32_t out[3]) {
    if (!h || !out) return set_err(h, GDB_ERR_ARG, "bad arguments");
    CK(cudaSetDevice(h->dev));
    int rc = read_ctrl(h);
    if (rc) return rc;
    out[0] = h->h_ctrl->rebuild ? 1 : 0;
    out[1] = h->h_ctrl->maxcount >= h->max_nbs ? h->h_ctrl->maxcount : 0;
    out[2] = h->h_ctrl->nrebuild;
    return GDB_OK;
}

uint32_t gdb_status_word(gdb_sim *h) {
    if (!h) return GDB_STATUS_BAD_ARG;
    if (cudaSetDevice(h->dev) != cudaSuccess || read_ctrl(h) != GDB_OK) return GDB_STATUS_BAD_ARG;
    uint32_t s = h->h_ctrl->status;
    if (h->max_nbs > 0 && h->h_ctrl->maxcount >= h->max_nbs) s |= GDB_STATUS_NBLIST_OVERFLOW;
    return s;
}

int gdb_clear_status(gdb_sim *h) {
    if (!h) return set_err(h, GDB_ERR_ARG, "NULL handle");
    CK(cudaSetDevice(h->dev));
    CK(cudaMemsetAsync(&h->ctrl->status, 0, sizeof(unsigned), h->st));
    CK(cudaStreamSynchronize(h->st));
    return GDB_OK;
}

int gdb_get_last_error(gdb_sim *h, char *buf, int n) {
    if (!buf || n < 1) return GDB_ERR_ARG;
    snprintf(buf, (size_t)n, "%s", h ? h->err : g_lib_error);
    return GDB_OK;
}

// accessors used by analysis.cu
const float4 *gdb_internal_pos(gdb_sim *h) { return h->pos[h->cur]; }
const int *gdb_internal_orig(gdb_sim *h) { return h->orig; }
cudaStream_t gdb_internal_stream(gdb_sim *h) { return h->st; }
const float *gdb_internal_box(gdb_sim *h) { return h->box; }
int gdb_internal_n(gdb_sim *h) { return h->n; }
int gdb_internal_ntypes(gdb_sim *h) { return h->ntypes; }
int gdb_internal_dev(gdb_sim *h) { return h->dev; }
int gdb_internal_uploaded(gdb_sim *h) { return h->uploaded ? 1 : 0; }
char *gdb_internal_err(gdb_sim *h) { return h ? h->err : g_lib_error; }

}  // extern "C"
