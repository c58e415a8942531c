// analysis.cu -- radial distribution function and structure factor on B200.
//
// RDF (calculators/calculator_radial_distribution.py:76-107): every ordered
// pair i != j with dist_sq < r_max^2 is counted in bin int(d / width) of its
// (type_i, type_j) histogram, with the reference's mixed precision: dist_sq
// in float32 (orthorhombic.py:59-73), the range test and d / width in
// float64, d = sqrt(dist_sq) in float32.  Counts are exact integers (uint64).
// dist_sq is symmetric bit for bit (the minimum image of -dr is -dr's), so
// each unordered pair is evaluated once and counted in both orders.
//   * r_max >= min(L)/3: all pairs, j tiles staged in shared memory.
//   * smaller r_max: particles sorted into cells of edge >= r_max (counting
//     sort), home cell and half shell of 13 neighbours.  Same pair set, so
//     the same counts.
// Pairs in range are queued per warp and binned 32 at a time.  Per-block
// histograms live in shared memory (uint32) and are flushed with 64-bit
// atomics.
//
// S(q) (calculators/calculator_structure_factor.py:131-156, :185-203):
// rho_q = N_f^-1/2 sum_i f_i exp(i q.r_i) with q = 2 pi n / L.  Because q is
// on the reciprocal lattice, exp(i q.r) = e_x(nx) e_y(ny) e_z(nz) with
// e_d(k) = exp(2 pi i k r_d / L_d); each block tabulates e_d(k) for a tile of
// particles in shared memory (sincospi, float32) and every thread accumulates
// its q-vectors with complex multiplies, float32 within a tile and float64
// across tiles.
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <mutex>
#include <vector>

#include "../../include/gamdb200.h"
#include "gdb_internal.cuh"

using namespace gdb;

extern "C" {
const float4 *gdb_internal_pos(gdb_sim *h);
const int *gdb_internal_orig(gdb_sim *h);
cudaStream_t gdb_internal_stream(gdb_sim *h);
const float *gdb_internal_box(gdb_sim *h);
int gdb_internal_n(gdb_sim *h);
int gdb_internal_ntypes(gdb_sim *h);
int gdb_internal_dev(gdb_sim *h);
int gdb_internal_uploaded(gdb_sim *h);
char *gdb_internal_err(gdb_sim *h);
cudaEvent_t gdb_internal_event(gdb_sim *h, int k);
void gdb_internal_set_analysis_ms(gdb_sim *h, float ms);
}

// Device time of one handle call: events on the handle's stream around its
// device work (nothing for the stand-alone calculators, h == NULL).
static cudaError_t timing_begin(gdb_sim *h, cudaStream_t st) {
    return h ? cudaEventRecord(gdb_internal_event(h, 0), st) : cudaSuccess;
}
static cudaError_t timing_end(gdb_sim *h, cudaStream_t st) {
    return h ? cudaEventRecord(gdb_internal_event(h, 1), st) : cudaSuccess;
}
static void timing_store(gdb_sim *h) {
    float ms = 0.f;
    if (h && cudaEventElapsedTime(&ms, gdb_internal_event(h, 0), gdb_internal_event(h, 1)) == cudaSuccess)
        gdb_internal_set_analysis_ms(h, ms);
}

static int aset(gdb_sim *h, int code, const char *msg, cudaError_t e = cudaSuccess) {
    snprintf(gdb_internal_err(h), 512, "%s%s%s", msg, e != cudaSuccess ? ": " : "",
             e != cudaSuccess ? cudaGetErrorString(e) : "");
    return code;
}

#define ACK(call)                                                     \
    do {                                                              \
        cudaError_t e_ = (call);                                      \
        if (e_ != cudaSuccess) return aset(h, GDB_ERR_CUDA, #call, e_); \
    } while (0)

namespace {

constexpr int RDF_THREADS = 256;
constexpr int RDF_WARPS = RDF_THREADS / 32;
constexpr int RDF_TILE = RDF_THREADS;     // j positions staged per block (all-pairs path)
constexpr int RDF_SMEM_MAX_BINS = 12288;  // uint32 entries kept in shared memory
constexpr int RDF_RING = 64;              // pending pairs per warp (< 32 + 32 before a drain)

struct RdfArgs {
    int n, nt, bins;
    float Lx, Ly, Lz;
    // smallest float32 >= r_max^2 and >= r_max: for a float32 x,
    // (double)x < r_max^2  <=>  x < r2f, so the range tests stay in float32
    float r2f, rf;
    double width, inv_width;  // r_max / bins and its rounded reciprocal
    unsigned long long *out;
};

// Pairs within range wait in a per-warp ring until 32 of them are pending;
// the square root, the float64 bin and the histogram increments then run with
// every lane busy instead of at the hit rate (about 15 % of candidates).
struct RdfRing {
    float d2[RDF_RING];
    int code[RDF_RING];  // t_i | t_j << 16
};

// int(d / width) as the float64 division gives it.  q = d * (1 / width) is
// within 2.3e-16 q of d / width and the rounded quotient within 1.2e-16, so
// their floors can differ only when an integer k >= 1 lies within
// 3.3e-16 k of q; such quotients (|q - k| <= 1e-12 k) take the division.
__device__ __forceinline__ int rdf_bin(const RdfArgs &a, float d) {
    const double q = (double)d * a.inv_width;
    const double k = rint(q);
    int b = (k >= 1.0 && fabs(q - k) <= 1e-12 * k) ? (int)__ddiv_rn((double)d, a.width) : (int)q;
    // d < r_max, yet d / width can round up to `bins`; the reference would
    // index past its array there, this keeps the count in range
    return b < a.bins ? b : a.bins - 1;
}

// One pending pair per lane (lane < take): both orders (i, j) and (j, i) of
// the pair are counted, in (t_i, t_j) and (t_j, t_i).
__device__ __forceinline__ void rdf_drain(const RdfArgs &a, const RdfRing &rg, int head, int take, int lane,
                                          unsigned *hist, bool sh) {
    __syncwarp();
    if (lane < take) {
        const int e = (head + lane) & (RDF_RING - 1);
        const float d = __fsqrt_rn(rg.d2[e]);
        if (d < a.rf) {
            const int b = rdf_bin(a, d);
            const int ti = rg.code[e] & 0xffff, tj = rg.code[e] >> 16;
            const int k1 = (ti * a.nt + tj) * a.bins + b, k2 = (tj * a.nt + ti) * a.bins + b;
            if (sh) {
                if (k1 == k2) {
                    atomicAdd(&hist[k1], 2u);
                } else {
                    atomicAdd(&hist[k1], 1u);
                    atomicAdd(&hist[k2], 1u);
                }
            } else {
                if (k1 == k2) {
                    atomicAdd(&a.out[k1], 2ull);
                } else {
                    atomicAdd(&a.out[k1], 1ull);
                    atomicAdd(&a.out[k2], 1ull);
                }
            }
        }
    }
    __syncwarp();
}

// Lane's particle i against jn <= 32 staged positions js[0..jn).  First pass:
// every candidate's dist_sq goes to the warp's d2s[q][lane] and in-range
// candidates set bit q of the lane's mask; bits q <= lim are dropped (j at or
// before i in the same cell or tile).  Second pass: lanes hand their hits to
// the ring one per round, and full rounds of 32 are binned.  MIC: minimum
// image per component, as the reference; without it the plain difference,
// which callers use only where it gives the same pairs in range and the same
// dist_sq for them.
template <bool FMA, bool MIC>
__device__ __forceinline__ float rdf_d2(const RdfArgs &a, float4 pj, float4 pi) {
    float dx = __fsub_rn(pj.x, pi.x), dy = __fsub_rn(pj.y, pi.y), dz = __fsub_rn(pj.z, pi.z);
    if (MIC) {
        dx = mic(dx, a.Lx);
        dy = mic(dy, a.Ly);
        dz = mic(dz, a.Lz);
    }
    float d2 = __fmul_rn(dx, dx);
    if (FMA) {
        d2 = __fmaf_rn(dy, dy, d2);
        d2 = __fmaf_rn(dz, dz, d2);
    } else {
        d2 = __fadd_rn(d2, __fmul_rn(dy, dy));
        d2 = __fadd_rn(d2, __fmul_rn(dz, dz));
    }
    return d2;
}

template <bool FMA, bool MIC>
__device__ __forceinline__ void rdf_warp_tile(const RdfArgs &a, float4 pi, int ti, bool act, const float4 *js, int jn,
                                              int lim, float *d2s, RdfRing &rg, int &head, int &tail, int lane,
                                              unsigned *hist, bool sh) {
    unsigned mask = 0;
    if (act) {
        if (jn == 32) {
#pragma unroll
            for (int q = 0; q < 32; q++) {
                const float d2 = rdf_d2<FMA, MIC>(a, js[q], pi);
                d2s[q * 32 + lane] = d2;
                if (d2 < a.r2f) mask |= 1u << q;
            }
        } else {
            for (int q = 0; q < jn; q++) {
                const float d2 = rdf_d2<FMA, MIC>(a, js[q], pi);
                d2s[q * 32 + lane] = d2;
                if (d2 < a.r2f) mask |= 1u << q;
            }
        }
        if (lim >= 31)
            mask = 0;
        else if (lim >= 0)
            mask &= ~0u << (lim + 1);
    }
    const unsigned below = (1u << lane) - 1u;
    for (;;) {
        const unsigned m = __ballot_sync(0xffffffffu, mask != 0);
        if (m == 0) break;
        if (mask) {
            const int q = __ffs(mask) - 1;
            mask &= mask - 1u;
            const int e = (tail + __popc(m & below)) & (RDF_RING - 1);
            rg.d2[e] = d2s[q * 32 + lane];
            rg.code[e] = ti | (ptype_of(js[q]) << 16);
        }
        tail += __popc(m);
        if (tail - head >= 32) {
            rdf_drain(a, rg, head, 32, lane, hist, sh);
            head += 32;
        }
    }
    __syncwarp();
}

__device__ __forceinline__ void rdf_clear(unsigned *hist, int total) {
    for (int k = threadIdx.x; k < total; k += blockDim.x) hist[k] = 0;
    __syncthreads();
}

__device__ __forceinline__ void rdf_flush(const RdfArgs &a, unsigned *hist, int total) {
    __syncthreads();
    for (int k = threadIdx.x; k < total; k += blockDim.x)
        if (hist[k]) atomicAdd(&a.out[k], (unsigned long long)hist[k]);
}

// All pairs, each unordered pair once.  Tiles of RDF_TILE particles; i-tile b
// meets j-tiles b + k (mod T) for k = 0 .. T/2 (k = 0: j > i; for even T the
// tile pair at distance T/2 belongs to the lower tile), so every i-tile has
// the same work; blockIdx.y takes slice y of that k range (small systems still
// fill the GPU).
template <bool FMA>
__global__ void __launch_bounds__(RDF_THREADS) k_rdf_allpairs(RdfArgs a, const float4 *pos) {
    extern __shared__ unsigned char smraw[];
    float4 *tile = (float4 *)smraw;
    float *d2s = (float *)(tile + RDF_TILE);  // [RDF_WARPS][32][32]
    RdfRing *rings = (RdfRing *)(d2s + RDF_WARPS * 1024);
    unsigned *hist = (unsigned *)(rings + RDF_WARPS);
    const int total = a.nt * a.nt * a.bins;
    const bool sh = total <= RDF_SMEM_MAX_BINS;
    if (sh) rdf_clear(hist, total);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    float *wd2 = d2s + w * 1024;
    RdfRing &rg = rings[w];
    int head = 0, tail = 0;
    const int T = (a.n + RDF_TILE - 1) / RDF_TILE;
    const int b = blockIdx.x;
    const int i = b * RDF_TILE + threadIdx.x;
    const bool act = i < a.n;
    const float4 pi = act ? pos[i] : make_float4(0.f, 0.f, 0.f, 0.f);
    const int ti = ptype_of(pi);
    const int kmax = (T % 2 == 0 && b >= T / 2) ? T / 2 - 1 : T / 2;
    const int per = (T / 2 + gridDim.y) / gridDim.y;  // ceil((T / 2 + 1) / S)
    const int k_end = min(kmax + 1, ((int)blockIdx.y + 1) * per);
    for (int k = blockIdx.y * per; k < k_end; k++) {
        const int jt = (b + k) % T;
        const int j0 = jt * RDF_TILE;
        const int jn = min(RDF_TILE, a.n - j0);
        __syncthreads();
        if (threadIdx.x < jn) tile[threadIdx.x] = pos[j0 + threadIdx.x];
        __syncthreads();
        for (int q0 = 0; q0 < jn; q0 += 32)
            rdf_warp_tile<FMA, true>(a, pi, ti, act, tile + q0, min(32, jn - q0), k == 0 ? i - (j0 + q0) : -1, wd2,
                                     rg, head, tail, lane, hist, sh);
    }
    rdf_drain(a, rg, head, tail - head, lane, hist, sh);
    if (sh) rdf_flush(a, hist, total);
}

// Cell search for r_max < L/3: particles sorted by cell (cells of edge >=
// r_max, at least 3 per side).  A unit of work is 32 home particles of one
// cell (unit u: cell u / K, particles 32 (u % K) on, K = chunks of the
// fullest cell; units past a cell's end are empty), taken a unit per warp,
// against the home cell (j > i) and the 13 neighbour cells of the half shell
// (offsets after the centre in z-y-x order).  Each pair of neighbouring cells
// is visited from exactly one side, each pair of particles once.
//
// Plain differences between cells that are both off the box faces (cell
// index 1 .. nc-2 in every dimension): such particles lie at least one cell
// edge inside the box, so a pair whose difference the minimum image would
// fold is more than two edges (>= 2 r_max) apart in that component in both
// images; pairs in range have |dr| < L/2 and are left unchanged by it.  When
// any position lies outside [-L/2, L/2] (*outside set by the binning) every
// cell takes the minimum image.
template <bool FMA>
__global__ void __launch_bounds__(RDF_THREADS) k_rdf_cells(RdfArgs a, const float4 *spos, const int *start,
                                                           const int *outside, int ncx, int ncy, int ncz) {
    extern __shared__ unsigned char smraw[];
    float4 *jbuf = (float4 *)smraw;  // [RDF_WARPS][32]
    float *d2s = (float *)(jbuf + RDF_THREADS);
    RdfRing *rings = (RdfRing *)(d2s + RDF_WARPS * 1024);
    unsigned *hist = (unsigned *)(rings + RDF_WARPS);
    const int total = a.nt * a.nt * a.bins;
    const bool sh = total <= RDF_SMEM_MAX_BINS;
    if (sh) rdf_clear(hist, total);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    float4 *js = jbuf + 32 * w;
    float *wd2 = d2s + w * 1024;
    RdfRing &rg = rings[w];
    int head = 0, tail = 0;
    const bool inside = *outside == 0;
    const int ncell = ncx * ncy * ncz;
    const int K = start[ncell + 1];
    const long long units = (long long)ncell * K;
    for (long long u = (long long)blockIdx.x * RDF_WARPS + w; u < units; u += (long long)gridDim.x * RDF_WARPS) {
        const int c = (int)(u / K);
        const int cx = c % ncx, cy = (c / ncx) % ncy, cz = c / (ncx * ncy);
        const int h1 = start[c + 1];
        const int i0 = start[c] + 32 * (int)(u % K);
        if (i0 >= h1) continue;
        const int i = i0 + lane;
        const bool act = i < h1;
        const float4 pi = act ? spos[i] : make_float4(0.f, 0.f, 0.f, 0.f);
        const int ti = ptype_of(pi);
        const bool home_in = inside && cx >= 1 && cx <= ncx - 2 && cy >= 1 && cy <= ncy - 2 && cz >= 1 &&
                             cz <= ncz - 2;
        for (int s = 13; s < 27; s++) {
            int j0, j1;
            bool plain = home_in;
            if (s == 13) {
                j0 = i0;
                j1 = h1;
            } else {
                const int x = cx + s % 3 - 1, y = cy + (s / 3) % 3 - 1, z = cz + s / 9 - 1;
                plain = plain && x >= 1 && x <= ncx - 2 && y >= 1 && y <= ncy - 2 && z >= 1 && z <= ncz - 2;
                const int nb = (((z + ncz) % ncz) * ncy + (y + ncy) % ncy) * ncx + (x + ncx) % ncx;
                j0 = start[nb];
                j1 = start[nb + 1];
            }
            for (; j0 < j1; j0 += 32) {
                const int jn = min(32, j1 - j0);
                __syncwarp();
                if (lane < jn) js[lane] = spos[j0 + lane];
                __syncwarp();
                const int lim = s == 13 ? i - j0 : -1;
                if (plain)
                    rdf_warp_tile<FMA, false>(a, pi, ti, act, js, jn, lim, wd2, rg, head, tail, lane, hist, sh);
                else
                    rdf_warp_tile<FMA, true>(a, pi, ti, act, js, jn, lim, wd2, rg, head, tail, lane, hist, sh);
            }
        }
    }
    rdf_drain(a, rg, head, tail - head, lane, hist, sh);
    if (sh) rdf_flush(a, hist, total);
}

// cell binning for the cell search: a counting sort of the positions;
// *outside = 1 when a coordinate is outside [-L/2, L/2] (or not a number)
__global__ void k_bin_cells(const float4 *pos, int n, float Lx, float Ly, float Lz, int ncx, int ncy, int ncz,
                            int *pcell, int *prank, int *count, int *outside) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 p = pos[i];
    const float r[3] = {p.x, p.y, p.z};
    const float L[3] = {Lx, Ly, Lz};
    const int nc[3] = {ncx, ncy, ncz};
    int c[3];
    bool out = false;
    for (int k = 0; k < 3; k++) {
        const float h = 0.5f * L[k];
        out = out || !(r[k] >= -h && r[k] <= h);
        float f = (r[k] / L[k] + 0.5f) * nc[k];
        int ci = (int)floorf(f);
        if (!(f == f)) ci = 0;
        ci %= nc[k];
        if (ci < 0) ci += nc[k];
        c[k] = ci;
    }
    if (out) *outside = 1;
    const int cid = (c[2] * ncy + c[1]) * ncx + c[0];
    pcell[i] = cid;
    prank[i] = atomicAdd(&count[cid], 1);
}
// exclusive prefix sum of the cell counts (start[ncell] = total) and the
// 32-particle chunks of the fullest cell (start[ncell + 1]), one block of
// 1024 threads, each over a contiguous run of cells
constexpr int SCAN_THREADS = 1024;
__global__ void __launch_bounds__(SCAN_THREADS) k_cells_scan(const int *count, int *start, int ncell) {
    __shared__ int wsum[SCAN_THREADS / 32];
    __shared__ int cmax;
    if (threadIdx.x == 0) cmax = 0;
    const int per = (ncell + SCAN_THREADS - 1) / SCAN_THREADS;
    const int c0 = min(ncell, (int)threadIdx.x * per), c1 = min(ncell, c0 + per);
    int s = 0, m = 0;
    for (int c = c0; c < c1; c++) {
        s += count[c];
        m = max(m, count[c]);
    }
    __syncthreads();
    atomicMax(&cmax, m);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int x = s;  // inclusive scan within the warp
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) wsum[w] = x;
    __syncthreads();
    if (w == 0) {
        int v = wsum[lane];
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, v, o);
            if (lane >= o) v += y;
        }
        wsum[lane] = v;
    }
    __syncthreads();
    int run = x - s + (w > 0 ? wsum[w - 1] : 0);
    for (int c = c0; c < c1; c++) {
        start[c] = run;
        run += count[c];
    }
    if (threadIdx.x == SCAN_THREADS - 1) {
        start[ncell] = run;
        start[ncell + 1] = (cmax + 31) / 32;
    }
}

__global__ void k_cells_scatter(const float4 *pos, const int *pcell, const int *prank, const int *start,
                                float4 *spos, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    spos[start[pcell[i]] + prank[i]] = pos[i];
}

// ---------------------------------------------------------------------------
// S(q)
// ---------------------------------------------------------------------------
constexpr int SQ_TILE = 32;      // particles per shared-memory tile
constexpr int SQ_THREADS = 256;  // q-vectors per block
constexpr int SQ_CHUNK = 8192;   // particles per block (grid y)

struct SqArgs {
    const float4 *pos;
    const int *orig;
    const float *ff;  // user order, may be null
    int n, nq;
    const int *nvec;  // nq x 3
    int kmin[3], klen[3];
    float invL[3];
    double *acc;  // nq x 2
};

// One (particle, q) term of rho_q: (e_x e_y) e_z, times the form factor w
// when weighted, added to (tr, ti).  The roundings are written out, so every
// kernel that sums with it gives the same float32 partial sums.
__device__ __forceinline__ void sq_term(float2 ex, float2 ey, float2 ez, float w, bool weighted, float &tr,
                                        float &ti) {
    const float xr = __fmaf_rn(ex.x, ey.x, -__fmul_rn(ex.y, ey.y));
    const float xi = __fmaf_rn(ex.x, ey.y, __fmul_rn(ex.y, ey.x));
    const float cr = __fmaf_rn(xr, ez.x, -__fmul_rn(xi, ez.y));
    const float ci = __fmaf_rn(xr, ez.y, __fmul_rn(xi, ez.x));
    if (weighted) {
        tr = __fmaf_rn(w, cr, tr);
        ti = __fmaf_rn(w, ci, ti);
    } else {
        tr = __fadd_rn(tr, cr);
        ti = __fadd_rn(ti, ci);
    }
}

// One block: QPT x SQ_THREADS q-vectors (q = blockIdx.x QPT 256 + k 256 + t)
// against SQ_CHUNK particles.  Per tile of SQ_TILE particles the block
// tabulates e_d(k) = exp(2 pi i k x_d / L_d) once (sincospif, float32) and
// every thread accumulates its QPT q-vectors from the table: two complex
// products per (particle, q), float32 within a tile, float64 across tiles.
template <int QPT, bool FF>
__global__ void __launch_bounds__(SQ_THREADS) k_sq(SqArgs a) {
    extern __shared__ float2 tab[];  // [SQ_TILE][klen0 + klen1 + klen2]
    __shared__ float wsh[SQ_TILE];
    __shared__ float4 psh[SQ_TILE];
    const int k0 = a.klen[0], k01 = a.klen[0] + a.klen[1];
    const int row = k01 + a.klen[2];
    int ix[QPT], iy[QPT], iz[QPT];
#pragma unroll
    for (int k = 0; k < QPT; k++) {
        const int q = (blockIdx.x * QPT + k) * SQ_THREADS + threadIdx.x;
        ix[k] = 0, iy[k] = 0, iz[k] = 0;  // inactive slots read entry 0 and are not stored
        if (q < a.nq) {
            ix[k] = a.nvec[3 * q] - a.kmin[0];
            iy[k] = a.nvec[3 * q + 1] - a.kmin[1] + k0;
            iz[k] = a.nvec[3 * q + 2] - a.kmin[2] + k01;
        }
    }
    double sr[QPT], si[QPT];
#pragma unroll
    for (int k = 0; k < QPT; k++) sr[k] = si[k] = 0.0;
    // this thread's table entries: (pl0, col0) then steps of SQ_THREADS
    const int dpl = SQ_THREADS / row, dcol = SQ_THREADS % row;
    const int pl0 = threadIdx.x / row, col0 = threadIdx.x % row;
    const int p_begin = blockIdx.y * SQ_CHUNK;
    const int p_end = min(a.n, p_begin + SQ_CHUNK);
    for (int p0 = p_begin; p0 < p_end; p0 += SQ_TILE) {
        const int np = min(SQ_TILE, p_end - p0);
        __syncthreads();
        if (threadIdx.x < np) {
            psh[threadIdx.x] = a.pos[p0 + threadIdx.x];
            if (FF) wsh[threadIdx.x] = a.ff[a.orig[p0 + threadIdx.x]];
        }
        __syncthreads();
        for (int pl = pl0, col = col0; pl < np;) {
            const int d = (col >= k0) + (col >= k01);
            const int kk = col - (d == 0 ? 0 : (d == 1 ? k0 : k01)) + a.kmin[d];
            const float4 p = psh[pl];
            const float x = d == 0 ? p.x : (d == 1 ? p.y : p.z);
            float sn, cs;
            sincospif(2.0f * (float)kk * (x * a.invL[d]), &sn, &cs);
            tab[pl * row + col] = make_float2(cs, sn);
            col += dcol;
            pl += dpl;
            if (col >= row) {
                col -= row;
                pl++;
            }
        }
        __syncthreads();
        float tr[QPT], ti[QPT];
#pragma unroll
        for (int k = 0; k < QPT; k++) tr[k] = ti[k] = 0.f;
        for (int pl = 0; pl < np; pl++) {
            const float2 *t = tab + pl * row;
            const float w = FF ? wsh[pl] : 1.0f;
#pragma unroll
            for (int k = 0; k < QPT; k++) {
                sq_term(t[ix[k]], t[iy[k]], t[iz[k]], w, FF, tr[k], ti[k]);
            }
        }
#pragma unroll
        for (int k = 0; k < QPT; k++) {
            sr[k] += tr[k];
            si[k] += ti[k];
        }
    }
#pragma unroll
    for (int k = 0; k < QPT; k++) {
        const int q = (blockIdx.x * QPT + k) * SQ_THREADS + threadIdx.x;
        if (q < a.nq) {
            atomicAdd(&a.acc[2 * q], sr[k]);
            atomicAdd(&a.acc[2 * q + 1], si[k]);
        }
    }
}

template <int QPT>
static void launch_sq(dim3 grid, size_t smem, cudaStream_t st, const SqArgs &a) {
    if (a.ff)
        k_sq<QPT, true><<<grid, SQ_THREADS, smem, st>>>(a);
    else
        k_sq<QPT, false><<<grid, SQ_THREADS, smem, st>>>(a);
}

// ---------------------------------------------------------------------------
// trajectory dynamics (tools/calc_dynamics.py:6-75)
// ---------------------------------------------------------------------------
constexpr int DYN_THREADS = 256;
constexpr int DYN_MAX_TYPES = 8;

// Frame pair p (frames f0 -> f1, each 2 x n x 3 float32: positions, then
// image counts): dR = (r1 - r0) + (i1 - i0) L in float32 as the reference,
// dR^2 summed over x, y, z in float32; per type the float64 sums of dR^2,
// (dR^2)^2 and cos(q_t dR_k) over particles and components, into
// acc[(p * nt + t) * 3 + {0, 1, 2}].
__global__ void __launch_bounds__(DYN_THREADS) k_dynamics(const float *frames, int n, const int *ptype, int nt,
                                                          float Lx, float Ly, float Lz, const int2 *pairs,
                                                          const double *q, double *acc) {
    __shared__ double red[DYN_MAX_TYPES * 3];
    for (int k = threadIdx.x; k < nt * 3; k += blockDim.x) red[k] = 0.0;
    __syncthreads();
    const int2 pr = pairs[blockIdx.y];
    const float *A = frames + (size_t)pr.x * 2 * n * 3;
    const float *B = frames + (size_t)pr.y * 2 * n * 3;
    const float L[3] = {Lx, Ly, Lz};
    double s[DYN_MAX_TYPES][3];
#pragma unroll
    for (int t = 0; t < DYN_MAX_TYPES; t++) s[t][0] = s[t][1] = s[t][2] = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int t = ptype[i];
        float d[3];
#pragma unroll
        for (int k = 0; k < 3; k++) {
            const float dr = __fsub_rn(B[3 * i + k], A[3 * i + k]);
            const float di = __fsub_rn(B[3 * n + 3 * i + k], A[3 * n + 3 * i + k]);
            d[k] = __fadd_rn(dr, __fmul_rn(di, L[k]));
        }
        const float sq = __fadd_rn(__fadd_rn(__fmul_rn(d[0], d[0]), __fmul_rn(d[1], d[1])), __fmul_rn(d[2], d[2]));
        const double qt = q[t];
        const double c = cos((double)d[0] * qt) + cos((double)d[1] * qt) + cos((double)d[2] * qt);
#pragma unroll
        for (int u = 0; u < DYN_MAX_TYPES; u++)
            if (u == t) {
                s[u][0] += sq;
                s[u][1] += (double)__fmul_rn(sq, sq);
                s[u][2] += c;
            }
    }
    for (int t = 0; t < nt; t++)
        for (int k = 0; k < 3; k++) {
            const double v = warp_sum(s[t][k]);
            if ((threadIdx.x & 31) == 0) atomicAdd(&red[t * 3 + k], v);
        }
    __syncthreads();
    for (int k = threadIdx.x; k < nt * 3; k += blockDim.x)
        atomicAdd(&acc[(size_t)blockIdx.y * nt * 3 + k], red[k]);
}

__global__ void k_pack_pos(int n, const float *r, const int *pt, float4 *pos, int *orig) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    pos[i] = make_float4(r[3 * i], r[3 * i + 1], r[3 * i + 2], __int_as_float(pt ? pt[i] : 0));
    orig[i] = i;
}

}  // namespace

// ---------------------------------------------------------------------------
// host implementations working on device-resident positions
// ---------------------------------------------------------------------------
// smallest float32 >= x
static float float_at_or_above(double x) {
    float f = (float)x;
    if ((double)f < x) f = nextafterf(f, INFINITY);
    return f;
}

static int rdf_device(gdb_sim *h, cudaStream_t st, const float4 *pos, int n, const float *box, int nt, int bins,
                      double r_max, uint64_t *out_host) {
    if (bins < 1 || nt < 1) return aset(h, GDB_ERR_ARG, "rdf: bins and ntypes must be positive");
    if (nt > 0xffff) return aset(h, GDB_ERR_ARG, "rdf: too many particle types");
    float minL = fminf(box[0], fminf(box[1], box[2]));
    // the reference: min_box_dim float32, (min_box_dim / 2) float64
    const double half = (double)minL / 2.0;
    if (r_max <= 0.0) r_max = half;
    if (r_max > half) return aset(h, GDB_ERR_ARG, "rdf: r_max must not exceed min(L)/2");
    RdfArgs a;
    a.n = n;
    a.nt = nt;
    a.bins = bins;
    a.Lx = box[0];
    a.Ly = box[1];
    a.Lz = box[2];
    a.r2f = float_at_or_above(r_max * r_max);
    a.rf = float_at_or_above(r_max);
    a.width = r_max / (double)bins;
    a.inv_width = 1.0 / a.width;
    const char *fm = getenv("GDB_NBLIST_FMA");
    const bool fma = !(fm && fm[0] == '0');
    const size_t total = (size_t)nt * nt * bins;
    ACK(timing_begin(h, st));
    unsigned long long *dout = nullptr;
    ACK(pool_alloc(&dout, total * sizeof(unsigned long long), st));
    ACK(cudaMemsetAsync(dout, 0, total * sizeof(unsigned long long), st));
    a.out = dout;
    const size_t hist_bytes = total <= (size_t)RDF_SMEM_MAX_BINS ? total * sizeof(unsigned) : 0;
    int nc[3];
    bool cells = true;
    for (int k = 0; k < 3; k++) {
        // edge slightly above r_max so float32 rounding of the cell
        // coordinate can never separate a pair closer than r_max by two cells
        nc[k] = (int)floor(box[k] / (r_max * (1.0 + 1e-4)));
        if (nc[k] < 3) cells = false;
    }
    const long long ncell = cells ? (long long)nc[0] * nc[1] * nc[2] : 0;
    if (ncell > (1LL << 28)) cells = false;  // r_max tiny against L: fall back to all pairs
    if (!cells) {
        const size_t smem = RDF_TILE * sizeof(float4) + RDF_WARPS * (1024 * sizeof(float) + sizeof(RdfRing)) +
                            hist_bytes;
        const int T = (n + RDF_TILE - 1) / RDF_TILE;
        int dev = 0, sms = 0, per_sm = 0;
        ACK(cudaGetDevice(&dev));
        ACK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        auto kern = fma ? k_rdf_allpairs<true> : k_rdf_allpairs<false>;
        ACK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        ACK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, RDF_THREADS, smem));
        // slices of the tile-distance range: about two waves of blocks in all
        const int slots = sms * std::max(per_sm, 1);
        const int S = std::max(1, std::min(T / 2 + 1, (2 * slots + T - 1) / T));
        kern<<<dim3(T, S), RDF_THREADS, smem, st>>>(a, pos);
        ACK(cudaGetLastError());
    } else {
        int *count = nullptr, *start = nullptr, *pcell = nullptr, *prank = nullptr;
        float4 *spos = nullptr;
        ACK(pool_alloc(&count, (ncell + 1) * sizeof(int), st));  // [ncell]: the outside flag
        ACK(pool_alloc(&start, (ncell + 2) * sizeof(int), st));
        ACK(pool_alloc(&pcell, (size_t)n * sizeof(int), st));
        ACK(pool_alloc(&prank, (size_t)n * sizeof(int), st));
        ACK(pool_alloc(&spos, (size_t)n * sizeof(float4), st));
        ACK(cudaMemsetAsync(count, 0, (ncell + 1) * sizeof(int), st));
        const int g = (n + 255) / 256;
        k_bin_cells<<<g, 256, 0, st>>>(pos, n, box[0], box[1], box[2], nc[0], nc[1], nc[2], pcell, prank, count,
                                      count + ncell);
        k_cells_scan<<<1, SCAN_THREADS, 0, st>>>(count, start, (int)ncell);
        k_cells_scatter<<<g, 256, 0, st>>>(pos, pcell, prank, start, spos, n);
        const size_t smem = RDF_THREADS * sizeof(float4) + RDF_WARPS * (1024 * sizeof(float) + sizeof(RdfRing)) +
                            hist_bytes;
        int dev = 0, sms = 0, per_sm = 0;
        ACK(cudaGetDevice(&dev));
        ACK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        auto kern = fma ? k_rdf_cells<true> : k_rdf_cells<false>;
        ACK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        ACK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, RDF_THREADS, smem));
        const int grid = sms * std::max(per_sm, 1);  // warps stride over the units
        kern<<<grid, RDF_THREADS, smem, st>>>(a, spos, start, count + ncell, nc[0], nc[1], nc[2]);
        ACK(cudaGetLastError());
        ACK(cudaFreeAsync(count, st));
        ACK(cudaFreeAsync(start, st));
        ACK(cudaFreeAsync(pcell, st));
        ACK(cudaFreeAsync(prank, st));
        ACK(cudaFreeAsync(spos, st));
    }
    std::vector<unsigned long long> tmp(total);
    ACK(timing_end(h, st));
    ACK(cudaMemcpyAsync(tmp.data(), dout, total * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
    ACK(cudaFreeAsync(dout, st));
    ACK(cudaStreamSynchronize(st));
    timing_store(h);
    for (size_t k = 0; k < total; k++) out_host[k] += tmp[k];
    return GDB_OK;
}

static int sq_device(gdb_sim *h, cudaStream_t st, const float4 *pos, const int *orig, int n, const float *ff_host,
                     const float *box, int nq, const int32_t *nvec_host, double *re, double *im) {
    if (nq < 1) return GDB_OK;
    SqArgs a;
    a.pos = pos;
    a.orig = orig;
    a.n = n;
    a.nq = nq;
    for (int d = 0; d < 3; d++) {
        int lo = nvec_host[d], hi = nvec_host[d];
        for (int q = 0; q < nq; q++) {
            lo = nvec_host[3 * q + d] < lo ? nvec_host[3 * q + d] : lo;
            hi = nvec_host[3 * q + d] > hi ? nvec_host[3 * q + d] : hi;
        }
        a.kmin[d] = lo;
        a.klen[d] = hi - lo + 1;
        a.invL[d] = 1.0f / box[d];
    }
    const int row = a.klen[0] + a.klen[1] + a.klen[2];
    const size_t smem = (size_t)SQ_TILE * row * sizeof(float2);
    if (smem > 200 * 1024) return aset(h, GDB_ERR_ARG, "sq: n_vectors span too wide");
    int *dn = nullptr;
    float *dff = nullptr;
    double *acc = nullptr;
    ACK(timing_begin(h, st));
    ACK(pool_alloc(&dn, (size_t)nq * 3 * sizeof(int), st));
    ACK(pool_alloc(&acc, (size_t)nq * 2 * sizeof(double), st));
    ACK(cudaMemcpyAsync(dn, nvec_host, (size_t)nq * 3 * sizeof(int), cudaMemcpyHostToDevice, st));
    ACK(cudaMemsetAsync(acc, 0, (size_t)nq * 2 * sizeof(double), st));
    double nf = 0.0;
    if (ff_host) {
        ACK(pool_alloc(&dff, (size_t)n * sizeof(float), st));
        ACK(cudaMemcpyAsync(dff, ff_host, (size_t)n * sizeof(float), cudaMemcpyHostToDevice, st));
        for (int i = 0; i < n; i++) nf += ff_host[i];
    } else {
        nf = n;
    }
    a.nvec = dn;
    a.ff = dff;
    a.acc = acc;
    // q-vectors per thread: up to 4, as few blocks along q as that allows,
    // spread evenly over them (2219 q: 3 blocks of 3 x 256)
    const int nbx = (nq + 4 * SQ_THREADS - 1) / (4 * SQ_THREADS);
    const int qpt = (nq + nbx * SQ_THREADS - 1) / (nbx * SQ_THREADS);
    const dim3 grid(nbx, (n + SQ_CHUNK - 1) / SQ_CHUNK);
    const void *fn = nullptr;
    switch (qpt) {
        case 1: fn = a.ff ? (const void *)k_sq<1, true> : (const void *)k_sq<1, false>; break;
        case 2: fn = a.ff ? (const void *)k_sq<2, true> : (const void *)k_sq<2, false>; break;
        case 3: fn = a.ff ? (const void *)k_sq<3, true> : (const void *)k_sq<3, false>; break;
        default: fn = a.ff ? (const void *)k_sq<4, true> : (const void *)k_sq<4, false>; break;
    }
    ACK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    switch (qpt) {
        case 1: launch_sq<1>(grid, smem, st, a); break;
        case 2: launch_sq<2>(grid, smem, st, a); break;
        case 3: launch_sq<3>(grid, smem, st, a); break;
        default: launch_sq<4>(grid, smem, st, a); break;
    }
    ACK(cudaGetLastError());
    std::vector<double> tmp((size_t)nq * 2);
    ACK(timing_end(h, st));
    ACK(cudaMemcpyAsync(tmp.data(), acc, tmp.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    ACK(cudaFreeAsync(dn, st));
    ACK(cudaFreeAsync(acc, st));
    if (dff) ACK(cudaFreeAsync(dff, st));
    ACK(cudaStreamSynchronize(st));
    timing_store(h);
    const double norm = 1.0 / sqrt(nf);
    for (int q = 0; q < nq; q++) {
        re[q] = tmp[2 * q] * norm;
        im[q] = tmp[2 * q + 1] * norm;
    }
    return GDB_OK;
}

// ---------------------------------------------------------------------------
// S(q) with no device allocation
//
// For callers that cannot let this library call cudaMalloc: applications
// whose own allocator or fixed memory pool owns the GPU's memory, code with
// a hard device-memory budget, and call sites where allocating is not
// allowed while they run.  The caller passes device inputs and outputs; the
// only scratch (the float64 accumulators) is the file-scope array below,
// which every GPU that loads this library holds until the process exits.
// ---------------------------------------------------------------------------
#define GDB_SQ_NOALLOC_MAX_Q 65536  // q-vectors per call
#define GDB_SQ_NOALLOC_MAX_N 48     // largest |n| component (shared table 32 x 291 float2 = 74.5 KB)
#define SQNA_TAIL (2 * GDB_SQ_NOALLOC_MAX_Q)

// [0, 2 nq): (re, im) accumulators; [TAIL]: sum of form factors; [TAIL+1]:
// 1.0 when an n-vector component is outside [-n_max, n_max].  Shared by all
// calls on a device: calls that overlap on the GPU race on it.
static __device__ __align__(256) double g_sq_scratch[SQNA_TAIL + 32];

namespace {

std::mutex g_sq_scratch_mu;
double *g_sq_scratch_addr[256] = {nullptr};

// Device address of g_sq_scratch on the current device, looked up once per
// device (host code cannot use the symbol itself as a device address).
int sq_scratch_address(int dev, double **out) {
    std::lock_guard<std::mutex> lock(g_sq_scratch_mu);
    if (dev < 0 || dev >= 256) return GDB_ERR_ARG;
    if (!g_sq_scratch_addr[dev]) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_sq_scratch) != cudaSuccess || !p) return GDB_ERR_CUDA;
        g_sq_scratch_addr[dev] = (double *)p;
    }
    *out = g_sq_scratch_addr[dev];
    return GDB_OK;
}

__global__ void k_sqna_clear(double *s, int nq) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < 2 * nq; k += gridDim.x * blockDim.x) s[k] = 0.0;
    if (blockIdx.x == 0 && threadIdx.x < 2) s[SQNA_TAIL + threadIdx.x] = 0.0;
}

__global__ void k_sqna_weight_sum(const float *ff, int n, double *s) {
    __shared__ double sm[32];
    double v = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) v += ff ? ff[i] : 1.0;
    v = warp_sum(v);
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
        double w = threadIdx.x < (blockDim.x >> 5) ? sm[threadIdx.x] : 0.0;
        w = warp_sum(w);
        if (threadIdx.x == 0) atomicAdd(&s[SQNA_TAIL], w);
    }
}

// Same tabulated-phase method as k_sq; positions are the caller's (n, 3)
// float32 array, n-vector components lie in [-nmax, nmax].
__global__ void __launch_bounds__(SQ_THREADS) k_sqna(const float *__restrict__ r, const float *__restrict__ ff, int n,
                                                     const int *__restrict__ nvec, int nq, int nmax, float ilx,
                                                     float ily, float ilz, double *s) {
    extern __shared__ float2 tab[];
    __shared__ float wsh[SQ_TILE];
    const int span = 2 * nmax + 1, row = 3 * span;
    const int q = blockIdx.x * SQ_THREADS + threadIdx.x;
    bool ok = q < nq;
    int nx = 0, ny = 0, nz = 0;
    if (ok) {
        const int a = nvec[3 * q], b = nvec[3 * q + 1], c = nvec[3 * q + 2];
        if (a < -nmax || a > nmax || b < -nmax || b > nmax || c < -nmax || c > nmax) {
            s[SQNA_TAIL + 1] = 1.0;
            ok = false;
        } else {
            nx = a + nmax;
            ny = b + nmax + span;
            nz = c + nmax + 2 * span;
        }
    }
    const float il[3] = {ilx, ily, ilz};
    double sr = 0.0, si = 0.0;
    const int p_begin = blockIdx.y * SQ_CHUNK;
    const int p_end = min(n, p_begin + SQ_CHUNK);
    for (int p0 = p_begin; p0 < p_end; p0 += SQ_TILE) {
        const int np = min(SQ_TILE, p_end - p0);
        __syncthreads();
        for (int e = threadIdx.x; e < np * row; e += SQ_THREADS) {
            const int pl = e / row, col = e % row;
            const int d = col / span, k = col % span - nmax;
            const float x = r[3 * (size_t)(p0 + pl) + d];
            float sn, cs;
            sincospif(2.0f * (float)k * (x * il[d]), &sn, &cs);
            tab[pl * row + col] = make_float2(cs, sn);
        }
        if (threadIdx.x < np) wsh[threadIdx.x] = ff ? ff[p0 + threadIdx.x] : 1.0f;
        __syncthreads();
        if (ok) {
            float tr = 0.f, ti = 0.f;
            for (int pl = 0; pl < np; pl++)
                sq_term(tab[pl * row + nx], tab[pl * row + ny], tab[pl * row + nz], wsh[pl], true, tr, ti);
            sr += tr;
            si += ti;
        }
    }
    if (ok) {
        atomicAdd(&s[2 * q], sr);
        atomicAdd(&s[2 * q + 1], si);
    }
}

__global__ void k_sqna_finish(const double *s, int nq, double *re, double *im) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nq) return;
    const double norm = 1.0 / sqrt(s[SQNA_TAIL]);
    re[q] = s[2 * q] * norm;
    im[q] = s[2 * q + 1] * norm;
}

}  // namespace

extern "C" {

int gdb_sq_compute_noalloc(int n, const float *r_dev, const float *ff_dev, const float box[3], int nq,
                           const int32_t *n_vectors_dev, int n_max, double *rho_re_dev, double *rho_im_dev,
                           void *stream) {
    gdb_sim *h = nullptr;
    if (n < 1 || nq < 1 || !r_dev || !box || !n_vectors_dev || !rho_re_dev || !rho_im_dev)
        return aset(h, GDB_ERR_ARG, "gdb_sq_compute_noalloc: bad arguments");
    if (nq > GDB_SQ_NOALLOC_MAX_Q)
        return aset(h, GDB_ERR_ARG, "gdb_sq_compute_noalloc: more than 65536 q-vectors");
    if (n_max < 0 || n_max > GDB_SQ_NOALLOC_MAX_N)
        return aset(h, GDB_ERR_ARG, "gdb_sq_compute_noalloc: n_max must be in [0, 48]");
    if (!(box[0] > 0.f && box[1] > 0.f && box[2] > 0.f))
        return aset(h, GDB_ERR_ARG, "gdb_sq_compute_noalloc: non-positive box length");
    int dev = 0;
    ACK(cudaGetDevice(&dev));
    double *s = nullptr;
    int rc = sq_scratch_address(dev, &s);
    if (rc) return aset(h, rc, "gdb_sq_compute_noalloc: scratch address lookup failed");
    cudaStream_t st = (cudaStream_t)stream;
    const int span = 2 * n_max + 1;
    const size_t smem = (size_t)SQ_TILE * 3 * span * sizeof(float2);
    ACK(cudaFuncSetAttribute(k_sqna, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_sqna_clear<<<(2 * nq + 255) / 256, 256, 0, st>>>(s, nq);
    k_sqna_weight_sum<<<64, 256, 0, st>>>(ff_dev, n, s);
    dim3 grid((nq + SQ_THREADS - 1) / SQ_THREADS, (n + SQ_CHUNK - 1) / SQ_CHUNK);
    k_sqna<<<grid, SQ_THREADS, smem, st>>>(r_dev, ff_dev, n, n_vectors_dev, nq, n_max, 1.0f / box[0],
                                           1.0f / box[1], 1.0f / box[2], s);
    k_sqna_finish<<<(nq + 255) / 256, 256, 0, st>>>(s, nq, rho_re_dev, rho_im_dev);
    ACK(cudaGetLastError());
    double flag = 0.0;
    ACK(cudaMemcpyAsync(&flag, s + SQNA_TAIL + 1, sizeof(double), cudaMemcpyDeviceToHost, st));
    ACK(cudaStreamSynchronize(st));
    if (flag != 0.0)
        return aset(h, GDB_ERR_ARG, "gdb_sq_compute_noalloc: an n-vector component is outside [-n_max, n_max]");
    return GDB_OK;
}

int gdb_rdf_update(gdb_sim *h, int bins, double r_max, uint64_t *out) {
    if (!h || !out) return aset(h, GDB_ERR_ARG, "gdb_rdf_update: NULL argument");
    if (!gdb_internal_uploaded(h)) return aset(h, GDB_ERR_STATE, "state not uploaded");
    ACK(cudaSetDevice(gdb_internal_dev(h)));
    return rdf_device(h, gdb_internal_stream(h), gdb_internal_pos(h), gdb_internal_n(h), gdb_internal_box(h),
                      gdb_internal_ntypes(h), bins, r_max, out);
}

int gdb_sq_update(gdb_sim *h, int nq, const int32_t *n_vectors, const float *ff, double *rho_re, double *rho_im) {
    if (!h || !n_vectors || !rho_re || !rho_im) return aset(h, GDB_ERR_ARG, "gdb_sq_update: NULL argument");
    if (!gdb_internal_uploaded(h)) return aset(h, GDB_ERR_STATE, "state not uploaded");
    ACK(cudaSetDevice(gdb_internal_dev(h)));
    return sq_device(h, gdb_internal_stream(h), gdb_internal_pos(h), gdb_internal_orig(h), gdb_internal_n(h), ff,
                     gdb_internal_box(h), nq, n_vectors, rho_re, rho_im);
}

int gdb_rdf_compute(int n, const float *r, const int32_t *ptype, const float box[3], int ntypes, int bins,
                    double r_max, uint64_t *out) {
    gdb_sim *h = nullptr;
    if (n < 1 || !r || !box || !out || ntypes < 1) return aset(h, GDB_ERR_ARG, "gdb_rdf_compute: bad arguments");
    if (ptype)
        for (int i = 0; i < n; i++)
            if (ptype[i] < 0 || ptype[i] >= ntypes) return aset(h, GDB_ERR_ARG, "gdb_rdf_compute: type out of range");
    cudaStream_t st;
    ACK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    float *dr = nullptr;
    int *dpt = nullptr, *orig = nullptr;
    float4 *pos = nullptr;
    int rc = GDB_OK;
    do {
        cudaError_t e;
        if ((e = pool_alloc(&dr, (size_t)n * 3 * sizeof(float), st)) ||
            (e = pool_alloc(&pos, (size_t)n * sizeof(float4), st)) ||
            (e = pool_alloc(&orig, (size_t)n * sizeof(int), st)) ||
            (ptype && (e = pool_alloc(&dpt, (size_t)n * sizeof(int), st))) ||
            (e = cudaMemcpyAsync(dr, r, (size_t)n * 3 * sizeof(float), cudaMemcpyHostToDevice, st)) ||
            (ptype && (e = cudaMemcpyAsync(dpt, ptype, (size_t)n * sizeof(int), cudaMemcpyHostToDevice, st)))) {
            rc = aset(h, GDB_ERR_CUDA, "gdb_rdf_compute: staging", e);
            break;
        }
        k_pack_pos<<<(n + 255) / 256, 256, 0, st>>>(n, dr, dpt, pos, orig);
        rc = rdf_device(h, st, pos, n, box, ntypes, bins, r_max, out);
    } while (0);
    if (dr) cudaFreeAsync(dr, st);
    if (pos) cudaFreeAsync(pos, st);
    if (orig) cudaFreeAsync(orig, st);
    if (dpt) cudaFreeAsync(dpt, st);
    cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
    return rc;
}

int gdb_sq_compute(int n, const float *r, const float *ff, const float box[3], int nq, const int32_t *n_vectors,
                   double *rho_re, double *rho_im) {
    gdb_sim *h = nullptr;
    if (n < 1 || !r || !box || !n_vectors || !rho_re || !rho_im) return aset(h, GDB_ERR_ARG, "gdb_sq_compute: bad arguments");
    cudaStream_t st;
    ACK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    float *dr = nullptr;
    int *orig = nullptr;
    float4 *pos = nullptr;
    int rc = GDB_OK;
    do {
        cudaError_t e;
        if ((e = pool_alloc(&dr, (size_t)n * 3 * sizeof(float), st)) ||
            (e = pool_alloc(&pos, (size_t)n * sizeof(float4), st)) ||
            (e = pool_alloc(&orig, (size_t)n * sizeof(int), st)) ||
            (e = cudaMemcpyAsync(dr, r, (size_t)n * 3 * sizeof(float), cudaMemcpyHostToDevice, st))) {
            rc = aset(h, GDB_ERR_CUDA, "gdb_sq_compute: staging", e);
            break;
        }
        k_pack_pos<<<(n + 255) / 256, 256, 0, st>>>(n, dr, nullptr, pos, orig);
        rc = sq_device(h, st, pos, orig, n, ff, box, nq, n_vectors, rho_re, rho_im);
    } while (0);
    if (dr) cudaFreeAsync(dr, st);
    if (pos) cudaFreeAsync(pos, st);
    if (orig) cudaFreeAsync(orig, st);
    cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
    return rc;
}

// Frames of the blocks from first_block on are uploaded in groups of whole
// blocks that fit a staging budget (1 GiB, GDB_DYN_STAGE_BYTES overrides it),
// plus one buffer with the first frame of every such block for the lags
// longer than a block; frame pairs are launched at most 65535 per grid
// (GDB_DYN_PAIR_CHUNK lowers it), the y extent of a CUDA grid.
static size_t env_size(const char *name, size_t dflt) {
    const char *v = getenv(name);
    if (!v || !*v) return dflt;
    const long long x = atoll(v);
    return x > 0 ? (size_t)x : dflt;
}

static cudaError_t dyn_launch(cudaStream_t st, int gx, const float *frames, int n, const int *dpt, int nt,
                              const float *box, const int2 *dpairs, const double *dq, double *dacc, int count,
                              int chunk) {
    for (int off = 0; off < count; off += chunk) {
        const int c = std::min(chunk, count - off);
        k_dynamics<<<dim3(gx, c), DYN_THREADS, 0, st>>>(frames, n, dpt, nt, box[0], box[1], box[2], dpairs + off, dq,
                                                        dacc + (size_t)off * nt * 3);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

int gdb_calc_dynamics(int num_blocks, int conf_per_block, int n, const float *frames, const int32_t *ptype,
                      int ntypes, const float box[3], int first_block, const double *qvalues, int total_times,
                      double *msd, double *m4d, double *fs, int32_t *count) {
    gdb_sim *h = nullptr;
    if (num_blocks < 1 || conf_per_block < 1 || n < 1 || !frames || !ptype || !box || !qvalues || !msd || !m4d ||
        !fs || !count || ntypes < 1)
        return aset(h, GDB_ERR_ARG, "gdb_calc_dynamics: bad arguments");
    if (ntypes > DYN_MAX_TYPES) return aset(h, GDB_ERR_ARG, "gdb_calc_dynamics: more than 8 particle types");
    if (first_block < 0 || first_block >= num_blocks)
        return aset(h, GDB_ERR_ARG, "gdb_calc_dynamics: first_block outside [0, num_blocks)");
    int extra = 0;  // int(log2(num_blocks - first_block)) - 1
    while ((2 << extra) <= num_blocks - first_block) extra++;
    extra -= 1;
    if (extra < 0)  // the reference indexes past its arrays there
        return aset(h, GDB_ERR_ARG, "gdb_calc_dynamics: needs at least two blocks from first_block on");
    if (total_times != conf_per_block - 1 + extra)
        return aset(h, GDB_ERR_ARG, "gdb_calc_dynamics: total_times must be conf_per_block - 1 + log2 term");
    std::vector<int> nper(ntypes, 0);
    for (int i = 0; i < n; i++) {
        if (ptype[i] < 0 || ptype[i] >= ntypes) return aset(h, GDB_ERR_ARG, "gdb_calc_dynamics: type out of range");
        nper[ptype[i]]++;
    }
    const int fb = first_block, nblk = num_blocks - first_block, cpb = conf_per_block;
    const size_t frame_floats = (size_t)2 * n * 3;
    const size_t block_bytes = (size_t)cpb * frame_floats * sizeof(float);
    const int group = (int)std::max<size_t>(1, std::min<size_t>(nblk, env_size("GDB_DYN_STAGE_BYTES", 1ull << 30) /
                                                                       block_bytes));
    const int chunk = (int)std::min<size_t>(65535, env_size("GDB_DYN_PAIR_CHUNK", 65535));
    // frame pairs in the reference's loop order (calc_dynamics.py:50-63),
    // as indices into the staging buffers: within-block lags into the
    // group's buffer, longer lags into the buffer of first frames
    std::vector<int2> pairs;
    std::vector<int> tindex;
    for (int k = 0; k < total_times; k++) count[k] = 0;
    for (int b = fb; b < num_blocks; b++) {
        const int base = ((b - fb) % group) * cpb;
        for (int i = 0; i < cpb - 1; i++) {
            count[i]++;
            pairs.push_back(make_int2(base + i + 1, base));
            tindex.push_back(i);
        }
    }
    const int np_in = (int)pairs.size();
    for (int b = fb; b < num_blocks; b++)
        for (int i = 0; i < extra; i++) {
            const int other = b + (2 << i);
            if (other < num_blocks) {
                count[cpb - 1 + i]++;
                pairs.push_back(make_int2(other - fb, b - fb));
                tindex.push_back(cpb - 1 + i);
            }
        }
    const int np_ = (int)pairs.size();
    for (int k = 0; k < total_times * ntypes; k++) msd[k] = m4d[k] = fs[k] = 0.0;
    cudaStream_t st;
    ACK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    float *dgroup = nullptr, *dfirst = nullptr;
    int *dpt = nullptr;
    int2 *dpairs = nullptr;
    double *dq = nullptr, *dacc = nullptr;
    std::vector<double> acc((size_t)std::max(np_, 1) * ntypes * 3);
    int rc = GDB_OK;
    do {
        cudaError_t e;
        if ((e = pool_alloc(&dgroup, (size_t)group * block_bytes, st)) ||
            (e = pool_alloc(&dfirst, (size_t)nblk * frame_floats * sizeof(float), st)) ||
            (e = pool_alloc(&dpt, (size_t)n * sizeof(int), st)) ||
            (e = pool_alloc(&dpairs, (size_t)std::max(np_, 1) * sizeof(int2), st)) ||
            (e = pool_alloc(&dq, (size_t)ntypes * sizeof(double), st)) ||
            (e = pool_alloc(&dacc, acc.size() * sizeof(double), st)) ||
            (e = cudaMemcpyAsync(dpt, ptype, (size_t)n * sizeof(int), cudaMemcpyHostToDevice, st)) ||
            (e = cudaMemcpyAsync(dpairs, pairs.data(), (size_t)np_ * sizeof(int2), cudaMemcpyHostToDevice, st)) ||
            (e = cudaMemcpyAsync(dq, qvalues, (size_t)ntypes * sizeof(double), cudaMemcpyHostToDevice, st)) ||
            (e = cudaMemsetAsync(dacc, 0, acc.size() * sizeof(double), st))) {
            rc = aset(h, GDB_ERR_CUDA, "gdb_calc_dynamics: staging", e);
            break;
        }
        const int gx = std::min((n + DYN_THREADS - 1) / DYN_THREADS, 64);
        // lags within a block, one group of blocks at a time (stream order
        // keeps a group's kernels ahead of the next group's upload)
        for (int g0 = 0; g0 < nblk && !e; g0 += group) {
            const int gb = std::min(group, nblk - g0);
            const float *src = frames + (size_t)(fb + g0) * cpb * frame_floats;
            if ((e = cudaMemcpyAsync(dgroup, src, (size_t)gb * block_bytes, cudaMemcpyHostToDevice, st))) break;
            for (int b = 0; b < gb && !e; b++) {
                const float *f0 = src + (size_t)b * cpb * frame_floats;
                e = cudaMemcpyAsync(dfirst + (size_t)(g0 + b) * frame_floats, f0, frame_floats * sizeof(float),
                                    cudaMemcpyHostToDevice, st);
            }
            if (e) break;
            const int p0 = g0 * (cpb - 1), pc = gb * (cpb - 1);
            e = dyn_launch(st, gx, dgroup, n, dpt, ntypes, box, dpairs + p0, dq, dacc + (size_t)p0 * ntypes * 3, pc,
                           chunk);
        }
        // lags of whole blocks, between first frames
        if (!e && np_ > np_in)
            e = dyn_launch(st, gx, dfirst, n, dpt, ntypes, box, dpairs + np_in, dq,
                           dacc + (size_t)np_in * ntypes * 3, np_ - np_in, chunk);
        if (e || (e = cudaMemcpyAsync(acc.data(), dacc, acc.size() * sizeof(double), cudaMemcpyDeviceToHost, st)) ||
            (e = cudaStreamSynchronize(st))) {
            rc = aset(h, GDB_ERR_CUDA, "gdb_calc_dynamics: kernel", e);
            break;
        }
        // per pair and type: the means over the type's particles (and, for
        // Fs, components) added at the pair's time index, then / count; a
        // type without particles is NaN, as numpy's mean of an empty array
        for (int p = 0; p < np_; p++)
            for (int t = 0; t < ntypes; t++) {
                if (nper[t] == 0) continue;
                const double *a = &acc[((size_t)p * ntypes + t) * 3];
                const size_t o = (size_t)tindex[p] * ntypes + t;
                msd[o] += a[0] / nper[t];
                m4d[o] += a[1] / nper[t];
                fs[o] += a[2] / (3.0 * nper[t]);
            }
        for (int k = 0; k < total_times; k++)
            for (int t = 0; t < ntypes; t++) {
                const size_t o = (size_t)k * ntypes + t;
                if (nper[t] == 0) {
                    msd[o] = m4d[o] = fs[o] = NAN;
                    continue;
                }
                msd[o] /= count[k];
                m4d[o] /= count[k];
                fs[o] /= count[k];
            }
    } while (0);
    if (dgroup) cudaFreeAsync(dgroup, st);
    if (dfirst) cudaFreeAsync(dfirst, st);
    if (dpt) cudaFreeAsync(dpt, st);
    if (dpairs) cudaFreeAsync(dpairs, st);
    if (dq) cudaFreeAsync(dq, st);
    if (dacc) cudaFreeAsync(dacc, st);
    cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
    return rc;
}

}  // extern "C"
