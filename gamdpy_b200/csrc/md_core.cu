// md_core.cu -- simulation handle, neighbour lists, fused force+integrate step.
//
// Replaces, B200-native, the numba.cuda kernels of gamdpy's hot path:
//   interactions/pair_potential.py:141-246   (forces, U, W, lapU)
//   interactions/nblist.py:57-143            (N^2 list: check + build)
//   interactions/nblist_linked_lists.py:84-218 (cell list: check, cells, build, clear)
//   integrators/NVE.py:59-105, integrators/NVT.py:75-124
//   runtime_actions/scalar_saver.py:161-197, runtime_actions/momentum_reset.py:44-103
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
//  * By default a timeblock is one launch of the persistent cooperative kernel
//    k_run (md_kernels.cuh), or of the thread-block-cluster kernel for small
//    systems (md_cluster.cu).  The fallback (GDB_PERSISTENT=0) captures the
//    launch sequence of a chunk of steps once in a CUDA graph and replays it.
#include <cuda_runtime.h>
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/gamdb200.h"
#include "gdb_internal.cuh"
#include "md_kernels.cuh"
#include "md_cluster.cuh"


using namespace gdb;

namespace {

char g_lib_error[512] = "";

}  // namespace

// The persistent kernel builds cell-kind lists with the N^2 build up to this
// many particles: the same sets in one phase instead of the cell build's
// seven phases and grid barriers (measured on B200, KA rho 1.2, TPS cell vs
// N^2 build: N 2048 56.6k vs 70.9k, N 4096 46.0k vs 43.0k, N 8192 38.2k vs
// 23.2k).  GDB_NSQ_AUTO=<N> moves the limit, 0 switches it off.
constexpr int NSQ_AUTO_MAX = 3072;
// persistent N^2 builds stage the positions in shared memory up to this N
// (48 KiB, the default dynamic limit)
constexpr int NSQ_SMEM_MAX = 3072;

// Systems from this many particles take the brick path on the persistent
// kernel (GDB_BRICK_MIN_N moves it; GDB_BRICKS=0 switches the path off).
constexpr int BRICK_MIN_N = 131073;

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
    // NPT_Atomic: masses without the temperature factor, target pressure
    float npt_mass_t = 0.f, npt_mass_p = 0.f;
    int pfunc = 0;
    float pparams[4] = {0, 0, 0, 0};
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
    unsigned long long *trace = nullptr;
    int trace_cap = 0;
    float *conf = nullptr;  // ConfigurationSaver frames
    int conf_per_block = 0;
    int cur = 0;
    int num_sms = 148;
    bool persistent = true;
    bool cluster_ok = true;  // small systems run resident in one thread-block cluster
    bool cluster_force = false;  // GDB_CLUSTER=1: the cluster path whenever it fits
    int nsq_auto_max = NSQ_AUTO_MAX;  // persistent kernel: N^2 build up to this N (GDB_NSQ_AUTO)
    bool nsq_stage = true;            // persistent N^2 build from staged positions (GDB_NSQ_STAGE=0: from L2)
    // the staged-halo path of large cell-list systems on the persistent
    // kernel (md_bricks.cuh): cells numbered in bricks of 4 x 4 x 4 cells,
    // each brick's halo staged in shared memory.  Off by default (measured
    // slower than the row path on B200); GDB_BRICKS=1 (or 2) switches it on.
    bool bricks_req = false;  // GDB_BRICKS
    bool staged_ok = true;    // cleared when a halo outgrew its stage
    bool bricks_ok = true;    // cleared for batches' cluster systems (they run the row phases)
    int order = 0;            // 0: row order; 2: the staged-halo path's brick order
    int nb[3] = {0, 0, 0};    // bricks per dimension
    int brick_min_n = BRICK_MIN_N;  // GDB_BRICK_MIN_N
    int brick_hcap = BRICK_HCAP;    // GDB_BRICK_HCAP lowers the stage the kernels may fill (tests of the fallback)
    int last_path = -1;      // 0 graph, 1 persistent grid, 2 cluster
    int grid_cap = 0;        // upper bound on the persistent grid (0: the whole GPU; GDB_GRID_CAP)
    // persistent grid of at most BAR_FLAT_MAX blocks: every block does the
    // step's bookkeeping after the step barrier (GDB_STEP_BARRIER=0: the last
    // block to arrive does it and releases the others)
    bool step_bar_all = true;
    ClusterJob *d_job = nullptr, *h_job = nullptr;
    bool uploaded = false;
    // graphs: [parity] for chunks of GRAPH_STEPS steps
    cudaGraphExec_t gexec[2] = {nullptr, nullptr};
    int graph_steps = 0;
    bool use_graphs = true;
    float analysis_ms = 0.f;  // device time of the last RDF / S(q) call
    // NVT_Langevin: per-particle generators and previous random forces (user index)
    ulonglong2 *rng = nullptr;
    float4 *lbeta = nullptr;
    float alpha = 0.f;
    // molecules: pair exclusions and harmonic bonds (by user index)
    int *excl = nullptr;
    int max_excl = 0;
    int *bond_cnt = nullptr, *bond_j = nullptr, *bond_t = nullptr;
    float2 *bond_prm = nullptr;
    int bond_max = 0;
    int *slot_of = nullptr;
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
// standalone kernels (one phase each; the rebuild chain returns at once
// unless the rebuild flag is set) -- launched in a CUDA graph
// ---------------------------------------------------------------------------
template <bool FMA>
__global__ void __launch_bounds__(GDB_BLOCK) k_nbl_nsq(SimArgs a, int cur) {
    if (!a.ctrl->rebuild) return;
    phase_nbl_nsq<FMA, true>(a, cur);
}
__global__ void __launch_bounds__(GDB_BLOCK) k_cell_assign(SimArgs a, int cur) {
    if (!a.ctrl->rebuild) return;
    phase_cell_assign<true>(a, cur);
}
__global__ void __launch_bounds__(GDB_BLOCK) k_scan_partial(SimArgs a) {
    if (!a.ctrl->rebuild) return;
    phase_scan_partial(a);
}
__global__ void __launch_bounds__(GDB_BLOCK) k_scan_top(SimArgs a) {
    if (!a.ctrl->rebuild) return;
    block_scan_chunks(a);
}
__global__ void __launch_bounds__(GDB_BLOCK) k_scan_final(SimArgs a) {
    if (!a.ctrl->rebuild) return;
    phase_scan_final(a);
}
__global__ void __launch_bounds__(GDB_BLOCK) k_scatter(SimArgs a) {
    if (!a.ctrl->rebuild) return;
    phase_scatter(a);
}
__global__ void __launch_bounds__(GDB_BLOCK) k_sort_cells(SimArgs a) {
    if (!a.ctrl->rebuild) return;
    phase_sort_cells(a);
}
__global__ void __launch_bounds__(GDB_BLOCK) k_gather(SimArgs a, int cur) {
    if (!a.ctrl->rebuild) return;
    phase_gather(a, cur);
}
template <bool FMA>
__global__ void __launch_bounds__(GDB_BLOCK) k_nbl_cells(SimArgs a) {
    if (!a.ctrl->rebuild) return;
    __shared__ NbScratch<GDB_BLOCK / 32> scr;
    phase_nbl_cells<FMA>(a, grid_span(), scr);
}
__global__ void __launch_bounds__(GDB_BLOCK) k_finish_cells(SimArgs a, int cur) {
    if (!a.ctrl->rebuild) return;
    phase_finish_cells(a, cur);
}
__global__ void k_rebuild_done(DevCtrl *ctrl) {
    if (ctrl->rebuild) rebuild_done(ctrl);
}

__global__ void k_block_begin(DevCtrl *ctrl, double time_zero) {
    ctrl->step = 0;
    ctrl->time_zero = time_zero;
    ctrl->bar_count = 0;
    for (int g = 0; g < 64; g++) ctrl->bar_group[g] = 0;
    ctrl->bar_all[0] = ctrl->bar_all[1] = ctrl->bar_all[2] = 0;
    ctrl->abort = 0;
    ctrl->ticket = 0;
    ctrl->work[0] = ctrl->work[1] = 0;
    if (ctrl->rebuild_next) {
        ctrl->rebuild = 1;
        ctrl->rebuild_next = 0;
    }
}

// Continue an abandoned timeblock: clear the abort and barrier state and keep
// the step counter and the block's start time.
__global__ void k_block_resume(DevCtrl *ctrl) {
    ctrl->bar_count = 0;
    for (int g = 0; g < 64; g++) ctrl->bar_group[g] = 0;
    ctrl->bar_all[0] = ctrl->bar_all[1] = ctrl->bar_all[2] = 0;
    ctrl->abort = 0;
    ctrl->ticket = 0;
    ctrl->work[0] = ctrl->work[1] = 0;
    ctrl->rebuild = 1;
    ctrl->rebuild_next = 0;
}

// slot of every user index, from the current order
__global__ void k_fill_slot_of(int n, const int *orig, int *slot_of) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < n) slot_of[orig[s]] = s;
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

// download of the whole state in gamdpy's host layouts, one pass: slot s ->
// user index i = orig[s]; vec (3, n, 3) r, v, f; im (n, 3); sc (n, nscal) with
// column cols[q] for U, W, lapU, K, Fsq and the mass (q = 0..5, -1 = absent)
struct UnpackCols {
    int c[6];
};
__global__ void k_unpack_all(int n, const float4 *pos, const float4 *vel, const float4 *frc, const int4 *img,
                             const float *pscal, const int *orig, float *vec, int *im, float *sc, int nscal,
                             UnpackCols cols) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const size_t i = (size_t)orig[s], N = (size_t)n;
    if (vec) {
        const float4 p = pos[s], v = vel[s], f = frc[s];
        float *r = vec + 3 * i, *vv = vec + 3 * (N + i), *ff = vec + 3 * (2 * N + i);
        r[0] = p.x, r[1] = p.y, r[2] = p.z;
        vv[0] = v.x, vv[1] = v.y, vv[2] = v.z;
        ff[0] = f.x, ff[1] = f.y, ff[2] = f.z;
    }
    if (im) {
        const int4 g = img[s];
        im[3 * i] = g.x, im[3 * i + 1] = g.y, im[3 * i + 2] = g.z;
    }
    if (sc) {
        float *row = sc + i * nscal;
#pragma unroll
        for (int q = 0; q < 5; q++)
            if (cols.c[q] >= 0) row[cols.c[q]] = pscal[q * N + s];
        if (cols.c[5] >= 0) row[cols.c[5]] = vel[s].w;
    }
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
    // about 131k lanes in flight (measured on B200: 1 lane per particle at
    // N = 1M, 2 at 65k; at 2k, 32 lanes on 256 blocks 100 k TPS against 93 k
    // with 16 lanes, once grids up to 320 blocks take the one-level barrier)
    int tp = 1;
    while (tp < 32 && (long long)h->n * tp < 131072) tp *= 2;
    return tp;
}

static int ensure_nblist(gdb_sim *h) {
    const int tp = choose_tp(h);
    const int stride = (h->n + 31) / 32 * 32;
    const size_t need = ((size_t)h->max_nbs + NB_CHUNK) * stride;
    if (need > h->nbl_elems) {
        if (h->nbl) cudaFree(h->nbl);
        h->nbl = nullptr;
        CK(cudaMalloc(&h->nbl, need * sizeof(int)));
        h->nbl_elems = need;
        free_graphs(h);
        if (h->uploaded) CK(cudaMemsetAsync(&h->ctrl->rebuild, 0xff, sizeof(int), h->st));  // nonzero
    }
    if (tp != h->tp) {
        h->tp = tp;
        free_graphs(h);
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
        // the brick path: a persistent large system whose grid holds the
        // 8-cell halo of a brick in every dimension and whose expected halo
        // fits the stage with a quarter to spare
        const double per_cell = (double)h->n / ((double)nc[0] * nc[1] * nc[2]);
        const bool use = h->bricks_req && h->bricks_ok && h->staged_ok && h->persistent && !h->excl &&
                         h->integ != GDB_INTEGRATOR_NPT &&
                         !h->bond_cnt &&
                         h->n >= h->brick_min_n && h->n > h->nsq_auto_max && nc[0] >= BRICK_W &&
                         nc[1] >= BRICK_W && nc[2] >= BRICK_W &&
                         per_cell * BRICK_W * BRICK_W * BRICK_W * 1.25 <= BRICK_HCAP;
        const int order = use ? 2 : 0;
        const bool want = order != 0;
        if (order != h->order) {
            h->order = order;
            free_graphs(h);
            if (h->uploaded) {
                int one = 1;
                CK(cudaMemcpyAsync(&h->ctrl->rebuild, &one, sizeof(int), cudaMemcpyHostToDevice, h->st));
            }
        }
        for (int k = 0; k < 3; k++) h->nb[k] = want ? (nc[k] + BRICK - 1) / BRICK : 0;
        const int ncell = want ? h->nb[0] * h->nb[1] * h->nb[2] * BRICK * BRICK * BRICK : nc[0] * nc[1] * nc[2];
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
            free_graphs(h);
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

static SimArgs make_args(gdb_sim *h) {
    SimArgs a;
    a.nsq_smem = 0;
    a.bar_all = h->step_bar_all ? 1 : 0;
    a.pos0 = h->pos[0];
    a.pos1 = h->pos[1];
    a.vel = h->vel;
    a.img = h->img;
    a.rref = h->rref;
    a.frc = h->frc;
    a.pos_tmp = h->pos_tmp;
    a.vel_tmp = h->vel_tmp;
    a.img_tmp = h->img_tmp;
    a.orig = h->orig;
    a.orig_tmp = h->orig_tmp;
    a.nbl = h->nbl;
    a.nbc = h->nbc;
    a.pscal = h->pscal;
    a.pscal_tmp = h->pscal_tmp;
    a.cell_count = h->cell_count;
    a.cell_start = h->cell_start;
    a.pcell = h->pcell;
    a.prank = h->prank;
    a.perm = h->perm;
    a.scell = h->scell;
    a.bsum = h->bsum;
    a.partials = h->partials;
    a.rows = h->rows;
    a.conf = h->conf;
    a.conf_box = h->conf ? h->conf + (size_t)h->conf_per_block * 2 * h->n * 3 : nullptr;
    a.ctrl = h->ctrl;
    a.n = h->n;
    a.stride = h->stride;
    a.max_nbs = h->max_nbs;
    a.ncell = h->nb_kind == GDB_NBLIST_CELLS ? h->ncell : 0;
    a.nchunks = (a.ncell + SCAN_CHUNK - 1) / SCAN_CHUNK;
    a.ncx = h->nc[0];
    a.ncy = h->nc[1];
    a.ncz = h->nc[2];
    const int order = h->nb_kind == GDB_NBLIST_CELLS ? h->order : 0;
    a.nbx = order ? h->nb[0] : 0;
    a.nby = order ? h->nb[1] : 0;
    a.nbz = order ? h->nb[2] : 0;
    a.brick_hcap = h->brick_hcap;
    a.nb_kind = h->nb_kind;
    a.fma = h->fma;
    a.Lx = h->box[0];
    a.Ly = h->box[1];
    a.Lz = h->box[2];
    const float cps = h->max_cut + h->skin;  // nblist.py:152 (max_cut+skin, float32)
    a.cps2 = cps * cps;
    a.skin2q = h->skin * h->skin * 0.25f;
    a.dt = h->dt;
    a.omega2 = h->integ == GDB_INTEGRATOR_NVT ? h->omega2 : 0.f;
    a.dof = 3LL * h->n - 3;
    a.tfunc = h->tfunc;
    a.tp0 = h->tparams[0];
    a.tp1 = h->tparams[1];
    a.tp2 = h->tparams[2];
    a.tp3 = h->tparams[3];
    a.npt_mass_t = h->npt_mass_t;
    a.npt_mass_p = h->npt_mass_p;
    a.pfunc = h->pfunc;
    a.pp0 = h->pparams[0];
    a.pp1 = h->pparams[1];
    a.pp2 = h->pparams[2];
    a.pp3 = h->pparams[3];
    a.min_cell = (h->max_cut + h->skin) / 2.0f;  // nblist_linked_lists.py:36
    a.ncx_max = h->nc[0];
    a.ncy_max = h->nc[1];
    a.ncz_max = h->nc[2];
    if (h->integ == GDB_INTEGRATOR_NPT && h->nb_kind == GDB_NBLIST_CELLS && a.ncell > 0) {
        // the grid of the current box, within the allocated one
        int nc[3];
        for (int k = 0; k < 3; k++) nc[k] = std::min(h->nc[k], std::max(1, (int)(h->box[k] / a.min_cell)));
        a.ncx = nc[0];
        a.ncy = nc[1];
        a.ncz = nc[2];
        a.ncell = nc[0] * nc[1] * nc[2];
        a.nchunks = (a.ncell + SCAN_CHUNK - 1) / SCAN_CHUNK;
    }
    a.every = h->scalar_every;
    a.reset_every = h->momentum_every;
    a.nrows = h->rows ? h->rows_cap : 0;
    a.conf_per_block = h->conf_per_block;
    a.rng = h->rng;
    a.lbeta = h->lbeta;
    a.alpha = h->alpha;
    a.excl = h->excl;
    a.max_excl = h->max_excl;
    a.bond_cnt = h->bond_cnt;
    a.bond_j = h->bond_j;
    a.bond_t = h->bond_t;
    a.bond_prm = h->bond_prm;
    a.bond_max = h->bond_max;
    a.slot_of = h->slot_of;
    return a;
}

// Enqueue the (flag-gated) rebuild chain for the current buffer.
static int enqueue_rebuild(gdb_sim *h) {
    const SimArgs a = make_args(h);
    const int n = h->n, cur = h->cur;
    if (h->nb_kind == GDB_NBLIST_NSQ) {
        if (h->fma)
            k_nbl_nsq<true><<<grid_for((long long)n * 32), GDB_BLOCK, 0, h->st>>>(a, cur);
        else
            k_nbl_nsq<false><<<grid_for((long long)n * 32), GDB_BLOCK, 0, h->st>>>(a, cur);
        CKL();
    } else {
        const int g = grid_for(n);
        k_cell_assign<<<g, GDB_BLOCK, 0, h->st>>>(a, cur);
        k_scan_partial<<<a.nchunks, GDB_BLOCK, 0, h->st>>>(a);
        k_scan_top<<<1, GDB_BLOCK, 0, h->st>>>(a);
        k_scan_final<<<a.nchunks, GDB_BLOCK, 0, h->st>>>(a);
        k_scatter<<<g, GDB_BLOCK, 0, h->st>>>(a);
        k_sort_cells<<<grid_for(a.ncell), GDB_BLOCK, 0, h->st>>>(a);
        k_gather<<<g, GDB_BLOCK, 0, h->st>>>(a, cur);
        // a warp per cell, or a thread per particle for large systems (the
        // build picks by threads per particle)
        const int gw = n >= 131072 ? grid_for(n) : grid_for((long long)a.ncell * 32);
        if (h->fma)
            k_nbl_cells<true><<<gw, GDB_BLOCK, 0, h->st>>>(a);
        else
            k_nbl_cells<false><<<gw, GDB_BLOCK, 0, h->st>>>(a);
        k_finish_cells<<<g, GDB_BLOCK, 0, h->st>>>(a, cur);
        CKL();
    }
    k_rebuild_done<<<1, 1, 0, h->st>>>(h->ctrl);
    CKL();
    return GDB_OK;
}

static int enqueue_step(gdb_sim *h, int mode) {
    const int grid = grid_for((long long)h->n * h->tp);
    int rc = ensure_partials(h, grid);
    if (rc) return rc;
    const SimArgs a = make_args(h);
    if (h->ntypes == 1)
        launch_step_nt1(a, h->table, h->st, h->tp, h->integ, mode, grid, h->cur);
    else if (h->ntypes == 2)
        launch_step_nt2(a, h->table, h->st, h->tp, h->integ, mode, grid, h->cur);
    else
        launch_step_ntg(a, h->table, h->st, h->tp, h->integ, mode, grid, h->cur);
    CKL();
    if (mode == MODE_STEP) h->cur ^= 1;
    return GDB_OK;
}

// Grid of the persistent kernel: every block resident (cooperative launch).
static int run_grid(gdb_sim *h, const void *fn, int *grid, size_t dsmem = 0) {
    int occ = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, GDB_BLOCK, dsmem));
    if (occ < 1) return set_err(h, GDB_ERR_CUDA, "persistent kernel cannot be resident");
    const int needed = grid_for((long long)h->n * h->tp);
    *grid = std::min(std::min(needed, occ * h->num_sms), 64 * BAR_GROUP);
    if (h->grid_cap > 0) *grid = std::min(*grid, h->grid_cap);
    return GDB_OK;
}

// One launch of k_run: `steps` steps from pos[cur], then the final evaluation.
static int launch_run_bricks(gdb_sim *h, int steps, int do_eval) {
    const void *fn = h->ntypes == 1   ? run_bricks_kernel_nt1(h->integ)
                     : h->ntypes == 2 ? run_bricks_kernel_nt2(h->integ)
                                      : run_bricks_kernel_ntg(h->integ);
    const size_t smem = sizeof(BrickSmem);
    CK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int occ = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, BRICK_THREADS, smem));
    if (occ < 1) return set_err(h, GDB_ERR_CUDA, "brick kernel cannot be resident");
    const int nbricks = h->nb[0] * h->nb[1] * h->nb[2];
    int grid = std::min(std::min(nbricks, occ * h->num_sms), 64 * BAR_GROUP);
    if (h->grid_cap > 0) grid = std::min(grid, h->grid_cap);
    int rc;
    if ((rc = ensure_partials(h, nbricks))) return rc;
    SimArgs a = make_args(h);
    int cur0 = h->cur, ns = steps, ev = do_eval;
    void *args[] = {(void *)&a, (void *)&h->table, (void *)&cur0, (void *)&ns, (void *)&ev};
    CK(cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(BRICK_THREADS), args, smem, h->st));
    h->cur ^= (steps & 1);
    return GDB_OK;
}

static int launch_run(gdb_sim *h, int steps, int do_eval) {
    if (h->order == 2 && h->nb_kind == GDB_NBLIST_CELLS) return launch_run_bricks(h, steps, do_eval);
    const void *fn = h->ntypes == 1   ? run_kernel_nt1(h->tp, h->integ)
                     : h->ntypes == 2 ? run_kernel_nt2(h->tp, h->integ)
                                      : run_kernel_ntg(h->tp, h->integ);
    SimArgs a = make_args(h);
    if (a.nb_kind == GDB_NBLIST_CELLS && h->n <= h->nsq_auto_max) {
        // same neighbour sets as the cell build (in another order), one phase
        a.nb_kind = GDB_NBLIST_NSQ;
        a.ncell = 0;
        a.nchunks = 0;
        a.nbx = a.nby = a.nbz = 0;
    }
    // small N^2 systems: every block stages the positions for the list build
    const size_t dsmem =
        (a.nb_kind == GDB_NBLIST_NSQ && h->n <= NSQ_SMEM_MAX && h->nsq_stage) ? (size_t)h->n * sizeof(float4) : 0;
    a.nsq_smem = dsmem > 0;
    // static plus dynamic shared memory above 48 KiB needs the opt-in
    if (dsmem > 0) CK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dsmem));
    int grid = 0;
    int rc = run_grid(h, fn, &grid, dsmem);
    if (rc) return rc;
    // a row per round, two steps' rows where every block keeps the books
    if ((rc = ensure_partials(h, std::max(grid, 2 * grid_for((long long)h->n * h->tp))))) return rc;
    a.partials = h->partials;
    int cur0 = h->cur, ns = steps, ev = do_eval;
    void *args[] = {(void *)&a, (void *)&h->table, (void *)&cur0, (void *)&ns, (void *)&ev};
    CK(cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(GDB_BLOCK), args, dsmem, h->st));
    h->cur ^= (steps & 1);
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
    if (h->h_ctrl->status & GDB_STATUS_BAD_INDEX)
        return set_err(h, GDB_ERR_NUMERIC, "cell sort produced a slot outside the particle range");
    if (h->h_ctrl->status & GDB_STATUS_BARRIER_TIMEOUT) {
        // an abandoned rebuild leaves counted cells behind: clear them and
        // rebuild before the next step
        if (h->cell_count) cudaMemsetAsync(h->cell_count, 0, (size_t)h->cell_cap * sizeof(int), h->st);
        int one = 1;
        cudaMemcpyAsync(&h->ctrl->rebuild, &one, sizeof(int), cudaMemcpyHostToDevice, h->st);
        cudaStreamSynchronize(h->st);
        return set_err(h, GDB_ERR_TIMEOUT, "grid barrier of the persistent step kernel timed out");
    }
    return GDB_OK;
}

// Cluster path or persistent grid for a system that fits a cluster: the
// cluster (at most 16 SMs, no grid barrier) wins while the list holds fewer
// than about 70 000 entries, N x (4 pi / 3) (max_cut + skin)^3 N / V;
// above that the whole GPU's grid kernel is faster despite its barriers
// (measured on B200 with every block keeping the step's books, TPS cluster
// vs grid: KA rho 1.2 N 512 142k vs 132k, N 768 120k vs 126k, N 1024 85k vs
// 126k; LJ rho 0.973 N 500 191k vs 154k, N 864 134k vs 150k).
constexpr double CL_LIST_ENTRIES_MAX = 70000.0;
static bool cluster_preferred(const gdb_sim *h) {
    if (h->cluster_force) return true;
    const double vol = (double)h->box[0] * h->box[1] * h->box[2];
    const double rl = (double)h->max_cut + (double)h->skin;
    const double per_particle = 4.0 / 3.0 * M_PI * rl * rl * rl * h->n / vol;
    return h->n * per_particle <= CL_LIST_ENTRIES_MAX;
}

// One timeblock resident in a thread-block cluster (md_cluster.cu).  Returns
// GDB_ERR_UNSUPPORTED (and disables the path for this handle) when the
// cluster launch is not possible on this device.
static int run_cluster(gdb_sim *h, int steps) {
    int C, tp;
    cluster_shape(h->n, h->pb_req, &C, &tp);
    SimArgs a = make_args(h);
    // the cell grid of the global cell build, whatever list kind was chosen
    // (both kinds give the same sets)
    const float min_cell = (h->max_cut + h->skin) / 2.0f;
    int nc[3];
    for (int k = 0; k < 3; k++) {
        nc[k] = (int)(h->box[k] / min_cell);
        if (nc[k] < 1) nc[k] = 1;
    }
    a.ncx = nc[0];
    a.ncy = nc[1];
    a.ncz = nc[2];
    const int ncell = nc[0] * nc[1] * nc[2];
    int cap, pingpong, sorted;
    size_t smem;
    if (!cluster_plan(h->n, C, ncell, h->max_nbs, &cap, &pingpong, &sorted, &smem)) {
        h->cluster_ok = false;
        return GDB_ERR_UNSUPPORTED;
    }
    if (!h->d_job) {
        CK(cudaMalloc(&h->d_job, sizeof(ClusterJob)));
        CK(cudaMallocHost(&h->h_job, sizeof(ClusterJob)));
    }
    CK(cudaStreamSynchronize(h->st));  // the pinned job buffer is rewritten below
    h->h_job->a = a;
    h->h_job->tab = h->table;
    h->h_job->cur = h->cur;
    h->h_job->step0 = 0;
    h->h_job->cap = cap;
    h->h_job->pingpong = pingpong;
    h->h_job->sorted = sorted;
    CK(cudaMemcpyAsync(h->d_job, h->h_job, sizeof(ClusterJob), cudaMemcpyHostToDevice, h->st));
    cudaError_t e = launch_clusters(h->d_job, 1, C, tp, h->ntypes, h->integ, smem, steps, 1, h->st);
    if (e != cudaSuccess) {
        cudaGetLastError();
        h->cluster_ok = false;
        return set_err(h, GDB_ERR_UNSUPPORTED, "cluster launch not possible: %s", cudaGetErrorString(e));
    }
    return GDB_OK;
}

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
namespace gdb {

namespace {
constexpr int POOL_DEVICES = 64;
std::mutex g_pool_mu;
cudaMemPool_t g_pool[POOL_DEVICES] = {};
}  // namespace

cudaError_t pool_alloc_raw(void **p, size_t bytes, cudaStream_t st) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= POOL_DEVICES) return cudaMallocAsync(p, bytes, st);
    cudaMemPool_t pool;
    {
        std::lock_guard<std::mutex> lock(g_pool_mu);
        if (!g_pool[dev]) {
            cudaMemPoolProps props = {};
            props.allocType = cudaMemAllocationTypePinned;
            props.location.type = cudaMemLocationTypeDevice;
            props.location.id = dev;
            cudaMemPool_t created = nullptr;
            if ((e = cudaMemPoolCreate(&created, &props)) != cudaSuccess) return e;
            uint64_t keep = 1ull << 30;
            if ((e = cudaMemPoolSetAttribute(created, cudaMemPoolAttrReleaseThreshold, &keep)) != cudaSuccess) {
                cudaMemPoolDestroy(created);
                return e;
            }
            g_pool[dev] = created;
        }
        pool = g_pool[dev];
    }
    return cudaMallocFromPoolAsync(p, bytes, pool, st);
}

}  // namespace gdb

extern "C" {

int gdb_version(void) { return 100; }

int gdb_device_count(int *count) {
    gdb_sim *h = nullptr;
    if (!count) return set_err(h, GDB_ERR_ARG, "NULL count");
    CK(cudaGetDeviceCount(count));
    return GDB_OK;
}

int gdb_device_name(int device, char *buf, int n) {
    gdb_sim *h = nullptr;
    if (!buf || n < 1) return set_err(h, GDB_ERR_ARG, "gdb_device_name: bad arguments");
    cudaDeviceProp prop;
    CK(cudaGetDeviceProperties(&prop, device));
    snprintf(buf, (size_t)n, "%s", prop.name);
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
    const char *ps = getenv("GDB_PERSISTENT");
    if (ps && ps[0] == '0') h->persistent = false;
    const char *cs = getenv("GDB_CLUSTER");
    if (cs && cs[0] == '0') h->cluster_ok = false;
    if (cs && cs[0] == '1') h->cluster_force = true;
    const char *na = getenv("GDB_NSQ_AUTO");
    if (na) h->nsq_auto_max = atoi(na);
    const char *bk = getenv("GDB_BRICKS");
    if (bk && (bk[0] == '1' || bk[0] == '2')) h->bricks_req = true;
    const char *bm = getenv("GDB_BRICK_MIN_N");
    if (bm) h->brick_min_n = atoi(bm);
    const char *st = getenv("GDB_NSQ_STAGE");
    if (st && st[0] == '0') h->nsq_stage = false;
    const char *gc = getenv("GDB_GRID_CAP");
    if (gc) h->grid_cap = std::max(0, atoi(gc));
    const char *sb = getenv("GDB_STEP_BARRIER");
    if (sb && sb[0] == '0') h->step_bar_all = false;
    const char *bh = getenv("GDB_BRICK_HCAP");
    if (bh) h->brick_hcap = std::max(1, std::min(atoi(bh), BRICK_HCAP));
    cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, device);
    int coop = 0;
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device);
    if (!coop) h->persistent = false;
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
                    h->bsum,   h->ctrl,   h->partials,   h->rows,  h->conf, h->trace, h->rng, h->lbeta,
                    h->excl,   h->bond_cnt, h->bond_j,   h->bond_t, h->bond_prm, h->slot_of};
    for (void *p : bufs)
        if (p) cudaFree(p);
    if (h->h_ctrl) cudaFreeHost(h->h_ctrl);
    if (h->h_job) cudaFreeHost(h->h_job);
    if (h->d_job) cudaFree(h->d_job);
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
    CK(cudaSetDevice(h->dev));
    CK(cudaMemcpyAsync(h->ctrl->box, h->box, sizeof(h->box), cudaMemcpyHostToDevice, h->st));
    if (h->uploaded) {
        int one = 1;
        CK(cudaMemcpyAsync(&h->ctrl->rebuild, &one, sizeof(int), cudaMemcpyHostToDevice, h->st));
    }
    CK(cudaStreamSynchronize(h->st));
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
    CK(pool_alloc(&stage, bytes, h->st));
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
    if (h->slot_of) {
        k_fill_slot_of<<<grid_for(h->n), GDB_BLOCK, 0, h->st>>>(h->n, h->orig, h->slot_of);
        CKL();
    }
    CK(cudaFreeAsync(stage, h->st));
    int one = 1;
    CK(cudaMemcpyAsync(&h->ctrl->rebuild, &one, sizeof(int), cudaMemcpyHostToDevice, h->st));
    CK(cudaMemcpyAsync(h->ctrl->box, h->box, sizeof(h->box), cudaMemcpyHostToDevice, h->st));
    CK(cudaStreamSynchronize(h->st));
    h->uploaded = true;
    return GDB_OK;
}

static int download_planes(gdb_sim *h, const void *src, int kind, void *dst) {
    // kind 0: float4 -> (N,3) float, 1: int4 -> (N,3) int, 2: float plane -> (N,) float
    const size_t N = h->n;
    const size_t bytes = (kind == 2 ? 1 : 3) * N * 4;
    void *tmp = nullptr;
    CK(pool_alloc(&tmp, bytes, h->st));
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

int gdb_download_table(gdb_sim *h, float *vectors, int32_t *r_im, float *scalars, int nscal, const int32_t cols[6]) {
    if (!h) return set_err(h, GDB_ERR_ARG, "NULL handle");
    if (!h->uploaded) return set_err(h, GDB_ERR_STATE, "state not uploaded");
    if (scalars && (nscal < 1 || !cols)) return set_err(h, GDB_ERR_ARG, "gdb_download_table: bad scalar table");
    UnpackCols uc;
    for (int q = 0; q < 6; q++) {
        uc.c[q] = scalars ? cols[q] : -1;
        if (uc.c[q] >= nscal) return set_err(h, GDB_ERR_ARG, "gdb_download_table: column %d outside the table", uc.c[q]);
    }
    CK(cudaSetDevice(h->dev));
    const size_t N = h->n;
    const size_t bv = vectors ? 9 * N * sizeof(float) : 0, bi = r_im ? 3 * N * sizeof(int) : 0,
                 bs = scalars ? N * nscal * sizeof(float) : 0;
    if (bv + bi + bs == 0) return GDB_OK;
    char *stage = nullptr;
    CK(pool_alloc(&stage, bv + bi + bs, h->st));
    float *dv = vectors ? (float *)stage : nullptr;
    int *di = r_im ? (int *)(stage + bv) : nullptr;
    float *ds = scalars ? (float *)(stage + bv + bi) : nullptr;
    k_unpack_all<<<grid_for(h->n), GDB_BLOCK, 0, h->st>>>(h->n, h->pos[h->cur], h->vel, h->frc, h->img, h->pscal,
                                                        h->orig, dv, di, ds, nscal, uc);
    CKL();
    if (vectors) CK(cudaMemcpyAsync(vectors, dv, bv, cudaMemcpyDeviceToHost, h->st));
    if (r_im) CK(cudaMemcpyAsync(r_im, di, bi, cudaMemcpyDeviceToHost, h->st));
    if (scalars) CK(cudaMemcpyAsync(scalars, ds, bs, cudaMemcpyDeviceToHost, h->st));
    CK(cudaFreeAsync(stage, h->st));
    CK(cudaStreamSynchronize(h->st));
    return GDB_OK;
}

int gdb_host_alloc(size_t bytes, void **out) {
    gdb_sim *h = nullptr;
    if (!out) return set_err(h, GDB_ERR_ARG, "gdb_host_alloc: NULL argument");
    *out = nullptr;
    CK(cudaHostAlloc(out, bytes ? bytes : 1, cudaHostAllocPortable));
    return GDB_OK;
}

int gdb_host_free(void *p) {
    gdb_sim *h = nullptr;
    if (p) CK(cudaFreeHost(p));
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

int gdb_set_exclusions(gdb_sim *h, const int32_t *excl, int max_excl) {
    if (!h) return set_err(h, GDB_ERR_ARG, "NULL handle");
    CK(cudaSetDevice(h->dev));
    if (h->excl) cudaFree(h->excl);
    h->excl = nullptr;
    h->max_excl = 0;
    if (excl) {
        if (max_excl < 1) return set_err(h, GDB_ERR_ARG, "gdb_set_exclusions: max_excl must be positive");
        const size_t w = (size_t)max_excl + 1;
        for (int i = 0; i < h->n; i++) {
            const int cnt = excl[(size_t)i * w + max_excl];
            if (cnt < 0 || cnt > max_excl)
                return set_err(h, GDB_ERR_ARG, "gdb_set_exclusions: particle %d has %d exclusions (room for %d)", i,
                               cnt, max_excl);
            for (int k = 0; k < cnt; k++) {
                const int j = excl[(size_t)i * w + k];
                if (j < 0 || j >= h->n)
                    return set_err(h, GDB_ERR_ARG, "gdb_set_exclusions: particle %d excludes %d", i, j);
            }
        }
        CK(cudaMalloc(&h->excl, (size_t)h->n * w * sizeof(int)));
        CK(cudaMemcpy(h->excl, excl, (size_t)h->n * w * sizeof(int), cudaMemcpyHostToDevice));
        h->max_excl = max_excl;
    }
    free_graphs(h);
    if (h->uploaded) {
        int one = 1;
        CK(cudaMemcpyAsync(&h->ctrl->rebuild, &one, sizeof(int), cudaMemcpyHostToDevice, h->st));
        CK(cudaStreamSynchronize(h->st));
    }
    return GDB_OK;
}

int gdb_set_bonds(gdb_sim *h, int nbonds, const int32_t *indices, int ntypes, const float *params) {
    if (!h || nbonds < 0 || (nbonds > 0 && (!indices || !params || ntypes < 1)))
        return set_err(h, GDB_ERR_ARG, "gdb_set_bonds: bad arguments");
    CK(cudaSetDevice(h->dev));
    int **bufs[] = {&h->bond_cnt, &h->bond_j, &h->bond_t};
    for (int **b : bufs) {
        if (*b) cudaFree(*b);
        *b = nullptr;
    }
    if (h->bond_prm) cudaFree(h->bond_prm);
    h->bond_prm = nullptr;
    h->bond_max = 0;
    free_graphs(h);
    if (nbonds == 0) return GDB_OK;
    // per-particle partner lists: every bond appears at both of its ends
    std::vector<int> cnt(h->n, 0);
    for (int b = 0; b < nbonds; b++) {
        const int i = indices[3 * b], j = indices[3 * b + 1], t = indices[3 * b + 2];
        if (i < 0 || i >= h->n || j < 0 || j >= h->n || i == j || t < 0 || t >= ntypes)
            return set_err(h, GDB_ERR_ARG, "gdb_set_bonds: bond %d (%d, %d, type %d) is invalid", b, i, j, t);
        cnt[i]++;
        cnt[j]++;
    }
    int bmax = 1;
    for (int c : cnt) bmax = std::max(bmax, c);
    std::vector<int> bj((size_t)h->n * bmax, 0), bt((size_t)h->n * bmax, 0), fill(h->n, 0);
    for (int b = 0; b < nbonds; b++) {
        const int i = indices[3 * b], j = indices[3 * b + 1], t = indices[3 * b + 2];
        bj[(size_t)i * bmax + fill[i]] = j;
        bt[(size_t)i * bmax + fill[i]++] = t;
        bj[(size_t)j * bmax + fill[j]] = i;
        bt[(size_t)j * bmax + fill[j]++] = t;
    }
    std::vector<float2> prm(ntypes);
    for (int t = 0; t < ntypes; t++) prm[t] = make_float2(params[2 * t], params[2 * t + 1]);
    CK(cudaMalloc(&h->bond_cnt, (size_t)h->n * sizeof(int)));
    CK(cudaMalloc(&h->bond_j, bj.size() * sizeof(int)));
    CK(cudaMalloc(&h->bond_t, bt.size() * sizeof(int)));
    CK(cudaMalloc(&h->bond_prm, prm.size() * sizeof(float2)));
    CK(cudaMemcpy(h->bond_cnt, cnt.data(), (size_t)h->n * sizeof(int), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(h->bond_j, bj.data(), bj.size() * sizeof(int), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(h->bond_t, bt.data(), bt.size() * sizeof(int), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(h->bond_prm, prm.data(), prm.size() * sizeof(float2), cudaMemcpyHostToDevice));
    h->bond_max = bmax;
    if (!h->slot_of) CK(cudaMalloc(&h->slot_of, (size_t)h->n * sizeof(int)));
    if (h->uploaded) {
        k_fill_slot_of<<<grid_for(h->n), GDB_BLOCK, 0, h->st>>>(h->n, h->orig, h->slot_of);
        CKL();
        CK(cudaStreamSynchronize(h->st));
    }
    return GDB_OK;
}

int gdb_set_plan(gdb_sim *h, int tp, int pb) {
    if (!h) return set_err(h, GDB_ERR_ARG, "NULL handle");
    if (tp != 0 && tp != 1 && tp != 2 && tp != 4 && tp != 8 && tp != 16 && tp != 32)
        return set_err(h, GDB_ERR_ARG, "tp must be 0 (auto), 1, 2, 4, 8, 16 or 32");
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

// numba.cuda.random.create_xoroshiro128p_states(n, seed) (numba/cuda/random.py:
// init_xoroshiro128p_state, xoroshiro128p_jump, init_xoroshiro128p_states_cpu):
// SplitMix64 of the seed for state 0, state i = state i-1 advanced 2^64 steps.
static void xoro_host_next(unsigned long long &s0, unsigned long long &s1) {
    const unsigned long long a = s0;
    unsigned long long b = s1;
    b ^= a;
    s0 = ((a << 55) | (a >> 9)) ^ b ^ (b << 14);
    s1 = (b << 36) | (b >> 28);
}
static void xoro_states(int n, uint64_t seed, std::vector<ulonglong2> &out) {
    out.resize(n);
    if (n < 1) return;
    unsigned long long z = seed + 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    z = z ^ (z >> 31);
    out[0] = make_ulonglong2(z, z);
    static const unsigned long long J[2] = {0xbeac0467eba5facbULL, 0xd86b048b86aa9922ULL};
    for (int i = 1; i < n; i++) {
        unsigned long long s0 = out[i - 1].x, s1 = out[i - 1].y, j0 = 0, j1 = 0;
        for (int w = 0; w < 2; w++)
            for (int b = 0; b < 64; b++) {
                if (J[w] & (1ULL << b)) {
                    j0 ^= s0;
                    j1 ^= s1;
                }
                xoro_host_next(s0, s1);
            }
        out[i] = make_ulonglong2(j0, j1);
    }
}

int gdb_set_integrator_langevin(gdb_sim *h, float dt, float alpha, uint64_t seed, int tfunc, const float *tparams) {
    if (!h || !(dt > 0.f) || !(alpha >= 0.f) || !tparams)
        return set_err(h, GDB_ERR_ARG, "gdb_set_integrator_langevin: bad arguments");
    if (tfunc != GDB_TFUNC_CONSTANT && tfunc != GDB_TFUNC_RAMP)
        return set_err(h, GDB_ERR_UNSUPPORTED, "unsupported temperature function %d", tfunc);
    CK(cudaSetDevice(h->dev));
    if (!h->rng) CK(cudaMalloc(&h->rng, (size_t)h->n * sizeof(ulonglong2)));
    if (!h->lbeta) CK(cudaMalloc(&h->lbeta, (size_t)h->n * sizeof(float4)));
    std::vector<ulonglong2> st;
    xoro_states(h->n, seed, st);
    CK(cudaMemcpyAsync(h->rng, st.data(), (size_t)h->n * sizeof(ulonglong2), cudaMemcpyHostToDevice, h->st));
    CK(cudaMemsetAsync(h->lbeta, 0, (size_t)h->n * sizeof(float4), h->st));
    CK(cudaStreamSynchronize(h->st));
    h->integ = GDB_INTEGRATOR_LANGEVIN;
    h->dt = dt;
    h->alpha = alpha;
    h->tfunc = tfunc;
    const int np_ = tfunc == GDB_TFUNC_RAMP ? 4 : 1;
    for (int k = 0; k < 4; k++) h->tparams[k] = k < np_ ? tparams[k] : 0.f;
    free_graphs(h);
    return GDB_OK;
}

int gdb_get_langevin_state(gdb_sim *h, uint64_t *states, float *old_beta) {
    if (!h) return set_err(h, GDB_ERR_ARG, "NULL handle");
    if (!h->rng || !h->lbeta) return set_err(h, GDB_ERR_STATE, "no Langevin integrator set");
    CK(cudaSetDevice(h->dev));
    const size_t n = h->n;
    if (states) CK(cudaMemcpyAsync(states, h->rng, n * sizeof(ulonglong2), cudaMemcpyDeviceToHost, h->st));
    std::vector<float4> b;
    if (old_beta) {
        b.resize(n);
        CK(cudaMemcpyAsync(b.data(), h->lbeta, n * sizeof(float4), cudaMemcpyDeviceToHost, h->st));
    }
    CK(cudaStreamSynchronize(h->st));
    for (size_t i = 0; old_beta && i < n; i++) {
        old_beta[3 * i] = b[i].x;
        old_beta[3 * i + 1] = b[i].y;
        old_beta[3 * i + 2] = b[i].z;
    }
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
    state[1] = 0.0f;  // the sum is consumed by every update, as NVT.py:123
    return GDB_OK;
}

int gdb_set_thermostat_state(gdb_sim *h, const float state[2]) {
    if (!h || !state) return set_err(h, GDB_ERR_ARG, "NULL argument");
    CK(cudaSetDevice(h->dev));
    CK(cudaMemcpyAsync(&h->ctrl->xi, &state[0], sizeof(float), cudaMemcpyHostToDevice, h->st));
    CK(cudaStreamSynchronize(h->st));
    return GDB_OK;
}

int gdb_set_integrator_npt(gdb_sim *h, float dt, float mass_t, float mass_p, int tfunc, const float *tparams,
                           int pfunc, const float *pparams) {
    if (!h || !(dt > 0.f) || !(mass_t > 0.f) || !(mass_p > 0.f) || !tparams || !pparams)
        return set_err(h, GDB_ERR_ARG, "gdb_set_integrator_npt: bad arguments");
    if (tfunc != GDB_TFUNC_CONSTANT && tfunc != GDB_TFUNC_RAMP)
        return set_err(h, GDB_ERR_UNSUPPORTED, "unsupported temperature function %d", tfunc);
    if (pfunc != GDB_TFUNC_CONSTANT && pfunc != GDB_TFUNC_RAMP)
        return set_err(h, GDB_ERR_UNSUPPORTED, "unsupported pressure function %d", pfunc);
    if (!h->persistent)
        return set_err(h, GDB_ERR_UNSUPPORTED, "NPT_Atomic runs on the persistent kernel (cooperative launch)");
    h->integ = GDB_INTEGRATOR_NPT;
    h->dt = dt;
    h->npt_mass_t = mass_t;
    h->npt_mass_p = mass_p;
    h->tfunc = tfunc;
    h->pfunc = pfunc;
    const int nt_ = tfunc == GDB_TFUNC_RAMP ? 4 : 1, np_ = pfunc == GDB_TFUNC_RAMP ? 4 : 1;
    for (int k = 0; k < 4; k++) {
        h->tparams[k] = k < nt_ ? tparams[k] : 0.f;
        h->pparams[k] = k < np_ ? pparams[k] : 0.f;
    }
    free_graphs(h);
    // state as a new NPT_Atomic: zeros, the volume of the box (NPT_Atomic.py:35-36, 49)
    const float ts[2] = {0.f, 0.f};
    const float bs[3] = {0.f, 0.f, h->box[0] * h->box[1] * h->box[2]};
    return gdb_set_npt_state(h, ts, bs);
}

int gdb_get_npt_state(gdb_sim *h, float ts[2], float bs[3]) {
    if (!h) return set_err(h, GDB_ERR_ARG, "NULL handle");
    CK(cudaSetDevice(h->dev));
    int rc = read_ctrl(h);
    if (rc) return rc;
    if (ts) {
        ts[0] = h->h_ctrl->npt_ts0;
        ts[1] = 0.f;
    }
    if (bs) {
        bs[0] = h->h_ctrl->npt_bs0;
        bs[1] = 0.f;
        bs[2] = h->h_ctrl->npt_vol;
    }
    return GDB_OK;
}

int gdb_set_npt_state(gdb_sim *h, const float ts[2], const float bs[3]) {
    if (!h) return set_err(h, GDB_ERR_ARG, "NULL handle");
    CK(cudaSetDevice(h->dev));
    if (ts) CK(cudaMemcpyAsync(&h->ctrl->npt_ts0, &ts[0], sizeof(float), cudaMemcpyHostToDevice, h->st));
    if (bs) {
        CK(cudaMemcpyAsync(&h->ctrl->npt_bs0, &bs[0], sizeof(float), cudaMemcpyHostToDevice, h->st));
        CK(cudaMemcpyAsync(&h->ctrl->npt_vol, &bs[2], sizeof(float), cudaMemcpyHostToDevice, h->st));
    }
    CK(cudaStreamSynchronize(h->st));
    return GDB_OK;
}

int gdb_get_box(gdb_sim *h, float lengths[3]) {
    if (!h || !lengths) return set_err(h, GDB_ERR_ARG, "NULL argument");
    memcpy(lengths, h->box, sizeof(h->box));
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
        // frames, then one box row (4 floats) per frame
        const size_t bytes = ((size_t)conf_per_block * 2 * h->n * 3 + (size_t)conf_per_block * 4) * sizeof(float);
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

int gdb_get_saved_boxes(gdb_sim *h, float *out, int conf_per_block) {
    if (!h || !out) return set_err(h, GDB_ERR_ARG, "NULL argument");
    if (conf_per_block != h->conf_per_block || !h->conf)
        return set_err(h, GDB_ERR_STATE, "configuration saver holds %d frames", h->conf_per_block);
    if (h->integ != GDB_INTEGRATOR_NPT) {
        // a box that no step changes
        for (int k = 0; k < conf_per_block; k++) memcpy(out + 3 * k, h->box, 3 * sizeof(float));
        return GDB_OK;
    }
    CK(cudaSetDevice(h->dev));
    std::vector<float> rows((size_t)conf_per_block * 4);
    CK(cudaMemcpyAsync(rows.data(), h->conf + (size_t)conf_per_block * 2 * h->n * 3, rows.size() * sizeof(float),
                       cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    for (int k = 0; k < conf_per_block; k++) memcpy(out + 3 * k, rows.data() + 4 * k, 3 * sizeof(float));
    return GDB_OK;
}

int gdb_eval_forces(gdb_sim *h) {
    int rc = check_ready(h);
    if (rc) return rc;
    CK(cudaMemsetAsync(&h->ctrl->maxcount, 0, sizeof(int), h->st));
    if (h->order == 2 && h->nb_kind == GDB_NBLIST_CELLS) {
        // the staged-halo path's evaluation: the persistent kernel with no steps
        k_block_begin<<<1, 1, 0, h->st>>>(h->ctrl, 0.0);
        CKL();
        if ((rc = launch_run(h, 0, 1))) return rc;
        if ((rc = read_ctrl(h))) return rc;
        return status_to_rc(h);
    }
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
    if ((rc = ensure_partials(h, grid_for((long long)h->n * h->tp)))) return rc;
    CK(cudaMemsetAsync(&h->ctrl->maxcount, 0, sizeof(int), h->st));
    CK(cudaEventRecord(h->ev0, h->st));
    k_block_begin<<<1, 1, 0, h->st>>>(h->ctrl, time_zero);
    CKL();
    if (h->cluster_ok && h->n <= CL_MAX_N && h->integ != GDB_INTEGRATOR_LANGEVIN && h->integ != GDB_INTEGRATOR_NPT &&
        !h->excl && !h->bond_cnt && cluster_preferred(h)) {
        rc = run_cluster(h, steps);
        if (rc == GDB_OK) {
            CK(cudaEventRecord(h->ev1, h->st));
            if ((rc = read_ctrl(h))) return rc;
            if (!(h->h_ctrl->status & GDB_STATUS_CLUSTER_CAPACITY)) {
                h->cur ^= (steps & 1);
                h->last_path = 2;
                if (ms) CK(cudaEventElapsedTime(ms, h->ev0, h->ev1));
                return status_to_rc(h);
            }
            // a list outgrew shared memory: nothing was written back; rerun
            // this timeblock (and the following ones) on the global path
            h->cluster_ok = false;
            const unsigned clear = h->h_ctrl->status & ~GDB_STATUS_CLUSTER_CAPACITY;
            CK(cudaMemcpyAsync(&h->ctrl->status, &clear, sizeof(unsigned), cudaMemcpyHostToDevice, h->st));
            int one = 1;
            CK(cudaMemcpyAsync(&h->ctrl->rebuild, &one, sizeof(int), cudaMemcpyHostToDevice, h->st));
            CK(cudaEventRecord(h->ev0, h->st));
            k_block_begin<<<1, 1, 0, h->st>>>(h->ctrl, time_zero);
            CKL();
        } else if (rc != GDB_ERR_UNSUPPORTED) {
            return rc;
        }
    }
    if (h->persistent) {
        const int cur0 = h->cur;
        const bool bricks = h->order == 2 && h->nb_kind == GDB_NBLIST_CELLS;
        if ((rc = launch_run(h, steps, 1))) return rc;
        h->last_path = bricks ? 4 : 1;
        if (bricks) {
            if ((rc = read_ctrl(h))) return rc;
            if (h->h_ctrl->status & GDB_STATUS_BRICK_CAPACITY) {
                // a brick's halo outgrew shared memory at a rebuild, before
                // any step used that list: go on without bricks from the step
                // reached, in the same timeblock
                const int done = h->h_ctrl->step;
                h->cur = cur0 ^ (done & 1);
                h->staged_ok = false;
                if ((rc = ensure_nblist(h))) return rc;
                const unsigned clear = h->h_ctrl->status & ~GDB_STATUS_BRICK_CAPACITY;
                CK(cudaMemcpyAsync(&h->ctrl->status, &clear, sizeof(unsigned), cudaMemcpyHostToDevice, h->st));
                if (h->cell_count) CK(cudaMemsetAsync(h->cell_count, 0, (size_t)h->cell_cap * sizeof(int), h->st));
                k_block_resume<<<1, 1, 0, h->st>>>(h->ctrl);
                CKL();
                if ((rc = launch_run(h, steps - done, 1))) return rc;
                h->last_path = 1;
            }
        }
    } else {
        h->last_path = 0;
        const int G = 16;
        int s = 0;
        if (h->use_graphs && steps >= G) {
            while (s + G <= steps) {
                if (!h->gexec[h->cur] && (rc = build_graph(h, h->cur, G))) return rc;
                CK(cudaGraphLaunch(h->gexec[h->cur], h->st));
                s += G;  // G is even: the current buffer is unchanged after a chunk
            }
        }
        for (; s < steps; s++) {
            if ((rc = enqueue_rebuild(h))) return rc;
            if ((rc = enqueue_step(h, MODE_STEP))) return rc;
        }
        if ((rc = enqueue_rebuild(h))) return rc;
        if ((rc = enqueue_step(h, MODE_EVAL))) return rc;
    }
    CK(cudaEventRecord(h->ev1, h->st));
    if ((rc = read_ctrl(h))) return rc;
    if (h->integ == GDB_INTEGRATOR_NPT) memcpy(h->box, h->h_ctrl->box, sizeof(h->box));  // the box the run left
    if (ms) CK(cudaEventElapsedTime(ms, h->ev0, h->ev1));
    return status_to_rc(h);
}

int gdb_set_trace(gdb_sim *h, int capacity) {
    if (!h || capacity < 0) return set_err(h, GDB_ERR_ARG, "bad trace capacity");
    CK(cudaSetDevice(h->dev));
    CK(cudaStreamSynchronize(h->st));
    if (h->trace) cudaFree(h->trace);
    h->trace = nullptr;
    h->trace_cap = 0;
    if (capacity > 0) {
        CK(cudaMalloc(&h->trace, (size_t)capacity * sizeof(unsigned long long)));
        h->trace_cap = capacity;
    }
    unsigned long long *p = h->trace;
    int cap = h->trace_cap, zero = 0;
    CK(cudaMemcpy(&h->ctrl->trace, &p, sizeof(p), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(&h->ctrl->trace_cap, &cap, sizeof(int), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(&h->ctrl->trace_len, &zero, sizeof(int), cudaMemcpyHostToDevice));
    return GDB_OK;
}

int gdb_get_trace(gdb_sim *h, unsigned long long *out, int capacity, int *count) {
    if (!h || !out || !count) return set_err(h, GDB_ERR_ARG, "NULL argument");
    CK(cudaSetDevice(h->dev));
    int rc = read_ctrl(h);
    if (rc) return rc;
    const int len = std::min(std::min(h->h_ctrl->trace_len, h->trace_cap), capacity);
    if (len > 0) CK(cudaMemcpy(out, h->trace, (size_t)len * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
    *count = len;
    int zero = 0;
    CK(cudaMemcpy(&h->ctrl->trace_len, &zero, sizeof(int), cudaMemcpyHostToDevice));
    return GDB_OK;
}

int gdb_time_step_kernel(gdb_sim *h, int reps, float *ms_per_launch) {
    int rc = check_ready(h);
    if (rc) return rc;
    if (reps < 1 || !ms_per_launch) return set_err(h, GDB_ERR_ARG, "bad arguments");
    if (h->order == 2 && h->nb_kind == GDB_NBLIST_CELLS) {
        // a list for the current positions (the persistent kernel's
        // evaluation), then `reps` standalone brick steps
        k_block_begin<<<1, 1, 0, h->st>>>(h->ctrl, 0.0);
        CKL();
        if ((rc = launch_run(h, 0, 1))) return rc;
        const void *fn = h->ntypes == 1   ? step_bricks_kernel_nt1(h->integ, MODE_STEP)
                         : h->ntypes == 2 ? step_bricks_kernel_nt2(h->integ, MODE_STEP)
                                          : step_bricks_kernel_ntg(h->integ, MODE_STEP);
        const size_t smem = sizeof(BrickSmem);
        CK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        int occ = 0;
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, BRICK_THREADS, smem));
        const int nbricks = h->nb[0] * h->nb[1] * h->nb[2];
        const int grid = std::max(1, std::min(nbricks, occ * h->num_sms));
        k_block_begin<<<1, 1, 0, h->st>>>(h->ctrl, 0.0);
        CKL();
        const int saved_every = h->scalar_every, saved_reset = h->momentum_every;
        h->scalar_every = 0;
        h->momentum_every = 0;
        float ms = 0.f;
        cudaError_t e = cudaSuccess;
        for (int r = 0; r <= reps && e == cudaSuccess; r++) {  // the first launch untimed
            if (r == 1) e = cudaEventRecord(h->ev0, h->st);
            SimArgs a = make_args(h);
            int cur = h->cur;
            void *args[] = {(void *)&a, (void *)&h->table, (void *)&cur};
            if (e == cudaSuccess) e = cudaLaunchKernel(fn, dim3(grid), dim3(BRICK_THREADS), args, smem, h->st);
            h->cur ^= 1;
        }
        h->scalar_every = saved_every;
        h->momentum_every = saved_reset;
        if (e != cudaSuccess) return set_err(h, GDB_ERR_CUDA, "brick step kernel: %s", cudaGetErrorString(e));
        CK(cudaEventRecord(h->ev1, h->st));
        CK(cudaEventSynchronize(h->ev1));
        CK(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
        *ms_per_launch = ms / reps;
        return GDB_OK;
    }
    const int grid = grid_for((long long)h->n * h->tp);
    if ((rc = ensure_partials(h, grid))) return rc;
    // a list for the current positions, then `reps` step kernels alone
    if ((rc = enqueue_rebuild(h))) return rc;
    k_block_begin<<<1, 1, 0, h->st>>>(h->ctrl, 0.0);
    CKL();
    const int saved_every = h->scalar_every, saved_reset = h->momentum_every;
    h->scalar_every = 0;
    h->momentum_every = 0;
    // one untimed launch: the module's lazy loading of this kernel happens here
    if ((rc = enqueue_step(h, MODE_STEP))) return rc;
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
    const size_t stride = h->stride;
    if (h->order == 2 && h->nb_kind == GDB_NBLIST_CELLS) {
        // 16-bit halo indices: map them back through every brick's runs
        const unsigned short *l16 = reinterpret_cast<const unsigned short *>(nbl.data());
        std::vector<int> cs((size_t)h->ncell + 1);
        CK(cudaMemcpy(cs.data(), h->cell_start, cs.size() * sizeof(int), cudaMemcpyDeviceToHost));
        const int nbr = h->nb[0] * h->nb[1] * h->nb[2];
        std::vector<int> dst, src;
        for (int r = 0; r < nbr; r++) {
            const BrickHalo hb = brick_halo(r, h->nc, h->nb);
            dst.clear();
            src.clear();
            int off = 0;
            for (int row = 0; row < hb.wy * hb.wz; row++)
                for_each_halo_run(hb, row % hb.wy, row / hb.wy, h->nc, h->nb, [&](int, int first, int last, int) {
                    const int len = cs[last + 1] - cs[first];
                    if (len == 0) return;
                    dst.push_back(off);
                    src.push_back(cs[first]);
                    off += len;
                });
            dst.push_back(off);
            for (int s = cs[(size_t)r * BRICK * BRICK * BRICK]; s < cs[(size_t)(r + 1) * BRICK * BRICK * BRICK]; s++) {
                const int i = orig[s];
                int32_t *row = out + (size_t)i * (max_nbs + 1);
                const int cnt = nbc[s];
                const int lim = std::min(std::min(cnt, h->max_nbs), max_nbs);
                for (int k = 0; k < lim; k++) {
                    const int e = l16[((size_t)(k >> 3) * stride + s) * NB16 + (k & 7)];
                    const int q = (int)(std::upper_bound(dst.begin(), dst.end() - 1, e) - dst.begin()) - 1;
                    row[k] = orig[src[q] + (e - dst[q])];
                }
                row[max_nbs] = cnt;
            }
        }
        return GDB_OK;
    }
    for (size_t s = 0; s < N; s++) {
        const int i = orig[s];
        int32_t *row = out + (size_t)i * (max_nbs + 1);
        const int cnt = nbc[s];
        const int lim = std::min(std::min(cnt, h->max_nbs), max_nbs);
        for (int k = 0; k < lim; k++) row[k] = orig[nbl[(size_t)(k >> 2) * stride * 4 + s * 4 + (k & 3)]];
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

int gdb_get_last_path(gdb_sim *h) { return h ? h->last_path : -1; }

}  // extern "C"

// ---------------------------------------------------------------------------
// batched replicas: many independent systems advanced together
// ---------------------------------------------------------------------------
// Every system of a batch runs in one thread-block cluster: up to 4096
// particles with the whole state in shared memory (k_cluster_run), larger
// ones with the state in global memory and the phases of the persistent
// kernel between cluster barriers (k_run_clusters).  Systems of one cluster
// shape share a launch, largest first; the launches run concurrently on
// their own streams.  Systems above CLG_MAX_N particles (a cluster is too
// small for them) run one after another on the persistent grid kernel once
// the clusters are done, so no cooperative grid shares the GPU.
constexpr int CLG_MAX_N = 1 << 17;

static const void *run_clusters_kernel(int ntypes, int tp, int integ) {
    return ntypes == 1   ? run_clusters_kernel_nt1(tp, integ)
           : ntypes == 2 ? run_clusters_kernel_nt2(tp, integ)
                         : run_clusters_kernel_ntg(tp, integ);
}

struct gdb_batch {
    struct Group {
        int kind = 0;  // 0 shared-memory clusters, 1 global-memory clusters
        int C = 0, tp = 0;
        size_t smem = 0;
        std::vector<int> idx, cap, pp;
        void *d_jobs = nullptr, *h_jobs = nullptr;
        cudaStream_t st = nullptr;
        cudaEvent_t done = nullptr;
    };
    std::vector<gdb_sim *> sims;
    std::vector<Group> groups;
    std::vector<int> solo;  // too large for a cluster
    int dev = 0, ntypes = 1, integ = 0;
    int clg_tp = 1;
    int clg_ppc = 4096;  // particles per CTA of the global-memory clusters
    cudaStream_t st = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    char err[512] = "";
};

static int bset(gdb_batch *b, int code, const char *fmt, ...) {
    char *dst = b ? b->err : g_lib_error;
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(dst, 512, fmt, ap);
    va_end(ap);
    return code;
}

#define BCK(call)                                                                                     \
    do {                                                                                              \
        cudaError_t e_ = (call);                                                                      \
        if (e_ != cudaSuccess)                                                                        \
            return bset(b, GDB_ERR_CUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, \
                        __LINE__);                                                                    \
    } while (0)

static void batch_free(gdb_batch *b) {
    if (!b) return;
    cudaSetDevice(b->dev);
    if (b->st) cudaStreamSynchronize(b->st);
    for (auto &g : b->groups) {
        if (g.st) cudaStreamSynchronize(g.st);
        if (g.d_jobs) cudaFree(g.d_jobs);
        if (g.h_jobs) cudaFreeHost(g.h_jobs);
        if (g.done) cudaEventDestroy(g.done);
        if (g.st) cudaStreamDestroy(g.st);
    }
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    if (b->st) cudaStreamDestroy(b->st);
    delete b;
}

static void cluster_grid_of(const gdb_sim *h, int nc[3]) {
    const float min_cell = (h->max_cut + h->skin) / 2.0f;
    for (int k = 0; k < 3; k++) {
        nc[k] = (int)(h->box[k] / min_cell);
        if (nc[k] < 1) nc[k] = 1;
    }
}

static gdb_batch::Group *batch_group(gdb_batch *b, int kind, int C, int tp) {
    for (auto &x : b->groups)
        if (x.kind == kind && x.C == C && x.tp == tp) return &x;
    b->groups.emplace_back();
    gdb_batch::Group *g = &b->groups.back();
    g->kind = kind;
    g->C = C;
    g->tp = tp;
    return g;
}

static cudaError_t launch_run_clusters(const void *fn, const ClusterRunJob *d_jobs, int count, int C, int nsteps,
                                       int do_eval, cudaStream_t st) {
    if (C > 8) {
        cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        if (e != cudaSuccess) return e;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(count * C);
    cfg.blockDim = dim3(CLG_BLOCK);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    void *args[] = {(void *)&d_jobs, (void *)&nsteps, (void *)&do_eval};
    return cudaLaunchKernelExC(&cfg, fn, args);
}

extern "C" {

int gdb_batch_create(gdb_sim *const *sims, int count, int particles_per_cta, gdb_batch **out) {
    return gdb_batch_create_ex(sims, count, particles_per_cta, 0, 0, out);
}

int gdb_batch_create_ex(gdb_sim *const *sims, int count, int particles_per_cta, int clg_particles_per_cta,
                        int clg_tp, gdb_batch **out) {
    gdb_batch *b = nullptr;
    if (!sims || count < 1 || !out || clg_particles_per_cta < 0 || clg_tp < 0 ||
        (clg_tp != 0 && clg_tp != 1 && clg_tp != 2 && clg_tp != 4 && clg_tp != 8))
        return bset(b, GDB_ERR_ARG, "gdb_batch_create: bad arguments");
    b = new gdb_batch();
    if (clg_tp > 0) b->clg_tp = clg_tp;
    b->sims.assign(sims, sims + count);
    b->dev = sims[0]->dev;
    b->ntypes = sims[0]->ntypes;
    b->integ = sims[0]->integ;
    for (int k = 0; k < count; k++) {
        gdb_sim *h = sims[k];
        if (!h || h->dev != b->dev || h->ntypes != b->ntypes || h->integ != b->integ) {
            batch_free(b);
            return bset(nullptr, GDB_ERR_ARG,
                        "gdb_batch_create: every system needs the same device, type count and integrator");
        }
        if (h->integ == GDB_INTEGRATOR_LANGEVIN) {
            batch_free(b);
            return bset(nullptr, GDB_ERR_UNSUPPORTED, "gdb_batch_create: Langevin systems run one at a time");
        }
        if (h->integ == GDB_INTEGRATOR_NPT) {
            batch_free(b);
            return bset(nullptr, GDB_ERR_UNSUPPORTED, "gdb_batch_create: NPT_Atomic systems run one at a time");
        }
        for (int q = 0; q < k; q++)
            if (sims[q] == h) {
                batch_free(b);
                return bset(nullptr, GDB_ERR_ARG, "gdb_batch_create: system %d appears twice", k);
            }
        int rc = check_ready(h);
        if (rc) {
            snprintf(g_lib_error, sizeof(g_lib_error), "gdb_batch_create: system %d: %.400s", k, h->err);
            batch_free(b);
            return rc;
        }
    }
    cudaError_t e;
    if ((e = cudaSetDevice(b->dev)) != cudaSuccess || (e = cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking)) ||
        (e = cudaEventCreate(&b->ev0)) || (e = cudaEventCreate(&b->ev1))) {
        batch_free(b);
        return bset(nullptr, GDB_ERR_CUDA, "gdb_batch_create: %s", cudaGetErrorString(e));
    }
    // largest first inside every launch: the long clusters start first
    std::vector<int> order(count);
    for (int k = 0; k < count; k++) order[k] = k;
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return sims[x]->n > sims[y]->n; });
    // which systems fit a shared-memory cluster
    std::vector<char> in_smem(count, 0);
    long long p_smem = 0, p_glob = 0;
    for (int k : order) {
        gdb_sim *h = sims[k];
        int nc[3];
        cluster_grid_of(h, nc);
        int C, tp, cap, pingpong, sorted;
        size_t smem;
        cluster_shape(h->n, particles_per_cta, &C, &tp);
        in_smem[k] = h->cluster_ok && h->n <= CL_MAX_N && !h->excl && !h->bond_cnt &&
                     cluster_plan(h->n, C, nc[0] * nc[1] * nc[2], h->max_nbs, &cap, &pingpong, &sorted, &smem);
        if (in_smem[k])
            p_smem += h->n;
        else if (h->n <= CLG_MAX_N)
            p_glob += h->n;
    }
    // particles per CTA of the global-memory clusters: given, or the smallest
    // (from 4096, in steps of 1.25x) whose CTAs (one per SM, 1 to 16 a system)
    // fit the SMs left for them by the shared-memory clusters' share of the
    // particles, so that the launch is one wave
    if (clg_particles_per_cta > 0) {
        b->clg_ppc = std::max(256, clg_particles_per_cta);
    } else if (p_glob > 0) {
        const int sms = std::max(1, sims[0]->num_sms);
        const int budget = std::max(1, (int)((double)sms * (double)p_glob / (double)(p_glob + p_smem)));
        int ppc = 4096;
        for (int it = 0; it < 40; it++) {
            long long ctas = 0;
            for (int k : order)
                if (!in_smem[k] && sims[k]->n <= CLG_MAX_N)
                    ctas += std::min(16, (sims[k]->n + ppc - 1) / ppc);
            if (ctas <= budget || ppc >= CLG_MAX_N) break;
            ppc = (int)(ppc * 1.25);
        }
        b->clg_ppc = ppc;
    }
    for (int k : order) {
        gdb_sim *h = sims[k];
        int nc[3];
        cluster_grid_of(h, nc);
        int C, tp, cap, pingpong, sorted;
        size_t smem;
        cluster_shape(h->n, particles_per_cta, &C, &tp);
        if (in_smem[k] &&
            cluster_plan(h->n, C, nc[0] * nc[1] * nc[2], h->max_nbs, &cap, &pingpong, &sorted, &smem)) {
            gdb_batch::Group *g = batch_group(b, 0, C, tp);
            g->idx.push_back(k);
            g->cap.push_back(cap);
            g->pp.push_back(pingpong | (sorted << 1));
            g->smem = std::max(g->smem, smem);
        } else if (h->n <= CLG_MAX_N) {
            // the global-memory cluster kernel runs the row phases
            h->bricks_ok = false;
            if (int rc = ensure_nblist(h)) {
                batch_free(b);
                return rc;
            }
            // about clg_ppc particles per CTA, 1 to 16 CTAs
            const int c = std::max(1, std::min(16, (h->n + b->clg_ppc - 1) / b->clg_ppc));
            gdb_batch::Group *g = batch_group(b, 1, c, b->clg_tp);
            g->idx.push_back(k);
            g->cap.push_back(0);
            g->pp.push_back(0);
        } else {
            b->solo.push_back(k);
        }
    }
    for (auto &g : b->groups) {
        const size_t bytes = g.idx.size() * (g.kind == 0 ? sizeof(ClusterJob) : sizeof(ClusterRunJob));
        if ((e = cudaMalloc(&g.d_jobs, bytes)) || (e = cudaMallocHost(&g.h_jobs, bytes)) ||
            (e = cudaStreamCreateWithFlags(&g.st, cudaStreamNonBlocking)) ||
            (e = cudaEventCreateWithFlags(&g.done, cudaEventDisableTiming))) {
            batch_free(b);
            return bset(nullptr, GDB_ERR_CUDA, "gdb_batch_create: %s", cudaGetErrorString(e));
        }
    }
    *out = b;
    return GDB_OK;
}

int gdb_batch_destroy(gdb_batch *b) {
    batch_free(b);
    return GDB_OK;
}

int gdb_batch_run(gdb_batch *b, double time_zero, int steps, float *ms) {
    if (!b || steps < 0) return bset(b, GDB_ERR_ARG, "gdb_batch_run: bad arguments");
    BCK(cudaSetDevice(b->dev));
    // per-system preparation on each system's own stream
    for (gdb_sim *h : b->sims) {
        int rc = check_ready(h);
        if (rc) return bset(b, rc, "gdb_batch_run: %s", h->err);
        const int rows = h->scalar_every > 0 ? steps / h->scalar_every : 0;
        if (rows > h->rows_cap) {
            if (h->rows) cudaFree(h->rows);
            h->rows = nullptr;
            BCK(cudaMalloc(&h->rows, (size_t)rows * GDB_NUM_SCALARS * sizeof(double)));
            h->rows_cap = rows;
            free_graphs(h);
        }
        if (rows > 0) BCK(cudaMemsetAsync(h->rows, 0, (size_t)rows * GDB_NUM_SCALARS * sizeof(double), h->st));
        // one partial row per round of the global-memory clusters too
        // (rounds of CLG_BLOCK / clg_tp particles)
        if ((rc = ensure_partials(h, std::max(std::max(grid_for((long long)h->n * h->tp), 16),
                                              grid_for((long long)h->n * b->clg_tp, CLG_BLOCK)))))
            return bset(b, rc, "%s", h->err);
        BCK(cudaMemsetAsync(&h->ctrl->maxcount, 0, sizeof(int), h->st));
        k_block_begin<<<1, 1, 0, h->st>>>(h->ctrl, time_zero);
        BCK(cudaGetLastError());
        BCK(cudaEventRecord(h->ev0, h->st));
        BCK(cudaStreamWaitEvent(b->st, h->ev0, 0));
    }
    BCK(cudaEventRecord(b->ev0, b->st));
    // one launch per cluster shape, concurrently
    for (auto &g : b->groups) {
        BCK(cudaStreamWaitEvent(g.st, b->ev0, 0));
        BCK(cudaStreamSynchronize(g.st));  // the pinned job buffer is rewritten below
        for (size_t q = 0; q < g.idx.size(); q++) {
            gdb_sim *h = b->sims[g.idx[q]];
            SimArgs a = make_args(h);
            if (g.kind == 0) {
                int nc[3];
                cluster_grid_of(h, nc);
                a.ncx = nc[0];
                a.ncy = nc[1];
                a.ncz = nc[2];
                ClusterJob &j = static_cast<ClusterJob *>(g.h_jobs)[q];
                j.a = a;
                j.tab = h->table;
                j.cur = h->cur;
                j.step0 = 0;
                j.cap = g.cap[q];
                j.pingpong = g.pp[q] & 1;
                j.sorted = (g.pp[q] >> 1) & 1;
            } else {
                ClusterRunJob &j = static_cast<ClusterRunJob *>(g.h_jobs)[q];
                j.a = a;
                j.tab = h->table;
                j.cur = h->cur;
            }
        }
        const int cnt = (int)g.idx.size();
        if (g.kind == 0) {
            BCK(cudaMemcpyAsync(g.d_jobs, g.h_jobs, cnt * sizeof(ClusterJob), cudaMemcpyHostToDevice, g.st));
            BCK(launch_clusters(static_cast<const ClusterJob *>(g.d_jobs), cnt, g.C, g.tp, b->ntypes, b->integ, g.smem,
                                steps, 1, g.st));
        } else {
            BCK(cudaMemcpyAsync(g.d_jobs, g.h_jobs, cnt * sizeof(ClusterRunJob), cudaMemcpyHostToDevice, g.st));
            BCK(launch_run_clusters(run_clusters_kernel(b->ntypes, g.tp, b->integ),
                                    static_cast<const ClusterRunJob *>(g.d_jobs), cnt, g.C, steps, 1, g.st));
        }
        BCK(cudaEventRecord(g.done, g.st));
        BCK(cudaStreamWaitEvent(b->st, g.done, 0));
    }
    // systems too large for a cluster: the persistent grid kernel, one at a
    // time, after the clusters
    for (int k : b->solo) {
        gdb_sim *h = b->sims[k];
        BCK(cudaEventRecord(b->ev1, b->st));
        BCK(cudaStreamWaitEvent(h->st, b->ev1, 0));
        int rc = launch_run(h, steps, 1);
        if (rc) return bset(b, rc, "gdb_batch_run: %s", h->err);
        h->last_path = 1;
        BCK(cudaEventRecord(h->ev1, h->st));
        BCK(cudaStreamWaitEvent(b->st, h->ev1, 0));
    }
    BCK(cudaEventRecord(b->ev1, b->st));
    BCK(cudaEventSynchronize(b->ev1));
    if (ms) BCK(cudaEventElapsedTime(ms, b->ev0, b->ev1));
    for (auto &g : b->groups)
        for (int k : g.idx) {
            gdb_sim *h = b->sims[k];
            h->cur ^= (steps & 1);
            h->last_path = g.kind == 0 ? 2 : 3;
        }
    // status; a shared-memory cluster whose lists outgrew shared memory
    // reruns alone on the global-memory path
    int first_rc = GDB_OK;
    for (size_t k = 0; k < b->sims.size(); k++) {
        gdb_sim *h = b->sims[k];
        int rc = read_ctrl(h);
        if (rc) return bset(b, rc, "gdb_batch_run: %s", h->err);
        if (h->h_ctrl->status & GDB_STATUS_CLUSTER_CAPACITY) {
            h->cur ^= (steps & 1);  // nothing was written back
            h->cluster_ok = false;
            const unsigned clear = h->h_ctrl->status & ~GDB_STATUS_CLUSTER_CAPACITY;
            BCK(cudaMemcpy(&h->ctrl->status, &clear, sizeof(unsigned), cudaMemcpyHostToDevice));
            int one = 1;
            BCK(cudaMemcpy(&h->ctrl->rebuild, &one, sizeof(int), cudaMemcpyHostToDevice));
            rc = gdb_sim_run(h, time_zero, steps, nullptr);
        } else {
            rc = status_to_rc(h);
        }
        if (rc && first_rc == GDB_OK) {
            first_rc = rc;
            bset(b, rc, "system %d: %s", (int)k, h->err);
        }
    }
    return first_rc;
}

int gdb_batch_get_last_error(gdb_batch *b, char *buf, int n) {
    if (!buf || n < 1) return GDB_ERR_ARG;
    snprintf(buf, (size_t)n, "%s", b ? b->err : g_lib_error);
    return GDB_OK;
}



// Self-test of the bounded grid barrier: two blocks, the second leaves
// without arriving, so the first block's wait runs out after `cycles`.
__global__ void k_barrier_selftest(DevCtrl *c) {
    if (blockIdx.x == 1) return;
    grid_barrier(c, [] {});
}

int gdb_selftest_barrier_timeout(int device, long long cycles, unsigned *status) {
    gdb_sim *h = nullptr;
    if (!status || cycles <= 0) return set_err(h, GDB_ERR_ARG, "gdb_selftest_barrier_timeout: bad arguments");
    CK(cudaSetDevice(device));
    DevCtrl *c = nullptr;
    CK(cudaMalloc(&c, sizeof(DevCtrl)));
    cudaError_t e = cudaMemset(c, 0, sizeof(DevCtrl));
    if (e == cudaSuccess) e = cudaMemcpy(&c->bar_timeout, &cycles, sizeof(cycles), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        k_barrier_selftest<<<2, GDB_BLOCK>>>(c);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(status, &c->status, sizeof(unsigned), cudaMemcpyDeviceToHost);
    cudaFree(c);
    if (e != cudaSuccess) return set_err(h, GDB_ERR_CUDA, "gdb_selftest_barrier_timeout: %s", cudaGetErrorString(e));
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
cudaEvent_t gdb_internal_event(gdb_sim *h, int k) { return k ? h->ev1 : h->ev0; }
void gdb_internal_set_analysis_ms(gdb_sim *h, float ms) { h->analysis_ms = ms; }

int gdb_last_analysis_ms(gdb_sim *h, float *ms) {
    if (!h || !ms) return set_err(h, GDB_ERR_ARG, "gdb_last_analysis_ms: NULL argument");
    *ms = h->analysis_ms;
    return GDB_OK;
}

}  // extern "C"
