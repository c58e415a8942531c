// md_bricks.cuh -- the brick path of the large-system step: particles kept in
// brick order, each brick's neighbourhood staged in shared memory by the
// bulk-copy (TMA) engine, neighbour lists as 16-bit indices into that stage.
//
// Bricks.  The cell grid is the reference's (cells of edge >= (max_cut +
// skin)/2, nblist_linked_lists.py:36-39).  Bricks are blocks of 4 x 4 x 4
// cells (smaller at the high faces when the cell count is not a multiple of
// 4); cells are numbered brick by brick, x fastest inside a brick, so after
// the counting sort every brick's particles are one contiguous slot range
// and every x-row of cells inside one brick is contiguous too.
//
// Halo.  The 5 x 5 x 5 stencil of any cell of a brick lies inside the brick
// grown by two cells on every side (8 x 8 x 8 cells for a full brick, about
// 1 700 particles for the Kob-Andersen liquid).  A halo row (fixed y, z) of
// cells is at most four runs of consecutive cells of one brick each, so the
// halo is at most 4 x 64 contiguous slot ranges of the position array; one
// cp.async.bulk per range copies them into shared memory, rows in (z, y)
// order and each row in x order, completing on one mbarrier.
//
// Step.  Each CTA takes a brick per round (atomic counter, one float64
// partial row per brick, so sums stay fixed-order), stages its halo,
// shifts the copies that sit across a periodic face into the brick's frame
// (x - L rint((x - centre) / L), exact for every particle within L/2 of its
// cell), and runs the pair loop over 16-bit halo indices: shared-memory
// loads instead of dependent global gathers, and half the index bytes.
//
// Build.  The list is built brick by brick over the same stage: a particle's
// 25 stencil rows are contiguous halo ranges; a row whose (y, z) extent lies
// farther than (max_cut + skin) plus a margin from the particle is skipped,
// and the row is trimmed to the cells within reach.  Skipped cells hold no
// particle within the distance by geometry (the margin covers float32
// rounding), and every candidate is tested with the exact distance
// expression of the row build, so the neighbour sets equal the reference's
// bit for bit.
#pragma once

#include "md_phases.cuh"

namespace gdb {

constexpr int BRICK = 4;                         // cells per brick edge
constexpr int BRICK_W = BRICK + 4;               // widest halo, in cells
constexpr int BRICK_ROWS = BRICK_W * BRICK_W;    // halo rows (y, z)
constexpr int BRICK_RUNS = 4;                    // contiguous runs per halo row, at most
constexpr int BRICK_SLOTS = BRICK_ROWS * BRICK_RUNS;
constexpr int BRICK_HCAP = 2816;                 // staged positions per buffer (44 KB), sentinel included
constexpr int BRICK_CONSUMERS = 256;             // threads that compute particles: warps 0-7
constexpr int BRICK_CWARPS = BRICK_CONSUMERS / 32;
constexpr int BRICK_THREADS = BRICK_CONSUMERS + 32;  // and one producer warp that stages halos
constexpr int NB16 = 8;                          // 16-bit indices per 16-byte list chunk
constexpr long long MBAR_WAIT_POLLS = 1LL << 26; // bounded wait for a stage (~seconds)
constexpr float BRICK_SENTINEL = 1.0e30f;        // coordinates of the padding entry: beyond every cut
static_assert(BRICK == 4, "phase_cell_assign numbers cells in bricks of 4 x 4 x 4");

// Brick-major number of cell (gx, gy, gz) of a grid with nbx x nby bricks in
// x and y.
__host__ __device__ __forceinline__ int brick_cell_id(int gx, int gy, int gz, int nbx, int nby) {
    const int bx = gx / BRICK, by = gy / BRICK, bz = gz / BRICK;
    return ((bz * nby + by) * nbx + bx) * (BRICK * BRICK * BRICK) +
           ((gz % BRICK) * BRICK + (gy % BRICK)) * BRICK + (gx % BRICK);
}

__host__ __device__ __forceinline__ int wrap_cell(int x, int n) { return ((x % n) + n) % n; }

// Halo geometry of brick r: origin (unwrapped cell of halo cell 0) and width
// per dimension.
struct BrickHalo {
    int ox, oy, oz;  // unwrapped cell coordinates of halo cell (0, 0, 0)
    int wx, wy, wz;  // halo widths in cells (brick width + 4)
    int bx, by, bz;
};

__host__ __device__ __forceinline__ BrickHalo brick_halo(int r, const int nc[3], const int nb[3]) {
    BrickHalo h;
    h.bx = r % nb[0];
    h.by = (r / nb[0]) % nb[1];
    h.bz = r / (nb[0] * nb[1]);
    h.ox = h.bx * BRICK - 2;
    h.oy = h.by * BRICK - 2;
    h.oz = h.bz * BRICK - 2;
    h.wx = min(BRICK, nc[0] - h.bx * BRICK) + 4;
    h.wy = min(BRICK, nc[1] - h.by * BRICK) + 4;
    h.wz = min(BRICK, nc[2] - h.bz * BRICK) + 4;
    return h;
}

// The runs of halo row (hy, hz): ranges of consecutive cells of one brick
// each (at most BRICK_RUNS for halo widths <= 8), in x order.  f(k, first,
// last, hx0) receives run k's first and last brick-major cell ids and the
// halo x of its first cell; returns the count.
template <class F>
__host__ __device__ __forceinline__ int for_each_halo_run(const BrickHalo &h, int hy, int hz, const int nc[3],
                                                          const int nb[3], F f) {
    const int gy = wrap_cell(h.oy + hy, nc[1]), gz = wrap_cell(h.oz + hz, nc[2]);
    int cnt = 0, pg = -2, first = 0, last = 0, hx0 = 0;
    for (int hx = 0; hx < h.wx; hx++) {
        const int gx = wrap_cell(h.ox + hx, nc[0]);
        const int id = brick_cell_id(gx, gy, gz, nb[0], nb[1]);
        if (hx > 0 && (gx != pg + 1 || gx / BRICK != pg / BRICK)) {
            f(cnt, first, last, hx0);
            cnt++;
        }
        if (hx == 0 || gx != pg + 1 || gx / BRICK != pg / BRICK) {
            first = id;
            hx0 = hx;
        }
        last = id;
        pg = gx;
    }
    f(cnt, first, last, hx0);
    return cnt + 1;
}

// One stage buffer: a brick's halo and the runs it was copied from.
struct BrickStage {
    float4 halo[BRICK_HCAP];
    int seg_src[BRICK_SLOTS];  // first slot of the run in the position array
    int seg_len[BRICK_SLOTS];  // particles in the run (0: unused slot)
    int seg_dst[BRICK_SLOTS];  // offset of the run in `halo`
    int seg_hx[BRICK_SLOTS];   // halo x of the run's first cell, -1: unused
    double part[BRICK_CWARPS][9];  // per-warp sums of the brick (step phase)
    int brick;  // brick staged here; -1: no more bricks in this phase; -2: the halo did not fit
    int total;  // staged positions; halo[total] holds the sentinel
    int face;   // the halo reaches a cell on a box face
    int done;   // warps that finished the brick (step phase)
};

// Shared memory of one CTA of the brick path: two stage buffers (the
// producer warp fills one while the consumer warps read the other), the
// per-cell offsets of the list build, and the mbarriers.
struct BrickSmem {
    BrickStage st[2];
    int hoff[BRICK_ROWS * (BRICK_W + 1)];  // list build: halo offset of every halo cell
    unsigned long long full[2];   // stage k ready (producer arrives once)
    unsigned long long empty[2];  // stage k read by every consumer thread
    unsigned long long copy[2];   // the producer's own wait for the copies into stage k
    unsigned long long bmbar;     // list build: the stage of st[0]
};

// Pipeline state of one thread (producer and consumers track their sides).
struct BrickPipe {
    int pk, ck;            // next stage the producer fills / the consumers read
    unsigned pe[2], pf[2];  // parities of the empty / full barrier waits
    unsigned pc[2];         // parities of the producer's copy waits
    unsigned bpar;          // parity of the list build's stage
};

__device__ __forceinline__ BrickPipe brick_pipe_init() {
    BrickPipe p;
    p.pk = p.ck = 0;
    p.pe[0] = p.pe[1] = 1;  // both stages start free
    p.pf[0] = p.pf[1] = 0;
    p.pc[0] = p.pc[1] = 0;
    p.bpar = 0;
    return p;
}

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long *m, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(m)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long *m, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(m)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long *m, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(m)), "r"(parity)
        : "memory");
    return ok != 0;
}
// One bulk copy global -> this CTA's shared memory, completing on mbarrier m
// (no multicast: the source is this GPU's own position array).
__device__ __forceinline__ void bulk_copy_g2s(void *dst, const void *src, unsigned bytes, unsigned long long *m) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(m))
                 : "memory");
}
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive(unsigned long long *m) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(m)) : "memory");
}
// Bounded wait for the phase of parity `parity` of mbarrier m; false when it
// gave up (the caller records the failure).
__device__ __forceinline__ bool mbar_wait(unsigned long long *m, unsigned parity) {
    long long polls = 0;
    while (!mbar_try_wait(m, parity)) {
        if (++polls > MBAR_WAIT_POLLS) return false;
        if (polls > 64) __nanosleep(64);
    }
    return true;
}
__device__ __forceinline__ void consumer_sync() {
    asm volatile("bar.sync 1, %0;" ::"n"(BRICK_CONSUMERS) : "memory");
}

__device__ __forceinline__ void brick_smem_init(BrickSmem &bs) {
    if (threadIdx.x == 0) {
        for (int k = 0; k < 2; k++) {
            mbar_init(&bs.full[k], 1);
            mbar_init(&bs.empty[k], BRICK_CONSUMERS);
            mbar_init(&bs.copy[k], 1);
            bs.st[k].done = 0;
        }
        mbar_init(&bs.bmbar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
}

// Record a failed bounded wait: status bit and abort for the whole grid.
__device__ __forceinline__ void brick_wait_failed(const SimArgs &a) {
    atomicOr(&a.ctrl->status, GDB_STATUS_BARRIER_TIMEOUT);
    a.ctrl->abort = 1;
}

// Stage the halo of brick r from `src` into st, run by the 32 lanes of one
// warp: the lanes list the runs (two halo rows each), scan their lengths and
// issue one bulk copy per run, completing on mbarrier m; lane 0 writes the
// sentinel after the last entry and arrives on m with the byte count.  With
// HOFF the halo offset of every halo cell goes to hoff too (list build).  A
// halo that does not fit (sentinel included) copies nothing and is marked
// st.brick = -2.
template <bool HOFF>
__device__ inline void stage_issue_warp(const SimArgs &a, BrickStage &st, int *hoff, const float4 *src, int r,
                                        unsigned long long *m) {
    const int nc[3] = {a.ncx, a.ncy, a.ncz}, nb[3] = {a.nbx, a.nby, a.nbz};
    const BrickHalo h = brick_halo(r, nc, nb);
    const int nrows = h.wy * h.wz;
    const int lane = threadIdx.x & 31;
    // the runs of rows 2 lane and 2 lane + 1, four slots each, straight into
    // the slot tables
    int mytot = 0;
    bool face = h.ox <= 0 || h.ox + h.wx - 1 >= a.ncx - 1;
    bool runs_ok = true;
    for (int q = 0; q < 2; q++) {
        const int row = 2 * lane + q;
        const int g0 = row * BRICK_RUNS;
        int cnt = 0;
        if (row < nrows) {
            const int hy = row % h.wy, hz = row / h.wy;
            cnt = for_each_halo_run(h, hy, hz, nc, nb, [&](int k, int first, int last, int hx0) {
                if (k >= BRICK_RUNS) return;  // not reached for grids of >= 8 cells; flagged below
                const int s0 = a.cell_start[first];
                const int len = a.cell_start[last + 1] - s0;
                st.seg_src[g0 + k] = s0;
                st.seg_len[g0 + k] = len;
                st.seg_hx[g0 + k] = hx0;
                mytot += len;
            });
            const int uy = h.oy + hy, uz = h.oz + hz;
            face |= uy <= 0 || uy >= a.ncy - 1 || uz <= 0 || uz >= a.ncz - 1;
            if (cnt > BRICK_RUNS) {
                runs_ok = false;
                cnt = BRICK_RUNS;
            }
        }
        for (int k = cnt; k < BRICK_RUNS; k++) {
            st.seg_src[g0 + k] = 0;
            st.seg_len[g0 + k] = 0;
            st.seg_hx[g0 + k] = -1;
        }
    }
    // exclusive scan of the lanes' totals
    int incl = mytot;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    const int total = __shfl_sync(0xffffffffu, incl, 31);
    const bool anyface = __any_sync(0xffffffffu, face);
    const bool fits = total + 1 <= a.brick_hcap && __all_sync(0xffffffffu, runs_ok);
    int dst = incl - mytot;
    for (int g = 2 * lane * BRICK_RUNS; g < 2 * (lane + 1) * BRICK_RUNS; g++) {
        const int len = st.seg_len[g];
        st.seg_dst[g] = dst;
        if (fits && len > 0)
            bulk_copy_g2s(&st.halo[dst], src + st.seg_src[g], (unsigned)len * (unsigned)sizeof(float4), m);
        dst += len;
    }
    if (HOFF) {
        // halo offset of every cell of this lane's rows (from the cell table)
        // and the end of each row
        for (int q = 0; q < 2; q++) {
            const int row = 2 * lane + q;
            if (row >= nrows) continue;
            const int g0 = row * BRICK_RUNS;
            const int hy = row % h.wy, hz = row / h.wy;
            const int gy = wrap_cell(h.oy + hy, a.ncy), gz = wrap_cell(h.oz + hz, a.ncz);
            int k = 0, kl = 0;
            for (int hx = 0; hx < h.wx; hx++) {
                while (k + 1 < BRICK_RUNS && st.seg_hx[g0 + k + 1] >= 0 && st.seg_hx[g0 + k + 1] <= hx) k++;
                const int gx = wrap_cell(h.ox + hx, a.ncx);
                const int id = brick_cell_id(gx, gy, gz, a.nbx, a.nby);
                hoff[row * (BRICK_W + 1) + hx] = st.seg_dst[g0 + k] + (a.cell_start[id] - st.seg_src[g0 + k]);
                kl = k;
            }
            hoff[row * (BRICK_W + 1) + h.wx] = st.seg_dst[g0 + kl] + st.seg_len[g0 + kl];
        }
    }
    __threadfence_block();
    __syncwarp();
    if (lane == 0) {
        st.total = total;
        st.face = anyface;
        st.brick = fits ? r : -2;
        if (fits)
            st.halo[total] = make_float4(BRICK_SENTINEL, BRICK_SENTINEL, BRICK_SENTINEL, __int_as_float(0));
        mbar_arrive_expect_tx(m, fits ? (unsigned)total * (unsigned)sizeof(float4) : 0u);
    }
    __syncwarp();
}

// Shift the staged copies of particles that sit across a periodic face into
// the brick's frame: x -> x - L rint((x - c) / L) with c the centre of the
// run's cells (every particle lies within L/2 of its cell's centre).  Only
// bricks whose halo reaches a face cell have such copies.  Run by the
// threads [t0, t0 + nt) of the block (nt a multiple of 32).
__device__ inline void brick_unwrap_halo(const SimArgs &a, BrickStage &st, int t0, int nt) {
    const int nc[3] = {a.ncx, a.ncy, a.ncz}, nb[3] = {a.nbx, a.nby, a.nbz};
    const BrickHalo h = brick_halo(st.brick, nc, nb);
    const float hx = a.Lx / a.ncx, hy = a.Ly / a.ncy, hz = a.Lz / a.ncz;
    const float ilx = 1.0f / a.Lx, ily = 1.0f / a.Ly, ilz = 1.0f / a.Lz;
    const int t = (int)threadIdx.x - t0;
    const int warp = t >> 5, lane = t & 31;
    for (int g = warp; g < BRICK_SLOTS; g += nt / 32) {
        const int len = st.seg_len[g];
        if (len == 0) continue;
        const int row = g / BRICK_RUNS;
        const int hyy = row % h.wy, hzz = row / h.wy;
        const int hx0 = st.seg_hx[g];
        // cells of the run: hx0 .. the next run's start (or the row end)
        int hx1 = h.wx;
        if (g % BRICK_RUNS + 1 < BRICK_RUNS && st.seg_hx[g + 1] > hx0) hx1 = st.seg_hx[g + 1];
        const float cx = 0.5f * (float)(h.ox + hx0 + h.ox + hx1) * hx - 0.5f * a.Lx;
        const float cy = ((float)(h.oy + hyy) + 0.5f) * hy - 0.5f * a.Ly;
        const float cz = ((float)(h.oz + hzz) + 0.5f) * hz - 0.5f * a.Lz;
        const int d0 = st.seg_dst[g];
        for (int e = d0 + lane; e < d0 + len; e += 32) {
            float4 p = st.halo[e];
            p.x -= a.Lx * rintf((p.x - cx) * ilx);
            p.y -= a.Ly * rintf((p.y - cy) * ily);
            p.z -= a.Lz * rintf((p.z - cz) * ilz);
            st.halo[e] = p;
        }
    }
}

// Pair term with the neighbour already in the particle's frame (no minimum
// image): the brick stage put every copy there.
template <bool REC, int NT>
__device__ __forceinline__ void pair_force_framed(const PairRow<NT> &pr, float4 pi, float4 pj, bool valid, float &fx,
                                                  float &fy, float &fz, float &u, float &w, float &l) {
    const float dx = pj.x - pi.x, dy = pj.y - pi.y, dz = pj.z - pi.z;
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

// Entry k of slot s of the 16-bit list: chunk k / 8 of slot s holds entries
// 8 (k / 8) ... + 7, chunks strided by `stride` slots (a warp of
// consecutive slots reads 512 contiguous bytes per chunk).
__device__ __forceinline__ size_t nbl16_index(int s, int k, int stride) {
    return ((size_t)(k >> 3) * (size_t)stride + (size_t)s) * NB16 + (size_t)(k & 7);
}

// Pair loop of slot s over its 16-bit list (pairs from the stage `halo`),
// pair_potential.py:223-231 with the full-list calculator :164-178.  Lists
// are padded to whole chunks with the index of the stage's sentinel entry,
// whose distance from any particle is beyond every cut, so every entry of a
// chunk is evaluated without a test.
template <int NT, bool REC>
__device__ __forceinline__ void brick_neighbour_loop(const SimArgs &a, const float4 *halo, const PairEntry *tab, int nt,
                                                     int s, float4 pi, float &fx, float &fy, float &fz, float &u,
                                                     float &w, float &l) {
    const PairRow<NT> pr(tab, nt, NT == 1 ? 0 : ptype_of(pi));
    const int cnt = min(a.nbc[s], a.max_nbs);
    const int nch = (cnt + NB16 - 1) / NB16;
    const uint4 *base = reinterpret_cast<const uint4 *>(a.nbl) + s;
    const size_t cstride = (size_t)a.stride;
    uint4 jn = nch > 0 ? base[0] : make_uint4(0, 0, 0, 0);
    uint4 jn2 = nch > 1 ? base[cstride] : make_uint4(0, 0, 0, 0);
    for (int ch = 0; ch < nch; ch++) {
        const uint4 c = jn;
        jn = jn2;
        if (ch + 2 < nch) jn2 = base[(size_t)(ch + 2) * cstride];
        const unsigned wds[4] = {c.x, c.y, c.z, c.w};
#pragma unroll
        for (int q = 0; q < 4; q++) {
            // an entry is at most its brick's staged total (the sentinel) by
            // construction; the clamp keeps even a stale list inside the stage
            const int ja = min((int)(wds[q] & 0xffffu), BRICK_HCAP - 1);
            const int jb = min((int)(wds[q] >> 16), BRICK_HCAP - 1);
            const float4 pa = halo[ja];
            const float4 pb = halo[jb];
            pair_force_framed<REC, NT>(pr, pi, pa, true, fx, fy, fz, u, w, l);
            pair_force_framed<REC, NT>(pr, pi, pb, true, fx, fy, fz, u, w, l);
        }
    }
}

// Force + integrate over bricks (MODE_STEP) or forces only (MODE_EVAL), from
// pos[cur] into pos[cur^1].  Warp 8 is the producer: it claims bricks (the
// atomic round counter when PERSIST, a stride by CTA otherwise), stages each
// halo into the free stage buffer, shifts face copies and marks the buffer
// full; after the last brick it passes an end marker.  Warps 0-7 consume:
// particle s0 + t of a brick belongs to consumer thread t mod 256, each warp
// sums its particles' shares, and the last warp to finish a brick adds the
// eight warp sums in a fixed order into partials[brick] -- no block-wide
// barrier per brick, and sums independent of timing.
template <int NT, int INTEG, int MODE, bool PERSIST>
__device__ inline bool phase_step_bricks(const SimArgs &a, BrickSmem &bs, BrickPipe &pp, const PairEntry *tab, int nt,
                                         int cur, int step, Span g = grid_span()) {
    DevCtrl *ctrl = a.ctrl;
    const float4 *pos = cur_pos(a, cur);
    float4 *pos_next = cur_pos(a, cur ^ 1);
    const bool rec = MODE == MODE_EVAL || (a.every > 0 && step % a.every == 0);
    const bool reset = MODE == MODE_STEP && a.reset_every > 0 && step % a.reset_every == 0;
    const int ppar = (step & 1) ^ 1;
    const bool shift_pending = ctrl->pending[ppar] != 0;
    float shx = 0.f, shy = 0.f, shz = 0.f;
    if (shift_pending) {
        shx = ctrl->shift[ppar][0];
        shy = ctrl->shift[ppar][1];
        shz = ctrl->shift[ppar][2];
    }
    const float xi = ctrl->xi;
    const bool full = rec || reset;
    const bool needk = full || INTEG == GDB_INTEGRATOR_NVT;
    const int nbricks = a.nbx * a.nby * a.nbz;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    bool moved = false, ok = true;
    if (warp == BRICK_CWARPS) {
        // ---- producer ----
        for (int j = 0;; j++) {
            int r;
            if (PERSIST) {
                r = 0;
                if (lane == 0) r = (int)atomicAdd(&ctrl->work[step & 1], 1u);
                r = __shfl_sync(0xffffffffu, r, 0);
            } else {
                r = g.b + j * g.nb;
            }
            const int k = pp.pk;
            if (!mbar_wait(&bs.empty[k], pp.pe[k])) {
                if (lane == 0) brick_wait_failed(a);
                ok = false;
                break;
            }
            pp.pe[k] ^= 1u;
            pp.pk ^= 1;
            BrickStage &st = bs.st[k];
            if (r >= nbricks) {  // end marker
                if (lane == 0) {
                    st.brick = -1;
                    mbar_arrive(&bs.full[k]);
                }
                __syncwarp();
                break;
            }
            fence_proxy_async_smem();
            stage_issue_warp<false>(a, st, nullptr, pos, r, &bs.copy[k]);
            const bool fits = st.brick >= 0;
            if (!mbar_wait(&bs.copy[k], pp.pc[k])) {
                if (lane == 0) brick_wait_failed(a);
                ok = false;
                break;
            }
            pp.pc[k] ^= 1u;
            if (fits && st.face) brick_unwrap_halo(a, st, BRICK_CONSUMERS, 32);
            __threadfence_block();
            __syncwarp();
            if (lane == 0) {
                if (!fits) {
                    atomicOr(&ctrl->status, GDB_STATUS_BRICK_CAPACITY);
                    ctrl->abort = 1;
                }
                mbar_arrive(&bs.full[k]);
            }
            __syncwarp();
            if (!fits) {
                ok = false;
                break;
            }
        }
    } else {
        // ---- consumers ----
        for (;;) {
            const int k = pp.ck;
            if (!mbar_wait(&bs.full[k], pp.pf[k])) {
                if (lane == 0) brick_wait_failed(a);
                ok = false;
                break;
            }
            pp.pf[k] ^= 1u;
            pp.ck ^= 1;
            BrickStage &st = bs.st[k];
            const int br = st.brick;
            if (br < 0) {
                ok = br == -1;
                fence_proxy_async_smem();
                mbar_arrive(&bs.empty[k]);
                break;
            }
            double red[NQ];
#pragma unroll
            for (int q = 0; q < NQ; q++) red[q] = 0.0;
            const int s0 = a.cell_start[br * BRICK * BRICK * BRICK];
            const int s1 = a.cell_start[(br + 1) * BRICK * BRICK * BRICK];
            const float hcx = a.Lx / a.ncx, hcy = a.Ly / a.ncy, hcz = a.Lz / a.ncz;
            for (int i = s0 + (int)threadIdx.x; i < s1; i += BRICK_CONSUMERS) {
                const float4 v = a.vel[i];
                const float4 rr = MODE == MODE_STEP ? a.rref[i] : make_float4(0.f, 0.f, 0.f, 0.f);
                const float4 pi = pos[i];
                // the particle in its cell's frame (it may have crossed a face
                // since the build); the integration uses the stored value
                const int c = a.scell[i];
                const int bidx = c / (BRICK * BRICK * BRICK);
                const int gx = (bidx % a.nbx) * BRICK + c % BRICK;
                const int gy = ((bidx / a.nbx) % a.nby) * BRICK + (c / BRICK) % BRICK;
                const int gz = (bidx / (a.nbx * a.nby)) * BRICK + (c / (BRICK * BRICK)) % BRICK;
                float4 pf = pi;
                const float cx = ((float)gx + 0.5f) * hcx - 0.5f * a.Lx, cy = ((float)gy + 0.5f) * hcy - 0.5f * a.Ly,
                            cz = ((float)gz + 0.5f) * hcz - 0.5f * a.Lz;
                pf.x -= a.Lx * rintf((pf.x - cx) / a.Lx);
                pf.y -= a.Ly * rintf((pf.y - cy) / a.Ly);
                pf.z -= a.Lz * rintf((pf.z - cz) / a.Lz);
                float fx = 0.f, fy = 0.f, fz = 0.f, u = 0.f, w = 0.f, l = 0.f;
                if (rec)
                    brick_neighbour_loop<NT, true>(a, st.halo, tab, nt, i, pf, fx, fy, fz, u, w, l);
                else
                    brick_neighbour_loop<NT, false>(a, st.halo, tab, nt, i, pf, fx, fy, fz, u, w, l);
                finish_particle<INTEG, MODE>(a, i, pi, v, rr, fx, fy, fz, u, w, l, rec, reset, step, shift_pending,
                                             shx, shy, shz, xi, pos_next, red, moved);
            }
            // this warp's sums, then the last warp of the brick adds the
            // eight in warp order into partials[brick]
            if (full || needk) {
#pragma unroll
                for (int q = 0; q < NQ; q++) {
                    if (!full && q > 0) break;
                    const double v = warp_sum(red[q]);
                    if (lane == 0) st.part[warp][q] = v;
                }
                int last = 0;
                if (lane == 0) {
                    __threadfence_block();
                    last = atomicAdd(&st.done, 1) == BRICK_CWARPS - 1;
                }
                last = __shfl_sync(0xffffffffu, last, 0);
                if (last) {
                    __threadfence_block();
                    if (lane < NQ && (full || lane == 0)) {
                        double t = 0.0;
                        for (int w8 = 0; w8 < BRICK_CWARPS; w8++) t += *(volatile double *)&st.part[w8][lane];
                        a.partials[(size_t)br * NQ + lane] = t;
                    }
                    if (lane == 0) st.done = 0;
                }
            }
            // every consumer thread's reads of the stage before the next copy
            fence_proxy_async_smem();
            mbar_arrive(&bs.empty[k]);
        }
    }
    if (MODE == MODE_STEP) {
        if (__syncthreads_or(moved) && threadIdx.x == 0) {
            if (PERSIST)
                ctrl->rebuild_next = 1;
            else
                ctrl->rebuild = 1;
        }
    }
    return __syncthreads_and(ok);
}

// Neighbour lists of the particles of every brick (after the counting sort
// into brick order: positions in pos_tmp, cells in scell), 16-bit halo
// indices padded with the sentinel's index to whole chunks.  SHIFTED as the
// row build: every grid dimension has >= 7 cells and no coordinate sits on a
// face, so the periodic shift of a candidate is fixed by its cell and the
// distance needs no comparisons.  Bricks are strided over the CTAs; warp 0
// stages each one into st[0], every thread of the block builds.
template <bool FMA, bool SHIFTED>
__device__ inline bool phase_nbl_bricks_t(const SimArgs &a, BrickSmem &bs, BrickPipe &pp, Span g) {
    const int nc[3] = {a.ncx, a.ncy, a.ncz}, nb[3] = {a.nbx, a.nby, a.nbz};
    const int nbricks = a.nbx * a.nby * a.nbz;
    const float Lx = a.Lx, Ly = a.Ly, Lz = a.Lz;
    const double hx = (double)Lx / a.ncx, hy = (double)Ly / a.ncy, hz = (double)Lz / a.ncz;
    // reach for the geometric pruning: sqrt(cps2) plus a margin well above
    // the float32 rounding of the exact distance (a few ulp of L/2)
    const double Lmax = fmax((double)Lx, fmax((double)Ly, (double)Lz));
    const double reach = sqrt((double)a.cps2) + 1e-3 + 1e-5 * Lmax;
    const double reach2 = reach * reach;
    const float cps2 = a.cps2;
    const int maxn = a.max_nbs;
    unsigned short *nbl = reinterpret_cast<unsigned short *>(a.nbl);
    BrickStage &st = bs.st[0];
    for (int r = g.b; r < nbricks; r += g.nb) {
        // every thread's earlier accesses of the stage before the copies
        fence_proxy_async_smem();
        __syncthreads();
        if (threadIdx.x < 32) stage_issue_warp<true>(a, st, bs.hoff, a.pos_tmp, r, &bs.bmbar);
        const bool done = mbar_wait(&bs.bmbar, pp.bpar);
        if (!__syncthreads_and(done)) {
            if (threadIdx.x == 0) brick_wait_failed(a);
            // copies of this stage may still be landing: wait again, bounded
            mbar_wait(&bs.bmbar, pp.bpar);
            __syncthreads();
            return false;
        }
        pp.bpar ^= 1u;
        if (st.brick < 0) {  // the halo does not fit the stage
            if (threadIdx.x == 0) {
                atomicOr(&a.ctrl->status, GDB_STATUS_BRICK_CAPACITY);
                a.ctrl->abort = 1;
            }
            __syncthreads();
            return false;
        }
        const int sentinel = st.total;
        const BrickHalo h = brick_halo(r, nc, nb);
        const int s0 = a.cell_start[r * BRICK * BRICK * BRICK];
        const int s1 = a.cell_start[(r + 1) * BRICK * BRICK * BRICK];
        for (int s = s0 + (int)threadIdx.x; s < s1; s += (int)blockDim.x) {
            const float4 pi = a.pos_tmp[s];
            const int c = a.scell[s];
            const int hxo = c % BRICK + 2, hyo = (c / BRICK) % BRICK + 2, hzo = (c / (BRICK * BRICK)) % BRICK + 2;
            const int own = bs.hoff[(hzo * h.wy + hyo) * (BRICK_W + 1) + hxo] + (s - a.cell_start[c]);
            // the particle in its cell's frame for the pruning geometry (a
            // coordinate on the +L/2 face belongs to cell 0 at -L/2); exact
            // in float64, the distance test below keeps the stored values
            const double cxo = (h.ox + hxo + 0.5) * hx - 0.5 * Lx, cyo = (h.oy + hyo + 0.5) * hy - 0.5 * Ly,
                         czo = (h.oz + hzo + 0.5) * hz - 0.5 * Lz;
            const double px = pi.x - (double)Lx * rint((pi.x - cxo) / Lx);
            const double py = pi.y - (double)Ly * rint((pi.y - cyo) / Ly);
            const double pz = pi.z - (double)Lz * rint((pi.z - czo) / Lz);
            int cnt = 0;
            for (int dz = -2; dz <= 2; dz++) {
                const int hzz = hzo + dz, uz = h.oz + hzz;
                const double zlo = uz * hz - 0.5 * Lz, zhi = zlo + hz;
                const double ez = pz < zlo ? zlo - pz : (pz > zhi ? pz - zhi : 0.0);
                if (ez * ez > reach2) continue;
                const float sz = SHIFTED ? (uz < 0 ? -Lz : (uz >= a.ncz ? Lz : 0.f)) : 0.f;
                for (int dy = -2; dy <= 2; dy++) {
                    const int hyy = hyo + dy, uy = h.oy + hyy;
                    const double ylo = uy * hy - 0.5 * Ly, yhi = ylo + hy;
                    const double ey = py < ylo ? ylo - py : (py > yhi ? py - yhi : 0.0);
                    const double eyz = ey * ey + ez * ez;
                    if (eyz > reach2) continue;
                    const float sy = SHIFTED ? (uy < 0 ? -Ly : (uy >= a.ncy ? Ly : 0.f)) : 0.f;
                    // cells of the row within reach: a contiguous x range
                    int x0 = hxo - 2, x1 = hxo + 2;
                    for (; x0 < hxo; x0++) {
                        const double ex = px - ((h.ox + x0 + 1) * hx - 0.5 * Lx);
                        if (ex * ex + eyz <= reach2) break;
                    }
                    for (; x1 > hxo; x1--) {
                        const double ex = ((h.ox + x1) * hx - 0.5 * Lx) - px;
                        if (ex * ex + eyz <= reach2) break;
                    }
                    const int rowo = (hzz * h.wy + hyy) * (BRICK_W + 1);
                    for (int xc = x0; xc <= x1; xc++) {
                        const int ux = h.ox + xc;
                        const float sx = SHIFTED ? (ux < 0 ? -Lx : (ux >= a.ncx ? Lx : 0.f)) : 0.f;
                        const int e0 = bs.hoff[rowo + xc], e1 = bs.hoff[rowo + xc + 1];
                        for (int e = e0; e < e1; e++) {
                            const float4 pj = st.halo[e];
                            const float d2 = SHIFTED ? dist_sq_shifted<FMA>(pj, pi, sx, sy, sz)
                                                     : dist_sq_exact<FMA>(pj, pi, Lx, Ly, Lz);
                            if (d2 < cps2 && e != own) {
                                if (cnt < maxn) nbl[nbl16_index(s, cnt, a.stride)] = (unsigned short)e;
                                cnt++;
                            }
                        }
                    }
                }
            }
            // pad the last chunk with the sentinel's index
            if (cnt < maxn)
                for (int k = cnt; k & (NB16 - 1); k++) nbl[nbl16_index(s, k, a.stride)] = (unsigned short)sentinel;
            a.nbc[s] = cnt;
            atomicMax(&a.ctrl->maxcount, cnt);
        }
    }
    fence_proxy_async_smem();
    __syncthreads();
    return true;
}

template <bool FMA>
__device__ inline bool phase_nbl_bricks(const SimArgs &a, BrickSmem &bs, BrickPipe &pp, Span g) {
    const bool shifted = a.ncx >= 7 && a.ncy >= 7 && a.ncz >= 7 && !*(volatile int *)&a.ctrl->cell_wrap;
    return shifted ? phase_nbl_bricks_t<FMA, true>(a, bs, pp, g) : phase_nbl_bricks_t<FMA, false>(a, bs, pp, g);
}

}  // namespace gdb
