// md_kernels.cuh -- the fused step kernel (k_step, one step per launch) and
// the persistent kernel (k_run, a timeblock per launch), instantiated per
// type-count path in md_inst_nt1.cu / md_inst_nt2.cu / md_inst_ntg.cu so the
// instantiations compile in parallel.
#pragma once

#include "md_bricks.cuh"
#include "md_phases.cuh"

namespace gdb {

__device__ __forceinline__ void load_table(const PairTable &tab, PairEntry *s_tab) {
    for (int t = threadIdx.x; t < tab.nt * tab.nt; t += blockDim.x) s_tab[t] = tab.e[t];
    __syncthreads();
}

// one step (or the force-only evaluation); the last block to finish does
// the float64 bookkeeping
// register budget: 64 per thread (4 blocks/SM) for one lane per particle,
// 80 (3 blocks/SM) when lanes share a particle (measured best on B200); the
// persistent kernel also holds the list-build phase
#define GDB_STEP_MINBLOCKS(TP) ((TP) == 1 ? 4 : 3)
#ifndef GDB_RUN_MINBLOCKS_TP1
#define GDB_RUN_MINBLOCKS_TP1 4
#endif
#define GDB_RUN_MINBLOCKS(TP) ((TP) == 1 ? GDB_RUN_MINBLOCKS_TP1 : 3)

template <int TP, int NT, int INTEG, int MODE>
__global__ void __launch_bounds__(GDB_BLOCK, GDB_STEP_MINBLOCKS(TP)) k_step(SimArgs a, PairTable tab, int cur) {
    __shared__ PairEntry s_tab[GDB_MAX_TYPES * GDB_MAX_TYPES];
    __shared__ double s_red[NQ * 32];
    __shared__ bool s_last;
    load_table(tab, s_tab);
    DevCtrl *ctrl = a.ctrl;
    const int step = ctrl->step;
    phase_step<TP, NT, INTEG, MODE, true, false>(a, s_tab, tab.nt, cur, step, s_red);
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) s_last = atomicAdd(&ctrl->ticket, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!s_last) return;
    finalize_step<MODE>(a, step, gridDim.x, s_red);
    if (threadIdx.x == 0) ctrl->ticket = 0;
}

// Synchronisation of the blocks that share one system, between phases.
// `last` runs on one whole block after every block has arrived and before
// any leaves; the call returns false when the wait was abandoned.
// With `flag`, a block reports that one of its particles moved more than
// skin/2; the block that runs `last` finds in *any whether any block did.
struct GridSync {  // bounded software barrier over a cooperative grid
    static constexpr bool kGrid = true;
    template <typename F>
    __device__ __forceinline__ bool operator()(DevCtrl *c, F last, bool flag = false, int *any = nullptr) const {
        return grid_barrier(c, last, flag, any);
    }
};

// Hardware barrier of a thread-block cluster; release/acquire at cluster scope
// orders the global-memory writes of every CTA of the cluster before the
// reads after it.  Rank 0 runs `last` between two barriers.
__device__ __forceinline__ void cluster_barrier() {
    asm volatile("barrier.cluster.arrive.release;\n\tbarrier.cluster.wait.acquire;" ::: "memory");
}
struct ClusterSync {
    static constexpr bool kGrid = false;
    int rank;
    template <typename F>
    __device__ __forceinline__ bool operator()(DevCtrl *c, F last, bool flag = false, int *any = nullptr) const {
        if (flag && threadIdx.x == 0) c->rebuild_next = 1;
        cluster_barrier();
        if (rank == 0) {
            if (any && threadIdx.x == 0) {
                *any = c->rebuild_next;
                c->rebuild_next = 0;
            }
            last();
        }
        cluster_barrier();
        return true;
    }
};

// Neighbour-list rebuild by the blocks of span g: the phases of the
// standalone chain with a synchronisation between them.
template <bool FMA, int WPB, class Sync>
__device__ inline bool rebuild_phases(const SimArgs &a, int cur, Span g, const Sync &sync, NbScratch<WPB> &scr,
                                      float4 *spos) {
    DevCtrl *c = a.ctrl;
    auto none = [] {};
    if (a.nb_kind == GDB_NBLIST_NSQ) {
        phase_nbl_nsq<FMA, false>(a, cur, g, spos);
        trace_mark(c, TR_REBUILD_PHASE);
        const bool ok = sync(c, [&] {
            if (threadIdx.x == 0) rebuild_done(c);
        });
        trace_mark(c, TR_REBUILD_DONE);
        return ok;
    }
    phase_cell_assign<false>(a, cur, g);
    if (!sync(c, none)) return false;
    trace_mark(c, TR_REBUILD_PHASE);
    phase_scan_partial(a, g);
    if (!sync(c, [&] { block_scan_chunks(a); })) return false;
    phase_scan_final(a, g);
    if (!sync(c, none)) return false;
    phase_scatter(a, g);
    if (!sync(c, none)) return false;
    trace_mark(c, TR_REBUILD_PHASE);
    phase_sort_cells(a, g);
    if (!sync(c, none)) return false;
    phase_gather(a, cur, g);
    if (!sync(c, none)) return false;
    trace_mark(c, TR_REBUILD_PHASE);
    phase_nbl_cells<FMA>(a, g, scr);
    if (!sync(c, none)) return false;
    trace_mark(c, TR_REBUILD_PHASE);
    phase_finish_cells(a, cur, g);
    const bool ok = sync(c, [&] {
        if (threadIdx.x == 0) rebuild_done(c);
    });
    trace_mark(c, TR_REBUILD_DONE);
    return ok;
}

// `nsteps` steps starting from pos[cur0], then (if do_eval) the force-only
// evaluation of the final state -- one timeblock of
// simulation/Simulation.py:306-328 -- by the blocks of span g.
// NPT_Atomic changes the box every step: the box of the step (ctrl->box,
// written by the previous step's bookkeeping), and at a list build the cell
// grid of that box as nblist_linked_lists.py:36-39 computes it, within the
// allocated grid.
__device__ __forceinline__ void npt_refresh_box(SimArgs &a) {
    a.Lx = *(volatile float *)&a.ctrl->box[0];
    a.Ly = *(volatile float *)&a.ctrl->box[1];
    a.Lz = *(volatile float *)&a.ctrl->box[2];
}
__device__ __forceinline__ void npt_cell_grid(SimArgs &a) {
    if (a.nb_kind != GDB_NBLIST_CELLS) return;
    a.ncx = min(a.ncx_max, max(1, (int)(a.Lx / a.min_cell)));
    a.ncy = min(a.ncy_max, max(1, (int)(a.Ly / a.min_cell)));
    a.ncz = min(a.ncz_max, max(1, (int)(a.Lz / a.min_cell)));
    a.ncell = a.ncx * a.ncy * a.ncz;
    a.nchunks = (a.ncell + SCAN_CHUNK - 1) / SCAN_CHUNK;
}

template <int TP, int NT, int INTEG, int WPB, class Sync>
__device__ inline void run_steps(const SimArgs &a0, const PairEntry *s_tab, int nt, int cur0, int nsteps, int do_eval,
                                 Span g, const Sync &sync, double *s_red, float4 *spos = nullptr) {
    __shared__ NbScratch<WPB> scr;
    // NPT_Atomic: a copy of the arguments follows the box
    SimArgs a_npt;
    if (INTEG == GDB_INTEGRATOR_NPT) a_npt = a0;
    const SimArgs &a = INTEG == GDB_INTEGRATOR_NPT ? a_npt : a0;
    DevCtrl *ctrl = a.ctrl;
    int cur = cur0;
    const int rounds = (a.n + (int)blockDim.x / TP - 1) / ((int)blockDim.x / TP);  // partial rows per step
    trace_mark(ctrl, TR_START);
    __shared__ StepCtl s_ctl;
    __shared__ int s_any;  // a particle moved beyond skin/2 (the block running `last`, or every block)
    // a grid of at most BAR_FLAT_MAX blocks: every block keeps the books of a
    // step (step_barrier_all, finalize_step_all), on rows double-buffered by
    // step parity, as a block may write the next step's rows while another
    // still sums this step's
    const bool all = Sync::kGrid && INTEG != GDB_INTEGRATOR_NPT && a.bar_all && (int)gridDim.x <= BAR_FLAT_MAX;
    unsigned seq = 0;  // step barriers of this launch
    for (int s = 0; s < nsteps + do_eval; s++) {
        if (INTEG == GDB_INTEGRATOR_NPT) npt_refresh_box(a_npt);
        // the rebuild flag, the step index and the state the step reads
        // (momentum shift, thermostat), loaded together by one thread: none
        // of them changes across a rebuild.  Where every block keeps the
        // books, its own copy is current after the first step.
        if (threadIdx.x == 0 && (!all || s == 0)) load_step_ctl(ctrl, &s_ctl);
        __syncthreads();
        const int rebuild = s_ctl.rebuild;
        const int step = s_ctl.step;
        if (rebuild) {
            if (INTEG == GDB_INTEGRATOR_NPT) npt_cell_grid(a_npt);
            const bool ok = a.fma ? rebuild_phases<true>(a, cur, g, sync, scr, spos)
                                  : rebuild_phases<false>(a, cur, g, sync, scr, spos);
            if (!ok) return;
        }
        bool ok;
        if (s < nsteps) {
            double *part = all ? a.partials + (size_t)(step & 1) * rounds * NQ : nullptr;
            const bool moved = phase_step<TP, NT, INTEG, MODE_STEP, false, true>(a, s_tab, nt, cur, step, s_red, g,
                                                                                   &s_ctl, part);
            trace_mark(ctrl, TR_STEP_PHASE);
            if (all) {
                ok = step_barrier_all(ctrl, seq++, moved, &s_any);
                if (ok) finalize_step_all<INTEG>(a, step, rounds, part, s_red, &s_ctl, s_any);
            } else {
                ok = sync(
                    ctrl,
                    [&] {
                        finalize_step<MODE_STEP, INTEG>(a, step, rounds, s_red);
                        if (threadIdx.x == 0 && s_any) ctrl->rebuild = 1;
                    },
                    moved, &s_any);
            }
            cur ^= 1;
            trace_mark(ctrl, TR_STEP);
        } else {
            phase_step<TP, NT, INTEG, MODE_EVAL, false, true>(a, s_tab, nt, cur, step, s_red, g, &s_ctl);
            ok = sync(ctrl, [&] {
                finalize_step<MODE_EVAL>(a, step, rounds, s_red);
                if (threadIdx.x == 0) ctrl->work[(step + 1) & 1] = 0;
            });
            trace_mark(ctrl, TR_EVAL);
        }
        if (!ok) return;
    }
}

// Neighbour-list rebuild of the brick path: the counting sort into brick
// order (the row rebuild's phases, cells numbered brick by brick), then the
// brick-wise list build over staged halos.
template <bool FMA, class Sync>
__device__ inline bool rebuild_phases_bricks(const SimArgs &a, int cur, Span g, const Sync &sync, BrickSmem &bs,
                                             BrickPipe &pp) {
    DevCtrl *c = a.ctrl;
    auto none = [] {};
    phase_cell_assign<false>(a, cur, g);
    if (!sync(c, none)) return false;
    trace_mark(c, TR_REBUILD_PHASE);
    phase_scan_partial(a, g);
    if (!sync(c, [&] { block_scan_chunks(a); })) return false;
    phase_scan_final(a, g);
    if (!sync(c, none)) return false;
    phase_scatter(a, g);
    if (!sync(c, none)) return false;
    trace_mark(c, TR_REBUILD_PHASE);
    phase_sort_cells(a, g);
    if (!sync(c, none)) return false;
    phase_gather(a, cur, g);
    if (!sync(c, none)) return false;
    trace_mark(c, TR_REBUILD_PHASE);
    if (!phase_nbl_bricks<FMA>(a, bs, pp, g)) return false;
    if (!sync(c, none)) return false;
    trace_mark(c, TR_REBUILD_PHASE);
    phase_finish_cells(a, cur, g);
    const bool ok = sync(c, [&] {
        if (threadIdx.x == 0) rebuild_done(c);
    });
    trace_mark(c, TR_REBUILD_DONE);
    return ok;
}

// Persistent cooperative kernel of the brick path: one timeblock of one
// system per launch (steps, rebuilds, thermostat), bricks as rounds, halos
// staged by bulk copies into dynamic shared memory (BrickSmem).
template <int NT, int INTEG>
__global__ void __launch_bounds__(BRICK_THREADS, 2)
    k_run_bricks(SimArgs a, PairTable tab, int cur0, int nsteps, int do_eval) {
    extern __shared__ __align__(128) unsigned char brick_dsm[];
    BrickSmem &bs = *reinterpret_cast<BrickSmem *>(brick_dsm);
    __shared__ PairEntry s_tab[GDB_MAX_TYPES * GDB_MAX_TYPES];
    __shared__ double s_red[NQ * 32];
    load_table(tab, s_tab);
    brick_smem_init(bs);
    DevCtrl *ctrl = a.ctrl;
    if (*(volatile int *)&ctrl->abort) return;
    const GridSync sync{};
    const Span g = grid_span();
    const int nbricks = a.nbx * a.nby * a.nbz;
    BrickPipe pp = brick_pipe_init();
    int cur = cur0;
    trace_mark(ctrl, TR_START);
    for (int s = 0; s < nsteps + do_eval; s++) {
        if (*(volatile int *)&ctrl->rebuild) {
            const bool ok = a.fma ? rebuild_phases_bricks<true>(a, cur, g, sync, bs, pp)
                                  : rebuild_phases_bricks<false>(a, cur, g, sync, bs, pp);
            if (!ok) return;
        }
        const int step = *(volatile int *)&ctrl->step;
        bool ok;
        if (s < nsteps) {
            if (!phase_step_bricks<NT, INTEG, MODE_STEP, true>(a, bs, pp, s_tab, tab.nt, cur, step)) return;
            trace_mark(ctrl, TR_STEP_PHASE);
            ok = sync(ctrl, [&] {
                finalize_step<MODE_STEP>(a, step, nbricks, s_red);
                if (threadIdx.x == 0 && ctrl->rebuild_next) {
                    ctrl->rebuild = 1;
                    ctrl->rebuild_next = 0;
                }
            });
            cur ^= 1;
            trace_mark(ctrl, TR_STEP);
        } else {
            if (!phase_step_bricks<NT, INTEG, MODE_EVAL, true>(a, bs, pp, s_tab, tab.nt, cur, step)) return;
            ok = sync(ctrl, [&] {
                finalize_step<MODE_EVAL>(a, step, nbricks, s_red);
                if (threadIdx.x == 0) ctrl->work[(step + 1) & 1] = 0;
            });
            trace_mark(ctrl, TR_EVAL);
        }
        if (!ok) return;
    }
}

// One brick-path step (or force-only evaluation) per launch, with the list
// already built; the last CTA to finish does the float64 bookkeeping.
template <int NT, int INTEG, int MODE>
__global__ void __launch_bounds__(BRICK_THREADS, 2) k_step_bricks(SimArgs a, PairTable tab, int cur) {
    extern __shared__ __align__(128) unsigned char brick_dsm[];
    BrickSmem &bs = *reinterpret_cast<BrickSmem *>(brick_dsm);
    __shared__ PairEntry s_tab[GDB_MAX_TYPES * GDB_MAX_TYPES];
    __shared__ double s_red[NQ * 32];
    __shared__ bool s_last;
    load_table(tab, s_tab);
    brick_smem_init(bs);
    DevCtrl *ctrl = a.ctrl;
    const int step = ctrl->step;
    BrickPipe pp = brick_pipe_init();
    phase_step_bricks<NT, INTEG, MODE, false>(a, bs, pp, s_tab, tab.nt, cur, step);
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) s_last = atomicAdd(&ctrl->ticket, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!s_last) return;
    finalize_step<MODE>(a, step, a.nbx * a.nby * a.nbz, s_red);
    if (threadIdx.x == 0) ctrl->ticket = 0;
}

// Persistent cooperative kernel: one timeblock of one system per launch.
// Small N^2-list systems stage their positions for the list build in dynamic
// shared memory (a.nsq_smem, n float4 per block).
template <int TP, int NT, int INTEG>
__global__ void __launch_bounds__(GDB_BLOCK, GDB_RUN_MINBLOCKS(TP)) k_run(SimArgs a, PairTable tab, int cur0, int nsteps, int do_eval) {
    extern __shared__ float4 run_dsm[];
    __shared__ PairEntry s_tab[GDB_MAX_TYPES * GDB_MAX_TYPES];
    __shared__ double s_red[NQ * 32];
    load_table(tab, s_tab);
    // a block that starts after others abandoned a barrier does no work
    if (*(volatile int *)&a.ctrl->abort) return;
    run_steps<TP, NT, INTEG, GDB_BLOCK / 32>(a, s_tab, tab.nt, cur0, nsteps, do_eval, grid_span(), GridSync{}, s_red,
                                             a.nsq_smem ? run_dsm : nullptr);
}

// One system per thread-block cluster, state in global memory: a batch of
// systems advances a timeblock in one launch, each cluster with hardware
// barriers between its phases (no cooperative launch, no software barrier).
struct ClusterRunJob {
    SimArgs a;
    PairTable tab;
    int cur;  // position buffer holding the current state
};

constexpr int CLG_BLOCK = 1024;  // one CTA per SM: a cluster of C CTAs spans C SMs

template <int TP, int NT, int INTEG>
__global__ void __launch_bounds__(CLG_BLOCK, 1)
    k_run_clusters(const ClusterRunJob *__restrict__ jobs, int nsteps, int do_eval) {
    __shared__ PairEntry s_tab[GDB_MAX_TYPES * GDB_MAX_TYPES];
    __shared__ double s_red[NQ * 32];
    __shared__ SimArgs s_a;
    unsigned rank, nrank;
    asm("mov.u32 %0, %%cluster_ctarank;" : "=r"(rank));
    asm("mov.u32 %0, %%cluster_nctarank;" : "=r"(nrank));
    const ClusterRunJob &job = jobs[blockIdx.x / nrank];
    if (threadIdx.x == 0) s_a = job.a;
    load_table(job.tab, s_tab);  // ends with __syncthreads
    run_steps<TP, NT, INTEG, CLG_BLOCK / 32>(s_a, s_tab, job.tab.nt, job.cur, nsteps, do_eval,
                                             Span{(int)rank, (int)nrank}, ClusterSync{(int)rank}, s_red);
}

// Entry points each instantiation unit exports to the host code.
#define GDB_DECLARE_NT(NTNAME)                                                                          \
    void launch_step_##NTNAME(const SimArgs &a, const PairTable &tab, cudaStream_t st, int tp, int integ, \
                              int mode, int grid, int cur);                                            \
    const void *run_kernel_##NTNAME(int tp, int integ);                                                  \
    const void *run_clusters_kernel_##NTNAME(int tp, int integ);                                         \
    const void *run_bricks_kernel_##NTNAME(int integ);                                                   \
    const void *step_bricks_kernel_##NTNAME(int integ, int mode);

GDB_DECLARE_NT(nt1)
GDB_DECLARE_NT(nt2)
GDB_DECLARE_NT(ntg)

#define GDB_DEFINE_NT(NTNAME, NT)                                                                            \
    template <int TP>                                                                                        \
    static void step_tp_##NTNAME(const SimArgs &a, const PairTable &tab, cudaStream_t st, int integ, int mode, \
                                 int grid, int cur) {                                                        \
        if (mode == MODE_EVAL)                                                                               \
            k_step<TP, NT, 0, MODE_EVAL><<<grid, GDB_BLOCK, 0, st>>>(a, tab, cur);                           \
        else if (integ == GDB_INTEGRATOR_NVT)                                                                \
            k_step<TP, NT, GDB_INTEGRATOR_NVT, MODE_STEP><<<grid, GDB_BLOCK, 0, st>>>(a, tab, cur);          \
        else if (integ == GDB_INTEGRATOR_LANGEVIN)                                                           \
            k_step<TP, NT, GDB_INTEGRATOR_LANGEVIN, MODE_STEP><<<grid, GDB_BLOCK, 0, st>>>(a, tab, cur);     \
        else                                                                                                 \
            k_step<TP, NT, GDB_INTEGRATOR_NVE, MODE_STEP><<<grid, GDB_BLOCK, 0, st>>>(a, tab, cur);          \
    }                                                                                                        \
    void launch_step_##NTNAME(const SimArgs &a, const PairTable &tab, cudaStream_t st, int tp, int integ,    \
                              int mode, int grid, int cur) {                                                 \
        switch (tp) {                                                                                        \
            case 1: step_tp_##NTNAME<1>(a, tab, st, integ, mode, grid, cur); break;                          \
            case 2: step_tp_##NTNAME<2>(a, tab, st, integ, mode, grid, cur); break;                          \
            case 4: step_tp_##NTNAME<4>(a, tab, st, integ, mode, grid, cur); break;                          \
            case 8: step_tp_##NTNAME<8>(a, tab, st, integ, mode, grid, cur); break;                          \
            case 16: step_tp_##NTNAME<16>(a, tab, st, integ, mode, grid, cur); break;                        \
            default: step_tp_##NTNAME<32>(a, tab, st, integ, mode, grid, cur); break;                       \
        }                                                                                                    \
    }                                                                                                        \
    template <int TP>                                                                                        \
    static const void *run_tp_##NTNAME(int integ) {                                                          \
        return integ == GDB_INTEGRATOR_NVT        ? (const void *)k_run<TP, NT, GDB_INTEGRATOR_NVT>          \
               : integ == GDB_INTEGRATOR_LANGEVIN ? (const void *)k_run<TP, NT, GDB_INTEGRATOR_LANGEVIN>     \
               : integ == GDB_INTEGRATOR_NPT      ? (const void *)k_run<TP, NT, GDB_INTEGRATOR_NPT>          \
                                                  : (const void *)k_run<TP, NT, GDB_INTEGRATOR_NVE>;         \
    }                                                                                                        \
    const void *run_kernel_##NTNAME(int tp, int integ) {                                                     \
        switch (tp) {                                                                                        \
            case 1: return run_tp_##NTNAME<1>(integ);                                                        \
            case 2: return run_tp_##NTNAME<2>(integ);                                                        \
            case 4: return run_tp_##NTNAME<4>(integ);                                                        \
            case 8: return run_tp_##NTNAME<8>(integ);                                                        \
            case 16: return run_tp_##NTNAME<16>(integ);                                                      \
            default: return run_tp_##NTNAME<32>(integ);                                                      \
        }                                                                                                    \
    } \
    template <int TP>                                                                                        \
    static const void *run_clusters_tp_##NTNAME(int integ) {                                                 \
        return integ == GDB_INTEGRATOR_NVT ? (const void *)k_run_clusters<TP, NT, GDB_INTEGRATOR_NVT>        \
                                           : (const void *)k_run_clusters<TP, NT, GDB_INTEGRATOR_NVE>;       \
    }                                                                                                        \
    const void *run_clusters_kernel_##NTNAME(int tp, int integ) {                                            \
        switch (tp) {                                                                                        \
            case 1: return run_clusters_tp_##NTNAME<1>(integ);                                               \
            case 2: return run_clusters_tp_##NTNAME<2>(integ);                                               \
            case 4: return run_clusters_tp_##NTNAME<4>(integ);                                               \
            default: return run_clusters_tp_##NTNAME<8>(integ);                                              \
        }                                                                                                    \
    }                                                                                                        \
    const void *run_bricks_kernel_##NTNAME(int integ) {                                                      \
        return integ == GDB_INTEGRATOR_NVT        ? (const void *)k_run_bricks<NT, GDB_INTEGRATOR_NVT>       \
               : integ == GDB_INTEGRATOR_LANGEVIN ? (const void *)k_run_bricks<NT, GDB_INTEGRATOR_LANGEVIN>  \
                                                  : (const void *)k_run_bricks<NT, GDB_INTEGRATOR_NVE>;      \
    }                                                                                                        \
    const void *step_bricks_kernel_##NTNAME(int integ, int mode) {                                           \
        if (mode == MODE_EVAL) return (const void *)k_step_bricks<NT, 0, MODE_EVAL>;                          \
        return integ == GDB_INTEGRATOR_NVT ? (const void *)k_step_bricks<NT, GDB_INTEGRATOR_NVT, MODE_STEP>  \
               : integ == GDB_INTEGRATOR_LANGEVIN                                                            \
                   ? (const void *)k_step_bricks<NT, GDB_INTEGRATOR_LANGEVIN, MODE_STEP>                     \
                   : (const void *)k_step_bricks<NT, GDB_INTEGRATOR_NVE, MODE_STEP>;                         \
    }

}  // namespace gdb
