// md_cluster.cuh -- job descriptor and shared-memory layout of the
// thread-block-cluster path (md_cluster.cu), shared with the host code.
#pragma once

#include "md_phases.cuh"

namespace gdb {

constexpr int CL_THREADS = 512;  // 128 registers a thread: the step keeps its state in registers
constexpr int CL_MAX_N = 4096;
constexpr int CL_CAP_MAX = 1024;    // neighbour slots per particle: upper bound
constexpr int CL_MAX_CELLS = 8192;  // shared cell table; sparser grids build N^2
constexpr int CL_NSQ_MAX = 768;     // up to this size the list build is N^2 (measured: 2x faster at 512, 1.5x slower at 2048)
constexpr int CL_NQ = 11;           // NQ sums + moved flag + max list length
constexpr size_t CL_SMEM_LIMIT = 208 * 1024;  // dynamic; the kernel's static arrays take under 16 KB

struct ClusterJob {
    SimArgs a;
    PairTable tab;
    int cur;       // position buffer holding the current state
    int step0;     // ctrl->step at the start (0 at a timeblock start)
    int cap;       // neighbour slots per particle in shared memory (multiple of 4)
    int pingpong;  // two position copies per CTA: one cluster barrier per step
    int sorted;    // a cell-ordered position copy for the list build
};

struct ClusterSmem {
    size_t pos, pos2, sorted, nbl, nbc, newp, part, tot, cstart, cell, crank, cperm, total;
};

__host__ __device__ inline ClusterSmem cluster_smem_layout(int n, int P, int ncell, int cap, int pingpong,
                                                           int sorted) {
    ClusterSmem s;
    size_t o = 0;
    s.pos = o;
    o += (size_t)n * sizeof(float4);
    s.pos2 = o;
    if (pingpong) o += (size_t)n * sizeof(float4);
    s.sorted = o;  // positions in cell order during a build (cell grids only)
    if (ncell > 0 && sorted) o += (size_t)n * sizeof(float4);
    s.newp = o;
    o += (size_t)P * sizeof(float4);
    s.nbl = o;
    o += (size_t)((cap + 3) / 4) * 4 * P * sizeof(unsigned short);
    o = (o + 15) & ~(size_t)15;
    s.nbc = o;
    o += (size_t)P * sizeof(int);
    o = (o + 15) & ~(size_t)15;
    s.part = o;  // two slots (by step parity when pingpong)
    o += 2 * CL_NQ * sizeof(double);
    s.tot = o;
    o += CL_NQ * sizeof(double);
    s.cstart = o;  // cell counts, then exclusive starts (ncell + 1)
    o += (size_t)(ncell + 1) * sizeof(int);
    o = (o + 15) & ~(size_t)15;
    s.cell = o;  // cell of every particle
    o += (size_t)n * sizeof(unsigned short);
    s.crank = o;  // rank of every particle inside its cell
    o += (size_t)n * sizeof(unsigned short);
    s.cperm = o;  // particles sorted by cell
    o += (size_t)n * sizeof(unsigned short);
    o = (o + 15) & ~(size_t)15;
    s.total = o;
    return s;
}

// Host side (md_cluster.cu).
const void *cluster_kernel(int tp, int ntypes, int integ);
// Cluster size C and lanes per particle for n particles, about `target`
// particles per CTA (0: spread over 16 CTAs, at least 32 each; at most 256),
// C <= 16.
void cluster_shape(int n, int target, int *C, int *tp);
// Neighbour slots per particle, position double-buffering, the sorted copy and
// dynamic shared memory for a system of n particles on C CTAs over ncell
// cells with lists of at most max_nbs: the largest capacity up to max_nbs
// that fits the shared-memory budget, with the optional copies as long as
// 160 slots (or max_nbs) remain.  Returns false when not even 64 slots fit.
bool cluster_plan(int n, int C, int ncell, int max_nbs, int *cap, int *pingpong, int *sorted, size_t *smem);
cudaError_t launch_clusters(const ClusterJob *d_jobs, int count, int C, int tp, int ntypes, int integ, size_t smem,
                            int nsteps, int do_eval, cudaStream_t st);

}  // namespace gdb
