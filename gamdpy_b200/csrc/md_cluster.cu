// md_cluster.cu -- small systems (N <= 4096) resident in one thread-block
// cluster, and many of them at once (batched replicas).
//
// One cluster of C CTAs (512 threads each, one per SM) owns one system for a
// whole timeblock:
//   * every CTA holds all N positions in shared memory; after each step a CTA
//     sends the new positions of its own particles to every CTA of the
//     cluster through distributed shared memory (st.shared::cluster);
//   * each CTA owns P = ceil(N / C) particles; their neighbour lists (uint16
//     indices, chunks of four) live in its shared memory; velocities, images
//     and the build reference positions stay in registers across steps;
//   * steps are separated by hardware cluster barriers -- one per step when
//     two position copies fit (new positions go straight into every CTA's
//     other copy), two otherwise; the per-CTA float64 partial sums (only
//     those a step needs) are read by every CTA from the others' shared
//     memory in a fixed order, so every CTA computes the same thermostat
//     update, flags and sums without another round trip.
// Global memory is read at the start of a timeblock and written at its end
// (plus ScalarSaver rows and ConfigurationSaver frames).  Lists are built in
// shared memory over the cell grid of the global cell build (counting sort of
// all N per CTA, 5x5x5 stencil) with the reference's exact distance, so the
// sets equal the global builds' sets.
// A list longer than the shared-memory capacity aborts the whole cluster
// before anything is written back; the host then reruns the timeblock on the
// global-memory path.
#include <algorithm>
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include "md_cluster.cuh"

namespace cg = cooperative_groups;

namespace gdb {

__device__ __forceinline__ int cl_nbl_index(int p, int k, int P) { return (k >> 2) * (P * 4) + p * 4 + (k & 3); }

template <int TP, int NT, int INTEG>
__global__ void __launch_bounds__(CL_THREADS, 1) k_cluster_run(const ClusterJob *__restrict__ jobs, int nsteps,
                                                             int do_eval) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ PairEntry s_tab[GDB_MAX_TYPES * GDB_MAX_TYPES];
    __shared__ double s_red[NQ * 32];
    __shared__ int s_flag[4];
    __shared__ double s_lmax;
    __shared__ double s_gather[16][CL_NQ];
    __shared__ int s_seg_lo[CL_THREADS / 32][64];
    __shared__ int s_seg_pre[CL_THREADS / 32][64];
    cg::cluster_group cl = cg::this_cluster();
    const int C = (int)cl.num_blocks();
    const int rank = (int)cl.block_rank();
    const ClusterJob &job = jobs[blockIdx.x / C];
    const SimArgs &a = job.a;
    DevCtrl *ctrl = a.ctrl;
    const int n = a.n;
    const int P = (n + C - 1) / C;
    const int ncx = a.ncx, ncy = a.ncy, ncz = a.ncz;
    const int ncell = ncx * ncy * ncz;
    const bool use_cells = n > CL_NSQ_MAX && ncell > 0 && ncell <= CL_MAX_CELLS;
    const int cap = job.cap;
    const bool pp = job.pingpong != 0;
    const bool sorted = use_cells && job.sorted != 0;
    const ClusterSmem L = cluster_smem_layout(n, P, use_cells ? ncell : 0, cap, job.pingpong, job.sorted);
    int *scs = reinterpret_cast<int *>(smem + L.cstart);
    unsigned short *scell = reinterpret_cast<unsigned short *>(smem + L.cell);
    unsigned short *srank = reinterpret_cast<unsigned short *>(smem + L.crank);
    unsigned short *sperm = reinterpret_cast<unsigned short *>(smem + L.cperm);
    float4 *const sposA = reinterpret_cast<float4 *>(smem + L.pos);
    float4 *const sposB = pp ? reinterpret_cast<float4 *>(smem + L.pos2) : sposA;
    float4 *spos = sposA;  // the current positions
    float4 *snew = reinterpret_cast<float4 *>(smem + L.newp);
    float4 *ssort = reinterpret_cast<float4 *>(smem + L.sorted);
    unsigned short *snbl = reinterpret_cast<unsigned short *>(smem + L.nbl);
    int *snbc = reinterpret_cast<int *>(smem + L.nbc);
    double *spart = reinterpret_cast<double *>(smem + L.part);
    double *stot = reinterpret_cast<double *>(smem + L.tot);
    const int tid = threadIdx.x, lane = tid & 31;
    const int p0 = rank * P;
    const int np = max(0, min(P, n - p0));
    const int lp = tid / TP, sub = tid % TP;
    const int i = p0 + lp;
    const bool active = lp < np;
    const bool owner = active && sub == 0;
    const int nt = job.tab.nt;

    for (int t = tid; t < nt * nt; t += CL_THREADS) s_tab[t] = job.tab.e[t];
    const float4 *gpos = cur_pos(a, job.cur);
    for (int k = tid; k < n; k += CL_THREADS) spos[k] = gpos[k];
    float4 v = make_float4(0.f, 0.f, 0.f, 1.f), rr = v;
    int4 im = make_int4(0, 0, 0, 0);
    if (owner) {
        v = a.vel[i];
        im = a.img[i];
        rr = a.rref[i];
    }
    float kin_last = 0.f, fsq_last = 0.f;
    float xi = ctrl->xi;
    bool rebuild = *(volatile int *)&ctrl->rebuild != 0;
    // momentum shift left pending by a previous timeblock (standalone path)
    const int ppar0 = (job.step0 & 1) ^ 1;
    if (owner && ctrl->pending[ppar0]) {
        v.x -= ctrl->shift[ppar0][0];
        v.y -= ctrl->shift[ppar0][1];
        v.z -= ctrl->shift[ppar0][2];
    }
    int maxcount = 0, nbuild = 0;
    const float Lx = a.Lx, Ly = a.Ly, Lz = a.Lz;
    const float ilx = 1.0f / Lx, ily = 1.0f / Ly, ilz = 1.0f / Lz;
    // cluster-wide maximum of a per-thread value (called by every thread)
    auto cluster_max = [&](int val) -> int {
        val = __reduce_max_sync(0xffffffffu, val);
        if (tid == 0) s_flag[0] = 0;
        __syncthreads();
        if (lane == 0) atomicMax(&s_flag[0], val);
        __syncthreads();
        if (tid == 0) s_lmax = (double)s_flag[0];
        cl.sync();
        if (tid < C) s_gather[tid][0] = *cl.map_shared_rank(&s_lmax, tid);
        __syncthreads();
        if (tid == 0) {
            int m = 0;
            for (int r = 0; r < C; r++) m = max(m, (int)s_gather[r][0]);
            s_flag[1] = m;
        }
        __syncthreads();
        const int m = s_flag[1];
        cl.sync();
        return m;
    };
    cl.sync();
    trace_mark(ctrl, TR_START);
    // Shared memory holds the lists only while this launch runs.  Without a
    // rebuild due, the current lists come from global memory, where the last
    // build (on either path) left them.
    if (!rebuild) {
        int lmax = 0;
        for (int q = tid >> 5; q < np; q += CL_THREADS / 32) {
            int cnt = a.nbc[p0 + q];
            const int lim = min(min(cnt, cap), a.max_nbs);
            bool bad = false;
            for (int k = lane; k < lim; k += 32) {
                const int j = a.nbl[nbl_index(p0 + q, k, a.stride)];
                bad |= (unsigned)j >= (unsigned)n;
                snbl[cl_nbl_index(q, k, P)] = (unsigned short)j;
            }
            if (__any_sync(0xffffffffu, bad)) {  // not a list of this system: no pairs, error status
                cnt = 0;
                if (lane == 0) atomicOr(&ctrl->status, GDB_STATUS_BAD_INDEX);
            }
            if (lane == 0) snbc[q] = cnt;
            lmax = max(lmax, cnt);
        }
        const int mx = cluster_max(lmax);
        if (mx > cap && mx < a.max_nbs) {
            if (rank == 0 && tid == 0) atomicOr(&ctrl->status, GDB_STATUS_CLUSTER_CAPACITY);
            return;  // uniform across the cluster: nothing was written back
        }
    }

    for (int s = 0; s < nsteps + do_eval; s++) {
        const int step = job.step0 + s;
        const bool eval = s == nsteps;
        // ---- neighbour list from shared memory -----------------------------
        // Every CTA bins all N particles into the cell grid of the global
        // build (nblist_linked_lists.py:36-39, :127), orders each cell by
        // index, copies the positions into cell order and builds the lists of
        // its own particles over the 5x5x5 stencil (a warp per particle,
        // candidates in stencil-row order as the global builds).  Grids with
        // more than CL_MAX_CELLS cells build N^2.
        if (rebuild) {
            int lmax = 0;
            if (use_cells) {
                for (int c = tid; c <= ncell; c += CL_THREADS) scs[c] = 0;
                __syncthreads();
                for (int k = tid; k < n; k += CL_THREADS) {
                    const float4 p = spos[k];
                    const int c = (cell_coord(p.z, Lz, ncz, ctrl) * ncy + cell_coord(p.y, Ly, ncy, ctrl)) * ncx +
                                  cell_coord(p.x, Lx, ncx, ctrl);
                    scell[k] = (unsigned short)c;
                    srank[k] = (unsigned short)atomicAdd(&scs[c], 1);
                }
                __syncthreads();
                // exclusive scan of the counts (one warp, 32-wide chunks)
                if (tid < 32) {
                    int carry = 0;
                    for (int base = 0; base <= ncell; base += 32) {
                        const int c = base + lane;
                        const int x = c <= ncell ? scs[c] : 0;
                        int incl = x;
#pragma unroll
                        for (int o = 1; o < 32; o <<= 1) {
                            const int y = __shfl_up_sync(0xffffffffu, incl, o);
                            if (lane >= o) incl += y;
                        }
                        if (c <= ncell) scs[c] = carry + incl - x;
                        carry += __shfl_sync(0xffffffffu, incl, 31);
                    }
                }
                __syncthreads();
                for (int k = tid; k < n; k += CL_THREADS) sperm[scs[scell[k]] + srank[k]] = (unsigned short)k;
                __syncthreads();
                for (int c = tid; c < ncell; c += CL_THREADS) {  // ascending index inside each cell
                    const int lo = scs[c], hi = scs[c + 1];
                    for (int x = lo + 1; x < hi; x++) {
                        const unsigned short vv = sperm[x];
                        int y = x - 1;
                        while (y >= lo && sperm[y] > vv) {
                            sperm[y + 1] = sperm[y];
                            y--;
                        }
                        sperm[y + 1] = vv;
                    }
                }
                __syncthreads();
                trace_mark(ctrl, TR_REBUILD_PHASE);
                // positions in cell order: the candidates of a stencil row
                // are one contiguous run, read conflict-free by a warp
                if (sorted) {
                    for (int x = tid; x < n; x += CL_THREADS) ssort[x] = spos[sperm[x]];
                    __syncthreads();
                }
                // per particle (a warp each): the x-contiguous ranges of the 25
                // stencil rows (two at the x wrap; whole rows for grids under 5
                // cells), walked as one packed candidate sequence, 32 at a time,
                // ballot-appended in order
                const int ry = ncy < 5 ? ncy : 5, rz = ncz < 5 ? ncz : 5;
                const int nrows = ry * rz, nseg = 2 * nrows;
                const float cps2 = a.cps2;
                const bool fma = a.fma != 0;
                int *lo_s = s_seg_lo[tid >> 5], *pre_s = s_seg_pre[tid >> 5];
                for (int q = tid >> 5; q < np; q += CL_THREADS / 32) {
                    const int ii = p0 + q;
                    const float4 pi = spos[ii];
                    const int c = scell[ii];
                    const int cx = c % ncx, cy = (c / ncx) % ncy, cz = c / (ncx * ncy);
                    int len0 = 0, len1 = 0, lo0 = 0, lo1 = 0;
                    if (lane < nrows) {
                        const int za = lane / ry, yb = lane % ry;
                        const int z = ncz < 5 ? za : ((cz - 2 + za) % ncz + ncz) % ncz;
                        const int y = ncy < 5 ? yb : ((cy - 2 + yb) % ncy + ncy) % ncy;
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
                            } else {
                                l0 = rowbase + x0;
                                h0 = rowbase + ncx;
                                l1 = rowbase;
                                h1 = rowbase + x1 - ncx + 1;
                            }
                        }
                        lo0 = scs[l0];
                        len0 = scs[h0] - lo0;
                        if (h1 > l1) {
                            lo1 = scs[l1];
                            len1 = scs[h1] - lo1;
                        }
                    }
                    const int tot = len0 + len1;
                    int incl = tot;
#pragma unroll
                    for (int o = 1; o < 32; o <<= 1) {
                        const int y = __shfl_up_sync(0xffffffffu, incl, o);
                        if (lane >= o) incl += y;
                    }
                    if (lane < nrows) {
                        lo_s[2 * lane] = lo0;
                        pre_s[2 * lane] = incl - tot;
                        lo_s[2 * lane + 1] = lo1;
                        pre_s[2 * lane + 1] = incl - tot + len0;
                    }
                    const int T = __shfl_sync(0xffffffffu, incl, 31);
                    __syncwarp();
                    int count = 0, seg = 0;
                    for (int v0 = 0; v0 < T; v0 += 32) {
                        const int vv = v0 + lane;
                        bool hit = false;
                        int j = 0;
                        if (vv < T) {
                            while (seg + 1 < nseg && pre_s[seg + 1] <= vv) seg++;
                            const int x = lo_s[seg] + (vv - pre_s[seg]);
                            j = sperm[x];
                            const float4 pj = sorted ? ssort[x] : spos[j];
                            if (j != ii) {
                                const float d2 = fma ? dist_sq_exact<true>(pj, pi, Lx, Ly, Lz)
                                                     : dist_sq_exact<false>(pj, pi, Lx, Ly, Lz);
                                hit = d2 < cps2;
                            }
                        }
                        const unsigned m = __ballot_sync(0xffffffffu, hit);
                        if (hit) {
                            const int k = count + __popc(m & ((1u << lane) - 1u));
                            if (k < cap && k < a.max_nbs) snbl[cl_nbl_index(q, k, P)] = (unsigned short)j;
                        }
                        count += __popc(m);
                    }
                    __syncwarp();
                    if (lane == 0) snbc[q] = count;
                    lmax = max(lmax, count);
                }
            } else {
                for (int q = tid >> 5; q < np; q += CL_THREADS / 32) {
                    const int ii = p0 + q;
                    const float4 pi = spos[ii];
                    int count = 0;
                    for (int j0 = 0; j0 < n; j0 += 32) {
                        const int j = j0 + lane;
                        bool hit = false;
                        if (j < n && j != ii) {
                            const float d2 = a.fma ? dist_sq_exact<true>(spos[j], pi, Lx, Ly, Lz)
                                                   : dist_sq_exact<false>(spos[j], pi, Lx, Ly, Lz);
                            hit = d2 < a.cps2;
                        }
                        const unsigned m = __ballot_sync(0xffffffffu, hit);
                        if (hit) {
                            const int k = count + __popc(m & ((1u << lane) - 1u));
                            if (k < cap && k < a.max_nbs) snbl[cl_nbl_index(q, k, P)] = (unsigned short)j;
                        }
                        count += __popc(m);
                    }
                    if (lane == 0) snbc[q] = count;
                    lmax = max(lmax, count);
                }
            }
            if (owner) rr = spos[i];
            trace_mark(ctrl, TR_REBUILD_PHASE);
            // cluster-wide longest list; beyond the shared capacity: abort
            const int mx = cluster_max(lmax);
            trace_mark(ctrl, TR_REBUILD_DONE);
            maxcount = max(maxcount, mx);
            nbuild++;
            rebuild = false;
            if (mx > cap && mx < a.max_nbs) {
                if (rank == 0 && tid == 0) atomicOr(&ctrl->status, GDB_STATUS_CLUSTER_CAPACITY);
                return;  // uniform across the cluster: nothing was written back
            }
        }
        // ---- ConfigurationSaver (prestep) ------------------------------------
        if (owner && a.conf) {
            const int si = conf_save_index(step);
            if (si >= 0 && si < a.conf_per_block) {
                const size_t N3 = (size_t)n * 3;
                const size_t u = (size_t)a.orig[i];
                const float4 pi = spos[i];
                float *fr = a.conf + (size_t)si * 2 * N3;
                fr[3 * u] = pi.x;
                fr[3 * u + 1] = pi.y;
                fr[3 * u + 2] = pi.z;
                fr[N3 + 3 * u] = (float)im.x;
                fr[N3 + 3 * u + 1] = (float)im.y;
                fr[N3 + 3 * u + 2] = (float)im.z;
            }
        }
        // ---- forces from shared memory ----------------------------------------
        const bool rec = eval || (a.every > 0 && step % a.every == 0);
        const bool reset = !eval && a.reset_every > 0 && step % a.reset_every == 0;
        float fx = 0.f, fy = 0.f, fz = 0.f, u = 0.f, w = 0.f, l = 0.f;
        float4 pi = make_float4(0.f, 0.f, 0.f, 0.f);
        if (active) {
            pi = spos[i];
            const PairRow<NT> pr(s_tab, nt, NT == 1 ? 0 : ptype_of(pi));
            const int cnt = min(min(snbc[lp], cap), a.max_nbs);
            const int nch = (cnt + 3) >> 2;
            for (int ch = sub; ch < nch; ch += TP) {
                const ushort4 jj = *reinterpret_cast<const ushort4 *>(snbl + cl_nbl_index(lp, ch * 4, P));
                const int k0 = ch * 4;
                const bool v1 = k0 + 1 < cnt, v2 = k0 + 2 < cnt, v3 = k0 + 3 < cnt;
                const float4 q0 = spos[jj.x];
                const float4 q1 = spos[v1 ? jj.y : i];
                const float4 q2 = spos[v2 ? jj.z : i];
                const float4 q3 = spos[v3 ? jj.w : i];
                if (rec) {
                    pair_force<true, NT>(pr, pi, q0, true, Lx, Ly, Lz, ilx, ily, ilz, fx, fy, fz, u, w, l);
                    pair_force<true, NT>(pr, pi, q1, v1, Lx, Ly, Lz, ilx, ily, ilz, fx, fy, fz, u, w, l);
                    pair_force<true, NT>(pr, pi, q2, v2, Lx, Ly, Lz, ilx, ily, ilz, fx, fy, fz, u, w, l);
                    pair_force<true, NT>(pr, pi, q3, v3, Lx, Ly, Lz, ilx, ily, ilz, fx, fy, fz, u, w, l);
                } else {
                    pair_force<false, NT>(pr, pi, q0, true, Lx, Ly, Lz, ilx, ily, ilz, fx, fy, fz, u, w, l);
                    pair_force<false, NT>(pr, pi, q1, v1, Lx, Ly, Lz, ilx, ily, ilz, fx, fy, fz, u, w, l);
                    pair_force<false, NT>(pr, pi, q2, v2, Lx, Ly, Lz, ilx, ily, ilz, fx, fy, fz, u, w, l);
                    pair_force<false, NT>(pr, pi, q3, v3, Lx, Ly, Lz, ilx, ily, ilz, fx, fy, fz, u, w, l);
                }
            }
        }
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
        // ---- integrate own particles (registers) ------------------------------
        double red[NQ];
#pragma unroll
        for (int q = 0; q < NQ; q++) red[q] = 0.0;
        bool moved = false;
        float4 *const sother = (spos == sposA) ? sposB : sposA;  // next positions (ping-pong)
        if (owner) {
            const float fsq = fx * fx + fy * fy + fz * fz;
            const size_t N = n;
            if (rec) {
                a.pscal[i] = u;
                a.pscal[N + i] = w;
                a.pscal[2 * N + i] = l;
            }
            red[1] = u;
            red[2] = w;
            red[3] = l;
            red[4] = fsq;
            if (eval) {
                a.frc[i] = make_float4(fx, fy, fz, 0.f);
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
                const float Lk[3] = {Lx, Ly, Lz};
                int dimg[3] = {0, 0, 0};
#pragma unroll
                for (int k = 0; k < 3; k++) {  // orthorhombic.py:75-86
                    if (r[k] * 2.0f > Lk[k]) {
                        r[k] -= Lk[k];
                        dimg[k] += 1;
                    }
                    if (r[k] * 2.0f < -Lk[k]) {
                        r[k] += Lk[k];
                        dimg[k] -= 1;
                    }
                }
                im.x += dimg[0];
                im.y += dimg[1];
                im.z += dimg[2];
                if (!(fabsf(r[0]) <= Lk[0] && fabsf(r[1]) <= Lk[1] && fabsf(r[2]) <= Lk[2]))
                    atomicOr(&ctrl->status, GDB_STATUS_NAN);
                const float4 pn = make_float4(r[0], r[1], r[2], pi.w);
                snew[lp] = pn;
                v = make_float4(vv[0], vv[1], vv[2], m);
                kin_last = kin;
                fsq_last = fsq;
                moved = dist_sq_exact<false>(pn, rr, Lx, Ly, Lz) > a.skin2q;
                red[0] = kin;
                if (reset) {
                    red[5] = (double)m * vv[0];
                    red[6] = (double)m * vv[1];
                    red[7] = (double)m * vv[2];
                    red[8] = m;
                }
            }
        }
        // ---- block partials: only the sums this step needs ----------------
        // every sum on saved and reset steps, the kinetic energy of the
        // thermostat (NVT) otherwise, and always the rebuild flag
        const bool full = rec || reset;
        const bool needk = full || INTEG == GDB_INTEGRATOR_NVT;
        double *slot = spart + (pp ? (s & 1) : 0) * CL_NQ;
        const int any_moved = __syncthreads_or(moved);  // also orders snew before the copies below
        if (full) {
            block_sum<NQ>(red, s_red);
        } else if (needk) {
            double rk[1] = {red[0]};
            block_sum<1>(rk, s_red);
            red[0] = rk[0];
        }
        if (tid == 0) {
            if (full) {
#pragma unroll
                for (int q = 0; q < NQ; q++) slot[q] = red[q];
            } else if (needk) {
                slot[0] = red[0];
            }
            slot[NQ] = any_moved ? 1.0 : 0.0;
        }
        // with two position copies, the new positions go straight into every
        // CTA's other copy, read only after the barrier below
        if (pp && !eval) {
            for (int k = tid; k < np * C; k += CL_THREADS) {
                const int r = k / np, q = k - r * np;
                cl.map_shared_rank(sother, r)[p0 + q] = snew[q];
            }
        }
        trace_mark(ctrl, TR_STEP_PHASE);
        cl.sync();  // every force phase done, every partial written (and, ping-pong, every position)
        if (!pp && !eval) {
            for (int k = tid; k < np * C; k += CL_THREADS) {
                const int r = k / np, q = k - r * np;
                cl.map_shared_rank(spos, r)[p0 + q] = snew[q];
            }
        }
        // the needed partials of every CTA, one remote load per thread, then
        // a fixed-order local sum
        const int ng = full ? NQ + 1 : (needk ? 2 : 1);
        if (tid < C * ng) {
            const int r = tid / ng, g = tid - r * ng;
            const int q = full ? g : (g == ng - 1 ? NQ : 0);
            s_gather[r][q] = cl.map_shared_rank(slot, r)[q];
        }
        __syncthreads();
        if (tid < NQ + 1 && (full || tid == NQ || (needk && tid == 0))) {
            double acc = 0.0;
            for (int r = 0; r < C; r++) acc += s_gather[r][tid];
            stot[tid] = acc;
        }
        __syncthreads();
        if (!eval) {
            const double time = ctrl->time_zero + (double)step * (double)a.dt;
            if (INTEG == GDB_INTEGRATOR_NVT) {  // NVT.py:113-124
                const double T = target_temperature(a, time);
                const double dev = 2.0 * stot[0] / ((double)a.dof * T) - 1.0;
                xi = (float)((double)xi + (double)(a.dt * a.omega2) * dev);
            }
            if (rank == 0 && tid == 0 && rec && step / a.every < a.nrows) {  // scalar_saver.py:165-179
                double *row = a.rows + (size_t)(step / a.every) * GDB_NUM_SCALARS;
                row[GDB_SCALAR_U] = stot[1];
                row[GDB_SCALAR_W] = stot[2];
                row[GDB_SCALAR_LAPU] = stot[3];
                row[GDB_SCALAR_K] = stot[0];
                row[GDB_SCALAR_FSQ] = stot[4];
            }
            if (reset && owner) {  // momentum_reset.py:64-78
                v.x -= (float)(stot[5] / stot[8]);
                v.y -= (float)(stot[6] / stot[8]);
                v.z -= (float)(stot[7] / stot[8]);
            }
            rebuild = stot[NQ] > 0.0;
            if (rank == 0 && tid == 0 && needk) ctrl->sumK = (float)stot[0];
        } else if (rank == 0 && tid == 0) {
            ctrl->evalU = stot[1];
            ctrl->evalW = stot[2];
        }
        if (pp) {
            if (!eval) spos = sother;
        } else {
            cl.sync();  // positions delivered; the partial slot is free again
        }
        trace_mark(ctrl, eval ? TR_EVAL : TR_STEP);
    }

    // ---- write the state back ----------------------------------------------
    const int cur_end = job.cur ^ (nsteps & 1);
    float4 *pend = cur_pos(a, cur_end);
    const size_t N = n;
    if (owner) {
        pend[i] = spos[i];
        a.vel[i] = v;
        a.img[i] = im;
        a.rref[i] = rr;
        if (nsteps > 0) {
            a.pscal[3 * N + i] = kin_last;
            a.pscal[4 * N + i] = fsq_last;
        }
    }
    // lists in the global chunked layout (int indices), for gdb_get_nblist
    if (nbuild > 0) {
        for (int q = tid >> 5; q < np; q += CL_THREADS / 32) {
            const int cnt = snbc[q];
            const int lim = min(min(cnt, cap), a.max_nbs);
            for (int k = lane; k < lim; k += 32) a.nbl[nbl_index(p0 + q, k, a.stride)] = snbl[cl_nbl_index(q, k, P)];
            if (lane == 0) a.nbc[p0 + q] = cnt;
        }
    }
    if (rank == 0 && tid == 0) {
        ctrl->xi = xi;
        ctrl->step = job.step0 + nsteps;
        ctrl->rebuild = rebuild ? 1 : 0;
        ctrl->rebuild_next = 0;
        ctrl->pending[0] = ctrl->pending[1] = 0;
        ctrl->nrebuild += nbuild;
        atomicMax(&ctrl->maxcount, maxcount);
    }
}

// ---------------------------------------------------------------------------
// host side: instantiation table and launch
// ---------------------------------------------------------------------------
template <int TP, int NT>
static const void *cluster_kernel_tp(int integ) {
    return integ == GDB_INTEGRATOR_NVT ? (const void *)k_cluster_run<TP, NT, GDB_INTEGRATOR_NVT>
                                       : (const void *)k_cluster_run<TP, NT, GDB_INTEGRATOR_NVE>;
}

template <int NT>
static const void *cluster_kernel_nt(int tp, int integ) {
    switch (tp) {
        case 2: return cluster_kernel_tp<2, NT>(integ);
        case 4: return cluster_kernel_tp<4, NT>(integ);
        case 8: return cluster_kernel_tp<8, NT>(integ);
        case 16: return cluster_kernel_tp<16, NT>(integ);
        default: return cluster_kernel_tp<32, NT>(integ);
    }
}

const void *cluster_kernel(int tp, int ntypes, int integ) {
    return ntypes == 1 ? cluster_kernel_nt<1>(tp, integ)
                       : (ntypes == 2 ? cluster_kernel_nt<2>(tp, integ) : cluster_kernel_nt<0>(tp, integ));
}

// Cluster size and lanes per particle for a system of n particles: about
// `target` particles per CTA (at most CL_THREADS / 2), at most 16 CTAs.
void cluster_shape(int n, int target, int *C, int *tp) {
    // default: spread the system over 16 CTAs, at least 32 particles each
    // (measured on B200, one KA system of 512: 6.7 us per step at 32
    // particles per CTA, 12.1 us at 128); batches of many systems run faster
    // with more particles per CTA (SimulationBatch.autotune)
    if (target <= 0) target = std::max(32, (n + 15) / 16);
    // every particle needs at least two lanes of the CTA (the kernel is
    // instantiated for 2..32 lanes per particle)
    target = std::min(target, CL_THREADS / 2);
    int c = 1;
    while (c < 16 && (n + c - 1) / c > target) c *= 2;
    const int P = (n + c - 1) / c;
    int t = 1;
    while (t < 32 && P * t * 2 <= CL_THREADS) t *= 2;
    if (t < 2) t = 2;
    *C = c;
    *tp = t;
}

bool cluster_plan(int n, int C, int ncell, int max_nbs, int *cap, int *pingpong, int *sorted, size_t *smem) {
    const int P = (n + C - 1) / C;
    if (2 * P > CL_THREADS) return false;  // not every particle would have its lanes
    const int nc = n > CL_NSQ_MAX && ncell > 0 && ncell <= CL_MAX_CELLS ? ncell : 0;
    const int want = std::min((std::max(max_nbs, 4) + 3) & ~3, CL_CAP_MAX);
    const int opts[3][2] = {{1, 1}, {0, 1}, {0, 0}};  // (pingpong, sorted), best first
    for (int o = 0; o < 3; o++) {
        const int pp = opts[o][0], so = opts[o][1];
        const int floor_cap = o < 2 ? std::min(want, 160) : 64;
        for (int c = want; c >= floor_cap; c -= 4) {
            const size_t bytes = cluster_smem_layout(n, P, nc, c, pp, so).total;
            if (bytes <= CL_SMEM_LIMIT) {
                *cap = c;
                *pingpong = pp;
                *sorted = so;
                *smem = bytes;
                return true;
            }
        }
    }
    return false;
}

// Launch `count` systems (one cluster each, all of cluster size C and lanes
// tp, `smem` >= the largest system's layout) for `nsteps` steps plus the
// final evaluation.
cudaError_t launch_clusters(const ClusterJob *d_jobs, int count, int C, int tp, int ntypes, int integ, size_t smem,
                            int nsteps, int do_eval, cudaStream_t st) {
    const void *fn = cluster_kernel(tp, ntypes, integ);
    if (smem > CL_SMEM_LIMIT) return cudaErrorInvalidValue;
    // one value for every launch of the function: launches of one kernel with
    // different shared-memory sizes may be in flight on several streams, and
    // the function attribute is shared by all of them
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)CL_SMEM_LIMIT);
    if (e != cudaSuccess) return e;
    if (C > 8) {
        e = cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        if (e != cudaSuccess) return e;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(count * C);
    cfg.blockDim = dim3(CL_THREADS);
    cfg.dynamicSmemBytes = smem;
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

}  // namespace gdb
