// adjoint.cu -- gradients of trajectory-averaged observables of an NVE
// leapfrog trajectory with respect to the Lennard-Jones pair parameters
// (sigma_ab, epsilon_ab), by a hand-written discrete adjoint.
//
// Forward (float32 state, float64 reductions), as integrators/NVE.py:78-97
// with the shifted-force LJ of LJ_12_6_sigma_epsilon.py:26-36 and
// apply_shifted_force_cutoff.py:30-37 (s -= s(rc), u += s(rc) rc (r - rc) - u(rc)):
//   f_n     = F(r_n)                       pair sum over all j (N^2, on the fly)
//   v_{n+1} = v_n + f_n dt / m
//   r_{n+1} = r_n + v_{n+1} dt             (periodic wrap; derivative identity)
//   U_n, W_n from r_n; K_n = sum m ((v_n + v_{n+1}) / 2)^2 / 2
//   g_b     = soft (Gaussian-kernel) A-A radial distribution on sampled steps
// Observables: time averages <U>, <W>, <K> over n = 0..T-1 and <g_b>.
//
// Backward: reverse sweep over the steps with the cotangents (R, V) of
// (r_{n+1}, v_{n+1}):
//   Vt   = V + dt R + gK dK_n/dv_{n+1}
//   R   <- R + (dt / m) J(r_n)^T Vt + gU dU_n/dr + gW dW_n/dr + sum_b gG_b dg_b/dr
//   V   <- Vt + gK dK_n/dv_n
//   dL/dtheta += (dt / m) (df/dtheta)^T Vt + gU dU_n/dtheta + gW dW_n/dtheta
// J^T Vt is the Hessian-vector product of the pair potential: for each pair
// (s I + s'/r d d^T)(Vt_i - Vt_j).  The sweep runs segment by segment: the
// forward keeps checkpoints of (r, v) every `checkpoint_every` steps and the
// backward recomputes each segment's states from its checkpoint with the
// same kernels (bit-identical) before sweeping it in reverse, in float64.
//
// Pairs come from a neighbour list (all j within the largest cut or the RDF
// kernel's reach plus a skin of 0.5, built N^2, rebuilt when a particle moves
// more than half the skin); 32 lanes per particle, lane L taking its column
// of the list, the neighbours j = L (mod 32) in ascending order.  Every per-lane sum
// is then the same as a loop over all j (the NbList2 pair set), whatever the
// list holds beyond the cutoff: results do not depend on when the list was
// built, so recomputed segments are bit-identical to the forward.  Every sum
// has a fixed order, so runs are reproducible.  Sized for the small systems
// this is meant for (N of a few thousand; the build is N^2).
#include <cuda_runtime.h>
#include <math.h>
#include <stdarg.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "../../include/gamdb200.h"
#include "gdb_internal.cuh"

namespace {

constexpr int ADJ_MAXT = 4;     // particle types
constexpr int ADJ_MAXB = 128;   // RDF bins
constexpr int ADJ_LANES = 32;   // lanes per particle
constexpr int ADJ_BLOCK = 256;  // 8 particles per block
constexpr int ADJ_PPB = ADJ_BLOCK / ADJ_LANES;
constexpr int ADJ_NTH = 2 * ADJ_MAXT * ADJ_MAXT;  // d/dsigma, d/depsilon per ordered type pair
constexpr double ADJ_FIX = 4294967296.0;          // fixed-point scale of the RDF kernel sums
constexpr double ADJ_KW = 8.0;                    // kernel support in widths (exp(-32): smooth to 1e-14)

// float32 pair entry, the same arithmetic as the plain kernels' PairEntry
struct Tab32 {
    float c, cu12, cu6, cs12, cs6, uc, sc, sccut, cut, cut2;
};
// float64 parameters and cutoff values for the backward sweep
struct Tab64 {
    double sig, eps, cut, cut2;
    double s_c;    // s0(rc)
    double dsds_c; // d s0 / d sigma at rc
    double u_c;    // u0(rc)
    double duds_c; // d u0 / d sigma at rc
};

struct Tables {
    int nt;
    Tab32 t32[ADJ_MAXT * ADJ_MAXT];
    Tab64 t64[ADJ_MAXT * ADJ_MAXT];
};

struct AdjArgs {
    int n, nt;
    float Lx, Ly, Lz;
    float dt;
    const int *type;
    const float *mass;
    int nbins;
    float r_lo, dr, width;  // bin centres r_lo + (b + 1/2) dr
    // neighbour list: all j within rl of i at the build; particle i's maxnb
    // entries at nbl + i * maxnb as 32 columns (entry c of column L at
    // c * 32 + L, the neighbours j = L (mod 32) ascending); nbc holds the 32
    // column counts of each particle; rebuilt when a particle moves more than
    // skin/2
    const int *nbl, *nbc;
    int maxnb;
    float rl2;      // (max cut or RDF reach + skin)^2
    float move2;    // (skin / 2 - margin)^2
    float4 *rref;   // positions at the last build
    int *flags;     // rebuild flags, by step parity
    unsigned *status;
};

constexpr float ADJ_SKIN = 0.5f;
constexpr unsigned ADJ_STATUS_OVERFLOW = 1u;

__device__ __forceinline__ float mic_rint(float d, float L, float iL) { return d - L * rintf(d * iL); }

template <typename T>
__device__ __forceinline__ T wsum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Forward step: forces at pos_in, integration into pos_out/vel_out, per-block
// float64 partial sums of U, W, K; on sampled steps the A-A kernel sums into
// gbins (fixed point, integer atomics: order-independent).
__global__ void __launch_bounds__(ADJ_BLOCK) k_adj_step(AdjArgs a, Tables tab, const float4 *__restrict__ pos_in,
                                                        const float4 *__restrict__ vel_in, float4 *pos_out,
                                                        float4 *vel_out, double *partials, unsigned long long *gbins,
                                                        int *flag_out) {
    __shared__ Tab32 s_tab[ADJ_MAXT * ADJ_MAXT];
    __shared__ double s_red[ADJ_PPB][3];
    __shared__ unsigned long long s_bins[ADJ_MAXB];
    const int nt = tab.nt;
    for (int t = threadIdx.x; t < nt * nt; t += blockDim.x) s_tab[t] = tab.t32[t];
    const bool rdf = gbins != nullptr;
    if (rdf)
        for (int b = threadIdx.x; b < a.nbins; b += blockDim.x) s_bins[b] = 0ull;
    __syncthreads();
    const int lane = threadIdx.x & 31, q = threadIdx.x >> 5;
    const int i = blockIdx.x * ADJ_PPB + q;
    const float iLx = 1.0f / a.Lx, iLy = 1.0f / a.Ly, iLz = 1.0f / a.Lz;
    float fx = 0.f, fy = 0.f, fz = 0.f, u = 0.f, w = 0.f;
    float4 pi = make_float4(0.f, 0.f, 0.f, 0.f);
    int ti = 0;
    if (i < a.n) {
        pi = pos_in[i];
        ti = a.type[i];
        const Tab32 *row = s_tab + ti * nt;
        const double rg_lo = (double)a.r_lo - ADJ_KW * a.width, rg_hi = (double)a.r_lo + a.nbins * (double)a.dr + ADJ_KW * a.width;
        // lane L takes its own column of the list: the neighbours j = L
        // (mod 32) in ascending order, the same per-lane sums as a loop over
        // all j whatever the list holds beyond the cutoff, so results do not
        // depend on when it was built
        const int *lst = a.nbl + (size_t)i * a.maxnb + lane;
        const int cnt = min(a.nbc[(size_t)i * ADJ_LANES + lane], a.maxnb / ADJ_LANES);
        for (int c = 0; c < cnt; c++) {
            const int j = lst[c * ADJ_LANES];
            const float4 pj = pos_in[j];
            const float dx = mic_rint(pj.x - pi.x, a.Lx, iLx);
            const float dy = mic_rint(pj.y - pi.y, a.Ly, iLy);
            const float dz = mic_rint(pj.z - pi.z, a.Lz, iLz);
            const float d2 = dx * dx + dy * dy + dz * dz;
            const int tj = a.type[j];
            const Tab32 &e = row[tj];
            if (d2 < e.cut2) {
                const float inv2 = 1.0f / d2;
                const float x2 = e.c * inv2;
                const float x6 = x2 * x2 * x2;
                const float x12 = x6 * x6;
                const float s = (e.cs12 * x12 + e.cs6 * x6) * inv2 - e.sc;
                fx -= dx * s;
                fy -= dy * s;
                fz -= dz * s;
                const float r = sqrtf(d2);
                u += 0.5f * (e.cu12 * x12 + e.cu6 * x6 - e.uc + e.sccut * (r - e.cut));
                w += d2 * s * (1.0f / 6.0f);
            }
            if (rdf && ti == 0 && tj == 0) {
                const double r = sqrt((double)d2);
                if (r > rg_lo && r < rg_hi) {
                    const double w2 = 2.0 * (double)a.width * a.width;
                    const double kn = 1.0 / (sqrt(2.0 * M_PI) * (double)a.width);
                    int b0 = (int)floor((r - ADJ_KW * a.width - a.r_lo) / a.dr);
                    int b1 = (int)floor((r + ADJ_KW * a.width - a.r_lo) / a.dr);
                    b0 = max(b0, 0);
                    b1 = min(b1, a.nbins - 1);
                    for (int b = b0; b <= b1; b++) {
                        const double x = r - ((double)a.r_lo + (b + 0.5) * (double)a.dr);
                        const double k = kn * exp(-x * x / w2);
                        atomicAdd(&s_bins[b], (unsigned long long)(k * ADJ_FIX + 0.5));
                    }
                }
            }
        }
    }
    fx = wsum(fx);
    fy = wsum(fy);
    fz = wsum(fz);
    u = wsum(u);
    w = wsum(w);
    double kin = 0.0;
    if (lane == 0 && i < a.n) {
        const float4 v = vel_in[i];
        const float m = a.mass[i];
        float vv[3] = {v.x, v.y, v.z};
        float r[3] = {pi.x, pi.y, pi.z};
        const float ff[3] = {fx, fy, fz};
        const float L[3] = {a.Lx, a.Ly, a.Lz};
        float k = 0.f;
#pragma unroll
        for (int c = 0; c < 3; c++) {  // integrators/NVE.py:78-97
            float vm = vv[c];
            vv[c] += ff[c] / m * a.dt;
            vm += vv[c];
            vm *= 0.5f;
            k += 0.5f * m * vm * vm;
            r[c] += vv[c] * a.dt;
            if (r[c] * 2.0f > L[c]) r[c] -= L[c];
            if (r[c] * 2.0f < -L[c]) r[c] += L[c];
        }
        pos_out[i] = make_float4(r[0], r[1], r[2], pi.w);
        vel_out[i] = make_float4(vv[0], vv[1], vv[2], 0.f);
        kin = k;
        if (flag_out) {
            const float4 q = a.rref[i];
            const float ex = mic_rint(r[0] - q.x, a.Lx, iLx), ey = mic_rint(r[1] - q.y, a.Ly, iLy),
                        ez = mic_rint(r[2] - q.z, a.Lz, iLz);
            if (ex * ex + ey * ey + ez * ez > a.move2) atomicOr(flag_out, 1);
        }
    }
    if (lane == 0) {
        s_red[q][0] = i < a.n ? (double)u : 0.0;
        s_red[q][1] = i < a.n ? (double)w : 0.0;
        s_red[q][2] = kin;
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        double acc = 0.0;
        for (int p = 0; p < ADJ_PPB; p++) acc += s_red[p][threadIdx.x];
        partials[(size_t)blockIdx.x * 3 + threadIdx.x] = acc;
    }
    if (rdf)
        for (int b = threadIdx.x; b < a.nbins; b += blockDim.x)
            if (s_bins[b]) atomicAdd(&gbins[b], s_bins[b]);
}

// Fixed-order sum of the block partials into the running time sums.
__global__ void k_adj_reduce(const double *partials, int nblocks, double *acc) {
    __shared__ double s[3][32];
    double v[3] = {0.0, 0.0, 0.0};
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x)
        for (int q = 0; q < 3; q++) v[q] += partials[(size_t)b * 3 + q];
    for (int q = 0; q < 3; q++) v[q] = wsum(v[q]);
    if ((threadIdx.x & 31) == 0)
        for (int q = 0; q < 3; q++) s[q][threadIdx.x >> 5] = v[q];
    __syncthreads();
    if (threadIdx.x < 3) {
        double t = 0.0;
        for (int k = 0; k < (int)(blockDim.x >> 5); k++) t += s[threadIdx.x][k];
        acc[threadIdx.x] += t;
    }
}

// Vt = V + dt R + gK dK_n/dv_{n+1},  dK_n/dv_{n+1} = m (v_n + v_{n+1}) / 4
__global__ void k_adj_vtot(int n, float dt, double gK, const float *mass, const double *R, const double *V,
                           const float4 *vn, const float4 *vn1, double *Vt) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double m = mass[i];
    const float4 a = vn[i], b = vn1[i];
    const double va[3] = {a.x, a.y, a.z}, vb[3] = {b.x, b.y, b.z};
    for (int c = 0; c < 3; c++) Vt[3 * i + c] = V[3 * i + c] + (double)dt * R[3 * i + c] + gK * m * (va[c] + vb[c]) * 0.25;
}

// Pair derivatives of one ordered type pair at distance r (float64).
struct PairD {
    double s, ds_dr_over_r;  // s_SF, s0'(r)/r
    double dsde, dsds;       // d s_SF / d eps, d s_SF / d sigma
    double dude, duds;       // d u_SF / d eps, d u_SF / d sigma
    double dudr_over_r;      // u_SF'(r)/r
};

__device__ __forceinline__ PairD pair_derivs(const Tab64 &e, double r2) {
    PairD p;
    const double r = sqrt(r2);
    const double ir2 = 1.0 / r2;
    const double sr2 = e.sig * e.sig * ir2;
    const double sr6 = sr2 * sr2 * sr2, sr12 = sr6 * sr6;
    const double s0 = e.eps * (48.0 * sr12 - 24.0 * sr6) * ir2;
    p.s = s0 - e.s_c;
    p.ds_dr_over_r = e.eps * (-672.0 * sr12 + 192.0 * sr6) * ir2 * ir2;
    p.dsde = p.s / e.eps;
    const double ds0ds = e.eps * (576.0 * sr12 - 144.0 * sr6) * ir2 / e.sig;
    p.dsds = ds0ds - e.dsds_c;
    const double u0 = 4.0 * e.eps * (sr12 - sr6);
    const double uSF = u0 - e.u_c + e.s_c * e.cut * (r - e.cut);
    p.dude = uSF / e.eps;
    const double du0ds = 4.0 * e.eps * (12.0 * sr12 - 6.0 * sr6) / e.sig;
    p.duds = du0ds - e.duds_c + e.dsds_c * e.cut * (r - e.cut);
    p.dudr_over_r = -s0 + e.s_c * e.cut / r;
    return p;
}

// Backward step at r_n: R += (dt/m) HVP(Vt) + gU dU/dr + gW dW/dr + dG/dr,
// V = Vt + gK dK_n/dv_n, per-block parameter cotangents accumulated.
__global__ void __launch_bounds__(ADJ_BLOCK) k_adj_back(AdjArgs a, Tables tab, const float4 *__restrict__ pos,
                                                        const double *__restrict__ Vt, double *R, double *V,
                                                        const float4 *vn, const float4 *vn1, double gU, double gW,
                                                        double gK, const double *gG, double *th_part) {
    __shared__ Tab64 s_tab[ADJ_MAXT * ADJ_MAXT];
    __shared__ double s_th[ADJ_PPB][ADJ_NTH];
    const int nt = tab.nt;
    for (int t = threadIdx.x; t < nt * nt; t += blockDim.x) s_tab[t] = tab.t64[t];
    __syncthreads();
    const int lane = threadIdx.x & 31, q = threadIdx.x >> 5;
    const int i = blockIdx.x * ADJ_PPB + q;
    double h[3] = {0, 0, 0}, du[3] = {0, 0, 0}, dw[3] = {0, 0, 0}, dg[3] = {0, 0, 0};
    double th[ADJ_NTH];
#pragma unroll
    for (int k = 0; k < ADJ_NTH; k++) th[k] = 0.0;
    double mi = 1.0;
    if (i < a.n) {
        const float4 pi = pos[i];
        const int ti = a.type[i];
        mi = a.mass[i];
        const double vi[3] = {Vt[3 * i], Vt[3 * i + 1], Vt[3 * i + 2]};
        // input of the Hessian-vector product: the kick's cotangent (dt / m) Vt
        const double ui[3] = {a.dt / mi * vi[0], a.dt / mi * vi[1], a.dt / mi * vi[2]};
        const float iLx = 1.0f / a.Lx, iLy = 1.0f / a.Ly, iLz = 1.0f / a.Lz;
        const double rg_lo = (double)a.r_lo - ADJ_KW * a.width, rg_hi = (double)a.r_lo + a.nbins * (double)a.dr + ADJ_KW * a.width;
        const double cdt = (double)a.dt / mi;
        const int *lst = a.nbl + (size_t)i * a.maxnb + lane;
        const int cnt = min(a.nbc[(size_t)i * ADJ_LANES + lane], a.maxnb / ADJ_LANES);
        for (int c = 0; c < cnt; c++) {  // lane L: the neighbours j = L (mod 32), ascending
            const int j = lst[c * ADJ_LANES];
            const float4 pj = pos[j];
            // same float32 displacement and cutoff test as the forward
            const float fdx = mic_rint(pj.x - pi.x, a.Lx, iLx);
            const float fdy = mic_rint(pj.y - pi.y, a.Ly, iLy);
            const float fdz = mic_rint(pj.z - pi.z, a.Lz, iLz);
            const float fd2 = fdx * fdx + fdy * fdy + fdz * fdz;
            const int tj = a.type[j];
            const Tab64 &e = s_tab[ti * nt + tj];
            // d = r_i - r_j (the forward's dx is r_j - r_i)
            const double d[3] = {-(double)fdx, -(double)fdy, -(double)fdz};
            const double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
            if (fd2 < (float)e.cut2) {
                const PairD p = pair_derivs(e, r2);
                const double cj = (double)a.dt / (double)a.mass[j];
                const double dv[3] = {ui[0] - cj * Vt[3 * j], ui[1] - cj * Vt[3 * j + 1], ui[2] - cj * Vt[3 * j + 2]};
                const double dd = d[0] * dv[0] + d[1] * dv[1] + d[2] * dv[2];
                const double vd = d[0] * vi[0] + d[1] * vi[1] + d[2] * vi[2];
                for (int c = 0; c < 3; c++) {
                    h[c] += p.s * dv[c] + p.ds_dr_over_r * dd * d[c];
                    du[c] += p.dudr_over_r * d[c];
                    dw[c] += (2.0 * p.s + r2 * p.ds_dr_over_r) * d[c] * (1.0 / 3.0);
                }
                const int k = ti * nt + tj;
                // force term (dt/m) (df_i/dtheta) . Vt_i, f_i = sum_j s d
                th[2 * k] += cdt * p.dsds * vd + gU * 0.5 * p.duds + gW * r2 * p.dsds * (1.0 / 6.0);
                th[2 * k + 1] += cdt * p.dsde * vd + gU * 0.5 * p.dude + gW * r2 * p.dsde * (1.0 / 6.0);
            }
            if (gG && ti == 0 && tj == 0) {
                const double r = sqrt(r2);
                if (r > rg_lo && r < rg_hi) {
                    const double w2 = (double)a.width * a.width;
                    const double kn = 1.0 / (sqrt(2.0 * M_PI) * (double)a.width);
                    int b0 = (int)floor((r - ADJ_KW * a.width - a.r_lo) / a.dr);
                    int b1 = (int)floor((r + ADJ_KW * a.width - a.r_lo) / a.dr);
                    b0 = max(b0, 0);
                    b1 = min(b1, a.nbins - 1);
                    double acc = 0.0;
                    for (int b = b0; b <= b1; b++) {
                        const double x = r - ((double)a.r_lo + (b + 0.5) * (double)a.dr);
                        acc += gG[b] * 2.0 * (-x / w2) * kn * exp(-0.5 * x * x / w2);
                    }
                    for (int c = 0; c < 3; c++) dg[c] += acc * d[c] / r;
                }
            }
        }
    }
    for (int c = 0; c < 3; c++) {
        h[c] = wsum(h[c]);
        du[c] = wsum(du[c]);
        dw[c] = wsum(dw[c]);
        dg[c] = wsum(dg[c]);
    }
    const int nth = 2 * nt * nt;
    for (int k = 0; k < nth; k++) th[k] = wsum(th[k]);
    if (lane == 0) {
        for (int k = 0; k < nth; k++) s_th[q][k] = i < a.n ? th[k] : 0.0;
        if (i < a.n) {
            const float4 va = vn[i], vb = vn1[i];
            const double sa[3] = {va.x, va.y, va.z}, sb[3] = {vb.x, vb.y, vb.z};
            for (int c = 0; c < 3; c++) {
                R[3 * i + c] += h[c] + gU * du[c] + gW * dw[c] + dg[c];
                V[3 * i + c] = Vt[3 * i + c] + gK * mi * (sa[c] + sb[c]) * 0.25;
            }
        }
    }
    __syncthreads();
    if (threadIdx.x < nth) {
        double acc = 0.0;
        for (int p = 0; p < ADJ_PPB; p++) acc += s_th[p][threadIdx.x];
        th_part[(size_t)blockIdx.x * ADJ_NTH + threadIdx.x] += acc;
    }
}

// Neighbour list (gated): rebuilt when `force` or when flags[rd] is set;
// block 0 clears flags[clr] for the next writer.  A warp per particle; lane L
// tests j = L, L + 32, ... and appends its hits to column L of the particle's
// rows (entry c of column L at c * 32 + L), so each column holds the
// neighbours j = L (mod 32) in ascending order.
__global__ void __launch_bounds__(ADJ_BLOCK) k_adj_build(AdjArgs a, const float4 *__restrict__ pos, int *nbl, int *nbc,
                                                         int force, int rd, int clr) {
    const bool go = force || *(volatile int *)&a.flags[rd] != 0;
    if (blockIdx.x == 0 && threadIdx.x == 0) a.flags[clr] = 0;
    if (!go) return;
    const int lane = threadIdx.x & 31;
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (i >= a.n) return;
    const float iLx = 1.0f / a.Lx, iLy = 1.0f / a.Ly, iLz = 1.0f / a.Lz;
    const float4 pi = pos[i];
    const int rows = a.maxnb / ADJ_LANES;
    int *col = nbl + (size_t)i * a.maxnb + lane;
    int count = 0;
    for (int j = lane; j < a.n; j += ADJ_LANES) {
        if (j == i) continue;
        const float4 pj = pos[j];
        const float dx = mic_rint(pj.x - pi.x, a.Lx, iLx);
        const float dy = mic_rint(pj.y - pi.y, a.Ly, iLy);
        const float dz = mic_rint(pj.z - pi.z, a.Lz, iLz);
        if (dx * dx + dy * dy + dz * dz < a.rl2) {
            if (count < rows) col[count * ADJ_LANES] = j;
            count++;
        }
    }
    nbc[(size_t)i * ADJ_LANES + lane] = count;
    if (count > rows) atomicOr(a.status, ADJ_STATUS_OVERFLOW);
    if (lane == 0) a.rref[i] = pi;
}

// Sets flags[wr] when a particle of pos has moved more than skin/2 since the
// last build (the backward sweep's positions come from a stored segment).
__global__ void k_adj_check(AdjArgs a, const float4 *__restrict__ pos, int wr) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const float4 p = pos[i], q = a.rref[i];
    const float ex = mic_rint(p.x - q.x, a.Lx, 1.0f / a.Lx), ey = mic_rint(p.y - q.y, a.Ly, 1.0f / a.Ly),
                ez = mic_rint(p.z - q.z, a.Lz, 1.0f / a.Lz);
    if (ex * ex + ey * ey + ez * ez > a.move2) atomicOr(&a.flags[wr], 1);
}

__global__ void k_adj_pack(int n, const float *r, const float *v, const int *type, float4 *pos, float4 *vel) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    pos[i] = make_float4(r[3 * i], r[3 * i + 1], r[3 * i + 2], 0.f);
    vel[i] = make_float4(v[3 * i], v[3 * i + 1], v[3 * i + 2], 0.f);
    (void)type;
}

char g_adj_error[512] = "";

}  // namespace

struct gdb_adj {
    int n = 0, nt = 0, dev = 0;
    float box[3] = {0, 0, 0};
    float dt = 0.f;
    int steps = 0, ckpt = 50;
    int nbins = 0, rdf_every = 0;
    int window = 0;  // 0: exact adjoint; W > 0: cotangents cut every W steps
    float r_lo = 0.f, r_hi = 0.f, width = 0.f;
    bool setup = false, forward_done = false;
    Tables tab{};
    int *d_type = nullptr;
    float *d_mass = nullptr;
    float4 *d_pos[2] = {nullptr, nullptr}, *d_vel[2] = {nullptr, nullptr};
    float4 *d_ck_pos = nullptr, *d_ck_vel = nullptr;  // checkpoints
    float4 *d_seg_pos = nullptr, *d_seg_vel = nullptr;  // one recomputed segment
    double *d_part = nullptr, *d_acc = nullptr;
    unsigned long long *d_bins = nullptr;
    double *d_R = nullptr, *d_V = nullptr, *d_Vt = nullptr, *d_th = nullptr, *d_gG = nullptr;
    int *d_nbl = nullptr, *d_nbc = nullptr, *d_flags = nullptr;
    float4 *d_rref = nullptr;
    unsigned *d_status = nullptr;
    int maxnb = 0;
    float rl = 0.f;
    int nsamples = 0;
    std::vector<double> obs;
    cudaStream_t st = nullptr;
    char err[512] = "";
};

namespace {

int aset(gdb_adj *h, int code, const char *fmt, ...) {
    char *dst = h ? h->err : g_adj_error;
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(dst, 512, fmt, ap);
    va_end(ap);
    return code;
}

#define ACK(call)                                                                                          \
    do {                                                                                                   \
        cudaError_t e_ = (call);                                                                           \
        if (e_ != cudaSuccess)                                                                             \
            return aset(h, GDB_ERR_CUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, \
                        __LINE__);                                                                         \
    } while (0)

void adj_free(gdb_adj *h) {
    if (!h) return;
    cudaSetDevice(h->dev);
    if (h->st) cudaStreamSynchronize(h->st);
    void *ptrs[] = {h->d_type, h->d_mass, h->d_pos[0], h->d_pos[1], h->d_vel[0], h->d_vel[1], h->d_ck_pos,
                    h->d_ck_vel, h->d_seg_pos, h->d_seg_vel, h->d_part, h->d_acc, h->d_bins, h->d_R,
                    h->d_V, h->d_Vt, h->d_th, h->d_gG, h->d_nbl, h->d_nbc, h->d_flags, h->d_rref,
                    h->d_status};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    if (h->st) cudaStreamDestroy(h->st);
}

AdjArgs adj_args(const gdb_adj *h) {
    AdjArgs a;
    a.n = h->n;
    a.nt = h->nt;
    a.Lx = h->box[0];
    a.Ly = h->box[1];
    a.Lz = h->box[2];
    a.dt = h->dt;
    a.type = h->d_type;
    a.mass = h->d_mass;
    a.nbins = h->nbins;
    a.r_lo = h->r_lo;
    a.dr = h->nbins > 0 ? (h->r_hi - h->r_lo) / h->nbins : 1.f;
    a.width = h->width;
    a.nbl = h->d_nbl;
    a.nbc = h->d_nbc;
    a.maxnb = h->maxnb;
    a.rl2 = h->rl * h->rl;
    const float mv = 0.5f * ADJ_SKIN - 0.01f;
    a.move2 = mv * mv;
    a.rref = h->d_rref;
    a.flags = h->d_flags;
    a.status = h->d_status;
    return a;
}

int nblocks_of(const gdb_adj *h) { return (h->n + ADJ_PPB - 1) / ADJ_PPB; }

int build_blocks(const gdb_adj *h) { return (h->n * 32 + ADJ_BLOCK - 1) / ADJ_BLOCK; }

// One forward step from buffers (pin, vin) into (pout, vout); step index s.
// The list is rebuilt first when the previous step flagged it (or `force`);
// step s flags into slot s & 1, which the build before it clears.
int forward_step(gdb_adj *h, const float4 *pin, const float4 *vin, float4 *pout, float4 *vout, int s,
                 bool accumulate, bool force) {
    const AdjArgs a = adj_args(h);
    k_adj_build<<<build_blocks(h), ADJ_BLOCK, 0, h->st>>>(a, pin, h->d_nbl, h->d_nbc, force ? 1 : 0, (s + 1) & 1,
                                                           s & 1);
    ACK(cudaGetLastError());
    const bool rdf = accumulate && h->nbins > 0 && h->rdf_every > 0 && s % h->rdf_every == 0;
    k_adj_step<<<nblocks_of(h), ADJ_BLOCK, 0, h->st>>>(a, h->tab, pin, vin, pout, vout, h->d_part,
                                                        rdf ? h->d_bins : nullptr, h->d_flags + (s & 1));
    ACK(cudaGetLastError());
    if (accumulate) {
        k_adj_reduce<<<1, 256, 0, h->st>>>(h->d_part, nblocks_of(h), h->d_acc);
        ACK(cudaGetLastError());
    }
    return GDB_OK;
}

// List reach (largest cut, or the RDF kernel's reach, plus the skin) and
// capacity (32 columns, each twice its mean count at this density plus 8).
int ensure_list(gdb_adj *h) {
    float reach = 0.f;
    for (int k = 0; k < h->nt * h->nt; k++) reach = std::max(reach, h->tab.t32[k].cut);
    if (h->nbins > 0)
        reach = std::max(reach, (float)((double)h->r_hi + ADJ_KW * h->width));
    h->rl = reach + ADJ_SKIN;
    const double vol = (double)h->box[0] * h->box[1] * h->box[2];
    const double mean = 4.0 / 3.0 * M_PI * (double)h->rl * h->rl * h->rl * h->n / vol;
    // 32 columns of rows entries: a column holds about mean / 32 neighbours
    const int rows = std::min((int)(2.0 * mean / ADJ_LANES) + 8, (h->n + ADJ_LANES - 1) / ADJ_LANES);
    const int want = rows * ADJ_LANES;
    if (want > h->maxnb || !h->d_nbl) {
        if (h->d_nbl) cudaFree(h->d_nbl);
        h->d_nbl = nullptr;
        ACK(cudaMalloc(&h->d_nbl, (size_t)h->n * want * sizeof(int)));
        h->maxnb = want;
    }
    if (!h->d_nbc) {
        ACK(cudaMalloc(&h->d_nbc, (size_t)h->n * ADJ_LANES * sizeof(int)));
        ACK(cudaMalloc(&h->d_rref, h->n * sizeof(float4)));
        ACK(cudaMalloc(&h->d_flags, 2 * sizeof(int)));
        ACK(cudaMalloc(&h->d_status, sizeof(unsigned)));
    }
    ACK(cudaMemsetAsync(h->d_flags, 0, 2 * sizeof(int), h->st));
    ACK(cudaMemsetAsync(h->d_status, 0, sizeof(unsigned), h->st));
    return GDB_OK;
}

void build_tables(gdb_adj *h, const double *params) {
    Tables &T = h->tab;
    T.nt = h->nt;
    for (int k = 0; k < h->nt * h->nt; k++) {
        const double sig = params[3 * k], eps = params[3 * k + 1], cut = params[3 * k + 2];
        Tab32 &e = T.t32[k];
        e.c = (float)(sig * sig);
        e.cu12 = (float)(4.0 * eps);
        e.cu6 = (float)(-4.0 * eps);
        e.cs12 = (float)(48.0 * eps);
        e.cs6 = (float)(-24.0 * eps);
        const double sr6 = pow(sig / cut, 6.0), sr12 = sr6 * sr6;
        const double uc = 4.0 * eps * (sr12 - sr6);
        const double sc = eps * (48.0 * sr12 - 24.0 * sr6) / (cut * cut);
        e.uc = (float)uc;
        e.sc = (float)sc;
        e.sccut = (float)(sc * cut);
        e.cut = (float)cut;
        e.cut2 = (float)cut * (float)cut;
        Tab64 &d = T.t64[k];
        d.sig = sig;
        d.eps = eps;
        d.cut = cut;
        d.cut2 = (double)e.cut2;
        d.s_c = sc;
        d.dsds_c = eps * (576.0 * sr12 - 144.0 * sr6) / (cut * cut) / sig;
        d.u_c = uc;
        d.duds_c = 4.0 * eps * (12.0 * sr12 - 6.0 * sr6) / sig;
    }
}

}  // namespace

extern "C" {

int gdb_adj_create(int n, int ntypes, int device, gdb_adj **out) {
    gdb_adj *h = nullptr;
    if (!out || n < 2 || ntypes < 1 || ntypes > ADJ_MAXT)
        return aset(nullptr, GDB_ERR_ARG, "gdb_adj_create: bad arguments (n=%d, ntypes=%d, max types %d)", n, ntypes,
                    ADJ_MAXT);
    h = new gdb_adj();
    h->n = n;
    h->nt = ntypes;
    h->dev = device;
    cudaError_t e;
    if ((e = cudaSetDevice(device)) != cudaSuccess || (e = cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking)) ||
        (e = cudaMalloc(&h->d_type, n * sizeof(int))) || (e = cudaMalloc(&h->d_mass, n * sizeof(float))) ||
        (e = cudaMalloc(&h->d_pos[0], n * sizeof(float4))) || (e = cudaMalloc(&h->d_pos[1], n * sizeof(float4))) ||
        (e = cudaMalloc(&h->d_vel[0], n * sizeof(float4))) || (e = cudaMalloc(&h->d_vel[1], n * sizeof(float4))) ||
        (e = cudaMalloc(&h->d_part, (size_t)((n + ADJ_PPB - 1) / ADJ_PPB) * 3 * sizeof(double))) ||
        (e = cudaMalloc(&h->d_acc, 3 * sizeof(double))) ||
        (e = cudaMalloc(&h->d_bins, ADJ_MAXB * sizeof(unsigned long long))) ||
        (e = cudaMalloc(&h->d_R, (size_t)n * 3 * sizeof(double))) ||
        (e = cudaMalloc(&h->d_V, (size_t)n * 3 * sizeof(double))) ||
        (e = cudaMalloc(&h->d_Vt, (size_t)n * 3 * sizeof(double))) ||
        (e = cudaMalloc(&h->d_th, (size_t)((n + ADJ_PPB - 1) / ADJ_PPB) * ADJ_NTH * sizeof(double))) ||
        (e = cudaMalloc(&h->d_gG, ADJ_MAXB * sizeof(double)))) {
        adj_free(h);
        delete h;
        return aset(nullptr, GDB_ERR_CUDA, "gdb_adj_create: %s", cudaGetErrorString(e));
    }
    *out = h;
    return GDB_OK;
}

int gdb_adj_destroy(gdb_adj *h) {
    if (!h) return GDB_OK;
    adj_free(h);
    delete h;
    return GDB_OK;
}

int gdb_adj_setup(gdb_adj *h, const float box[3], const int32_t *ptype, const float *mass, float dt, int steps,
                  int checkpoint_every, int rdf_bins, float rdf_lo, float rdf_hi, float rdf_width, int rdf_every) {
    if (!h || !box || !ptype || !mass || !(dt > 0.f) || steps < 1 || checkpoint_every < 1 || rdf_bins < 0 ||
        rdf_bins > ADJ_MAXB || (rdf_bins > 0 && !(rdf_hi > rdf_lo && rdf_lo >= 0.f && rdf_width > 0.f)))
        return aset(h, GDB_ERR_ARG, "gdb_adj_setup: bad arguments");
    for (int k = 0; k < 3; k++)
        if (!(box[k] > 0.f)) return aset(h, GDB_ERR_ARG, "gdb_adj_setup: box lengths must be positive");
    for (int i = 0; i < h->n; i++) {
        if (ptype[i] < 0 || ptype[i] >= h->nt) return aset(h, GDB_ERR_ARG, "gdb_adj_setup: type out of range");
        if (!(mass[i] > 0.f)) return aset(h, GDB_ERR_ARG, "gdb_adj_setup: masses must be positive");
    }
    ACK(cudaSetDevice(h->dev));
    memcpy(h->box, box, sizeof(h->box));
    h->dt = dt;
    h->steps = steps;
    h->ckpt = checkpoint_every;
    h->nbins = rdf_bins;
    h->r_lo = rdf_lo;
    h->r_hi = rdf_hi;
    h->width = rdf_width;
    h->rdf_every = rdf_every;
    ACK(cudaMemcpyAsync(h->d_type, ptype, h->n * sizeof(int), cudaMemcpyHostToDevice, h->st));
    ACK(cudaMemcpyAsync(h->d_mass, mass, h->n * sizeof(float), cudaMemcpyHostToDevice, h->st));
    const int nck = (steps + checkpoint_every - 1) / checkpoint_every;
    if (h->d_ck_pos) cudaFree(h->d_ck_pos);
    if (h->d_ck_vel) cudaFree(h->d_ck_vel);
    if (h->d_seg_pos) cudaFree(h->d_seg_pos);
    if (h->d_seg_vel) cudaFree(h->d_seg_vel);
    h->d_ck_pos = h->d_ck_vel = h->d_seg_pos = h->d_seg_vel = nullptr;
    ACK(cudaMalloc(&h->d_ck_pos, (size_t)nck * h->n * sizeof(float4)));
    ACK(cudaMalloc(&h->d_ck_vel, (size_t)nck * h->n * sizeof(float4)));
    ACK(cudaMalloc(&h->d_seg_pos, (size_t)(checkpoint_every + 1) * h->n * sizeof(float4)));
    ACK(cudaMalloc(&h->d_seg_vel, (size_t)(checkpoint_every + 1) * h->n * sizeof(float4)));
    ACK(cudaStreamSynchronize(h->st));
    h->setup = true;
    h->forward_done = false;
    return GDB_OK;
}

int gdb_adj_forward(gdb_adj *h, const double *params, const float *r0, const float *v0, double *obs) {
    if (!h || !params || !r0 || !v0 || !obs) return aset(h, GDB_ERR_ARG, "gdb_adj_forward: bad arguments");
    if (!h->setup) return aset(h, GDB_ERR_STATE, "gdb_adj_forward: call gdb_adj_setup first");
    for (int k = 0; k < h->nt * h->nt; k++) {
        const double sig = params[3 * k], eps = params[3 * k + 1], cut = params[3 * k + 2];
        if (!(sig > 0.0 && eps > 0.0 && cut > 0.0))
            return aset(h, GDB_ERR_ARG, "gdb_adj_forward: sigma, epsilon and cut must be positive");
        if (2.0 * cut >= std::min(std::min(h->box[0], h->box[1]), h->box[2]))
            return aset(h, GDB_ERR_ARG, "gdb_adj_forward: cut must be below half the box");
    }
    ACK(cudaSetDevice(h->dev));
    build_tables(h, params);
    const int n = h->n;
    int rc = ensure_list(h);
    if (rc) return rc;
    float *dr = nullptr, *dv = nullptr;
    ACK(gdb::pool_alloc(&dr, (size_t)n * 3 * sizeof(float), h->st));
    ACK(gdb::pool_alloc(&dv, (size_t)n * 3 * sizeof(float), h->st));
    ACK(cudaMemcpyAsync(dr, r0, (size_t)n * 3 * sizeof(float), cudaMemcpyHostToDevice, h->st));
    ACK(cudaMemcpyAsync(dv, v0, (size_t)n * 3 * sizeof(float), cudaMemcpyHostToDevice, h->st));
    k_adj_pack<<<(n + 255) / 256, 256, 0, h->st>>>(n, dr, dv, h->d_type, h->d_pos[0], h->d_vel[0]);
    ACK(cudaGetLastError());
    ACK(cudaFreeAsync(dr, h->st));
    ACK(cudaFreeAsync(dv, h->st));
    ACK(cudaMemsetAsync(h->d_acc, 0, 3 * sizeof(double), h->st));
    ACK(cudaMemsetAsync(h->d_bins, 0, ADJ_MAXB * sizeof(unsigned long long), h->st));
    int cur = 0;
    h->nsamples = 0;
    for (int s = 0; s < h->steps; s++) {
        if (s % h->ckpt == 0) {
            const size_t off = (size_t)(s / h->ckpt) * n;
            ACK(cudaMemcpyAsync(h->d_ck_pos + off, h->d_pos[cur], n * sizeof(float4), cudaMemcpyDeviceToDevice, h->st));
            ACK(cudaMemcpyAsync(h->d_ck_vel + off, h->d_vel[cur], n * sizeof(float4), cudaMemcpyDeviceToDevice, h->st));
        }
        rc = forward_step(h, h->d_pos[cur], h->d_vel[cur], h->d_pos[cur ^ 1], h->d_vel[cur ^ 1], s, true, s == 0);
        if (rc) return rc;
        if (h->nbins > 0 && h->rdf_every > 0 && s % h->rdf_every == 0) h->nsamples++;
        cur ^= 1;
    }
    double acc[3];
    std::vector<unsigned long long> bins(ADJ_MAXB);
    ACK(cudaMemcpyAsync(acc, h->d_acc, sizeof(acc), cudaMemcpyDeviceToHost, h->st));
    ACK(cudaMemcpyAsync(bins.data(), h->d_bins, ADJ_MAXB * sizeof(unsigned long long), cudaMemcpyDeviceToHost, h->st));
    unsigned status = 0;
    ACK(cudaMemcpyAsync(&status, h->d_status, sizeof(unsigned), cudaMemcpyDeviceToHost, h->st));
    ACK(cudaStreamSynchronize(h->st));
    if (status & ADJ_STATUS_OVERFLOW)
        return aset(h, GDB_ERR_NBLIST, "gdb_adj_forward: a list column outgrew %d entries (reach %.3f)",
                    h->maxnb / ADJ_LANES, h->rl);
    h->obs.assign(3 + h->nbins, 0.0);
    for (int q = 0; q < 3; q++) h->obs[q] = acc[q] / h->steps;
    if (h->nbins > 0 && h->nsamples > 0) {
        // g_b = sum K / (samples * N_A * rho_A * 4 pi r_b^2)
        std::vector<int> types(n);
        ACK(cudaMemcpy(types.data(), h->d_type, n * sizeof(int), cudaMemcpyDeviceToHost));
        const double na = (double)std::count(types.begin(), types.end(), 0);
        const double vol = (double)h->box[0] * h->box[1] * h->box[2];
        const double dr_ = (double)(h->r_hi - h->r_lo) / h->nbins;
        for (int b = 0; b < h->nbins; b++) {
            const double rb = h->r_lo + (b + 0.5) * dr_;
            const double norm = 1.0 / (h->nsamples * na * (na / vol) * 4.0 * M_PI * rb * rb);
            h->obs[3 + b] = (double)bins[b] / ADJ_FIX * norm;
        }
    }
    memcpy(obs, h->obs.data(), h->obs.size() * sizeof(double));
    h->forward_done = true;
    return GDB_OK;
}

int gdb_adj_backward(gdb_adj *h, const double *grad_obs, double *grad_params) {
    if (!h || !grad_obs || !grad_params) return aset(h, GDB_ERR_ARG, "gdb_adj_backward: bad arguments");
    if (!h->forward_done) return aset(h, GDB_ERR_STATE, "gdb_adj_backward: run gdb_adj_forward first");
    ACK(cudaSetDevice(h->dev));
    const int n = h->n, T = h->steps;
    const double gU = grad_obs[0] / T, gW = grad_obs[1] / T, gK = grad_obs[2] / T;
    // dL/dr contributions of g_b on a sampled step: grad_g_b * norm_b
    std::vector<double> gG(ADJ_MAXB, 0.0);
    bool any_g = false;
    if (h->nbins > 0 && h->nsamples > 0) {
        std::vector<int> types(n);
        ACK(cudaMemcpy(types.data(), h->d_type, n * sizeof(int), cudaMemcpyDeviceToHost));
        const double na = (double)std::count(types.begin(), types.end(), 0);
        const double vol = (double)h->box[0] * h->box[1] * h->box[2];
        const double dr_ = (double)(h->r_hi - h->r_lo) / h->nbins;
        for (int b = 0; b < h->nbins; b++) {
            const double rb = h->r_lo + (b + 0.5) * dr_;
            gG[b] = grad_obs[3 + b] / (h->nsamples * na * (na / vol) * 4.0 * M_PI * rb * rb);
            any_g |= gG[b] != 0.0;
        }
        ACK(cudaMemcpyAsync(h->d_gG, gG.data(), ADJ_MAXB * sizeof(double), cudaMemcpyHostToDevice, h->st));
    }
    const int nb = nblocks_of(h);
    ACK(cudaMemsetAsync(h->d_R, 0, (size_t)n * 3 * sizeof(double), h->st));
    ACK(cudaMemsetAsync(h->d_V, 0, (size_t)n * 3 * sizeof(double), h->st));
    ACK(cudaMemsetAsync(h->d_th, 0, (size_t)nb * ADJ_NTH * sizeof(double), h->st));
    const AdjArgs a = adj_args(h);
    const int nseg = (T + h->ckpt - 1) / h->ckpt;
    for (int sg = nseg - 1; sg >= 0; sg--) {
        const int s0 = sg * h->ckpt, len = std::min(h->ckpt, T - s0);
        // recompute the segment's states (bit-identical to the forward)
        const size_t off = (size_t)sg * n;
        ACK(cudaMemcpyAsync(h->d_seg_pos, h->d_ck_pos + off, n * sizeof(float4), cudaMemcpyDeviceToDevice, h->st));
        ACK(cudaMemcpyAsync(h->d_seg_vel, h->d_ck_vel + off, n * sizeof(float4), cudaMemcpyDeviceToDevice, h->st));
        for (int k = 0; k < len; k++) {
            int rc = forward_step(h, h->d_seg_pos + (size_t)k * n, h->d_seg_vel + (size_t)k * n,
                                  h->d_seg_pos + (size_t)(k + 1) * n, h->d_seg_vel + (size_t)(k + 1) * n, s0 + k,
                                  false, k == 0);
            if (rc) return rc;
        }
        // reverse sweep of the segment; the list follows the positions
        // backwards (check -> gated build), slots by step parity
        ACK(cudaMemsetAsync(h->d_flags, 0, 2 * sizeof(int), h->st));
        for (int k = len - 1; k >= 0; k--) {
            const int s = s0 + k;
            {
                const float4 *pk = h->d_seg_pos + (size_t)k * n;
                k_adj_check<<<(n + 255) / 256, 256, 0, h->st>>>(a, pk, s & 1);
                ACK(cudaGetLastError());
                k_adj_build<<<build_blocks(h), ADJ_BLOCK, 0, h->st>>>(a, pk, h->d_nbl, h->d_nbc, k == len - 1 ? 1 : 0,
                                                                       s & 1, (s + 1) & 1);
                ACK(cudaGetLastError());
            }
            if (h->window > 0 && (s + 1) % h->window == 0) {
                // last step of a window: nothing flows back across its end
                ACK(cudaMemsetAsync(h->d_R, 0, (size_t)n * 3 * sizeof(double), h->st));
                ACK(cudaMemsetAsync(h->d_V, 0, (size_t)n * 3 * sizeof(double), h->st));
            }
            const float4 *pn = h->d_seg_pos + (size_t)k * n;
            const float4 *vn = h->d_seg_vel + (size_t)k * n, *vn1 = h->d_seg_vel + (size_t)(k + 1) * n;
            k_adj_vtot<<<(n + 255) / 256, 256, 0, h->st>>>(n, h->dt, gK, h->d_mass, h->d_R, h->d_V, vn, vn1, h->d_Vt);
            ACK(cudaGetLastError());
            const bool rdf = any_g && h->rdf_every > 0 && s % h->rdf_every == 0;
            k_adj_back<<<nb, ADJ_BLOCK, 0, h->st>>>(a, h->tab, pn, h->d_Vt, h->d_R, h->d_V, vn, vn1, gU, gW, gK,
                                                     rdf ? h->d_gG : nullptr, h->d_th);
            ACK(cudaGetLastError());
        }
    }
    std::vector<double> th((size_t)nb * ADJ_NTH);
    unsigned status = 0;
    ACK(cudaMemcpyAsync(th.data(), h->d_th, th.size() * sizeof(double), cudaMemcpyDeviceToHost, h->st));
    ACK(cudaMemcpyAsync(&status, h->d_status, sizeof(unsigned), cudaMemcpyDeviceToHost, h->st));
    ACK(cudaStreamSynchronize(h->st));
    if (status & ADJ_STATUS_OVERFLOW)
        return aset(h, GDB_ERR_NBLIST, "gdb_adj_backward: a list column outgrew %d entries (reach %.3f)",
                    h->maxnb / ADJ_LANES, h->rl);
    // fixed-order sum over blocks; a parameter of the unordered pair {a, b}
    // collects the (a, b) and (b, a) entries
    const int nt = h->nt;
    std::vector<double> g(2 * nt * nt, 0.0);
    for (int b = 0; b < nb; b++)
        for (int k = 0; k < 2 * nt * nt; k++) g[k] += th[(size_t)b * ADJ_NTH + k];
    for (int x = 0; x < nt; x++)
        for (int y = 0; y < nt; y++) {
            const int k = x * nt + y, kt = y * nt + x;
            const double gs = x == y ? g[2 * k] : g[2 * k] + g[2 * kt];
            const double ge = x == y ? g[2 * k + 1] : g[2 * k + 1] + g[2 * kt + 1];
            grad_params[3 * k] = gs;
            grad_params[3 * k + 1] = ge;
            grad_params[3 * k + 2] = 0.0;
        }
    return GDB_OK;
}

int gdb_adj_set_window(gdb_adj *h, int window) {
    if (!h || window < 0) return aset(h, GDB_ERR_ARG, "gdb_adj_set_window: bad arguments");
    h->window = window;
    return GDB_OK;
}

int gdb_adj_final_state(gdb_adj *h, float *r, float *v) {
    if (!h || !h->forward_done) return aset(h, GDB_ERR_STATE, "gdb_adj_final_state: no forward run");
    ACK(cudaSetDevice(h->dev));
    const int cur = h->steps & 1;
    std::vector<float4> p(h->n), q(h->n);
    ACK(cudaMemcpy(p.data(), h->d_pos[cur], h->n * sizeof(float4), cudaMemcpyDeviceToHost));
    ACK(cudaMemcpy(q.data(), h->d_vel[cur], h->n * sizeof(float4), cudaMemcpyDeviceToHost));
    for (int i = 0; i < h->n; i++) {
        if (r) {
            r[3 * i] = p[i].x;
            r[3 * i + 1] = p[i].y;
            r[3 * i + 2] = p[i].z;
        }
        if (v) {
            v[3 * i] = q[i].x;
            v[3 * i + 1] = q[i].y;
            v[3 * i + 2] = q[i].z;
        }
    }
    return GDB_OK;
}

int gdb_adj_get_last_error(gdb_adj *h, char *buf, int n) {
    if (!buf || n < 1) return GDB_ERR_ARG;
    snprintf(buf, (size_t)n, "%s", h ? h->err : g_adj_error);
    return GDB_OK;
}

}  // extern "C"
