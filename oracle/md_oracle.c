/*
 * md_oracle.c -- CPU restatement of gamdpy's simulation hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA library in
 * gamdpy_b200/csrc: only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline / --impl reference leg may load it.  The product path never
 * calls it and has no CPU fallback.
 *
 * Every function restates one piece of the reference (gamdpy, pure Python +
 * numba) and cites the file:line it follows, relative to the gamdpy project
 * root.  Arithmetic is float32 where gamdpy's numba kernels are float32 and
 * float64 where numba's typing rules promote (Python int/float literals mixed
 * with float32 give float64 under numba).  Compile with -ffp-contract=off so
 * that no multiply-add is fused implicitly; the one place where the GPU build
 * of gamdpy may fuse (the distance accumulation) is selected explicitly by the
 * `fma` argument.
 *
 * Parity of this restatement is pinned against outputs of gamdpy itself run
 * on the CPU (the .npz fixtures in tests/golden, generated by tests/golden/make_golden.py).
 *
 * Reductions the reference does with float32 atomics (ScalarSaver sums, the
 * Nose-Hoover kinetic-energy sum) are accumulated here in float64 in a fixed
 * order; the CUDA library does the same, so both are run-to-run deterministic.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_POT_LJ_SIGMA_EPSILON 0 /* potential_functions/LJ_12_6_sigma_epsilon.py:6-36 */
#define ORC_POT_LJ_12_6 1          /* potential_functions/LJ_12_6.py:3-41 */
#define ORC_CUT_SF 0               /* apply_shifted_force_cutoff.py:30-37 */
#define ORC_CUT_SP 1               /* apply_shifted_potential_cutoff.py:42-47 */
#define ORC_CUT_NONE 2             /* potential used unwrapped */

int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void orc_set_num_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

/* numba lowers `x ** k` with an integer literal k by binary exponentiation in
 * the operand's type (numba/cpython/numbers.py static_power_impl); this is
 * that loop for float32. */
static float powi_f32(float a, int k) {
    float result = 1.0f;
    while (k) {
        if (k & 1) result = result * a;
        a = a * a;
        k >>= 1;
    }
    return result;
}

/* LJ_12_6_sigma_epsilon.py:26-36: params (sigma, epsilon, ...). */
static void lj_sigma_epsilon(float dist, const float *p, float *u, float *s, float *umm) {
    float sigma = p[0], epsilon = p[1];
    float OneOdist = 1.0f / dist;
    float sigmaOdist = sigma * OneOdist;
    float x12 = powi_f32(sigmaOdist, 12), x6 = powi_f32(sigmaOdist, 6);
    float o2 = powi_f32(OneOdist, 2);
    *u = 4.0f * epsilon * (x12 - x6);
    *s = 24.0f * epsilon * (2.0f * x12 - x6) * o2;
    *umm = 24.0f * epsilon * (26.0f * x12 - 7.0f * x6) * o2;
}

/* LJ_12_6.py:34-41: params (A12, A6, ...). */
static void lj_12_6(float dist, const float *p, float *u, float *s, float *umm) {
    float A12 = p[0], A6 = p[1];
    float inv = 1.0f / dist;
    *u = A12 * powi_f32(inv, 12) + A6 * powi_f32(inv, 6);
    *s = 12.0f * A12 * powi_f32(inv, 14) + 6.0f * A6 * powi_f32(inv, 8);
    *umm = 156.0f * A12 * powi_f32(inv, 14) + 42.0f * A6 * powi_f32(inv, 8);
}

static void raw_pot(int kind, float dist, const float *p, float *u, float *s, float *umm) {
    if (kind == ORC_POT_LJ_12_6) lj_12_6(dist, p, u, s, umm);
    else lj_sigma_epsilon(dist, p, u, s, umm);
}

/* Cutoff wrappers.  The cut is the last parameter (params[-1]); np = number
 * of parameters including the cut.
 *   SF: apply_shifted_force_cutoff.py:30-37   u -= u_c - s_c*cut*(r-cut); s -= s_c
 *   SP: apply_shifted_potential_cutoff.py:42-47  u -= u_c
 * Both re-evaluate the potential at the cut on every call, as the reference. */
void orc_pair_potential(int kind, int cutmode, float dist, const float *p, int np, float out[3]) {
    float u, s, umm;
    raw_pot(kind, dist, p, &u, &s, &umm);
    if (cutmode != ORC_CUT_NONE) {
        float cut = p[np - 1];
        float uc, sc, ummc;
        raw_pot(kind, cut, p, &uc, &sc, &ummc);
        if (cutmode == ORC_CUT_SF) {
            u -= uc - sc * cut * (dist - cut);
            s -= sc;
        } else {
            u -= uc;
        }
    }
    out[0] = u;
    out[1] = s;
    out[2] = umm;
}

/* simulation_boxes/orthorhombic.py:43-57 (dist_sq_dr_function) and :59-73
 * (dist_sq_function): dr = ri - rj, minimum image via 2*dr vs +-L, and
 * dist_sq accumulated in k order.  fma=1 evaluates the accumulation as
 * fmaf(dr, dr, dist_sq), the form libNVVM produces with its default
 * contraction; fma=0 rounds the product first (numba on the CPU). */
static inline float dist_sq_dr(const float *ri, const float *rj, const float *box, float *dr, int fma) {
    float dsq = 0.0f;
    for (int k = 0; k < 3; k++) {
        float d = ri[k] - rj[k];
        float L = box[k];
        d += (2.0f * d > L) ? -L : ((2.0f * d < -L) ? L : 0.0f);
        if (dr) dr[k] = d;
        if (fma) dsq = fmaf(d, d, dsq);
        else {
            float p = d * d;
            dsq = dsq + p;
        }
    }
    return dsq;
}

float orc_dist_sq(const float *ri, const float *rj, const float *box, float *dr, int fma) {
    return dist_sq_dr(ri, rj, box, dr, fma);
}

/* orthorhombic.py:75-86 */
void orc_apply_pbc(float *r, int *img, const float *box) {
    for (int k = 0; k < 3; k++) {
        if (r[k] * 2.0f > box[k]) { r[k] -= box[k]; img[k] += 1; }
        if (r[k] * 2.0f < -box[k]) { r[k] += box[k]; img[k] -= 1; }
    }
}

/* nblist.py:88-127 (NbList2.nblist_update, full list, no exclusions):
 * j != i and dist_sq < (max_cut+skin)^2.  Output in gamdpy's layout: row i of
 * nbl (n x (max_nbs+1)) holds the neighbours, the count is in the last column.
 * Neighbours are appended in ascending j (the reference's order is set by
 * atomics and is not deterministic; only the set is compared).
 * Returns the largest count seen (overflow when >= max_nbs, nblist.py:140). */
int orc_nblist_nsq(int n, const float *r, const float *box, float cut_plus_skin, int max_nbs,
                   int32_t *nbl, int fma) {
    int maxcount = 0;
    const float cps2 = cut_plus_skin * cut_plus_skin;
#pragma omp parallel for schedule(dynamic, 16) reduction(max : maxcount)
    for (int i = 0; i < n; i++) {
        int32_t *row = nbl + (size_t)i * (max_nbs + 1);
        int c = 0;
        for (int j = 0; j < n; j++) {
            if (j == i) continue;
            float d2 = dist_sq_dr(r + 3 * (size_t)j, r + 3 * (size_t)i, box, NULL, fma);
            if (d2 < cps2) {
                if (c < max_nbs) row[c] = j;
                c++;
            }
        }
        row[max_nbs] = c;
        if (c > maxcount) maxcount = c;
    }
    return maxcount;
}

/* nblist_linked_lists.py:36-42: cells per dimension = int(L / ((max_cut+skin)/2)),
 * asserted > 4 (and > 6 in x).  Returns 0 and fills nc, or -1 when the assert
 * of the reference would fail. */
int orc_cells_per_dimension(const float *box, float max_cut, float skin, int *nc) {
    /* max_cut and skin are np.float32 (pair_potential.py:49, compute_plan);
     * (max_cut + skin)/2 is float32 arithmetic divided by a Python int ->
     * numpy float32 on the host; lengths[i] / that -> float32; int() truncates. */
    float min_cell = (max_cut + skin) / 2.0f;
    for (int k = 0; k < 3; k++) {
        float q = box[k] / min_cell;
        nc[k] = (int)q;
        if (nc[k] <= 4) return -1;
        if (k == 0 && nc[k] <= 6) return -1;
    }
    return 0;
}

/* nblist_linked_lists.py:127: cell = int(floor((x + 0.5*L) * nc / L)) % nc.
 * 0.5 is a float64 literal, so numba evaluates the whole expression in
 * float64; % on integers follows Python (result has the divisor's sign). */
static inline int cell_coord(float x, float L, int nc) {
    double v = ((double)x + 0.5 * (double)L) * (double)nc / (double)L;
    long long c = (long long)floor(v);
    long long m = c % nc;
    if (m < 0) m += nc;
    return (int)m;
}

void orc_cell_coords(int n, const float *r, const float *box, const int *nc, int32_t *cells_out) {
    for (int i = 0; i < n; i++)
        for (int k = 0; k < 3; k++) cells_out[3 * i + k] = cell_coord(r[3 * i + k], box[k], nc[k]);
}

/* NbListLinkedLists: put_particles_in_cells (nblist_linked_lists.py:117-131)
 * pushes every particle on the head of its cell's chain; the build
 * (:133-183) walks a 5x5x5 stencil of cells and the chains in them; clear
 * (:196-218) resets.  The chain order of the reference depends on atomics;
 * here particles are pushed in ascending index, so each chain is in
 * descending index.  Only the per-particle sets are compared.  Returns the
 * largest count, or -1 if the cell grid fails the reference's asserts. */
int orc_nblist_cells(int n, const float *r, const float *box, float max_cut, float skin, int max_nbs,
                     int32_t *nbl, int fma) {
    int nc[3];
    if (orc_cells_per_dimension(box, max_cut, skin, nc) != 0) return -1;
    size_t ncell = (size_t)nc[0] * nc[1] * nc[2];
    int32_t *head = (int32_t *)malloc(ncell * sizeof(int32_t));
    int32_t *next = (int32_t *)malloc((size_t)n * sizeof(int32_t));
    int32_t *mc = (int32_t *)malloc((size_t)n * 3 * sizeof(int32_t));
    for (size_t c = 0; c < ncell; c++) head[c] = -1;
    for (int i = 0; i < n; i++) {
        for (int k = 0; k < 3; k++) mc[3 * i + k] = cell_coord(r[3 * i + k], box[k], nc[k]);
        size_t idx = ((size_t)mc[3 * i] * nc[1] + mc[3 * i + 1]) * nc[2] + mc[3 * i + 2];
        next[i] = head[idx];
        head[idx] = i;
    }
    const float cut_plus_skin = max_cut + skin;
    const float cps2 = cut_plus_skin * cut_plus_skin;
    int maxcount = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(max : maxcount)
    for (int i = 0; i < n; i++) {
        int32_t *row = nbl + (size_t)i * (max_nbs + 1);
        int c = 0;
        for (int ix = -2; ix < 3; ix++)
            for (int iy = -2; iy < 3; iy++)
                for (int iz = -2; iz < 3; iz++) {
                    int cx = ((mc[3 * i] + ix) % nc[0] + nc[0]) % nc[0];
                    int cy = ((mc[3 * i + 1] + iy) % nc[1] + nc[1]) % nc[1];
                    int cz = ((mc[3 * i + 2] + iz) % nc[2] + nc[2]) % nc[2];
                    int j = head[((size_t)cx * nc[1] + cy) * nc[2] + cz];
                    while (j >= 0) {
                        if (j != i) {
                            float d2 = dist_sq_dr(r + 3 * (size_t)j, r + 3 * (size_t)i, box, NULL, fma);
                            if (d2 < cps2) {
                                c++;
                                if (c < max_nbs) row[c - 1] = j;
                            }
                        }
                        j = next[j];
                    }
                }
        row[max_nbs] = c;
        if (c > maxcount) maxcount = c;
    }
    free(head);
    free(next);
    free(mc);
    return maxcount;
}

/* pair_potential.py:164-178 (full-list pairpotential_calculator) inside
 * calc_forces (:185-246): for each listed neighbour j with
 * dist_sq < cut_ij^2: f_i -= dr*s; W_i += dr_k^2*s*(0.5/D); U_i += u/2;
 * lapU_i += (1-D)*s + umm.  Per-particle sums are float32 in list order.
 * params: nt*nt rows of np floats (last = cut).  Any output pointer may be
 * NULL.  Fsq (a scalar the integrator computes, NVE.py:79-80) is returned
 * for the forces just computed if fsq != NULL. */
void orc_forces(int n, const float *r, const int32_t *ptype, const float *box, const float *params,
                int np, int nt, int kind, int cutmode, const int32_t *nbl, int max_nbs, float *f,
                float *U, float *W, float *lapU, float *fsq, int fma) {
    const float virial_factor = 0.5f / 3.0f; /* numba.float32(0.5/D) */
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; i++) {
        const int32_t *row = nbl + (size_t)i * (max_nbs + 1);
        int cnt = row[max_nbs];
        if (cnt > max_nbs) cnt = max_nbs;
        int ti = ptype ? ptype[i] : 0;
        float fi[3] = {0.0f, 0.0f, 0.0f};
        float u_i = 0.0f, w_i = 0.0f, l_i = 0.0f;
        for (int a = 0; a < cnt; a++) {
            int j = row[a];
            int tj = ptype ? ptype[j] : 0;
            const float *p = params + ((size_t)ti * nt + tj) * np;
            float cut = p[np - 1];
            float dr[3];
            float d2 = dist_sq_dr(r + 3 * (size_t)j, r + 3 * (size_t)i, box, dr, fma);
            if (d2 < cut * cut) {
                float o[3];
                orc_pair_potential(kind, cutmode, sqrtf(d2), p, np, o);
                float s = o[1];
                for (int k = 0; k < 3; k++) {
                    fi[k] = fi[k] - dr[k] * s;
                    w_i += dr[k] * dr[k] * s * virial_factor;
                }
                u_i += 0.5f * o[0];
                l_i += (1.0f - 3.0f) * s + o[2];
            }
        }
        if (f) for (int k = 0; k < 3; k++) f[3 * (size_t)i + k] = fi[k];
        if (U) U[i] = u_i;
        if (W) W[i] = w_i;
        if (lapU) lapU[i] = l_i;
        if (fsq) fsq[i] = fi[0] * fi[0] + fi[1] * fi[1] + fi[2] * fi[2];
    }
}

/* integrators/NVE.py:59-105: leapfrog; K from the mean of the two half-step
 * velocities; PBC with image counters.  m is per particle. */
void orc_nve_step(int n, float *r, float *v, const float *f, const float *m, int32_t *img, const float *box,
                  float dt, float *K, float *fsq) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; i++) {
        float my_m = m[i];
        float k_i = 0.0f, fsq_i = 0.0f;
        for (int k = 0; k < 3; k++) {
            float fk = f[3 * (size_t)i + k];
            fsq_i += fk * fk;
            float v_mean = 0.0f;
            v_mean += v[3 * (size_t)i + k];
            v[3 * (size_t)i + k] += fk / my_m * dt;
            v_mean += v[3 * (size_t)i + k];
            v_mean /= 2.0f;
            k_i += 0.5f * my_m * v_mean * v_mean;
            r[3 * (size_t)i + k] += v[3 * (size_t)i + k] * dt;
        }
        orc_apply_pbc(r + 3 * (size_t)i, img + 3 * (size_t)i, box);
        if (K) K[i] = k_i;
        if (fsq) fsq[i] = fsq_i;
    }
}

/* Random numbers of integrators/NVT_Langevin.py:48 and :105, which are
 * numba.cuda.random's (numba 0.65.0, numba/cuda/random.py; a dependency of the
 * reference, not vendored in it): xoroshiro128+ with the (55, 14, 36) update
 * (xoroshiro128p_next); state 0 from SplitMix64 of the seed
 * (init_xoroshiro128p_state), state i = state i-1 advanced 2^64 steps by the
 * jump polynomial (init_xoroshiro128p_states_cpu, xoroshiro128p_jump);
 * uniform float32 = float32((x >> 11) * 2^-53) (uint64_to_unit_float32);
 * normal = sqrt(-2 log u1) cos(2 pi u2), float32, the first Box-Muller value
 * of two draws (xoroshiro128p_normal_float32). */
static uint64_t xr_rotl(uint64_t x, unsigned k) { return (x << k) | (x >> (64 - k)); }

uint64_t orc_xoro_next(uint64_t *s) {
    uint64_t s0 = s[0], s1 = s[1];
    uint64_t result = s0 + s1;
    s1 ^= s0;
    s[0] = xr_rotl(s0, 55) ^ s1 ^ (s1 << 14);
    s[1] = xr_rotl(s1, 36);
    return result;
}

static void xoro_jump(uint64_t *s) {
    static const uint64_t J[2] = {0xbeac0467eba5facbULL, 0xd86b048b86aa9922ULL};
    uint64_t a = 0, b = 0;
    for (int i = 0; i < 2; i++)
        for (int k = 0; k < 64; k++) {
            if (J[i] & (1ULL << k)) {
                a ^= s[0];
                b ^= s[1];
            }
            orc_xoro_next(s);
        }
    s[0] = a;
    s[1] = b;
}

/* states: n x 2 uint64 (s0, s1) */
void orc_xoro_init(int n, uint64_t seed, uint64_t *states) {
    if (n < 1) return;
    uint64_t z = seed + 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    z = z ^ (z >> 31);
    states[0] = z;
    states[1] = z;
    for (int i = 1; i < n; i++) {
        states[2 * (size_t)i] = states[2 * (size_t)i - 2];
        states[2 * (size_t)i + 1] = states[2 * (size_t)i - 1];
        xoro_jump(states + 2 * (size_t)i);
    }
}

float orc_xoro_uniform_f32(uint64_t *s) {
    return (float)((double)(orc_xoro_next(s) >> 11) * (1.0 / 9007199254740992.0));
}

float orc_xoro_normal_f32(uint64_t *s) {
    const float u1 = orc_xoro_uniform_f32(s);
    const float u2 = orc_xoro_uniform_f32(s);
    const float two_pi = (float)(2.0 * M_PI);
    return sqrtf(-2.0f * logf(u1)) * cosf(two_pi * u2);
}

/* integrators/NVT_Langevin.py:86-128: leap-frog Langevin (Gronbech-Jensen and
 * Farago, Eq. 16), per particle i (user order) and component k: one normal
 * from state i, beta = sqrt(2 alpha T dt) z, K from the velocity before the
 * update, v = a v + (b/m) f dt + (b/m) (beta + beta_old) / 2, r += v dt; then
 * periodic boundaries.  T is the thermostat temperature (float32). */
void orc_langevin_step(int n, float *r, float *v, const float *f, const float *m, int32_t *img, const float *box,
                       float dt, float alpha, float T, uint64_t *states, float *old_beta, float *K) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; i++) {
        const float my_m = m[i];
        float k_i = 0.0f;
        for (int k = 0; k < 3; k++) {
            const size_t e = 3 * (size_t)i + k;
            const float z = orc_xoro_normal_f32(states + 2 * (size_t)i);
            const float beta = sqrtf(2.0f * alpha * T * dt) * z;
            const float numerator = 2.0f * my_m - alpha * dt;
            const float denominator = 2.0f * my_m + alpha * dt;
            const float a = numerator / denominator;
            const float b_over_m = 2.0f / denominator;
            k_i += 0.5f * my_m * v[e] * v[e];
            v[e] = a * v[e] + b_over_m * f[e] * dt + b_over_m * 0.5f * (beta + old_beta[e]);
            old_beta[e] = beta;
            r[e] += v[e] * dt;
        }
        orc_apply_pbc(r + 3 * (size_t)i, img + 3 * (size_t)i, box);
        if (K) K[i] = k_i;
    }
}

/* integrators/NPT_Atomic.py (Martyna, Tobias and Klein thermostat-barostat,
 * leap-frog), its three parts in order.  State as the reference's float32
 * arrays: ts[0] = p_xi/Q, bs[0] = p_eps/W, bs[2] = volume; the K and W sums
 * (ts[1], bs[1] there, float32 atomics) are float64 sums here, rounded to
 * float32 where the reference reads the float32 accumulators.
 *
 * step (:104-136), per particle: factor = 0.5 dt ((1 + 3/degrees) bs0 + ts0)
 * in float64, plus = 1/(1 + factor) and minus = 1 - factor in float32,
 * rfactor = bs0 dt; v = plus (minus v + f/m dt), K += m v^2 / 2 (the new
 * half-step velocity), r += v dt + rfactor r, then periodic boundaries in the
 * box of the step.  Returns sum K; *wsum = sum W (the virial the force
 * evaluation wrote per particle). */
double orc_npt_step(int n, float *r, float *v, const float *f, const float *m, int32_t *img, const float *box,
                    float dt, float ts0, float bs0, long long degrees, const float *W, float *K, double *wsum) {
    const double factor = (double)(0.5f * dt) * ((1.0 + 3.0 / (double)degrees) * (double)bs0 + (double)ts0);
    const float plus = 1.0f / (float)(1.0 + factor);
    const float minus = (float)(1.0 - factor);
    const float rfactor = bs0 * dt;
    float *kbuf = (float *)malloc((size_t)n * sizeof(float));
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; i++) {
        const float my_m = m[i];
        float k_i = 0.0f;
        for (int k = 0; k < 3; k++) {
            const size_t e = 3 * (size_t)i + k;
            v[e] = plus * (minus * v[e] + f[e] / my_m * dt);
            k_i += 0.5f * my_m * v[e] * v[e];
            r[e] += v[e] * dt + rfactor * r[e];
        }
        orc_apply_pbc(r + 3 * (size_t)i, img + 3 * (size_t)i, box);
        kbuf[i] = k_i;
        if (K) K[i] = k_i;
    }
    double ks = 0.0, ws = 0.0;
    for (int i = 0; i < n; i++) {
        ks += kbuf[i];
        ws += W[i];
    }
    free(kbuf);
    *wsum = ws;
    return ks;
}

/* scale_box (:168-181): every coordinate times (1 + dt D bs0)^(1/3), in
 * float64, stored float32. */
void orc_npt_scale(int n, float *r, float dt, float bs0) {
    const double sf3 = 1.0 + (double)dt * 3.0 * (double)bs0;
    const double sf = pow(sf3, 1.0 / 3.0);
    for (size_t e = 0; e < 3 * (size_t)n; e++) r[e] = (float)(sf * (double)r[e]);
}

/* update_thermostat_barostat_state (:138-166) with the sums of the step: box
 * and volume scaled by the factor of scale_box, then the state equations of
 * the reference in its float32/float64 typing.  T_target, P_target: the
 * target functions at the step's time. */
void orc_npt_update(float *ts, float *bs, float *box, int n, long long degrees, float dt, float mass_t0,
                    float mass_p0, double ksum, double wsum, double T_target, double P_target) {
    const float ts1 = (float)ksum, bs1 = (float)wsum;
    const double temperature = 2.0 * (double)ts1 / (double)degrees;
    const double sf3 = 1.0 + (double)dt * 3.0 * (double)bs[0];
    const double mass_t = (double)mass_t0 * temperature;
    const double mass_p = (double)mass_p0 * temperature;
    bs[2] = (float)((double)bs[2] * sf3);
    const double sf = pow(sf3, 1.0 / 3.0);
    for (int k = 0; k < 3; k++) box[k] = (float)((double)box[k] * sf);
    const double p_inst = (temperature * (double)n + (double)bs1) / (double)bs[2];
    const double ke_dev = ((double)(2.0f * ts1) + (double)(bs[0] * bs[0]) * mass_p) /
                              ((double)(degrees + 1) * T_target) - 1.0;
    const double p_dev = 3.0 * ((double)bs[2] * (p_inst - P_target) + (double)(0.5f * ts1) / (double)degrees);
    ts[0] = (float)((double)ts[0] + (double)dt * ke_dev * (double)(degrees + 1) * T_target / mass_t);
    bs[0] = (float)((double)bs[0] + (double)dt * (p_dev / mass_p + (double)(ts[0] * bs[0])));
    ts[1] = 0.0f;
    bs[1] = 0.0f;
}

/* NPT state for orc_run_timeblock's integrator 3 (set before the call):
 * ts (2) and bs (3) float32 arrays, masses without the temperature factor
 * (NPT_Atomic.py:45-48), constant target pressure. */
static float *g_npt_ts = NULL, *g_npt_bs = NULL;
static float g_npt_mass_t = 0.0f, g_npt_mass_p = 0.0f, g_npt_P = 0.0f;
void orc_set_npt(float *ts, float *bs, float mass_t, float mass_p, float P) {
    g_npt_ts = ts;
    g_npt_bs = bs;
    g_npt_mass_t = mass_t;
    g_npt_mass_p = mass_p;
    g_npt_P = P;
}

/* Langevin state for orc_run_timeblock's integrator 2 (set before the call) */
static uint64_t *g_lv_states = NULL;
static float *g_lv_beta = NULL;
static float g_lv_alpha = 0.0f;
void orc_set_langevin(uint64_t *states, float *old_beta, float alpha) {
    g_lv_states = states;
    g_lv_beta = old_beta;
    g_lv_alpha = alpha;
}

/* integrators/NVT.py:75-111 (step) and :113-124 (update_thermostat_state).
 * state[0] = xi (float32), the kinetic-energy sum is returned in float64
 * (the reference accumulates it with float32 atomics into state[1]).
 * Returns sum_i K_i. */
double orc_nvt_step(int n, float *r, float *v, const float *f, const float *m, int32_t *img, const float *box,
                    float dt, float xi, float *K, float *fsq) {
    float factor = 0.5f * xi * dt;
    float plus = 1.0f / (1.0f + factor);
    float minus = 1.0f - factor;
    double ksum = 0.0;
    float *kbuf = (float *)malloc((size_t)n * sizeof(float));
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; i++) {
        float my_m = m[i];
        float k_i = 0.0f, fsq_i = 0.0f;
        for (int k = 0; k < 3; k++) {
            float fk = f[3 * (size_t)i + k];
            fsq_i += fk * fk;
            float vk = v[3 * (size_t)i + k];
            vk = plus * (minus * vk + fk / my_m * dt);
            v[3 * (size_t)i + k] = vk;
            k_i += 0.5f * my_m * vk * vk;
            r[3 * (size_t)i + k] += vk * dt;
        }
        orc_apply_pbc(r + 3 * (size_t)i, img + 3 * (size_t)i, box);
        kbuf[i] = k_i;
        if (K) K[i] = k_i;
        if (fsq) fsq[i] = fsq_i;
    }
    for (int i = 0; i < n; i++) ksum += kbuf[i];
    free(kbuf);
    return ksum;
}

/* NVT.py:119-123: ke_deviation = 2*sumK/(degrees*T) - 1 (float64 under
 * numba: degrees is an int64), xi += dt*omega2*ke_deviation stored float32. */
float orc_nvt_thermostat_update(float xi, double ksum, float dt, float omega2, long long degrees, float T) {
    double ke_dev = 2.0 * ksum / ((double)degrees * (double)T) - 1.0;
    double nx = (double)xi + (double)(dt * omega2) * ke_dev;
    return (float)nx;
}

/* runtime_actions/momentum_reset.py:57-78: v -= (sum m v)/(sum m). */
void orc_momentum_reset(int n, float *v, const float *m) {
    double p[3] = {0, 0, 0}, M = 0;
    for (int i = 0; i < n; i++) {
        for (int k = 0; k < 3; k++) p[k] += (double)m[i] * v[3 * (size_t)i + k];
        M += m[i];
    }
    float vcm[3];
    for (int k = 0; k < 3; k++) vcm[k] = (float)(p[k] / M);
    for (int i = 0; i < n; i++)
        for (int k = 0; k < 3; k++) v[3 * (size_t)i + k] -= vcm[k];
}

/*
 * One timeblock of the composed step loop (simulation/Simulation.py:330-346,
 * the kernel-launch form of :306-328): for step in 0..steps:
 *   neighbour-list check (nblist.py:57-86 / nblist_linked_lists.py:84-115)
 *   and rebuild; forces; if step < steps: integrate, then post-step actions
 *   ScalarSaver (scalar_saver.py:161-197) and MomentumReset
 *   (momentum_reset.py:84-103) in that order.
 *
 * integrator: 0 = NVE, 1 = NVT, 2 = NVT_Langevin (state from orc_set_langevin),
 * 3 = NPT_Atomic (state from orc_set_npt; box is updated in place).
 * nvt_state[0] = xi (in/out).
 * nblist_kind: 0 = N squared, 1 = linked lists.  r_ref / have_list carry the
 * list state across calls (have_list = 0 forces a build).
 * scal_out: (steps/every) x 4 doubles: U, W, K, lapU sums per saved step
 * (every = 0 disables saving).  Returns the number of rebuilds, or -1 on a
 * cell-grid error, -2 on neighbour-list overflow.
 */
int orc_run_timeblock(int n, float *r, float *v, float *f, const float *m, int32_t *img, const int32_t *ptype,
                      float *box, const float *params, int np, int nt, int kind, int cutmode,
                      int nblist_kind, float skin, int max_nbs, int32_t *nbl, float *r_ref, int *have_list,
                      int integrator, float dt, float *nvt_state, float omega2, float T, int steps, int every,
                      int reset_every, float *U, float *W, float *K, double *scal_out, int fma) {
    float max_cut = 0.0f;
    for (int a = 0; a < nt * nt; a++)
        if (params[(size_t)a * np + np - 1] > max_cut) max_cut = params[(size_t)a * np + np - 1];
    int rebuilds = 0;
    long long degrees = 3LL * n - 3;
    float *lap = (float *)malloc((size_t)n * sizeof(float));
    for (int step = 0; step <= steps; step++) {
        int need = !*have_list;
        if (!need) {
            for (int i = 0; i < n && !need; i++) {
                float d2 = dist_sq_dr(r + 3 * (size_t)i, r_ref + 3 * (size_t)i, box, NULL, fma);
                if (d2 > skin * skin * 0.25f) need = 1;
            }
        }
        if (need) {
            int mx;
            if (nblist_kind == 0) mx = orc_nblist_nsq(n, r, box, max_cut + skin, max_nbs, nbl, fma);
            else mx = orc_nblist_cells(n, r, box, max_cut, skin, max_nbs, nbl, fma);
            if (mx < 0) { free(lap); return -1; }
            if (mx >= max_nbs) { free(lap); return -2; }
            memcpy(r_ref, r, (size_t)n * 3 * sizeof(float));
            *have_list = 1;
            rebuilds++;
        }
        orc_forces(n, r, ptype, box, params, np, nt, kind, cutmode, nbl, max_nbs, f, U, W, lap, NULL, fma);
        if (step < steps) {
            if (integrator == 0) {
                orc_nve_step(n, r, v, f, m, img, box, dt, K, NULL);
            } else if (integrator == 2) {
                orc_langevin_step(n, r, v, f, m, img, box, dt, g_lv_alpha, T, g_lv_states, g_lv_beta, K);
            } else if (integrator == 3) {
                double ws = 0.0;
                const double ks = orc_npt_step(n, r, v, f, m, img, box, dt, g_npt_ts[0], g_npt_bs[0], degrees, W, K,
                                               &ws);
                orc_npt_scale(n, r, dt, g_npt_bs[0]);
                orc_npt_update(g_npt_ts, g_npt_bs, box, n, degrees, dt, g_npt_mass_t, g_npt_mass_p, ks, ws, (double)T,
                               (double)g_npt_P);
            } else {
                double ks = orc_nvt_step(n, r, v, f, m, img, box, dt, nvt_state[0], K, NULL);
                nvt_state[0] = orc_nvt_thermostat_update(nvt_state[0], ks, dt, omega2, degrees, T);
            }
            if (every > 0 && step % every == 0) {
                double su = 0, sw = 0, sk = 0, sl = 0;
                for (int i = 0; i < n; i++) { su += U[i]; sw += W[i]; sk += K[i]; sl += lap[i]; }
                double *row = scal_out + (size_t)(step / every) * 4;
                row[0] = su; row[1] = sw; row[2] = sk; row[3] = sl;
            }
            if (reset_every > 0 && step % reset_every == 0) orc_momentum_reset(n, v, m);
        }
    }
    free(lap);
    return rebuilds;
}

/* calculators/calculator_radial_distribution.py:76-107: all ordered pairs
 * i != j with dist_sq < (Lmin/2)^2 counted into bins[ti][tj][int(d/width)].
 * numba types: min_box_dim float32; (min_box_dim/2)/bins float64; the
 * comparison against (min_box_dim/2)**2 in float64; dist = sqrt(float32)
 * in float32; d/width in float64.  Counts are exact integers. */
void orc_rdf(int n, const float *r, const int32_t *ptype, const float *box, int nt, int bins, uint64_t *out,
             int fma, double r_max) {
    float minL = box[0] < box[1] ? box[0] : box[1];
    minL = minL < box[2] ? minL : box[2];
    /* r_max <= 0: the reference's range min(L)/2; otherwise a shorter range
     * with the same arithmetic (used to check the library's cell search) */
    double half = r_max > 0.0 ? r_max : (double)minL / 2.0;
    double width = half / (double)bins;
    double half_sq = half * half;
    size_t tot = (size_t)nt * nt * bins;
    memset(out, 0, tot * sizeof(uint64_t));
#pragma omp parallel
    {
        uint64_t *loc = (uint64_t *)calloc(tot, sizeof(uint64_t));
#pragma omp for schedule(dynamic, 16)
        for (int i = 0; i < n; i++) {
            int ti = ptype ? ptype[i] : 0;
            for (int j = 0; j < n; j++) {
                if (j == i) continue;
                float d2 = dist_sq_dr(r + 3 * (size_t)j, r + 3 * (size_t)i, box, NULL, fma);
                if ((double)d2 < half_sq) {
                    float d = sqrtf(d2);
                    if ((double)d < half) {
                        long long b = (long long)((double)d / width);
                        if (b >= bins) b = bins - 1;
                        int tj = ptype ? ptype[j] : 0;
                        loc[((size_t)ti * nt + tj) * bins + b] += 1;
                    }
                }
            }
        }
#pragma omp critical
        for (size_t a = 0; a < tot; a++) out[a] += loc[a];
        free(loc);
    }
}

/* calculators/calculator_structure_factor.py:185-196 ('CPU multi core'):
 * rho_q = N_f^-1/2 sum_n f_n exp(i q.r_n), N_f = sum f_n.  Evaluated here
 * in float64 throughout (the reference: float32 q.r, complex64 sums).
 * ff may be NULL (all ones). */
void orc_sq(int n, const float *r, const float *ff, int nq, const float *q, double *re, double *im) {
    double nf = 0.0;
    for (int i = 0; i < n; i++) nf += ff ? ff[i] : 1.0;
    double norm = 1.0 / sqrt(nf);
#pragma omp parallel for schedule(dynamic, 4)
    for (int a = 0; a < nq; a++) {
        double sr = 0.0, si = 0.0;
        double qx = q[3 * a], qy = q[3 * a + 1], qz = q[3 * a + 2];
        for (int i = 0; i < n; i++) {
            double ph = qx * r[3 * (size_t)i] + qy * r[3 * (size_t)i + 1] + qz * r[3 * (size_t)i + 2];
            double w = ff ? ff[i] : 1.0;
            sr += w * cos(ph);
            si += w * sin(ph);
        }
        re[a] = sr * norm;
        im[a] = si * norm;
    }
}
