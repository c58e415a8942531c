/*
 * gamdb200.h -- C ABI of libgamdb200.so, the B200 (sm_100a) implementation of
 * gamdpy's simulation hot path: pair-potential forces/virial/energy over a
 * neighbour list (N-squared or cell-list build), the NVE leapfrog, NVT
 * Nose-Hoover and NVT Langevin steps, the ScalarSaver/MomentumReset runtime
 * actions, and the radial-distribution and structure-factor calculators.
 *
 * Plain C: opaque handles, host pointers and sizes, int status codes
 * (GDB_OK == 0).  No torch or CUDA types appear in the signatures.  A handle
 * owns all of its device memory and one CUDA stream; calls on one handle must
 * come from one host thread at a time.
 *
 * Host arrays use gamdpy's layout (gamdpy/configuration/Configuration.py:
 * 141-146, colarray.py:45): positions/velocities/forces (N, 3) float32 row
 * major, masses (N,) float32, types (N,) int32, images (N, 3) int32, all in
 * the user's particle order.  Internally particles are kept in cell order
 * (cell-list mode); every download returns the user's order.
 *
 * Each entry point names the reference interface it replaces (paths relative
 * to the gamdpy project root).
 */
#ifndef GAMDB200_H
#define GAMDB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GDB_OK 0
#define GDB_ERR_ARG 1      /* bad argument (shape, kind, NULL handle) */
#define GDB_ERR_CUDA 2     /* a CUDA runtime call failed; see gdb_get_last_error */
#define GDB_ERR_STATE 3    /* call order (e.g. run before upload) */
#define GDB_ERR_NBLIST 4   /* neighbour-list overflow (count >= max_nbs) */
#define GDB_ERR_NUMERIC 5  /* non-finite position seen by a kernel */
#define GDB_ERR_UNSUPPORTED 6
#define GDB_ERR_TIMEOUT 7  /* a bounded wait inside a kernel gave up (status bit BARRIER_TIMEOUT) */

/* status-word bits (gdb_status_word), set by kernels, cleared by gdb_clear_status */
#define GDB_STATUS_NBLIST_OVERFLOW 0x1u
#define GDB_STATUS_BARRIER_TIMEOUT 0x2u
#define GDB_STATUS_NAN 0x4u
#define GDB_STATUS_BAD_ARG 0x8u
#define GDB_STATUS_CLUSTER_CAPACITY 0x10u /* a list outgrew the cluster path's shared memory (rerun on the global path) */
#define GDB_STATUS_BAD_INDEX 0x20u /* a cell-sort slot outside [0, n): the access was skipped */
#define GDB_STATUS_BRICK_CAPACITY 0x40u /* a brick's halo outgrew shared memory (the run goes on without bricks) */

/* potentials: gamdpy/interactions/potential_functions/ */
#define GDB_POT_LJ_SIGMA_EPSILON 0 /* LJ_12_6_sigma_epsilon.py:6-36, params (sigma, epsilon, cut) */
#define GDB_POT_LJ_12_6 1          /* LJ_12_6.py:3-41, params (A12, A6, cut) */
/* cutoff wrappers */
#define GDB_CUT_SHIFTED_FORCE 0     /* apply_shifted_force_cutoff.py:30-37 */
#define GDB_CUT_SHIFTED_POTENTIAL 1 /* apply_shifted_potential_cutoff.py:42-47 */
/* neighbour lists */
#define GDB_NBLIST_NSQ 0   /* interactions/nblist.py NbList2 */
#define GDB_NBLIST_CELLS 1 /* interactions/nblist_linked_lists.py NbListLinkedLists */
/* integrators */
#define GDB_INTEGRATOR_NVE 0 /* integrators/NVE.py */
#define GDB_INTEGRATOR_NVT 1 /* integrators/NVT.py */
#define GDB_INTEGRATOR_LANGEVIN 2 /* integrators/NVT_Langevin.py */
#define GDB_INTEGRATOR_NPT 3 /* integrators/NPT_Atomic.py */
/* NVT target temperature T(t): misc/make_function.py */
#define GDB_TFUNC_CONSTANT 0 /* make_function_constant :6-13, tparams = {T} */
#define GDB_TFUNC_RAMP 1     /* make_function_ramp :16-34, tparams = {T0, t0, T1, t1} */

/* column order of gdb_get_scalar_rows: sums over particles per saved step */
#define GDB_SCALAR_U 0
#define GDB_SCALAR_W 1
#define GDB_SCALAR_LAPU 2
#define GDB_SCALAR_K 3
#define GDB_SCALAR_FSQ 4
#define GDB_SCALAR_VOL 5 /* box volume after the step: NPT_Atomic runs only (zero otherwise) */
#define GDB_NUM_SCALARS 6

typedef struct gdb_sim gdb_sim;

/* Library version (major*10000 + minor*100 + patch). */
int gdb_version(void);

/* Number of visible CUDA devices. */
int gdb_device_count(int *count);
/* Name of CUDA device `device` (for the autotuner's per-GPU cache; no
 * reference counterpart). */
int gdb_device_name(int device, char *buf, int n);

/* Create a simulation of n particles and ntypes particle types on `device`.
 * Replaces Configuration.copy_to_device's allocations and the per-object
 * cuda.to_device calls of PairPotential/NbList/integrators
 * (configuration/Configuration.py:227-234, interactions/nblist.py:14-18). */
int gdb_sim_create(int n, int ntypes, int device, gdb_sim **out);
int gdb_sim_destroy(gdb_sim *h);

/* Orthorhombic box lengths (simulation_boxes/orthorhombic.py:25-29). */
int gdb_set_box(gdb_sim *h, const float lengths[3]);

/* Host -> device copy of the full state (Configuration.copy_to_device,
 * configuration/Configuration.py:227-234).  r_im may be NULL (zeros).
 * Marks the neighbour list for rebuild. */
int gdb_upload_state(gdb_sim *h, const float *r, const float *v, const float *m, const int32_t *ptype,
                     const int32_t *r_im);

/* Device -> host copy (Configuration.copy_to_host, Configuration.py:236-243).
 * Any pointer may be NULL.  Synchronises the handle's stream. */
int gdb_download_state(gdb_sim *h, float *r, float *v, float *f, int32_t *r_im);

/* Per-particle scalars of the last force evaluation / integration step in
 * gamdpy's columns (Configuration.py:109-131).  Any pointer may be NULL. */
int gdb_download_scalars(gdb_sim *h, float *U, float *W, float *lapU, float *K, float *Fsq);

/* The whole state in one call, in the host arrays of gamdpy's Configuration
 * (Configuration.copy_to_host, configuration/Configuration.py:236-243):
 * vectors is the (3, n, 3) float32 r, v, f column array (colarray.py:45),
 * r_im (n, 3) int32, scalars the (n, nscal) float32 table whose columns
 * cols[0..5] hold U, W, lapU, K, Fsq and the mass (-1 = column absent;
 * Configuration.py:109-131).  One kernel unpacks every plane into device
 * staging laid out as those arrays, then one copy per array; from pinned
 * host memory (gdb_host_alloc) the copies run at DMA speed.  Any array may
 * be NULL.  Synchronises the handle's stream. */
int gdb_download_table(gdb_sim *h, float *vectors, int32_t *r_im, float *scalars, int nscal, const int32_t cols[6]);

/* Page-locked host memory (cudaHostAlloc, portable across devices) for the
 * host arrays of a Configuration attached to a device, so uploads and
 * downloads copy without staging through pageable pages.  No counterpart in
 * the reference, whose host arrays are numpy's (numba copies through its own
 * staging).  gdb_host_free releases it. */
int gdb_host_alloc(size_t bytes, void **out);
int gdb_host_free(void *p);

/* Pair potential table (PairPotential.convert_user_params,
 * interactions/pair_potential.py:23-51): params is ntypes*ntypes rows of
 * nparams float32 (row-major [i][j][p]); the last parameter is the cut. */
int gdb_set_pair_potential(gdb_sim *h, int kind, int cutmode, int ntypes, const float *params, int nparams);

/* Neighbour-list algorithm, skin and capacity (PairPotential.get_params,
 * pair_potential.py:84-97; compute_plan['nblist'], ['skin']). */
int gdb_set_nblist(gdb_sim *h, int kind, float skin, int max_nbs);

/* Pair exclusions (PairPotential(..., exclusions), interactions/
 * pair_potential.py:12-20, tested in the list builds at
 * interactions/nblist.py:120-123 and nblist_linked_lists.py:174-178): excl is
 * the (n, max_excl + 1) int32 table of user indices with the count last, as
 * Bonds.get_exclusions returns it (interactions/bonds.py:137-150); excluded
 * pairs never enter the neighbour list.  NULL removes the table.  Systems with
 * exclusions or bonds run on the grid kernels, not the thread-block-cluster
 * or staged-halo paths. */
int gdb_set_exclusions(gdb_sim *h, const int32_t *excl, int max_excl);

/* Harmonic bonds (interactions/bonds.py:12-135 with
 * potential_functions/harmonic_bond_function.py:6-43): indices (nbonds, 3)
 * int32 rows (i, j, bond type) of user indices, params (ntypes, 2) float32
 * rows (r0, k).  u = k (r - r0)^2 / 2 per bond, half to each end; the bond
 * forces are added in the fused step before the integration.  nbonds = 0
 * removes them. */
int gdb_set_bonds(gdb_sim *h, int nbonds, const int32_t *indices, int ntypes, const float *params);

/* Threads per particle (compute_plan['tp'], simulation/get_default_compute_plan.py:55-63):
 * 1, 2, 4, 8, 16 or 32 lanes share one particle's neighbours; 0 = choose.
 * pb (particles per block): for systems on the thread-block-cluster path
 * (N <= 4096), about pb particles per CTA (at most 256); 0 = choose (spread
 * over 16 CTAs). */
int gdb_set_plan(gdb_sim *h, int tp, int pb);

/* Integrators: NVE.get_params (integrators/NVE.py:29-31);
 * NVT.get_params (integrators/NVT.py:33-37). */
int gdb_set_integrator_nve(gdb_sim *h, float dt);
int gdb_set_integrator_nvt(gdb_sim *h, float dt, float tau, int tfunc, const float *tparams);

/* NVT_Langevin (integrators/NVT_Langevin.py:44-53 get_params, :86-128 step):
 * leap-frog Langevin with friction alpha and temperature tfunc/tparams (as
 * gdb_set_integrator_nvt).  One xoroshiro128+ generator per particle (user
 * index), seeded as numba.cuda.random.create_xoroshiro128p_states(N, seed);
 * the stored random forces start at zero.  Runs on the persistent and graph
 * paths (not on thread-block clusters, not in batches). */
int gdb_set_integrator_langevin(gdb_sim *h, float dt, float alpha, uint64_t seed, int tfunc, const float *tparams);

/* The Langevin state in user order (no counterpart in the reference, whose
 * rng_states and old_beta device arrays live inside the integrator's
 * parameters, NVT_Langevin.py:48-50): states n x 2 uint64 (s0, s1) and the
 * previous random forces n x 3 float32; either pointer may be NULL. */
int gdb_get_langevin_state(gdb_sim *h, uint64_t *states, float *old_beta);
/* NVT.thermostat_state = {xi, sumK} (integrators/NVT.py:30). */
int gdb_get_thermostat_state(gdb_sim *h, float state[2]);
int gdb_set_thermostat_state(gdb_sim *h, const float state[2]);

/* NPT_Atomic (integrators/NPT_Atomic.py:38-50 get_params, :104-136 step,
 * :138-166 thermostat/barostat update, :168-181 box scaling): leap-frog with
 * the Martyna-Tobias-Klein thermostat and barostat.  mass_t and mass_p are
 * the reference's masses without the temperature factor (float32, computed
 * by the caller as get_params does); target temperature tfunc/tparams and
 * target pressure pfunc/pparams take the forms of gdb_set_integrator_nvt.
 * The box changes every step (gdb_get_box reads it back); the cell grid is
 * recomputed from the current box at every list build, within the grid
 * allocated for the box at gdb_set_nblist (the reference keeps the initial
 * grid).  Runs on the persistent kernel only (not on thread-block clusters,
 * not in batches); per-particle virials are evaluated every step. */
int gdb_set_integrator_npt(gdb_sim *h, float dt, float mass_t, float mass_p, int tfunc, const float *tparams,
                           int pfunc, const float *pparams);
/* NPT_Atomic.thermostat_state = {p_xi/Q, 0} and barostat_state =
 * {p_eps/W, 0, volume} (integrators/NPT_Atomic.py:35-36); set_npt_state
 * with a NULL pointer leaves that part unchanged.  The volume of a new
 * simulation is the box's. */
int gdb_get_npt_state(gdb_sim *h, float ts[2], float bs[3]);
int gdb_set_npt_state(gdb_sim *h, const float ts[2], const float bs[3]);
/* The current box lengths (changed by NPT runs). */
int gdb_get_box(gdb_sim *h, float lengths[3]);

/* Runtime actions compiled into the step: ScalarSaver(steps_between_output)
 * (runtime_actions/scalar_saver.py:161-197) and MomentumReset(steps_between_reset)
 * (runtime_actions/momentum_reset.py:84-103); 0 disables. */
int gdb_set_runtime_actions(gdb_sim *h, int scalar_every, int momentum_every);

/* ConfigurationSaver (runtime_actions/configuration_saver.py:21-141): keep
 * positions and images at steps 0, 1, 2, 4, ..., 2^k of every timeblock
 * (log-spaced, taken before that step's integration) in conf_per_block frames
 * of layout (conf_per_block, 2, n, 3) float32 = {r, r_im as float} in user
 * order.  conf_per_block = int(log2(steps_per_timeblock)) + 2; 0 disables. */
int gdb_set_configuration_saver(gdb_sim *h, int conf_per_block);
/* Frames saved during the last timeblock (same layout as above). */
int gdb_get_saved_configurations(gdb_sim *h, float *out, int conf_per_block);
/* The box of each saved frame (ConfigurationSaver(include_simbox=True),
 * configuration_saver.py:47-51, 137-139): conf_per_block x 3 float32, the
 * box lengths at the step the frame was taken (they change under NPT_Atomic). */
int gdb_get_saved_boxes(gdb_sim *h, float *out, int conf_per_block);

/* One evaluation of the interactions on the current state: neighbour-list
 * check/rebuild, then forces, U, W, lapU (Evaluator.evaluate,
 * tools/Evaluator.py:82-94; interactions/pair_potential.py:250-268). */
int gdb_eval_forces(gdb_sim *h);

/* One timeblock: `steps` integration steps plus the final force evaluation
 * (simulation/Simulation.py:306-346 via integrate_self :271-282).  time_zero
 * is the simulated time at the block start.  Returns GDB_ERR_NBLIST on
 * overflow and GDB_ERR_NUMERIC on non-finite positions.  If ms != NULL the
 * block's device time (CUDA events) is stored there. */
int gdb_sim_run(gdb_sim *h, double time_zero, int steps, float *ms);

/* Measurement: build a list for the current state, then launch the fused
 * step kernel `reps` times alone (no rebuild chain, runtime actions off)
 * between CUDA events on the handle's stream; *ms_per_launch = average
 * duration.  Advances the state; intended for benchmarks (the reference
 * times whole timeblocks with CUDA events, simulation/Simulation.py:404-448). */
int gdb_time_step_kernel(gdb_sim *h, int reps, float *ms_per_launch);

/* Phase trace of the persistent step kernel (tracing aid; no counterpart in
 * the reference, which times whole timeblocks only): with capacity > 0,
 * every grid barrier appends (tag << 56 | globaltimer ns); tags: 1 step,
 * 2 final evaluation, 3 rebuild phase, 4 rebuild done, 5 kernel start.
 * gdb_get_trace copies up to `capacity` entries, sets *count and restarts
 * the trace.  capacity 0 switches tracing off. */
int gdb_set_trace(gdb_sim *h, int capacity);
int gdb_get_trace(gdb_sim *h, unsigned long long *out, int capacity, int *count);

/* Mean and maximum neighbour count of the current list (per particle). */
int gdb_nblist_stats(gdb_sim *h, double *mean_count, int *max_count);

/* ScalarSaver rows of the last timeblock: rows x GDB_NUM_SCALARS doubles
 * (sums over particles, float64).  rows = steps / scalar_every. */
int gdb_get_scalar_rows(gdb_sim *h, double *out, int rows);

/* Neighbour list in gamdpy's layout (interactions/nblist.py:8): (n, max_nbs+1)
 * int32, user indices, count in the last column. */
int gdb_get_nblist(gdb_sim *h, int32_t *out, int max_nbs);

/* gamdpy's nbflag (nblist.py:9): {update pending, max count if overflowed
 * else 0, number of rebuilds}. */
int gdb_get_nbflag(gdb_sim *h, int32_t out[3]);

/* Which implementation ran the last gdb_sim_run: 0 CUDA-graph launch
 * sequence, 1 persistent cooperative kernel, 2 thread-block cluster
 * (N <= 4096 with fewer than about 160 000 list entries, N x the neighbours
 * expected from the density; environment GDB_CLUSTER=1: whenever N <= 4096
 * fits, GDB_CLUSTER=0: never), 3 global-memory cluster (batches), 4 the
 * persistent kernel with staged halos (environment GDB_BRICKS=1: cells
 * numbered in bricks of 4 x 4 x 4, each brick's halo copied into shared
 * memory by bulk copies, 16-bit lists; cell lists from 131 073 particles,
 * GDB_BRICK_MIN_N moves the size; off by default, measured slower than the
 * row path on B200), -1 none yet.
 * Diagnostic; no counterpart in the reference. */
int gdb_get_last_path(gdb_sim *h);

/* Status bits set by kernels since the last clear; gdb_clear_status resets. */
uint32_t gdb_status_word(gdb_sim *h);
int gdb_clear_status(gdb_sim *h);

/* Last error message of the handle (or of the library when h == NULL). */
int gdb_get_last_error(gdb_sim *h, char *buf, int n);

/* Radial distribution counts of the current state, added into out
 * (ntypes x ntypes x bins uint64, exact integer counts).  r_max <= 0 means
 * min(L)/2, the reference's range (calculators/calculator_radial_distribution.py:
 * 76-107, update :111-119). */
int gdb_rdf_update(gdb_sim *h, int bins, double r_max, uint64_t *out);

/* Collective density of the current state for q = 2 pi n / L
 * (calculators/calculator_structure_factor.py:131-156 GPU kernel, :185-203
 * CPU backends): rho_q = N_f^-1/2 sum_i f_i exp(i q.r_i), N_f = sum f_i.
 * n_vectors: nq x 3 int32; ff: n float32 in user order or NULL (all 1). */
int gdb_sq_update(gdb_sim *h, int nq, const int32_t *n_vectors, const float *ff, double *rho_re,
                  double *rho_im);

/* Device time in ms (CUDA events on the handle's stream) of the handle's
 * last gdb_rdf_update or gdb_sq_update call: its device work, from the first
 * copy or kernel to the last kernel (the result's copy back not included).  A measurement aid with no
 * counterpart in the reference, which times its calculators with wall
 * clocks around update() (e.g. examples/structure_factor.py). */
int gdb_last_analysis_ms(gdb_sim *h, float *ms);

/* Stand-alone calculators on host arrays (no handle): same semantics as the
 * two calls above, for callers that only hold a configuration
 * (CalculatorRadialDistribution.update / CalculatorStructureFactor.update). */
int gdb_rdf_compute(int n, const float *r, const int32_t *ptype, const float box[3], int ntypes, int bins,
                    double r_max, uint64_t *out);
int gdb_sq_compute(int n, const float *r, const float *ff, const float box[3], int nq, const int32_t *n_vectors,
                   double *rho_re, double *rho_im);

/* Trajectory dynamics (tools/calc_dynamics.py:6-75) of ConfigurationSaver
 * frames: frames num_blocks x conf_per_block x 2 x n x 3 float32 (positions,
 * then image counts; the `block` dataset), ptype n int32 in [0, ntypes),
 * ntypes <= 8, box the initial box, qvalues ntypes float64.  Lags as the
 * reference: frame i+1 against frame 0 of each block from first_block on,
 * then first frames 2^(i+1) blocks apart; total_times = conf_per_block - 1 +
 * int(log2(num_blocks - first_block)) - 1.  Outputs total_times x ntypes
 * float64 msd, m4d (mean dr^4) and fs (mean cos(q dr) over particles and
 * components), already divided by count (total_times int32). */
int gdb_calc_dynamics(int num_blocks, int conf_per_block, int n, const float *frames, const int32_t *ptype,
                      int ntypes, const float box[3], int first_block, const double *qvalues, int total_times,
                      double *msd, double *m4d, double *fs, int32_t *count);

/* Batched replicas (no counterpart in the reference, whose users loop over
 * state points one Simulation at a time, e.g. examples/isomorph.py:27-82):
 * advance many independent, fully configured and uploaded systems together.
 * Systems of up to 4096 particles run one thread-block cluster each, grouped
 * into one launch per cluster shape; larger systems run their persistent
 * kernels concurrently on their own streams with a share of the GPU.  All
 * systems need the same device, number of types and integrator; sizes,
 * boxes, parameters and temperatures may differ.  gdb_batch_run is one
 * timeblock for every system (as gdb_sim_run) and returns the first error;
 * per-system results are read from each handle as usual. */
typedef struct gdb_batch gdb_batch;
/* particles_per_cta: cluster shaping target (about that many particles per
 * CTA, at most 256, up to 16 CTAs per system); 0 = the single-system default
 * (spread over 16 CTAs, at least 32 particles each), so a system gives the
 * same bits in a batch as alone.  Tuned by SimulationBatch.autotune. */
int gdb_batch_create(gdb_sim *const *sims, int count, int particles_per_cta, gdb_batch **out);
/* As gdb_batch_create, with the shape of the systems above 4096 particles
 * (which run the persistent phases on thread-block clusters with state in
 * global memory, one 1024-thread CTA per SM): about clg_particles_per_cta
 * particles per CTA (1 to 16 CTAs a system; 0 = the smallest count from 4096
 * up whose CTAs fit the SMs left by the smaller systems' share of the
 * particles) and clg_tp lanes per particle (1, 2, 4 or 8; 0 = 1).  Tuned by
 * SimulationBatch.autotune. */
int gdb_batch_create_ex(gdb_sim *const *sims, int count, int particles_per_cta, int clg_particles_per_cta,
                        int clg_tp, gdb_batch **out);
int gdb_batch_run(gdb_batch *b, double time_zero, int steps, float *ms);
int gdb_batch_destroy(gdb_batch *b);
int gdb_batch_get_last_error(gdb_batch *b, char *buf, int n);

/* S(q) without any device allocation.  No counterpart in the reference: it
 * serves callers that cannot let the library call cudaMalloc -- programs whose
 * own allocator or pre-reserved pool owns the GPU's memory, code under a hard
 * device-memory budget, and call sites where allocating is not allowed.
 * Inputs and outputs are the caller's DEVICE arrays: r_dev (n, 3) float32,
 * ff_dev (n,) float32 or NULL (all 1), n_vectors_dev (nq, 3) int32 with every
 * component in [-n_max, n_max], rho_re_dev / rho_im_dev (nq,) float64.  box is
 * a host array.  stream is a cudaStream_t (NULL = default stream).  Every
 * call synchronizes `stream` before it returns: it reads back a flag that
 * reports n-vector components outside [-n_max, n_max].  Limits: nq <= 65536,
 * n_max <= 48.  Scratch is one static device array of 0.5 MiB that every GPU
 * loading the library keeps until exit; it is shared by all calls on a
 * device, so calls that overlap on the GPU (other streams, other host
 * threads) race and must be serialized by the caller.  The first call on a
 * device looks up the array's address and should come before any stream
 * capture; the address is kept for the life of the process, so the device's
 * primary context must not be reset (cudaDeviceReset) between calls. */
int gdb_sq_compute_noalloc(int n, const float *r_dev, const float *ff_dev, const float box[3], int nq,
                           const int32_t *n_vectors_dev, int n_max, double *rho_re_dev, double *rho_im_dev,
                           void *stream);

/* Self-test of the bounded wait of the persistent kernels' grid barrier (no
 * reference counterpart): a two-block kernel whose second block never
 * arrives; the first gives up after `cycles` SM clock cycles and sets
 * GDB_STATUS_BARRIER_TIMEOUT, returned in *status.  The device stays usable. */
int gdb_selftest_barrier_timeout(int device, long long cycles, unsigned *status);

/* ---- adjoint: gradients of trajectory averages w.r.t. pair parameters ----
 * No counterpart in the reference (gamdpy has no differentiation).  The
 * forward is the NVE leapfrog of integrators/NVE.py:78-97 with the
 * shifted-force Lennard-Jones of LJ_12_6_sigma_epsilon.py:26-36 and
 * apply_shifted_force_cutoff.py:30-37, pairs over all j (the NbList2 set),
 * float32 state with float64 sums.  Observables (time averages over the
 * `steps` steps n = 0..steps-1): obs[0] = <U>, obs[1] = <W>, obs[2] = <K>
 * (sums over particles; K from the mean of the half-step velocities, as NVE),
 * obs[3 + b] = <g_AA(r_b)>, a Gaussian-kernel radial distribution of type-0
 * pairs on every rdf_every-th step, bin centres r_lo + (b + 1/2)(r_hi - r_lo)/bins.
 * The backward is the discrete adjoint of that forward: a reverse sweep with
 * Hessian-vector products of the pair forces, recomputing each segment from
 * checkpoints kept every checkpoint_every steps. */
typedef struct gdb_adj gdb_adj;
int gdb_adj_create(int n, int ntypes, int device, gdb_adj **out);
int gdb_adj_destroy(gdb_adj *h);
/* box lengths, types (n int32), masses (n float32), time step, steps,
 * checkpoint interval; RDF bins (0 = none, at most 128), range, kernel width
 * and sampling interval. */
int gdb_adj_setup(gdb_adj *h, const float box[3], const int32_t *ptype, const float *mass, float dt, int steps,
                  int checkpoint_every, int rdf_bins, float rdf_lo, float rdf_hi, float rdf_width, int rdf_every);
/* params: ntypes*ntypes rows of (sigma, epsilon, cut) as double, symmetric;
 * r0, v0: (n, 3) float32 host arrays.  obs: 3 + rdf_bins doubles. */
int gdb_adj_forward(gdb_adj *h, const double *params, const float *r0, const float *v0, double *obs);
/* grad_obs: dL/dobs (3 + rdf_bins doubles) -> grad_params, ntypes*ntypes rows
 * of (dL/dsigma, dL/depsilon, 0); entry (a, b) holds the derivative with
 * respect to the shared parameter of the unordered pair {a, b}. */
int gdb_adj_backward(gdb_adj *h, const double *grad_obs, double *grad_params);
/* Truncated adjoint: window W > 0 treats the state at every multiple of W
 * steps as a constant, so each observable term is differentiated through at
 * most W steps of the trajectory (the exact gradient of a chaotic trajectory
 * grows like exp(lambda t)); 0 (the default) = the exact adjoint. */
int gdb_adj_set_window(gdb_adj *h, int window);
/* State after the forward's last step (either pointer may be NULL). */
int gdb_adj_final_state(gdb_adj *h, float *r, float *v);
int gdb_adj_get_last_error(gdb_adj *h, char *buf, int n);

#ifdef __cplusplus
}
#endif
#endif
