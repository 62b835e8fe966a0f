/*
 * lemc.h -- C-ABI boundary of the LaughlinEdge B200 engine (sm_100a).
 *
 * Every entry point takes plain pointers and sizes and returns an int status
 * (LEMC_OK == 0, negative on failure).  Nothing here calls exit(); the C++
 * drop-in layer (include/modules/*.h) maps a non-zero status back onto the
 * reference's print-and-exit(1) behaviour.
 *
 * Citations name the reference interface each entry point replaces, as
 * <file within the LaughlinEdge project>:<line>.
 *
 * Conventions
 *  - Complex matrices are row-major, interleaved (re, im) doubles, D x D.
 *  - Positions are interleaved (x, y) floats, walker-major: xy[(w*N + i)*2 + c].
 *  - A context owns its device buffers and one CUDA stream; it is not
 *    thread-safe.  Host buffers are always owned by the caller.
 */
#ifndef LEMC_H
#define LEMC_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define LEMC_API __attribute__((visibility("default")))
#else
#define LEMC_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define LEMC_OK 0
#define LEMC_ERR_ARG (-1)       /* invalid argument / configuration          */
#define LEMC_ERR_CAPACITY (-2)  /* a size exceeds a compiled capacity bound  */
#define LEMC_ERR_CUDA (-3)      /* a CUDA runtime call failed                */
#define LEMC_ERR_TIMEOUT (-4)   /* a bounded device wait gave up             */
#define LEMC_ERR_NUMERIC (-5)   /* non-positive metric / failed factorisation */
#define LEMC_ERR_STATE (-6)     /* call made in the wrong order              */
#define LEMC_ERR_NODEVICE (-7)  /* no CUDA device visible                    */
#define LEMC_ERR_IO (-8)        /* file could not be read or written         */

/* ---- compiled capacity bounds ------------------------------------------ */
#define LEMC_MAX_DEGREE 24      /* largest power-sum degree k (max Delta L)  */
#define LEMC_MAX_PARTICLES 1024
#define LEMC_MAX_GUIDE_PARTS 8  /* distinct parts of a guide partition       */
#define LEMC_MAX_PROBES 8       /* angular probes l of the cos/sin planes      */

/* ---- enumerations ------------------------------------------------------ */
enum lemc_guide {
  LEMC_GUIDE_LAUGHLIN = 0, /* sample |Psi_m|^2; all rows share one chain       */
  LEMC_GUIDE_ROW = 1       /* sample |P_a Psi_m|^2 per basis row a (reference) */
};
enum lemc_gram_mode {
  LEMC_GRAM_FP64 = 0,   /* SIMT FP64 accumulation (the exact accumulation)     */
  LEMC_GRAM_BF16X3 = 1, /* tcgen05 kind::f16, hi/lo split, 3 products         */
  LEMC_GRAM_BF16X4 = 2, /* tcgen05 kind::f16, hi/lo split, 4 products         */
  LEMC_GRAM_TF32X3 = 3  /* tcgen05 kind::tf32, hi/lo split, 3 products        */
};
/* weight planes recorded per measurement (rows of the record buffer) */
enum lemc_weight {
  LEMC_W_ONE = 0,    /* sample weight of the guide (1 for the Laughlin guide)  */
  LEMC_W_R2 = 1,     /* sum_i |z_i|^2                                           */
  LEMC_W_R4 = 2,     /* sum_i |z_i|^4                                           */
  LEMC_W_USER = 3,   /* caller-supplied per-sample potential U(z) (hook)        */
  LEMC_W_PROBE0 = 4, /* plane 4+2q: sum_i cos(l_q theta_i); 5+2q: sin(l_q theta_i) */
  LEMC_N_WEIGHTS = LEMC_W_PROBE0 + 2 * LEMC_MAX_PROBES
};

/* ---- configuration ------------------------------------------------------ */
typedef struct lemc_config {
  int32_t particles;        /* N                                              */
  int32_t inverse_filling;  /* m (nu = 1/m)                                   */
  int32_t n_walkers;        /* W, independent Markov chains                  */
  int32_t lanes_per_walker; /* G in {1,2,4,8,16,32}; 0 = heuristic, -1 = autotuned at
                               lemc_init_walkers by timing every feasible G, and
                               (tensor-core modes) the contraction's walker split
                               at the first measured sweep                      */
  float step_sigma;         /* Gaussian single-particle step (l_B)           */
  int32_t guide;            /* enum lemc_guide                               */
  uint64_t seed;            /* Philox-4x32-10 key                            */
  double radius_scale;      /* R of (z/R)^k in p_k; <= 0 selects sqrt(2 m N) */
  double init_radius;       /* walkers start uniform in this disk; <=0: sqrt(2mN) */
  int32_t gram_mode;        /* enum lemc_gram_mode                           */
  int32_t graph_batch;      /* >0: measured sweeps run as CUDA-graph replays of this
                               many sweeps (sweep, basis, contraction each); results
                               are identical to direct launches.  0: direct launches */
  int32_t flush_every;      /* tcgen05 path: K-chunks per FP64 flush (0=auto) */
  int32_t profile;          /* 1: time each kernel family with CUDA events   */
} lemc_config;

/* Statistics of a context after lemc_run(). */
typedef struct lemc_stats {
  uint64_t sweeps;          /* sweeps executed per walker                     */
  uint64_t measurements;    /* measurements accumulated per walker            */
  double acceptance;        /* accepted / proposed single-particle moves       */
  double tau_int;           /* max integrated autocorrelation time of p_1..p_4 (sweeps) */
  double tau_int_each[4];   /* per observable |p_k|, k = 1..4                 */
  double ms_sweep;          /* device time of the sweep kernels (ms, total)   */
  double ms_basis;          /* device time of the basis build (ms, total)     */
  double ms_gram;           /* device time of the S/H contraction (ms, total) */
  double reverse_fraction;  /* learned proposal: share of proposed moves whose reverse
                               density was evaluated (the others could not be accepted
                               whatever it is); 0 for the Gaussian step                */
} lemc_stats;

/* One row of the basis returned by lemc_partitions(): the compressed partition
 * (part, multiplicity) pairs, in the reference's order.                     */
typedef struct lemc_partition_row {
  int32_t dL;        /* angular momentum carried by the partition           */
  int32_t sector_size;
  int32_t n_pairs;   /* number of distinct parts                             */
  int32_t pairs_off; /* offset into the pairs array (2 ints per pair)        */
} lemc_partition_row;

typedef struct lemc_ctx lemc_ctx;

/* ---- library / device ---------------------------------------------------- */
LEMC_API int lemc_version(void);
LEMC_API const char* lemc_status_string(int status);
/* Number of visible CUDA devices (0 with LEMC_ERR_NODEVICE when none). */
LEMC_API int lemc_device_count(int* count);

/* ---- basis enumeration (host only) ------------------------------------------
 * Replaces iparts::integer_partitions (modules/integer_partitions.h:25-93,
 * modules/partitions/integer_partitions.cu:10-47, :79-140, :199-226): the
 * partitions of each dL, restricted to at most `particles` parts, compressed
 * to (part, multiplicity) pairs ordered by ascending multiplicity, listed in
 * accelerated-ascending generation order.  Call with rows == NULL to size.  */
LEMC_API int lemc_partitions(int particles, const int32_t* sectors, int n_sectors,
                    lemc_partition_row* rows, int max_rows, int32_t* pairs,
                    int max_pair_ints, int* n_rows, int* n_pair_ints,
                    int* max_degree, int* longest_compressed);

/* ---- context ------------------------------------------------------------
 * Replaces the per-call set-up of edgeMC::spectrum_compute
 * (modules/edge_mc/em_spectrum.cu:210-252): device limits, RNG states,
 * partitions on the device and the capacity checks.                         */
LEMC_API int lemc_create(const lemc_config* cfg, lemc_ctx** out);
LEMC_API int lemc_destroy(lemc_ctx* ctx);
/* Gaussian step sigma of subsequent sweeps (step tuning). */
LEMC_API int lemc_set_step(lemc_ctx* ctx, float sigma);
/* Tune the Gaussian step to an acceptance within tol of target: measure the
 * acceptance of `moves` unmeasured sweeps of the live chain at the current
 * step, double or halve the step until the target is bracketed, then regula
 * falsi on the bracket (at most 40 + 60 measurements).  The walkers advance and
 * the accumulators are reset.  On success the context keeps the step, and
 * *sigma / *acceptance (may be NULL) receive it and its last measured
 * acceptance; LEMC_ERR_NUMERIC when the search fails.  Replaces optimal_step
 * and mcmc_acceptanceBisection (modules/edge_mc/em_bisection.cu:7-153). */
LEMC_API int lemc_tune_step(lemc_ctx* ctx, double target, double tol, int moves, float* sigma,
                            double* acceptance);
/* Walker width G in use (after autotuning). */
LEMC_API int lemc_lanes_per_walker(const lemc_ctx* ctx, int* lanes);
/* Walker split of the tensor-core contraction (jobs = tiles x split; 0 before
 * the first contraction without autotuning). */
LEMC_API int lemc_gram_splits(const lemc_ctx* ctx, int* splits);
/* Select the angular-momentum sectors whose basis is sampled. */
LEMC_API int lemc_set_sectors(lemc_ctx* ctx, const int32_t* sectors, int n_sectors);
/* Guide rows for LEMC_GUIDE_ROW: walker w samples |P_{rows[w % n]}|^2 |Psi|^2,
 * rows index the basis of the selected sectors.  NULL selects every row. */
LEMC_API int lemc_set_guide_rows(lemc_ctx* ctx, const int32_t* rows, int n_rows);
/* Angular probes l_0..l_{n-1} (n <= LEMC_MAX_PROBES): every measurement records
 * sum_i cos(l_q theta_i) and sum_i sin(l_q theta_i), and the cross-sector blocks
 * between sectors whose dL differ by l_q are accumulated with those weights
 * (edge density Fourier components, reference em_edgeResponse.tpp:136-163,
 * and the dynamic structure factor, em_dsf.cu:101-117). */
LEMC_API int lemc_set_probes(lemc_ctx* ctx, const int32_t* l, int n);
/* Built-in excitation potential for the USER weight plane, in place of a hook:
 * U(z) = amplitude * sum_i r_i^k cos(k theta_i) = amplitude * Re sum_i z_i^k,
 * formed on the device from the recorded power sums at every measured sweep
 * (k <= the basis' largest degree; k = 0 switches it off).  The cross-sector
 * sums of lemc_read_cross then hold <f|U|g>.  This is the multipole drive
 * delta V = eps r^k cos(k theta) f(t) of the edge-response pipeline (the
 * reference's excitationResponse_compute with such a lambda,
 * em_edgeResponse.tpp:26-194); the temporal profile f enters the evolution. */
LEMC_API int lemc_set_multipole_potential(lemc_ctx* ctx, int k, double amplitude);
/* Initial walker positions; host_xy == NULL draws them uniformly in the
 * init disk from the Philox stream (replaces particle_positions_initialize,
 * modules/edge_mc/em_markovchain.cu:223-263). */
LEMC_API int lemc_init_walkers(lemc_ctx* ctx, const float* host_xy);
/* Advance every walker n_sweeps sweeps.  measure != 0 records a sample after
 * each sweep and accumulates S, H2, H4 (and the row sums for LEMC_GUIDE_ROW).
 * Replaces burnin + hamiltonian_sampler (em_markovchain.cu:266-334,
 * em_spectrum.cu:16-136) and the mcmc_* launches (em_spectrum.cu:139-208). */
LEMC_API int lemc_run(lemc_ctx* ctx, int n_sweeps, int measure);
/* Per-step hook for a caller-defined potential U(z): after each measured
 * sweep the library calls hook(user, xy, u, W, N, stream) with device
 * pointers to the walker positions (W x N interleaved x,y floats) and to the
 * LEMC_W_USER weight plane (W floats, to be written with U of each walker) on
 * the context's stream, before the S/H/cross accumulation of that step.  A
 * non-zero return aborts the run with that status.  Replaces the device
 * lambda argument of excitationResponse_compute (em_edgeResponse.tpp:26-194). */
typedef int (*lemc_step_hook)(void* user, const float* dev_xy, float* dev_user_plane, int W,
                              int N, void* stream);
LEMC_API int lemc_run_hooked(lemc_ctx* ctx, int n_sweeps, lemc_step_hook hook, void* user);
/* Zero every accumulator (samples, Gram matrices, series, acceptance) and the
 * context's device error word (after LEMC_ERR_TIMEOUT the context is usable
 * again once reset). */
LEMC_API int lemc_reset_accumulators(lemc_ctx* ctx);
/* Bounded waits of the tensor-core contraction.  Every mbarrier wait of
 * gram_tc_kernel gives up after `cycles` SM clocks (0 restores the default,
 * about 2 s); the kernel then records LEMC_ERR_TIMEOUT in the context's error
 * word, waits (bounded) for its own copies and MMAs in flight, frees its
 * tensor memory and exits, and lemc_synchronize / the read calls return
 * LEMC_ERR_TIMEOUT.  hold_loads != 0 keeps the kernel's loader from issuing
 * any copy, so that every wait expires: a test hook for that path (process
 * wide, for launches made afterwards).  No counterpart in the reference. */
LEMC_API int lemc_debug_gram_wait(long long cycles, int hold_loads);
LEMC_API int lemc_synchronize(lemc_ctx* ctx);
/* The context's CUDA stream (cudaStream_t), for callers that order their own
 * work or device timers after the context's kernels. */
LEMC_API int lemc_stream(lemc_ctx* ctx, void** stream);

/* Basis dimension of a selected sector and of all selected sectors. */
LEMC_API int lemc_sector_dim(const lemc_ctx* ctx, int sector_index, int* dim);
LEMC_API int lemc_total_dim(const lemc_ctx* ctx, int* dim);

/* Raw Gram sums of one selected sector, complex D x D interleaved:
 *   S[a][b]  = sum_samples w1 * conj(v_a) v_b
 *   H2[a][b] = sum_samples w1 * (sum_i |z_i|^2) conj(v_a) v_b
 *   H4[a][b] = sum_samples w1 * (sum_i |z_i|^4) conj(v_a) v_b
 * with v_a = prod_j p_{lambda_j}, p_k = sum_i (z_i / R)^k.  Any output may be
 * NULL.  *n_samples receives the number of accumulated samples.
 * Range: the device holds each state's values times a range factor c_a (the
 * inverse geometric mean of |v_a| over the walkers at the first measured sweep
 * of the basis, Laughlin guide), so that FP32 values and accumulations stay
 * O(1) in every sector; the sums returned here are divided by c_a c_b.  A
 * non-finite sum is returned with LEMC_ERR_NUMERIC (outputs still written).
 * Replaces the device->host copy and block averaging of em_spectrum.cu:256-359. */
LEMC_API int lemc_read_gram(lemc_ctx* ctx, int sector_index, double* S, double* H2,
                   double* H4, double* n_samples);
/* Raw cross-sector sums between two different selected sectors (Da x Db):
 *   Cuser[a][b] = sum w1 U conj(v_a) v_b,
 *   Ccos[a][b]  = sum w1 (sum_i cos l theta_i) conj(v_a) v_b,
 *   Csin[a][b]  = sum w1 (sum_i sin l theta_i) conj(v_a) v_b,
 * l = |dL_b - dL_a|; Ccos/Csin are zero unless l is a probe.  Any output may
 * be NULL.  Range factors are undone and non-finite sums reported as in
 * lemc_read_gram.  Used by the dynamic structure factor (em_dsf.cu:18-158) and the
 * excitation response (em_edgeResponse.tpp:26-194). */
LEMC_API int lemc_read_cross(lemc_ctx* ctx, int sector_a, int sector_b, double* Cuser,
                             double* Ccos, double* Csin);
/* Reference-estimator row averages (LEMC_GUIDE_ROW), D x D over all selected
 * rows, each averaged over the samples of the walkers guided by row a:
 *   fg[a][b] = <v_b/v_a>, gg[a][b] = <|v_b/v_a|^2> (real),
 *   fh[a][b] = <V(z) v_b/v_a> with V = omega r^2 + kappa r^4 given here,
 *   fcos/fsin[a][b] = <sum_i cos/sin(l_0 theta_i) v_b/v_a> (first probe),
 *   fuser[a][b] = <U(z) v_b/v_a> (hooked runs).  Outputs may be NULL.
 * Replaces results.fg_ff/gg_ff/fHg_ff (modules/edge_montecarlo.h:15-33). */
LEMC_API int lemc_read_rows(lemc_ctx* ctx, double omega, double kappa, double* fg,
                   double* gg, double* fh, double* fcos, double* fsin, double* fuser,
                   double* n_samples_per_row);
LEMC_API int lemc_read_stats(lemc_ctx* ctx, lemc_stats* st);
LEMC_API int lemc_read_positions(lemc_ctx* ctx, float* host_xy);
/* Walker-mean series of Re/Im p_1..p_4 per measurement: series[m*8 + 2(k-1) + c]. */
LEMC_API int lemc_read_series(lemc_ctx* ctx, double* series, int max_meas, int* n_meas);

/* ---- bins and jackknife error bars -------------------------------------------
 * The reference leaves error bars to repetitions of whole runs, each saved as
 * a numbered .tsv (main.cu:18-20, em_spectrum.cu:393-414).  Here one run is cut
 * into bins: lemc_close_bin ends the current bin at the measurements made
 * since the previous close (LEMC_GUIDE_LAUGHLIN; a bin must hold at least one
 * measurement, and should span many autocorrelation times).  Bins are kept on
 * the host (3 D_s^2 complex FP64 per sector each) until
 * lemc_reset_accumulators. */
LEMC_API int lemc_close_bin(lemc_ctx* ctx);
LEMC_API int lemc_n_bins(const lemc_ctx* ctx, int* n_bins);
/* Raw Gram sums of one bin and sector, as lemc_read_gram. */
LEMC_API int lemc_read_gram_bin(lemc_ctx* ctx, int bin, int sector_index, double* S, double* H2,
                                double* H4, double* n_samples);
/* Jackknife (leave one bin out) over n_bins bins of raw Gram sums of one
 * sector (S, H2, H4: [n_bins][D][D] complex, interleaved): evals of the full
 * sums (normalised as lemc_normalise, solved as lemc_geneig) and their
 * standard errors; M_err, H_err (D x D real, may be NULL) the errors of the
 * normalised matrix entries (modulus of the complex deviation).  Host only. */
LEMC_API int lemc_jackknife_spectrum(int D, int n_bins, const double* S, const double* H2,
                                     const double* H4, double omega, double kappa, double eps,
                                     double* evals, double* evals_err, double* M_err,
                                     double* H_err);

/* ---- error analysis of a scalar Monte Carlo series (host only) -------------
 * The reference leaves error bars to post-processing of repeated runs
 * (main.cu:18-20, em_spectrum.cu:393-414); these give them from one run.
 * Sokal's windowed integrated autocorrelation time: tau = 1/2 + sum_{t<=M}
 * rho(t) with the smallest window M >= c tau (c <= 0 selects 5).  *tau is NaN
 * when no window up to T/2 qualifies, T < 100 or T < 50 max(tau, 1): the series is too short
 * for its own autocorrelation time, and no estimate is claimed.  lemc_stats
 * reports this estimate (max over Re/Im p_1..p_4), NaN under the same rule. */
LEMC_API int lemc_tau_sokal(const double* x, int T, double c, double* tau);
/* Binning analysis: bins of length 2^k while at least min_bins bins remain
 * (<= 0 selects 16); tau(b) = b s_b^2 / (2 s_1^2) at the last level, its error,
 * the standard error of the series mean from that level, and *converged = 1
 * when the last two levels agree within twice the error (or 5 %). */
LEMC_API int lemc_tau_binning(const double* x, int T, int min_bins, double* tau,
                              double* tau_err, double* err_of_mean, int* converged);

/* ---- device-buffer entry points (the hot path, for integrators/tests) ------
 * All pointers are device pointers; `stream` is a cudaStream_t (NULL = legacy).
 * One sweep-kernel launch: n_sweeps sweeps of W walkers starting at global
 * sweep index sweep0, then (measure != 0) one measurement record.
 *   pos      [W][N] float2, in/out
 *   rec_p    [K][W] float2, p_k for k = 1..K  (out, measure != 0)
 *   rec_w    [4 + 2 n_probes][W] float       (out, measure != 0; USER plane = 0)
 *   accepted [W] uint32, accumulated          (in/out, may be NULL)       */
LEMC_API int lemc_sweep_device(void* pos, int W, int N, int m, float sigma,
                      uint64_t seed, uint32_t sweep0, int n_sweeps, int K,
                      double radius_scale, int lanes_per_walker, int measure,
                      const int32_t* probes, int n_probes, void* rec_p, void* rec_w,
                      void* accepted, void* stream);
/* Basis build: V[row][w] (float, row stride ldv >= W) for the rows of the
 * selected sectors of ctx, from records rec_p [K][W]. */
LEMC_API int lemc_basis_device(lemc_ctx* ctx, const void* rec_p, int W, void* V,
                      int ldv, void* stream);
/* Accumulate raw Gram sums of ctx's sectors from V (rows x ldv) and rec_w
 * into the device accumulator of ctx using the given mode. */
LEMC_API int lemc_gram_device(lemc_ctx* ctx, const void* V, const void* rec_w, int W,
                     int ldv, int gram_mode, void* stream);

/* ---- learned proposal (DeepSets network, exact Metropolis-Hastings) ---------
 * No counterpart in the reference, whose sampler moves one particle by an
 * isotropic Gaussian step.  A lemc_proposal holds the weights of a small
 * permutation-invariant network: the 16 nearest-neighbour displacements of
 * the moving particle in its local radial/tangential frame -> phi (2 -> 64,
 * ReLU) -> mean, with r/R - 1 appended -> rho (65 -> 64, ReLU -> 4) =
 * (mu_r, mu_t, log s_r, log s_t) of the proposed move z' = z + Rot(theta)(mu
 * + s eps).  A context using it (lemc_set_proposal) accepts with the exact
 * ratio |Psi(z')|^2 q(z|z') / (|Psi(z)|^2 q(z'|z)), so it samples |Psi_m|^2
 * for any weights.  The scales are clamped to s in [1, 4] (units of l_B); the
 * lower bound gives ln q(z|z') <= 0, so a sweep skips the reverse network for
 * moves that ln u already rejects (lemc_stats.reverse_fraction reports the
 * share it evaluated) with unchanged decisions.  Weights: FP32 master copy,
 * BF16 copy used by the kernels.  particles <= 256; Laughlin guide only. */
typedef struct lemc_proposal lemc_proposal;
typedef struct lemc_train_config {
  int32_t steps;      /* Adam steps */
  int32_t batch;      /* (configuration, particle, eps) samples per objective estimate */
  int32_t pairs;      /* antithetic parameter perturbations per step */
  float lr;           /* Adam learning rate */
  float es_sigma;     /* perturbation scale of the evolution-strategies gradient */
  uint64_t seed;      /* Philox key of samples and perturbations */
} lemc_train_config;
/* Number of network parameters (FP32 layout W1[64][2], b1[64], W2[64][65], b2[64],
 * W3[4][64], b3[4]). */
LEMC_API int lemc_proposal_n_params(int* n);
/* New proposal initialised to the plain isotropic step init_sigma (clamped to
 * [1, 4]; hidden weights random from seed, output weights near zero). */
LEMC_API int lemc_proposal_create(int particles, int inverse_filling, float init_sigma,
                                  uint64_t seed, lemc_proposal** out);
LEMC_API int lemc_proposal_destroy(lemc_proposal* p);
LEMC_API int lemc_proposal_get_params(const lemc_proposal* p, float* host, int n);
/* Replace the weights (also resets the Adam state). */
LEMC_API int lemc_proposal_set_params(lemc_proposal* p, const float* host, int n);
/* For n (configuration, particle, eps) samples (host arrays: xy [n][particles][2],
 * particle [n], eps [n][2]) write out[s][8] = {mu_r, mu_t, log s_r, log s_t,
 * z'.x, z'.y, ln A, |z'-z|^2} as the sampler computes them (BF16 weights). */
LEMC_API int lemc_proposal_eval(const lemc_proposal* p, const float* host_xy, int n,
                                const int32_t* particle, const float* eps, float* out);
/* Maximise E[min(1, A) |z'-z|^2] over configurations `configs` (device array
 * [n_cfg][particles] of float2, e.g. snapshots of a plain-proposal context via
 * lemc_copy_positions_device): per step 2*pairs antithetic weight
 * perturbations evaluated on `batch` common samples give an
 * evolution-strategies gradient for one Adam step.  trace[s] (host, may be NULL)
 * receives the mean objective of step s. */
LEMC_API int lemc_proposal_train(lemc_proposal* p, const void* configs, int n_cfg,
                                 const lemc_train_config* cfg, double* trace);
/* Use proposal p for the context's sweeps (NULL: the plain Gaussian step).
 * p must outlive its use; particles and inverse filling must match. */
LEMC_API int lemc_set_proposal(lemc_ctx* ctx, const lemc_proposal* p);
/* Copy the context's walker positions ([W][N] float2) to device memory dst,
 * ordered on the context stream. */
LEMC_API int lemc_copy_positions_device(lemc_ctx* ctx, void* dst);

/* ---- occupation numbers (two-state walker) -------------------------------
 * <f_L| a^dagger_l a_l |f_R> for every ordered pair (L, R) of basis rows of
 * sector dL, l < l_cutoff.  Each walker carries N+1 particles: particle 0
 * belongs to the bra only, particle N to the ket only, 1..N-1 to both; the
 * sampled weight is |f_L(z_0..z_{N-1})| |f_R(z_1..z_N)| and the estimator per
 * sample is sum_l exp(-ln(2 pi l!) + l ln(z_0 conj(z_N) / 2)
 * - (|z_0|^2 + |z_N|^2)/4 + i phase), phase = arg(P_R/P_L)
 * + m arg prod_{i=1}^{N-1} (z_i - z_N)/(z_0 - z_i).
 * out[((L*D + R)*l_cutoff + l)*2 + {0,1}] receives the per-pair averages (not
 * normalised to N).  Walkers are split into equal contiguous blocks per pair.
 * Replaces greenFunctionMC::occupation_numbers_sampler and on_compute
 * (modules/green_function/gf_occupation_numbers.cu:16-239, :309-544). */
typedef struct lemc_occupation_config {
  int32_t particles, inverse_filling, dL, l_cutoff;
  int32_t n_walkers;
  float step_sigma;
  uint64_t seed;
  int32_t burn_in, sweeps;
} lemc_occupation_config;
LEMC_API int lemc_occupation(const lemc_occupation_config* cfg, double* out, double* acceptance);

/* Allocation-free form of lemc_occupation.  It has no counterpart in the
 * reference: the reference allocates and frees its device buffers inside
 * every call.  This form is for callers that must not allocate device memory
 * during the call, for example a process whose device memory is already
 * owned by a caching allocator (cudaMalloc would fail there), or a loop that
 * cannot take the device-wide synchronisation of cudaFree.
 *
 * Same arguments, kernels, results and status codes as lemc_occupation (the
 * same seed gives the same output).  All device memory it uses is one fixed
 * static device array of LEMC_OCC_STATIC_SCRATCH_BYTES per device, holding:
 *   - the row table;
 *   - 4*W bytes of acceptance counters;
 *   - 16*l_cutoff*W bytes of per-walker sums;
 *   - 16*D*D*l_cutoff bytes of per-pair sums (D = basis size of sector dL).
 * Each part is rounded up to 256 bytes.  A configuration that needs more
 * returns LEMC_ERR_CAPACITY before any device work.  The call makes no
 * cudaMalloc or cudaFree and no allocating library call.
 *
 * Set-up: the first call on each device resolves the array's device address
 * with that device current (cudaGetSymbolAddress), which can load the module
 * onto the device.  Make that first call before any stream capture.
 *
 * Footprint: the array is part of the library's device module, so its
 * LEMC_OCC_STATIC_SCRATCH_BYTES are reserved on every device where the module
 * is loaded (by any entry point of the library, not only this one), until the
 * process exits.
 *
 * Concurrency: every call on one device uses the same array, so calls that
 * overlap on the same device (from several host threads) race and corrupt
 * each other's results.  Serialise them.  The call itself is synchronous, as
 * lemc_occupation is. */
#define LEMC_OCC_STATIC_SCRATCH_BYTES (64u << 20)
LEMC_API int lemc_occupation_static(const lemc_occupation_config* cfg, double* out,
                                    double* acceptance);

/* Edge spectral function of sector dL as energy-resolved orbital occupations:
 * the occupation matrices occ (lemc_occupation's per-pair averages, D x D x
 * Lc complex) normalised with the metric as the reference normalises them
 * (gf_occupation_numbers.cu:432-445) and Hermitised per l, rotated onto the
 * generalized eigenvectors c_j of H c = E M c (normalised H, M of the same
 * sector, c^H M c = 1):
 *   weights[j][l] = Re c_j^H n_l c_j,  sum_l weights[j][l] = N,
 * with energies[j] ascending (*n_modes = kept rank; later rows NaN).
 * A(l, E) = sum_j weights[j][l] delta(E - E_j) is the spectral weight of
 * angular-momentum orbital l at edge energy E.  The reference announces a
 * spectral function on its two-state walker but leaves it unimplemented
 * (README.md:14-15; the commented spectral_function_sampler,
 * green_function.h:90); this is the rotation onto the eigenvector basis that
 * its occupation output asks for (gf_occupation_numbers.cu:512).  Host only. */
LEMC_API int lemc_spectral_weights(int D, int Lc, const double* occ, const double* H,
                                   const double* M, int N, double eps, double* energies,
                                   double* weights, int* n_modes);

/* ---- FP64 dense tail ----------------------------------------------------
 * Generalized Hermitian eigenproblem H c = E M c (complex D x D, interleaved).
 * Eigenvalues ascending; eigenvectors (optional, column j = vector j) are
 * M-normalised (c^H M c = 1).  M is factorised by Cholesky; when M is not
 * positive definite the directions with eigenvalues below eps * max are
 * dropped and *rank reports the kept dimension (evals beyond rank = NaN).
 * Replaces ges::generalizedEigenproblem::extract_spectrum and
 * extract_dsf_coefficients (modules/eigensolver/generalized_eigenproblem.cpp:45-95). */
LEMC_API int lemc_geneig(int D, const double* H, const double* M, double eps,
                double* evals, double* evecs, int* rank);

/* Edge dynamic structure factor from the normalised matrices of the sectors
 * {0, dL} (D = 1 + D_dL, row 0 the Laughlin state; complex D x D, interleaved):
 * the generalized problem of the dL block, H[1:,1:] c = E M[1:,1:] c with
 * c^H M c = 1 (eigenvalues ascending), and the weight of mode j,
 * |sum_a (Vc - i Vs)[0][a+1] c_j[a]|^2 (Vc, Vs: the cos / sin(dL theta)
 * excitation matrices).  energies and weights receive D - 1 entries, *n_modes
 * the kept rank (weights beyond it NaN).  Replaces
 * ges::generalizedEigenproblem::extract_dsf_coefficients
 * (modules/eigensolver/generalized_eigenproblem.cpp:54-95). */
LEMC_API int lemc_dsf_weights(int D, const double* H, const double* M, const double* Vc,
                              const double* Vs, double eps, double* energies, double* weights,
                              int* n_modes);

/* Generalized spectra of one sector for n confinement strengths, computed on
 * the GPU in FP64 (the kappa sweep of the batched form).  S, H2, H4 are the raw
 * Gram sums of lemc_read_gram (D x D complex, interleaved); for each j the
 * problem is H_j c = E M c with M and H_j normalised and Hermitised as in
 * lemc_normalise, H_j = omega[j] H2 + kappa[j] H4.  M is factorised once by
 * canonical orthogonalisation: directions with metric eigenvalue <= eps * max
 * are dropped (*rank = kept dimension; evals beyond it are NaN).
 * evals[j*D + k] ascending.  Replaces ges::generalizedEigenproblem
 * (modules/eigensolver/generalized_eigenproblem.cpp:38-95) called once per
 * strength. */
LEMC_API int lemc_geneig_sweep(int D, const double* S, const double* H2, const double* H4,
                               const double* omega, const double* kappa, int n, double eps,
                               double* evals, int* rank);

/* Normalised matrices from raw Gram sums (reference convention,
 * em_spectrum.cu:331-335 and the Hermitisation at :383-390):
 *   M[a][b] = S[a][b] / sqrt(S[a][a] S[b][b]),
 *   H[a][b] = (omega H2 + kappa H4)[a][b] / sqrt(S[a][a] S[b][b]),
 * both made Hermitian as (X + X^H)/2.  Any output may be NULL. */
LEMC_API int lemc_normalise(int D, const double* S, const double* H2, const double* H4,
                   double omega, double kappa, double* M, double* H);

/* ---- time evolution (FP64) ------------------------------------------------
 * dC/dt = -i M^-1 (H + f(t) U) C, C(0) = e_0, integrated by the embedded
 * Cash-Karp RK5(4) pair with error control (abs 1e-10, rel 1e-8) and sampled
 * at t = s * save_step, s < ceil(end_time / save_step):
 *   out[s][l] = C^H rho_l C (complex), norms[s] = Re C^H M C.
 * rho holds L matrices D x D.  f(t, user) is the temporal profile.
 * Replaces timeEvolution::edgeDensityResponse_compute
 * (modules/dynamics/dynamics.cpp:24-53, :73-125, :280-290). */
typedef double (*lemc_profile_fn)(double t, void* user);
LEMC_API int lemc_evolve(int D, const double* M, const double* H, const double* U,
                int L, const double* rho, lemc_profile_fn f, void* user,
                double end_time, double save_step, double* out, double* norms,
                int* n_save);

/* The same evolution on the GPU in FP64, in the S-orthonormal basis of the
 * canonical orthogonalisation of M (directions with metric eigenvalue <=
 * eps * max dropped; *rank = kept dimension): C = X y, dy/dt = -i (X^H H X
 * + f(t) X^H U X) y with the trace mean of X^H H X removed as a global phase,
 * classical RK4 with step save_step / substeps.  f is evaluated on the host at
 * every stage time before the integration starts.  Outputs as lemc_evolve.
 * Replaces the host integration of timeEvolution::edgeDensityResponse_compute
 * (modules/dynamics/dynamics.cpp:149-308) for fixed-step propagation. */
LEMC_API int lemc_evolve_device(int D, const double* M, const double* H, const double* U,
                                int L, const double* rho, lemc_profile_fn f, void* user,
                                double end_time, double save_step, int substeps, double eps,
                                double* out, double* norms, int* n_save, int* rank);

/* Edge density response on an angular grid, from the Fourier components
 * <rho_l>(t) = C^H rho_l C of the evolution (rho_t: [n_times][L] complex,
 * interleaved, angular momenta l[q] >= 0):
 *   out[t][g] = (1/2pi) [ d_0 + 2 Re sum_{l>0} e^{-i l theta_g} d_l(t) ],
 *   d_l(t) = <rho_l>(t) - rho_ref[l], theta_g = 2 pi g / n_theta,
 * rho_ref (L complex) NULL selects rho_t[0] (the response to the drive).
 * Computed on the GPU in FP64.  Completes the reference's
 * edgeDensityResponse_compute, which stops at the components
 * (modules/dynamics/dynamics.cpp:110-125, :293-306). */
LEMC_API int lemc_edge_density_grid(int L, const int32_t* l, int n_times, const double* rho_t,
                                    const double* rho_ref, int n_theta, double* out);

#ifdef __cplusplus
}
#endif
#endif /* LEMC_H */
