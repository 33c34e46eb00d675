/*
 * plomgpu: C ABI of the sm_100a sequential Monte Carlo engine for one
 * generated plom model.
 *
 * One shared library is built per model (libplomgpu_<model>.so), as the
 * reference builds one libplomtpl.a per model (model_builder/C/templates/
 * Makefile:9-14).  Every library exports the same symbols; the model's
 * dimensions are compile-time constants reported by plomgpu_get_model_info().
 *
 * All arrays are plain host pointers in row-major order; sizes follow from
 * the descriptor's J / n_obs / n_sub and from plomgpu_get_model_info().  No call
 * exits the process: every entry point returns a status code
 * (PLOMGPU_OK = 0) and plomgpu_last_error() describes the last failure of
 * the calling thread.  The reference terminates with print_err + exit
 * (model_builder/C/core/print.c:247-268) instead.
 */
#ifndef PLOMGPU_H
#define PLOMGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum plomgpu_status {
    PLOMGPU_OK = 0,
    PLOMGPU_EINVAL = 1,      /* bad argument or size */
    PLOMGPU_ECUDA = 2,       /* CUDA runtime error */
    PLOMGPU_ENOMEM = 3,      /* device allocation failed */
    PLOMGPU_ETIMEOUT = 4,    /* a bounded device wait ran out (the filter result is invalid) */
    PLOMGPU_ENODEV = 5       /* no CUDA device */
};

/* noises_off bits, same values as enum plom_noises_off (model_builder/C/core/plom.h:66) */
enum plomgpu_noises_off {
    PLOMGPU_NO_DEM_STO = 1 << 0,
    PLOMGPU_NO_ENV_STO = 1 << 1,
    PLOMGPU_NO_DRIFT = 1 << 2
};

typedef struct plomgpu_model_info {
    int n_par_sv, n_c, n_ac, n_cac;
    int n_ts, n_ts_inc_unique, n_obs_inc, n_obs_prev;
    int n_drift;          /* drifted parameters; each owns n_cac state words */
    int off_drift, off_inc, n_state;   /* state layout: [sv*cac | drift*cac | incidences] */
    int n_par_proc, n_par_obs, n_cov_cac, n_cov_ts;
    int n_reac, n_white_noise;
    int coupled;          /* 1 if the model reads a cac x cac coupling matrix */
    int pop_size_eq_sum_sv;
    const char *name;
    int n_hat;            /* rows of the filtered summaries: n_par_sv*n_cac [+ n_cac remainders] + n_ts + n_drift*n_cac */
} plomgpu_model_info;

/* Back-transform of one group of a drifted parameter (back_transform_x,
 * model_builder/C/core/transform.c:462-481). f_inv: 0 id, 1 exp, 2 inv-logit,
 * 3 inv-logit_ab; scale: 0 id, 1 pow10, 2 pow10 of the negative. */
typedef struct plomgpu_back_transform {
    int f_inv;
    int scale;
    int is_duration;
    int pad;
    double a, b;
    double multiplier;
} plomgpu_back_transform;

/* One particle filter (the arguments of run_SMC, model_builder/C/core/smc.c:204-210,
 * flattened to arrays). */
typedef struct plomgpu_smc_desc {
    int J;                    /* particles */
    int n_obs;                /* observation intervals (nb_obs) */
    const int *n_sub;         /* [n_obs] Euler substeps in interval n */
    const double *t_sub;      /* [sum n_sub] start time of every substep (t += dt replayed on the host) */
    const double *t_obs;      /* [n_obs] end time t1 of interval n (time of observation n) */
    double dt;                /* integration step (1/round(1/dt), build.c:1303) */
    const double *data;       /* [n_obs][n_ts]; NaN = missing */
    const double *par_cac;    /* [n_par_proc][n_cac] natural process parameters */
    const double *par_ts;     /* [n_par_obs][n_ts] natural observation parameters */
    const double *cov_cac;    /* [sum n_sub][n_cov_cac][n_cac] covariates at the substep times */
    const double *cov_ts;     /* [n_obs][n_cov_ts][n_ts] observation covariates at t_obs */
    const double *coupling;   /* [n_cac][n_cac] or NULL when the model is not coupled */
    const int *drift_group;   /* [n_drift][n_cac] group of each cac, or NULL */
    const int *drift_ngroups; /* [n_drift] */
    const plomgpu_back_transform *drift_bt;  /* [n_drift][n_cac] per group */
    const double *drift_vol;  /* [n_drift][n_cac] volatility per group (natural) */
    const double *x0;         /* [n_state] initial particle (replicated to all J) */
    int noises_off;           /* plomgpu_noises_off bits */
    int filter;               /* 0 = propagate only (smc -t) */
    double like_min;          /* LIKE_MIN (smc -l), default 1e-17 */
    uint64_t seed;            /* Philox key; ignored with CRN draws */
    int precision;            /* 32: FP32 state and log-weights; 64: FP64 everywhere */
                              /* (with CRN draws in precision 32 the injected normals are rounded to FP32) */
    /* Common random numbers (optional): when crn_normals is set, every normal
     * is read from it: [n][j][k][d] for interval n, particle j, substep k and
     * draw d < plomgpu_draws_per_substep(noises_off) in the reference's draw
     * order (cac-major, dem_sto__* then white_noise__*, then drift words
     * [n_drift][n_cac]).  crn_uniforms[n] in [0,1) gives the systematic
     * resampling offset U = u/J of interval n. */
    const double *crn_normals;
    const double *crn_uniforms;
    /* Inputs of the filtered summaries, read only when result.hat or
     * result.pred_res is requested:
     * [n_obs + 1][n_cac] population size N at 0 and at every t_obs, for the
     * remainder rows (models with a remainder compartment);
     * [n_cov_ts][n_ts] observation covariates at time 0 (models with
     * observation covariates). */
    const double *pop_size;
    const double *cov_ts0;
    /* Deterministic skeleton, the reference's "ode" implementation
     * (f_prediction_ode, model_builder/C/core/prediction_util.c:176-193): when
     * ode is 1 the process is integrated without noise by an embedded
     * Runge-Kutta-Fehlberg 4(5) pair with step control (eps_abs, eps_rel;
     * every interval starts from the step dt) and noises_off is ignored.  The
     * process covariates are then evaluated at every stage time from their
     * interpolants: cov_spline_meta [n_cov_cac * n_cac][3] = kind (0 constant,
     * 1 linear, 2 natural cubic), number of knots, offset into the knot
     * arrays x / y / m2 (second derivatives) of total length cov_spline_knots. */
    int ode;
    double eps_abs, eps_rel;
    const int *cov_spline_meta;
    const double *cov_spline_x;
    const double *cov_spline_y;
    const double *cov_spline_m2;
    int cov_spline_knots;
    /* 1: Poisson system with stochastic rates, the reference's default "psr"
     * implementation (step_psr, model_builder/C/templates/core_template.c:
     * 105-209): multinomial splits of the integer compartments, Poisson
     * arrivals, Gamma white noise (off with PLOMGPU_NO_ENV_STO; the
     * demographic flag has no effect).  Philox draws only. */
    int psr;
    /* Paired draws, for measuring the precision error (no counterpart in the
     * reference): 1 makes a filter without crn_normals consume the normals
     * of the precision-64 Philox filter of the same seed, rounded to the
     * state precision, and its resampling uniforms, so that an FP32 filter
     * and the FP64 filter of one seed see the same draws.  sde only. */
    int paired_draws;
    /* Optional initial particles, one per particle: [off_inc][J] (FP64),
     * used instead of x0 replicated (x0 must still be given).  Plain filters
     * only (no iterated filtering). */
    const double *x0_particles;
} plomgpu_smc_desc;

typedef struct plomgpu_smc_result {
    double loglik;            /* Llike_best */
    int n_all_fail;
    int status;
    double *llike_n;          /* [n_obs] optional: log(mean weight) per interval (0 when not weighted) */
    double *ess_n;            /* [n_obs] optional */
    uint32_t *ancestors;      /* [n_obs][J] optional: select[n][j] (identity when not resampled) */
    double *x_pred;           /* [n_obs][n_state][J] optional: propagated particles before resampling */
    double *x_final;          /* [n_state][J] optional: particles after the last interval (resampled) */
    /* [n_obs + 1][n_hat][3] optional: filtered summaries at time 0 and after
     * every interval (compute_hat / compute_hat_nn, model_builder/C/core/hat.c:68-260):
     * for every compartment state, remainder, series observation mean and
     * drifted parameter (natural scale, f_inv of the state word; word
     * i*n_cac + g for drift i, group g): the weighted 2.5 % quantile, mean,
     * 97.5 % quantile.  Weights are the interval's normalised weights where it
     * was weighted, 1/J elsewhere.  Requires a single run. */
    double *hat;
    /* [n_obs][n_ts][2] optional: prediction mean and standardised residual per
     * series over the resampled particles (print_prediction_residuals,
     * model_builder/C/core/print.c:632-711); written for intervals that were
     * weighted */
    double *pred_res;
} plomgpu_smc_result;

/* Model dimensions of this library. */
int plomgpu_get_model_info(plomgpu_model_info *out);

/* Normals one particle draws per substep for a noises_off value. */
int plomgpu_draws_per_substep(int noises_off);

/* Runs one filter: replaces run_SMC (model_builder/C/core/smc.c:204-307) and
 * the per-particle loop of worker_routine_smc_inproc
 * (model_builder/C/core/worker_inproc.c:21-102).  Host buffers in and out;
 * its device workspace comes from the library's memory pool for the call
 * (see plomgpu_release_memory). */
int plomgpu_smc_run(const plomgpu_smc_desc *desc, plomgpu_smc_result *result);

/* Reusable plan: device buffers, uploaded inputs and a CUDA graph of the
 * whole time loop, for callers that evaluate many likelihoods of the same
 * shape (pmcmc, C/pmcmc/pmcmc.c:214; mif, C/mif/mif.c:128-200). */
typedef struct plomgpu_plan plomgpu_plan;

int plomgpu_plan_create(const plomgpu_smc_desc *desc, plomgpu_plan **out);
/* flags: PLOMGPU_PLAN_TIMING records CUDA events around every propagate
 * launch inside the graph, read back with plomgpu_plan_propagate_time();
 * PLOMGPU_PLAN_TRAJ keeps the genealogy and the propagated particles of every
 * interval (FP64, n_obs * n_state * J doubles) for plomgpu_plan_sample_traj
 * and for result.ancestors / result.x_pred; PLOMGPU_PLAN_SUMMARIES computes
 * result.hat and result.pred_res on every launch. */
enum { PLOMGPU_PLAN_TIMING = 1, PLOMGPU_PLAN_TRAJ = 2, PLOMGPU_PLAN_SUMMARIES = 4 };
int plomgpu_plan_create_ex(const plomgpu_smc_desc *desc, int flags, plomgpu_plan **out);
/* One trajectory of the last launch drawn from its genealogy
 * (sample_traj_and_print, model_builder/C/core/print.c:715-784, with the same
 * indexing): u in [0, 1) picks the final particle by the last weighted
 * interval's normalised weights.  Writes n_rows (<= n_obs + 2) rows in the
 * reference's print order, last time first: rows_t[r] is the time row
 * (0 = time 0, n + 1 = t_obs[n]) and states[r][n_state] the particle.  Needs
 * PLOMGPU_PLAN_TRAJ and at least two intervals with data. */
int plomgpu_plan_sample_traj(plomgpu_plan *plan, double u, int *n_rows, int *rows_t, double *states);
/* Device time of the propagate launches of the last plomgpu_plan_launch
 * (sum over launches, milliseconds) and their number. */
int plomgpu_plan_propagate_time(plomgpu_plan *plan, double *total_ms, int *launches);
/* Uploads new parameters / initial state / seed from host memory (pinned or
 * pageable) on the plan's stream; pointers may be NULL to keep the previous
 * values. */
int plomgpu_plan_update(plomgpu_plan *plan, const double *par_cac, const double *par_ts,
                        const double *x0, uint64_t seed);
/* Uploads a new volatility table of the drifted parameters ([n_drift][n_cac],
 * indexed like smc_desc.drift_vol); synchronous. */
int plomgpu_plan_update_drift(plomgpu_plan *plan, const double *drift_vol);
/* Enqueues one filter run on the plan's stream; inputs must be resident. */
int plomgpu_plan_launch(plomgpu_plan *plan);
/* Waits for the plan's stream and copies the results to host memory. */
int plomgpu_plan_results(plomgpu_plan *plan, plomgpu_smc_result *result);
/* Stream of the plan (a cudaStream_t), for timing with CUDA events. */
void *plomgpu_plan_stream(plomgpu_plan *plan);
/* Kernels launched by one plomgpu_plan_launch. */
int plomgpu_plan_kernel_count(plomgpu_plan *plan);
void plomgpu_plan_destroy(plomgpu_plan *plan);

/* Plans and one-shot filters take their device buffers from a memory pool of
 * the library (one per device, stream-ordered) that keeps the memory of
 * destroyed plans for the next ones.  This returns the pool's unused memory
 * on the current device to the driver. */
int plomgpu_release_memory(void);

/* Test hook (host only, no GPU needed): the largest double whose exponential
 * is <= thresh, which the filters compare log-weights with for the failure
 * test of weight() (exp(loglik) <= LIKE_MIN^N_TS, smc.c:44). */
double plomgpu_debug_fail_boundary(double thresh);

/* Test hook: the first J systematic-resampling points of offset U computed by
 * the device-side closed form (GPU) into out[J]. */
int plomgpu_debug_systematic_points(double U, int J, double *out);

/* Test hook: draws of the library's own generators on the device, as the
 * filters compile them (single precision with the special-function-unit
 * elementary functions), for distribution tests.  streams independent
 * Philox streams (the particle slot of the counter) of per_stream draws each
 * into out[streams * per_stream] (host).  kind 0: normals of the sde step
 * (Box-Muller); 1: binomial(n = a, p = b); 2: Poisson(mean a); 3: Gamma
 * (shape a, scale b); 4: normals of the psr uniform stream.  precision 32 or
 * 64 picks the generators of FP32 or FP64 particle states. */
int plomgpu_debug_draws(int kind, int precision, double a, double b, uint64_t seed, int streams, int per_stream,
                        double *out);

/* ------------------------------------------------------------------------
 * Iterated filtering (mif, model_builder/C/mif/mif.c:21-247): R independent
 * runs of J particles, each particle carrying its own transformed
 * parameters theta[q], q < n_theta (<= 16).  Per observation interval the
 * particles are propagated with their back-transformed parameters, weighted,
 * the weighted mean and prediction variance of every component are recorded
 * (mean_var_theta_theoretical_mif, C/mif/methods.c:133-192), and the
 * parameters are resampled with the particles and perturbed by a Gaussian
 * random walk on the estimated components (resample_and_mut_theta_mif,
 * methods.c:261-367).  The theta-hat update between iterations is left to
 * the host (update_theta_best_*, methods.c:394-467). */
typedef struct plomgpu_mif_desc {
    int n_runs;
    int n_theta;
    const int *proc_slot;   /* [n_par_proc] component of each process parameter, -1: from par_cac */
    const int *obs_slot;    /* [n_par_obs] component of each observation parameter, -1: from par_ts */
    const plomgpu_back_transform *theta_bt; /* [n_theta] transformed -> natural scale */
    const int *estimated;   /* [n_theta] 1: perturbed by the random walk */
    /* Parameters fitted per group: a slot of -2 above means that the
     * component depends on the population (process, [n_par_proc][n_cac]) or
     * series (observation, [n_par_obs][n_ts]) through these tables; null when
     * no slot is -2. */
    const int *proc_cac_slot;
    const int *obs_ts_slot;
    /* Fixed-lag smoothing of the initial conditions and drift start values
     * (update_fixed_lag_smoothing, model_builder/C/mif/methods.c:370-392) and
     * the --prior patch (patch_likelihood_prior, methods.c:469-520); every
     * field below is optional (NULL / 0: off). */
    const int *fls;          /* [n_theta] 1: component fitted by fixed-lag smoothing: proposed
                                with the others at the start of an iteration, resampled, never
                                perturbed by the random walk */
    const int *x0_slot;      /* [off_inc] component giving each initial state word, -1: the
                                descriptor's x0.  Compartment words take the component's
                                natural value (a proportion) times pop0 of their cac, drift
                                words its transformed value (theta_driftIC2Xdrift) */
    const double *pop0;      /* [n_cac] population size at t = 0 (with x0_slot) */
    const int *vol_slot;     /* [n_drift][n_cac] component giving the volatility of drift i,
                                group g; -1: the descriptor's drift_vol */
    int lag;                 /* L: the fixed-lag means are the weighted means of the
                                resampled components at interval L (L >= n_obs: none) */
    int prior;               /* 1: weights times prior^(1/n_obs) for the random-walk
                                components, prior^(1/lag) for the fixed-lag ones while
                                n < lag (before the failure test and the normalisation) */
    const int *prior_kind;   /* [n_theta] 0 flat on [lo, hi), 1 normal of mean (lo+hi)/2 and
                                sd (hi-lo)/4, 2 pseudo-uniform (metropolis_hastings_prior.c) */
    const double *prior_lo;  /* [n_theta] */
    const double *prior_hi;  /* [n_theta] */
    const plomgpu_back_transform *prior_finv; /* [n_theta] transformed -> scale of the prior */
} plomgpu_mif_desc;

typedef struct plomgpu_plan plomgpu_mif;

/* base: the filter problem (data, grid, covariates, fixed parameters, x0,
 * J particles per run); captures one iteration as a CUDA graph. */
int plomgpu_mif_create(const plomgpu_smc_desc *base, const plomgpu_mif_desc *mif, plomgpu_mif **out);
/* One iteration of all runs.  theta_hat [n_runs][n_theta] (transformed
 * scale); sd_init [n_theta] sd of the initial proposal around theta_hat;
 * sd_mut [n_obs][n_theta] random-walk sd applied after the resampling of
 * interval n; vt_add [n_obs][n_theta] theoretical variance added to the
 * prediction variance of interval n.  Outputs: loglik [n_runs],
 * n_all_fail [n_runs], bart / vt [n_runs][n_obs][n_theta] (rows of intervals
 * without data are not written). */
int plomgpu_mif_iteration(plomgpu_mif *mif, const double *theta_hat, const double *sd_init, const double *sd_mut,
                          const double *vt_add, uint64_t seed, double *loglik, int *n_all_fail, double *bart,
                          double *vt);
/* Fixed-lag means [n_runs][n_theta] of the last iteration (NaN for the
 * components not fitted by fixed-lag smoothing); *updated = 0 when the
 * filter never reached interval L (L >= n_obs). */
int plomgpu_mif_fls_means(plomgpu_mif *mif, double *out, int *updated);
void plomgpu_mif_destroy(plomgpu_mif *mif);

/* ------------------------------------------------------------------------
 * Batched filters: many independent filters of one model (different
 * parameters, particle counts, series lengths and data) in one persistent
 * launch.  Serves the callers that evaluate many likelihoods at once (mif
 * particles over parameter sets, concurrent pmcmc chains; C/mif/mif.c,
 * C/pmcmc/pmcmc.c).  Filter i with seed[i] consumes exactly the draws of a
 * single plomgpu_smc_run with seed = seed[i]. */
typedef struct plomgpu_batch_desc {
    int n_filters;
    const int *J;              /* [n] particles of each filter */
    const int *n_obs;          /* [n] intervals of each filter (<= max_obs) */
    const long long *data_row; /* [n] first row of each filter in data */
    const double *data;        /* [n_rows][n_ts], NaN = missing */
    long long n_rows;
    const double *par_cac;     /* [n][n_par_proc][n_cac] */
    const double *par_ts;      /* [n][n_par_obs][n_ts] */
    const double *x0;          /* [n][n_state] */
    const uint64_t *seed;      /* [n] */
    /* time grid and covariates of the longest filter, shared by all */
    int max_obs;
    const int *n_sub;          /* [max_obs] */
    const double *t_sub;       /* [sum n_sub] */
    const double *t_obs;       /* [max_obs] */
    double dt;
    const double *cov_cac;     /* [sum n_sub][n_cov_cac][n_cac] */
    const double *cov_ts;      /* [max_obs][n_cov_ts][n_ts] */
    const double *coupling;
    const int *drift_group;
    const int *drift_ngroups;
    const plomgpu_back_transform *drift_bt;
    const double *drift_vol;
    int noises_off;
    int filter;
    double like_min;
    int precision;             /* 32 or 64 */
    int block_threads;         /* 0: autotuned among 128 / 256 / 512 */
    int particles_per_thread;  /* particles a thread advances together: 0 autotuned among 1 / 2 (FP64: 1) */
} plomgpu_batch_desc;

typedef struct plomgpu_batch plomgpu_batch;

/* Uploads the batch, sizes the per-CTA workspaces and (block_threads or
 * particles_per_thread == 0) times the candidate (block size, particles per
 * thread) pairs on a sample of the batch, keeping the fastest. */
int plomgpu_batch_create(const plomgpu_batch_desc *desc, plomgpu_batch **out);
int plomgpu_batch_launch(plomgpu_batch *batch);
int plomgpu_batch_results(plomgpu_batch *batch, double *loglik, int *n_all_fail, double *ess_min);
void *plomgpu_batch_stream(plomgpu_batch *batch);
/* The configuration in use: threads per block, particles per thread, CTAs. */
int plomgpu_batch_config(plomgpu_batch *batch, int *block_threads, int *particles_per_thread, int *grid);
void plomgpu_batch_destroy(plomgpu_batch *batch);
/* One-shot: create, launch, results, destroy. */
int plomgpu_batch_run(const plomgpu_batch_desc *desc, double *loglik, int *n_all_fail);

/* ------------------------------------------------------------------------
 * Likelihood server for concurrent callers (pmcmc chains, C/pmcmc/pmcmc.c:
 * 186-266): requests (parameters, initial state, seed, J) on one data set
 * are queued, admitted while their HBM footprint fits the memory budget,
 * and run concurrently on a device-resident loop: a persistent kernel takes
 * requests from a ring in mapped host memory (continuous batching).  Models
 * whose particle fits registers run one CTA per request; larger models
 * (shared-memory particles) split every request into tiles of particles,
 * one tile of one interval being the unit of work, so that tiles of
 * different requests share the SMs.  A result does not depend on what else
 * runs: each request is computed by the same deterministic arithmetic alone
 * or in the mix.  Thread-safe. */
typedef struct plomgpu_server_opts {
    int max_J;              /* largest particle count of a request */
    double memory_budget;   /* bytes of HBM the requests may hold (0: 150e9) */
    int ring_slots;         /* requests in flight on the device loop (0: 1024) */
    int plan_pool;          /* concurrent plans for models served per plan (0: 4; one SEIR 20x2 filter of
                             * 2e4 particles fills half of a B200's resident slots: 2 / 3 / 4 plans run
                             * 1.6 / 2.0 / 2.1x the filters per second of one) */
    int precision;          /* 32 or 64 */
    int use_plan_pool;      /* 1: models with shared-memory particles run on the plan pool instead of the
                             * device loop (one captured whole filter per request, for comparison) */
    int task_budget;        /* tiles a CTA of the tiled loop runs before it returns and frees its SM slot
                             * for other kernels (0: 64; < 0: no limit) */
} plomgpu_server_opts;

typedef struct plomgpu_server_stats {
    long long pending, in_flight, completed, launches, peak_in_flight;
    double bytes_in_use, peak_bytes;
    int persistent_loop;    /* 1: device-resident loop, 0: plan pool */
} plomgpu_server_stats;

typedef struct plomgpu_server plomgpu_server;

/* base: the shared data set, time grid, covariates and default parameters
 * (base->J is ignored). */
int plomgpu_server_create(const plomgpu_smc_desc *base, const plomgpu_server_opts *opts, plomgpu_server **out);
/* par_cac / par_ts / x0 may be NULL to use the base values. */
int plomgpu_server_submit(plomgpu_server *server, int J, const double *par_cac, const double *par_ts,
                          const double *x0, uint64_t seed, long long *ticket);
int plomgpu_server_poll(plomgpu_server *server, long long ticket, int *done, double *loglik, int *n_all_fail,
                        double *latency_s);
int plomgpu_server_wait(plomgpu_server *server, long long ticket, double timeout_s, double *loglik,
                        int *n_all_fail, double *latency_s);
int plomgpu_server_get_stats(plomgpu_server *server, plomgpu_server_stats *stats);
void plomgpu_server_destroy(plomgpu_server *server);

/* Resamples one observation interval without allocating device memory.
 *
 * No counterpart in the reference.  For callers that cannot allocate: a
 * plug-in inside a runtime whose caching allocator owns the GPU memory, or a
 * latency-bounded serving loop in which cudaMalloc / cudaFree would
 * synchronise the device.  Runs the weighting (failure rule, log-sum-exp
 * normalisation, ESS), the cumulative weights and the systematic ancestor
 * search of one interval (smc.c:27-112 semantics) on caller-owned device
 * buffers:
 *   log_weights  device, J values (float when precision == 32, double when 64)
 *   u            uniform in [0, 1): the systematic offset is U = u / J
 *   ancestors    device, J values written
 *   out          device, 4 doubles written: log mean weight, ESS, all-fail
 *                flag (1.0 when every particle failed: identity ancestors),
 *                error flags (nonzero: a bounded wait ran out, result invalid)
 *   stream       cudaStream_t the work is queued on (NULL: legacy stream)
 * The work is asynchronous on `stream`; read `out` after synchronising it.
 * Scratch is one fixed array of this library (about 2.1 MB, held on every
 * GPU that loads the library until exit), so J is limited to 262144
 * (PLOMGPU_EINVAL beyond).  Calls that overlap on the GPU, on any stream of
 * the same device, race on that array and must be serialised by the caller.
 * Every call looks up the array's device address in the CUDA context current
 * at the call, so the address is valid for that context only; the first call
 * in a context also loads the library's device code there: make it before
 * any stream capture on that device. */
int plomgpu_resample_noalloc(const void *log_weights, int precision, int J, double like_min, double u,
                             uint32_t *ancestors, double *out, void *stream);

/* Per-particle values of the printed quantities: particle i is X[:, i]
 * (X [n_state][P], host, FP64) at time row rows[i] (0 = time 0, n + 1 =
 * t_obs[n]).  out ([n_hat + n_ts][P], host) holds the rows of the filtered
 * summaries (states, remainders, observation means, drifted parameters on
 * the natural scale) followed by the observation variances: the columns of
 * print_p_X (model_builder/C/core/print.c:301-357) apart from its random
 * observation draws. */
int plomgpu_particle_values(const plomgpu_smc_desc *desc, const double *X, int P, const int *rows, double *out);

const char *plomgpu_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* PLOMGPU_H */
