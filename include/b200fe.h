/*
 * b200fe.h -- C ABI of the B200 fixed-effects absorber (libb200fe.so).
 *
 * Every entry point takes plain pointers and sizes, returns an int status and
 * never throws.  Status codes follow the reference's GPU status semantics
 * (docs/gpu.md:159-161, src/fe_absorption.cpp:361-381):
 *
 *   B200FE_OK             0  solved; outputs written
 *   B200FE_NOT_CONVERGED  1  outputs written, tolerance not reached (status 3 upstream)
 *   B200FE_UNAVAILABLE    2  no usable CUDA device (status 2 upstream)
 *   B200FE_CUDA_ERROR     3  a CUDA call or allocation failed (status 4 upstream)
 *   B200FE_INVALID_ARG    4  bad sizes, ids out of range, non-finite input
 *
 * There is no CPU fallback behind any of these calls: a failure is returned
 * to the caller, which decides (the reference's fail-closed contract,
 * src/fe_absorption.cpp:9227-9237).
 *
 * Problem solved by every absorb call: for each column v of [y X] return the
 * weighted within transform  v~ = v - D a,  where a solves the normal
 * equations  D'W D a = D'W v  of the stacked FE dummies D = [D_1 ... D_m]
 * (the projection the reference's absorbers compute; fe_absorption.hpp).
 *
 * Group ids are dense 0..G_d-1 per dimension (the reference's GpuFeInput
 * contract, include/fe_absorption_cuda.hpp:12-22); X is column-major with
 * leading dimension n (the reference rejects ld != n,
 * src/fe_absorption_cuda.cu:2303-2306).
 */
#ifndef B200FE_H
#define B200FE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define B200FE_OK 0
#define B200FE_NOT_CONVERGED 1
#define B200FE_UNAVAILABLE 2
#define B200FE_CUDA_ERROR 3
#define B200FE_INVALID_ARG 4

#define B200FE_PREC_FP64 0   /* plain FP64 preconditioned CG                   */
#define B200FE_PREC_MIXED 1  /* FP32 inner CG inside FP64 iterative refinement */

#define B200FE_MAX_DIMS 8

typedef struct b200fe_context b200fe_context;

typedef struct b200fe_options {
    double tol;            /* stop when max_c ||b_c - S a_c|| <= tol * ||b_c|| (default 1e-8)   */
    int max_iter;          /* cap on PCG iterations, all refinement rounds together (10000)   */
    int precision;         /* B200FE_PREC_FP64 or B200FE_PREC_MIXED (default MIXED)           */
    int certify;           /* 1: compute abs_residual / abs_residual_rel on the device (1)    */
    int check_interval;    /* PCG iterations between host convergence checks (default 4)      */
    int reuse_structure;   /* 1: ids and weights equal those of the previous call (0)         */
    double inner_tol;      /* MIXED: relative tolerance of each FP32 inner solve (1e-5)       */
    int tolerance_mode;    /* certificate limit as the reference: 0 xhdfe-fast,
                              1 reghdfe-comparable (tol_eff = min(tol, 1e-9)), 2 strict (1)  */
    int max_outer;         /* MIXED: cap on refinement rounds (default 12)                    */
    int profile;           /* 1: time every kernel category with CUDA events (default 0)      */
    int pass_kernel;       /* CG matvec pass: 0 auto (block level when at most one large and
                              one small FE dim besides the largest; with a small dim, its
                              dense coupling rows when they are small; with one large dim,
                              its Schur block built explicitly as a sparse matrix when the
                              movers' pairs are few), 1 general tile pass, 2 block level
                              without the dense coupling, 3 as 0 but the large dim through
                              its runs (no explicit block); for the slope absorber 1 forces
                              block Jacobi over every dimension                              */
    double fe_linf_tol;    /* > 0: a column also needs every group's weighted mean of its
                              within transform (non-primary dims) at most this before it
                              stops -- the check recover_fixed_effects applies to saved FEs
                              (src/fe_absorption.cpp:15527-15548); a refinement round that
                              raises the residual (the bound lies below what rounding
                              allows) is undone and the L2 rule alone decides; 0 off      */
} b200fe_options;

/* Kernel categories of the profile arrays in b200fe_result. */
#define B200FE_PROF_PASS 0      /* alpha-space primary-segment pass (S x), the CG hot kernel */
#define B200FE_PROF_GATHER 1    /* run gather-sum per large FE dimension                    */
#define B200FE_PROF_FINALIZE 2  /* multi-chunk groups, small-dim bins, dot reduction        */
#define B200FE_PROF_VECTOR 3    /* CG vector updates and column dots                        */
#define B200FE_PROF_RHS 4       /* data pass forming the projected right-hand side          */
#define B200FE_PROF_FINAL 5     /* data pass writing the within transform (+ certificate)   */
#define B200FE_PROF_SETUP 6     /* FE structure build                                        */
#define B200FE_PROF_COUPLE 7    /* dense small-dim coupling product C_fy' x_f (CG matvec)    */
#define B200FE_PROF_CATEGORIES 8
/* b200fe_absorb_slopes fills the same slots: PASS the per-dim chunk sums of
 * w r and w z r (with the residual update), GATHER the image D p, FINALIZE the
 * per-group gradient and block preconditioner, VECTOR the CG scalars and
 * directions, RHS / FINAL the load into and store out of the row-major
 * residual, SETUP the sorts, chunks and block inverses. */

typedef struct b200fe_result {
    int status;
    int iterations;          /* PCG iterations over all refinement rounds                  */
    int outer_iterations;    /* FP64 refinement rounds (1 for FP64)                        */
    int converged;
    int precision_certified; /* converged and abs_residual_rel <= max(8 tol_eff, 64 eps)    */
    int primary_dim;         /* FE dimension eliminated exactly (the largest)              */
    int num_levels_present[B200FE_MAX_DIMS];
    double abs_residual;     /* max_c ||D'W v~_c||_2  (src/fe_absorption.cpp:14942-15190) */
    double abs_residual_rel; /* max_c ||D'W v~_c|| / (||D'W||_F ||v_c||)                   */
    double rel_residual;     /* max_c ||b_c - S a_c|| / ||b_c|| at exit                      */
    double setup_ms;         /* FE structure build (0 when reused)                          */
    double solve_ms;         /* RHS pass + PCG + output pass (+ certificate)                */
    double h2d_ms;
    double d2h_ms;
    long long kernel_launches;   /* this library's own kernels launched by the call     */
    long long library_calls;     /* CUB device-primitive calls (setup sorts and scans)   */
    /* profile == 1: per category, summed CUDA-event time, launches, and the
       algorithmic bytes those launches had to move (HBM roofline numerator). */
    double prof_ms[B200FE_PROF_CATEGORIES];
    double prof_bytes[B200FE_PROF_CATEGORIES];
    long long prof_launches[B200FE_PROF_CATEGORIES];
    int warm_columns;        /* columns started from the learned warm start's prediction  */
} b200fe_result;

/* Library version, e.g. 10000 for 1.0.0. */
int b200fe_version(void);

/* 1 when a CUDA device is usable.
 * Replaces hdfe::detail::cuda_backend_available()
 * (include/fe_absorption_cuda.hpp:125, src/fe_absorption_cuda.cu:2281). */
int b200fe_device_available(void);

void b200fe_default_options(b200fe_options* opts);

/* A context owns one CUDA stream and a grow-only device workspace.  One
 * context per host thread (the reference keeps its workspace thread_local,
 * src/fe_absorption_cuda.cu:1536). */
int b200fe_context_create(int device, b200fe_context** out);
void b200fe_context_destroy(b200fe_context* ctx);
const char* b200fe_last_error(const b200fe_context* ctx);
/* The context's cudaStream_t, as void*. */
void* b200fe_context_stream(b200fe_context* ctx);

/* Absorb host arrays: copies in, solves on the device, copies out.
 * y: n doubles; X: n*k doubles column-major (may be NULL when k == 0);
 * group_ids[d]: n int32 dense ids; num_groups[d]: G_d; weights: n doubles or
 * NULL.  y_out / X_out receive the within transforms.
 * Replaces hdfe::detail::absorb_fixed_effects_cuda
 * (include/fe_absorption_cuda.hpp:127-134, src/fe_absorption_cuda.cu:2294). */
int b200fe_absorb(b200fe_context* ctx, const double* y, const double* X,
                  int64_t n, int k, int num_dims,
                  const int32_t* const* group_ids, const int32_t* num_groups,
                  const double* weights, const b200fe_options* opts,
                  double* y_out, double* X_out, b200fe_result* res);

/* b200fe_absorb that also returns the fixed-effect coefficients (saved FEs):
 * fe_out[d] is a host array of num_groups[d] x (k + 1) doubles, column-major,
 * column 0 for y and column j for X column j.  On return, for every row i,
 * v_i - v~_i = sum_d fe_out[d][gid_d(i), :] (to rounding): the primary
 * dimension's coefficients are its weighted group means of v - (other FEs),
 * the others the refined solution of the reduced system.  As in any
 * multi-way FE model the split between dimensions is identified only up to
 * the usual normalisations (a constant moved between dimensions); the sum is
 * unique.  Groups without observations get 0.
 * Replaces the retain_fixed_effects outputs (fe_alpha_y / fe_alpha_X) of
 * hdfe::detail::absorb_fixed_effects_cuda (src/fe_absorption_cuda.cu:4663-4690),
 * which the reference's recover_fixed_effects consumes
 * (src/fe_absorption.cpp:15484-15520). */
int b200fe_absorb_fe(b200fe_context* ctx, const double* y, const double* X,
                     int64_t n, int k, int num_dims,
                     const int32_t* const* group_ids, const int32_t* num_groups,
                     const double* weights, const b200fe_options* opts,
                     double* y_out, double* X_out, double* const* fe_out,
                     b200fe_result* res);

/* Absorb device arrays (no host copies).  d_v: column-major n x cols with the
 * outcome in column 0; d_out: same shape (may alias nothing of the inputs).
 * stream: a cudaStream_t as void*, or NULL for the context's stream.
 * Same solver as b200fe_absorb. */
int b200fe_absorb_device(b200fe_context* ctx, const double* d_v, int64_t n,
                         int cols, int num_dims,
                         const int32_t* const* d_group_ids,
                         const int32_t* num_groups, const double* d_weights,
                         const b200fe_options* opts, double* d_out,
                         b200fe_result* res, void* stream);

/* Absorption with heterogeneous slopes.  Dimension d spans, per group g, the
 * intercept 1_g when slope_values[d] is NULL (a plain FE); otherwise the slope
 * z_d 1_g (z_d = slope_values[d], n doubles) and, when
 * slope_has_intercept[d] is nonzero, also 1_g.  slope_values may be NULL
 * (all plain).  A group's 2x2 block is inverted with the reference's rule:
 * determinant above 1e-12 max(1, W ZZ), else the intercept alone.  FP64
 * CGLS; when the dimension with the most groups (primary_dim in res) has no
 * slope, it is eliminated exactly (Schur form) and the other blocks are
 * preconditioned by the exact block diagonal of the Schur complement;
 * opts->pass_kernel == 1 forces block Jacobi over every dimension instead.
 * At most 256 columns.
 * Replaces the is_slope path of hdfe::detail::absorb_fixed_effects_cuda
 * (GpuFeInput.is_slope / slope_has_intercept / slope_values,
 * include/fe_absorption_cuda.hpp:12-22; src/fe_absorption_cuda.cu:2316-2420,
 * 586-650) and the slopes argument of absorb_fixed_effects_v6
 * (include/fe_absorption.hpp:95-101). */
int b200fe_absorb_slopes(b200fe_context* ctx, const double* y, const double* X,
                         int64_t n, int k, int num_dims,
                         const int32_t* const* group_ids, const int32_t* num_groups,
                         const double* const* slope_values,
                         const unsigned char* slope_has_intercept,
                         const double* weights, const b200fe_options* opts,
                         double* y_out, double* X_out, b200fe_result* res);

/* b200fe_absorb_slopes on device arrays (d_v / d_out as b200fe_absorb_device;
 * d_slope_values[d] device pointers or NULL). */
int b200fe_absorb_slopes_device(b200fe_context* ctx, const double* d_v, int64_t n,
                                int cols, int num_dims,
                                const int32_t* const* d_group_ids,
                                const int32_t* num_groups,
                                const double* const* d_slope_values,
                                const unsigned char* slope_has_intercept,
                                const double* d_weights, const b200fe_options* opts,
                                double* d_out, b200fe_result* res, void* stream);

/* Group/individual structure (host arrays), the reference's
 * GroupIndividualStructure (include/fe_absorption.hpp:13-21): every row of the
 * data is a group; group g holds the individuals
 * group_individual[group_ptr[g] .. group_ptr[g+1]), individual i appears in the
 * groups individual_group[individual_ptr[i] .. individual_ptr[i+1]) (both CSR
 * arrays list the same num_edges edges), and the basis column of individual i
 * is group_scale[g] at every group g that holds i (1 for sum aggregation,
 * 1 / group size for mean aggregation). */
typedef struct b200fe_group_individual {
    int32_t num_individuals;
    int64_t num_edges;
    const int32_t* group_ptr;         /* n + 1            */
    const int32_t* group_individual;  /* num_edges        */
    const int32_t* individual_ptr;    /* num_individuals + 1 */
    const int32_t* individual_group;  /* num_edges        */
    const double* group_scale;        /* n                */
} b200fe_group_individual;

/* Absorption of the standard FE dims (group_ids, num_dims >= 0) together with
 * the individual FEs of a group/individual design, on host arrays.  The CSR
 * arrays are range-checked on the host before any device work
 * (B200FE_INVALID_ARG when inconsistent).  Same solver as b200fe_absorb_slopes
 * with the individual dimension as one more block (diagonal preconditioner
 * sum over its groups of w scale^2); primary_dim is -1 when num_dims == 0.
 * Replaces hdfe::detail::absorb_fixed_effects_group_individual_cuda
 * (include/fe_absorption_cuda.hpp:136-145, src/fe_absorption_cuda.cu:4740). */
int b200fe_absorb_group_individual(b200fe_context* ctx, const double* y, const double* X,
                                   int64_t n, int k, int num_dims,
                                   const int32_t* const* group_ids,
                                   const int32_t* num_groups,
                                   const b200fe_group_individual* gi,
                                   const double* weights, const b200fe_options* opts,
                                   double* y_out, double* X_out, b200fe_result* res);

/* In-place demean of host arrays, the raw interface of the reference's
 * block-PCG absorber: Y (n) and X (n x k column-major) are overwritten with
 * their within transforms; iters_out receives the PCG iteration count.
 * Returns 0 on success.  Unlike the reference it has no column limit.
 * Replaces xhdfe::schwarz_demean_raw (include/schwarz_demean.hpp:30-34,
 * src/schwarz_demean.cpp:419-438). */
int b200fe_demean_raw(double* Y, double* X, int64_t n, int k, int num_dims,
                      const int32_t* const* fe, const int32_t* nlev,
                      double tol, int max_iter, int* iters_out);

/* Max over FE dims of max_g |weighted mean_g(residual)| after a Gauss-Seidel
 * pass over the dims in sweep_order (NULL: 0..m-1), each dim's means
 * subtracted before the next.  Used to check that a recovered residual is
 * orthogonal to every FE basis.
 * Replaces hdfe::detail::fe_recovery_max_delta_cuda
 * (include/fe_absorption_cuda.hpp:152-156, src/fe_absorption_cuda.cu:5227). */
int b200fe_fe_recovery_max_delta(b200fe_context* ctx, const double* residual,
                                 int64_t n, int num_dims,
                                 const int32_t* const* group_ids,
                                 const int32_t* num_groups,
                                 const double* weights,
                                 const int32_t* sweep_order,
                                 double* out_max_delta);

/* ---------------------------------------------------------------------------
 * Learned warm start (no counterpart in the reference, which always starts its
 * solves from zero).  A 3-hidden-layer, 64-wide MLP with BF16 weights and
 * activations and FP32 accumulation maps per-level features of the Schur
 * system (its first three Jacobi iterates, the level's weight and mobility)
 * to a correction of the third Jacobi iterate and a log-scaling of the level's
 * Jacobi diagonal.  Parameters: b200fe_mlp_num_params() FP32 values, layout
 * W1 (64x8, row-major), b1, W2 (64x64), b2, W3 (64x64), b3, W4 (2x64), b4.
 * The plain FP64-checked solver still runs to the stated tolerance from the
 * predicted start: only the iteration count changes.
 * ------------------------------------------------------------------------- */
int b200fe_mlp_num_params(void);
/* y[n][2] = MLP(x[n][8]) on tensor cores (device arrays). */
int b200fe_mlp_forward(b200fe_context* ctx, const float* d_params, const float* d_x, int64_t n,
                       float* d_y);
/* Loss L = (1/n) sum_s sum_o w_so (y_so - t_so)^2 over targets
 * d_targets[n][4] = (t0, t1, w0, w1), and its gradient with respect to the
 * FP32 master parameters (BF16 roundings straight-through):
 * d_grad_loss[0 .. P) = gradient, d_grad_loss[P] = loss (FP64, P = num_params).
 * Deterministic (fixed-order reductions). */
int b200fe_mlp_grad(b200fe_context* ctx, const float* d_params, const float* d_x,
                    const float* d_targets, int64_t n, double* d_grad_loss);
/* One Adam step (beta1 0.9, beta2 0.999, eps 1e-8) on the FP32 master
 * parameters from a gradient of b200fe_mlp_grad; step counts from 1. */
int b200fe_mlp_adam(b200fe_context* ctx, float* d_params, float* d_m, float* d_v,
                    const double* d_grad, int step, double lr);
/* Installs trained parameters (host array) in the context: mode bit 0 starts
 * every later absorption's refinement from the network's prediction (a column
 * whose predicted start has a larger residual than zero starts cold), bit 1
 * scales the Jacobi diagonal by the network's per-level factor.  params NULL
 * or mode 0 turns the warm start off. */
int b200fe_warmstart_set(b200fe_context* ctx, const float* params, int mode);
/* Training samples: runs b200fe_absorb_device on the given problem with the
 * plain solver (the installed warm start is not used) and writes, for every
 * level of the non-primary dims and every column, the network's 8 features
 * (d_features[count][8]) and the targets from the converged solution
 * (d_targets[count][4]); capacity rows at most (B200FE_INVALID_ARG beyond). */
int b200fe_warmstart_samples(b200fe_context* ctx, const double* d_v, int64_t n, int cols,
                             int num_dims, const int32_t* const* d_group_ids,
                             const int32_t* num_groups, const double* d_weights,
                             const b200fe_options* opts, double* d_out, float* d_features,
                             float* d_targets, int64_t capacity, int64_t* count,
                             b200fe_result* res);

/* One-way within transform that allocates no device memory, for callers that
 * cannot call cudaMalloc while they use this library: a host application that
 * keeps all device memory in its own pool, or a plugin that must not grow its
 * CUDA footprint in the middle of a session.  The caller passes every input
 * and output as a device pointer: d_v column-major n x cols, d_group_ids dense
 * ids in [0, num_groups) sorted non-decreasing (data ordered by the FE, e.g. a
 * panel sorted by worker), d_weights n doubles or NULL, d_out n x cols (not
 * aliasing d_v).  d_out receives v minus the weighted group mean of v, per
 * column.  The only scratch is a fixed array inside the library: at most 2^20
 * groups (a larger num_groups returns B200FE_INVALID_ARG before any GPU work),
 * kept until the process exits by every GPU on which it was placed.  CUDA loads
 * device code lazily: b200fe_context_create places the array on its device,
 * so after a context exists on a device no-alloc calls there load nothing;
 * without one, the first no-alloc call on a device loads this code (the array
 * and its kernels) unless CUDA_MODULE_LOADING=EAGER is set.  All calls on one
 * device share that array, so calls whose GPU work overlaps race on it.  The
 * array's address is looked up once per device with that device current (at
 * context creation or by the first call); make that first call before any
 * stream capture.  Each call waits once for its stream (the id check's status
 * is read back).  A CUDA error pending from earlier work returns
 * B200FE_CUDA_ERROR (and is cleared).  Unsorted or out-of-range ids return
 * B200FE_INVALID_ARG.  stream: a cudaStream_t as void*, or NULL.
 * This entry point has no counterpart in the reference, which always
 * allocates its device workspace. */
int b200fe_demean_sorted_noalloc(const double* d_v, int64_t n, int cols,
                                 const int32_t* d_group_ids, int32_t num_groups,
                                 const double* d_weights, double* d_out,
                                 void* stream);

/* ---------------------------------------------------------------------------
 * Preprocessing on the device (the reference does these on the host).
 * ------------------------------------------------------------------------- */
/* Dense group ids from raw int32 ids (device arrays), the rule of the
 * reference's build_indexer (src/fe_absorption.cpp:845-940): if the raw range
 * R = max - min + 1 is at most 50,000,000 and at most 2n, id = raw - min with
 * num_groups = R, compacted in raw order (num_groups = distinct values) when
 * fewer than 90% of the range is present; otherwise id = rank of the raw value
 * among the distinct values.  num_levels_present = distinct values. */
int b200fe_dense_ids_device(b200fe_context* ctx, const int32_t* d_raw, int64_t n,
                            int32_t* d_out, int32_t* num_groups,
                            int32_t* num_levels_present);
/* Iterative singleton drop (device arrays): d_keep[i] = 0 for the rows removed
 * by rounds that drop every kept row alone in its group of some dimension,
 * until a round drops nothing or max_iter rounds (<= 0: 100, the reference's
 * cap) ran; the reference's compute_keep_mask_drop_singletons
 * (src/hdfe_regressor_v11.cpp:4056-4290).  ids dense in [0, num_groups[d]). */
int b200fe_drop_singletons_device(b200fe_context* ctx, int num_dims,
                                  const int32_t* const* d_ids,
                                  const int32_t* num_groups, int64_t n,
                                  uint8_t* d_keep, int max_iter, int64_t* dropped,
                                  int* rounds);

/* Mobility groups of the first FE pair (device arrays of raw int32 ids, each
 * ranked as build_indexer does): the connected components of the bipartite
 * graph whose nodes are the groups of both dims and whose edges are the
 * observations.  Returns the number of components with observations, the
 * largest one's observation count and share, and its weight share (the largest
 * component weight over the total; weights must be finite and positive, NULL
 * for the observation share).  Replaces hdfe::v11::compute_first_pair_component_stats
 * (include/hdfe/hdfe_regressor_v11.hpp:68-79, src/hdfe_regressor_v11.cpp:7192-7270). */
int b200fe_first_pair_components_device(b200fe_context* ctx, const int32_t* d_fe1,
                                        const int32_t* d_fe2, int64_t n,
                                        const double* d_weights, int* num_components,
                                        int64_t* largest_component_n_obs,
                                        double* largest_component_obs_share,
                                        double* largest_component_weight_share);

/* ---------------------------------------------------------------------------
 * OLS on within-transformed data: the reference's hdfe::detail::run_ols
 * (include/ols.hpp:40-51, src/ols.cpp:1237-1520) with its covariance
 * conventions (compute_covariance, src/ols.cpp:495-700): coefficients from
 * X'WX b = X'Wy, residuals e = y - X b, RSS = sum w e^2, df_resid =
 * max(0, n_eff - p), and
 *   se_type 0 (homoskedastic): cov = RSS/df_resid (X'WX)^-1;
 *   se_type 1 (robust):        cov = (X'WX)^-1 [sum (w e)^2 x x'] (X'WX)^-1
 *                              (frequency weights: sum w e^2 x x');
 *   se_type 2 (cluster):       cov = scale (X'WX)^-1 [sum_g s_g s_g'] (X'WX)^-1,
 *                              s_g = sum_{i in g} w e x, scale =
 *                              G/(G-1) (n_eff-1)/df_resid, G = non-empty clusters.
 * The data-sized moments (Gram, residual pass, cluster scores in cluster
 * order) run on the device with fixed-order sums; the p x p algebra on the
 * host.  X is n x p column-major (ld = n), p <= B200FE_OLS_MAX_P; cluster ids
 * dense in [0, num_clusters).  n_effective <= 0 means n.
 * ------------------------------------------------------------------------- */
#define B200FE_OLS_MAX_P 32

typedef struct b200fe_ols_result {
    int p;
    int num_clusters;
    double rss, sigma2, df_resid, cov_scale, cluster_u2;
    double coef[B200FE_OLS_MAX_P];
    double se[B200FE_OLS_MAX_P];
    double cov[B200FE_OLS_MAX_P * B200FE_OLS_MAX_P];      /* p x p column-major */
    double xtx_inv[B200FE_OLS_MAX_P * B200FE_OLS_MAX_P];  /* p x p column-major */
} b200fe_ols_result;

/* Device arrays (e.g. the output of b200fe_absorb_device: y = column 0, X =
 * the next p columns).  Returns B200FE_INVALID_ARG when X'WX is not
 * positive definite (the reference throws "Failed to factorize X'X"). */
int b200fe_ols_device(b200fe_context* ctx, const double* d_y, const double* d_X,
                      int64_t n, int p, const double* d_weights,
                      const int32_t* d_clusters, int32_t num_clusters, int se_type,
                      double n_effective, int weights_are_frequencies,
                      b200fe_ols_result* out);
/* Host arrays (copied in on the context's stream). */
int b200fe_ols(b200fe_context* ctx, const double* y, const double* X, int64_t n, int p,
               const double* weights, const int32_t* clusters, int32_t num_clusters,
               int se_type, double n_effective, int weights_are_frequencies,
               b200fe_ols_result* out);

/* ---------------------------------------------------------------------------
 * AKM/KSS two-way solver: Jacobi-PCG on the grounded worker-partialled firm
 * Laplacian S = Df - B' Dw^{-1} B over the match (worker-firm pair) structure,
 * the firm-side system of the leave-out (KSS) variance decomposition.  The
 * ground firm is the last one (J - 1): its rhs entry is ignored and its
 * solution entry is zero.  FP64 throughout; reductions have a fixed order, so
 * results are bitwise reproducible on a device.
 * ------------------------------------------------------------------------- */
typedef struct b200fe_kss b200fe_kss;

/* Builds a solver context on the current device from host arrays: matches
 * m = 0..n_matches-1 sorted by worker (m_w non-decreasing) with firms m_f and
 * weights m_c; w_ptr[N+1] / f_ptr[J+1] the worker and firm CSR offsets;
 * f_matches[n_matches] the match ids in firm order; Dw[N], Df[J] the worker
 * and firm weight sums; inv_diagS[J] the Jacobi preconditioner (0 at the
 * ground).  The arrays are copied; the caller may free them on return.
 * Replaces hdfe::akm::akm_cuda_create (include/hdfe/akm_kss_cuda.hpp:30-36,
 * src/akm_kss_cuda.cu:330-380). */
int b200fe_kss_create(int n_workers, int n_firms, const int32_t* m_w,
                      const int32_t* m_f, const double* m_c, int64_t n_matches,
                      const int64_t* w_ptr, const int64_t* f_ptr,
                      const int64_t* f_matches, const double* Dw,
                      const double* Df, const double* inv_diagS,
                      b200fe_kss** out);
/* Replaces akm_cuda_destroy (akm_kss_cuda.hpp:38). */
void b200fe_kss_destroy(b200fe_kss* kss);
const char* b200fe_kss_last_error(const b200fe_kss* kss);
/* Largest nb of b200fe_kss_solve_multi.  Replaces akm_cuda_max_lanes
 * (akm_kss_cuda.hpp:62-64). */
int b200fe_kss_max_lanes(void);
/* Page-locked host buffer of nb * J doubles owned by the context (NULL if
 * pinned memory is unavailable); valid until a larger nb is requested or the
 * context is destroyed.  It may serve as both rhs_pack and z_pack.
 * Replaces akm_cuda_pack_buffer (akm_kss_cuda.hpp:66-76). */
double* b200fe_kss_pack_buffer(b200fe_kss* kss, int nb);
/* nb independent grounded solves S z_l = rhs_l, lane-major packs (lane l at
 * offset l*J); x0 = 0; lane l stops when ||r_l||^2 <= tol^2 ||rhs_l||^2
 * (rhs with its ground entry zeroed) and iters_out[l] receives its
 * iteration count, or -1 (its z zeroed) when it does not converge within
 * max_iter or its curvature p'Sp is not positive and finite.  Returns
 * B200FE_OK (individual lane failures are reported per lane) or an error
 * status.  rhs_pack and z_pack may be the same buffer.
 * Replaces akm_cuda_solve_S_multi (akm_kss_cuda.hpp:49-60,
 * src/akm_kss_cuda.cu:530-650). */
int b200fe_kss_solve_multi(b200fe_kss* kss, const double* rhs_pack, double* z_pack,
                           int nb, double tol, int max_iter, int* iters_out);
/* One solve; *iterations receives the count.  Returns B200FE_OK,
 * B200FE_NOT_CONVERGED (z zeroed) or an error status.
 * Replaces akm_cuda_solve_S (akm_kss_cuda.hpp:40-44, src/akm_kss_cuda.cu:655-700). */
int b200fe_kss_solve(b200fe_kss* kss, const double* rhs, double* z, double tol,
                     int max_iter, int* iterations);
/* JLA leverages of the leave-out decomposition for `draws` Rademacher draws,
 * on the device: per draw d, working row r gets the sign bit r % 64 of the
 * SplitMix64 stream (seed, 3d, r / 64), match m the sum of m_cnt[m] signs of
 * the stream (seed, 3d + 1, m); the worker/firm scatters of row_sw[r] * sign
 * (row_sw NULL: 1) and of the centred match sums solve K z = (tw1, tf1),
 * (0, tf2), (tw2, 0) in batches of `block` draws (three lanes each; 0: 8),
 * and every row accumulates, in ascending draw order, the sums of the
 * ratio estimator and its nonlinearity correction.  Rows are given by
 * their worker row_w and firm row_f (0-based, the context's numbering) in
 * the caller's row order, which indexes the streams; m_cnt[M] are the
 * person-year counts of the matches, n_py their total.  Outputs (host, R
 * each, any may be NULL): pii, mii (ratio estimates), corr (nonlinearity
 * correction), bfe, bpe, bcov (sums over draws of W2^2, W1^2, W1 W2).  The
 * solves stop as b200fe_kss_solve_multi (tol, max_iter); *failed_lanes
 * counts lanes that did not converge (B200FE_NOT_CONVERGED when > 0) and
 * *iterations sums the others' iterations.
 * Replaces the JLA draw loop of hdfe::akm::akm_kss_decompose
 * (src/akm_kss.cpp:2753-3160, the ratio estimator :3275-3289), whose solves
 * go through akm_cuda_solve_S_multi. */
int b200fe_kss_jla(b200fe_kss* kss, int64_t n_rows, const int32_t* row_w, const int32_t* row_f,
                   const double* row_sw, const int64_t* m_cnt, double n_py, uint64_t seed, int draws,
                   int block, double tol, int max_iter, double* pii, double* mii, double* corr,
                   double* bfe, double* bpe, double* bcov, int* failed_lanes, long long* iterations);
/* Stable ascending sort of host uint64 keys: order_out[i] is the input row of
 * the i-th smallest key, equal keys in input order.
 * Replaces akm_cuda_stable_sort_u64 (akm_kss_cuda.hpp:21-28). */
int b200fe_stable_sort_u64(const uint64_t* keys, int64_t* order_out, int64_t n);

#ifdef __cplusplus
}
#endif

#endif /* B200FE_H */
