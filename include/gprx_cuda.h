/*
 * gprx_cuda.h — C ABI of the B200 (sm_100a) backend for gprx's exact-GPR and
 * VFE-SGPR objective-and-prediction path.
 *
 * The reference (gprx 0.2.0, a Rust crate) has no FFI layer: its seams are
 * Rust traits.  Each entry point below names the reference function whose
 * work it takes over; a Rust `cuda` backend calls it from that seam through
 * an `extern "C"` block that mirrors these declarations.
 *
 * Conventions
 *  - Every call returns a gprx_status.  No exception, abort or panic crosses
 *    this boundary.  A failed call leaves the handle as it was before the call
 *    unless the entry point says otherwise; gprx_last_error() gives details.
 *  - Host buffers are owned by the caller and only read or written during the
 *    call.  Points are column-major: x[i + f*n] is feature f of point i
 *    (gprx `data::pack_points`, src/data.rs).
 *  - Hyperparameters are in log space, kernel parameters first in depth-first
 *    leaf order, then log σn² (src/gpr/exact_fit.rs:212-236; docs/design.md
 *    §"parameter order").
 *  - One handle owns one CUDA stream and its device state; a handle is not
 *    re-entrant, distinct handles may be used from distinct threads.
 */
#ifndef GPRX_CUDA_H
#define GPRX_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GPRX_CUDA_ABI_VERSION 1

/* ---- status codes: each maps onto a gprx GprError variant (src/error.rs:308-500) ---- */
typedef int32_t gprx_status;
enum {
  GPRX_OK = 0,
  GPRX_CHOLESKY_FAILED = 1,        /* GprError::CholeskyFailed{jitter, matrix_size, stage} */
  GPRX_NONFINITE_KERNEL = 2,       /* GprError::NonFiniteKernelValue */
  GPRX_SHAPE_MISMATCH = 3,         /* ShapeMismatch / LengthMismatch / DimensionMismatch */
  GPRX_INVALID_POINT_ID = 4,       /* IndexOutOfRange on an unknown PointId (src/points.rs:156) */
  GPRX_INSUFFICIENT_DATA = 5,      /* InsufficientData{n, min: 2} (src/gpr/online.rs:565) */
  GPRX_CUDA_ERROR = 6,             /* no gprx counterpart: a CUDA runtime error */
  GPRX_TIMEOUT = 7,                /* no gprx counterpart: a bounded device wait ran out */
  GPRX_INVALID_HYPERPARAMETER = 8, /* InvalidHyperparameter / IntervalError::OutOfRange */
  GPRX_NONFINITE_INPUT = 9,        /* NonFiniteInput */
  GPRX_EMPTY_INPUT = 10,           /* EmptyInput */
  GPRX_OUT_OF_MEMORY = 11,         /* no gprx counterpart: device allocation or HBM budget */
  GPRX_INVALID_CONFIG = 12,        /* InvalidConfig */
  GPRX_NOT_CONVERGED = 13,         /* OptimizationNotConverged{iterations} */
  GPRX_INVALID_ARGUMENT = 14,      /* null handle / null pointer / bad enum */
  GPRX_STALE_FACTOR = 15,          /* internal: the factor was consumed by a gradient */
  GPRX_CAPACITY = 16,              /* a fixed-size buffer was too small for the request */
  GPRX_NOT_POSITIVE_DEFINITE = 17, /* GprError::NonPositiveDefiniteMatrix (a leave-one-out [K⁻¹]_ii ≤ 0) */
  GPRX_PERSIST_FAILED = 18,        /* GprError::PersistFailed{kind, reason} (src/persist/mod.rs) */
  GPRX_UNSUPPORTED_PERSIST_VERSION = 19 /* GprError::UnsupportedPersistVersion */
};

/* CholeskyStage (src/error.rs:31-39) */
enum {
  GPRX_STAGE_FIT = 0,
  GPRX_STAGE_PREDICT = 1,
  GPRX_STAGE_ONLINE_INSERT = 2,
  GPRX_STAGE_ONLINE_DELETE = 3
};

typedef struct {
  gprx_status status;
  double jitter;          /* CHOLESKY_FAILED: the last offset j tried */
  uint64_t matrix_size;   /* CHOLESKY_FAILED: order of the matrix */
  int32_t stage;          /* CHOLESKY_FAILED: GPRX_STAGE_* */
  int32_t cuda_error;     /* CUDA_ERROR: the cudaError_t value */
  uint64_t iterations;    /* NOT_CONVERGED: iterations run */
  char message[256];
} gprx_error_info;

/* ---- kernel description: a flattened KernelSpec tree (src/kernel/spec.rs:106) ----
 * Nodes are listed in prefix order.  SUM and PRODUCT give their arity in
 * `arg`; RBF_ARD gives its number of dimensions in `arg`.  θ for the leaves is
 * passed separately, in the same (depth-first) order:
 *   RBF        1 param  log ℓ               k = exp(-r²/(2ℓ²))        (src/kernel/rbf.rs:18)
 *   RBF_ARD    d params log ℓ_1..log ℓ_d    k = exp(-½ Σ Δ_f²/ℓ_f²)   (src/kernel/rbf_ard.rs:16)
 *   CONSTANT   1 param  log c               k = c                     (src/kernel/constant.rs:12)
 *   PERIODIC   2 params log ℓ, log p        k = exp(-2 sin²(π r/p)/ℓ²) (src/kernel/periodic.rs:598) */
enum {
  GPRX_NODE_SUM = 1,
  GPRX_NODE_PRODUCT = 2,
  GPRX_LEAF_RBF = 10,
  GPRX_LEAF_RBF_ARD = 11,
  GPRX_LEAF_CONSTANT = 12,
  GPRX_LEAF_PERIODIC = 13
};

typedef struct {
  int32_t kind;
  int32_t arg;
} gprx_kernel_node;

/* Upper limits of the device kernel evaluator. */
#define GPRX_MAX_NODES 16
#define GPRX_MAX_PARAMS 40
#define GPRX_MAX_DIM 32

enum { GPRX_PRECISION_FP64 = 0, GPRX_PRECISION_MIXED = 1 };
enum { GPRX_VARIANCE_LATENT = 0, GPRX_VARIANCE_OBSERVATION = 1 }; /* src/prediction.rs */
enum { GPRX_JITTER_FIXED = 0, GPRX_JITTER_ADAPTIVE = 1 };          /* src/policy.rs:245,266 */

/* Model options.  gprx_options_default() fills the reference's defaults:
 * FP64, JitterPolicy::fixed(0.0) for exact models (src/policy.rs:230) and
 * JitterPolicy::adaptive(1e-8, 10, 5, 1e-3) for the Sgpr K_mm factor. */
typedef struct {
  int32_t precision;
  int32_t jitter_kind;
  double jitter_initial;
  double jitter_multiplier;
  int32_t jitter_max_retries;
  double jitter_max;
  int32_t device;
  int32_t block_size;     /* 0 = autotuned panel width of the blocked factor */
} gprx_options;

/* L-BFGS settings (src/optimizer/lbfgs.rs:28-46): history 10, ≤100 iterations,
 * gradient tolerance √ε, logit map onto (1e-5, 1e5) per parameter. */
typedef struct {
  uint64_t max_iterations;
  double tolerance;
  int32_t history_size;
  int32_t restarts;       /* extra starts (0 = none) */
  uint64_t seed;          /* seed of the extra starts */
  double interval_lo;     /* open interval of every parameter, user units */
  double interval_hi;
} gprx_lbfgs_options;

/* TrustRegion settings (src/optimizer/trust_region.rs:32-51): ≤100
 * iterations, gradient tolerance √ε, initial radius 1, maximum radius 100
 * (logit coordinates), the same logit map as L-BFGS. */
typedef struct {
  uint64_t max_iterations;
  double tolerance;
  double initial_radius;  /* 0 < initial_radius <= max_radius < inf */
  double max_radius;
  int32_t restarts;       /* extra starts (0 = none) */
  uint64_t seed;
  double interval_lo;
  double interval_hi;
} gprx_trust_region_options;

typedef struct {
  double nlml;
  uint64_t iterations;
  uint64_t evaluations;
  double grad_norm;
  int32_t converged;
} gprx_fit_report;

/* ------------------------------------------------------------------ */
/* common                                                               */
/* ------------------------------------------------------------------ */
int32_t gprx_abi_version(void);
void gprx_options_default(gprx_options* opt);
void gprx_options_default_sparse(gprx_options* opt);
void gprx_lbfgs_options_default(gprx_lbfgs_options* opt);
void gprx_trust_region_options_default(gprx_trust_region_options* opt);
/* Details of the last failed call on this thread. */
gprx_status gprx_last_error(gprx_error_info* out);
/* Number of kernels this library launched since load (instrumentation). */
uint64_t gprx_launch_count(void);

/* ------------------------------------------------------------------ */
/* exact GPR (src/gpr/)                                                 */
/* ------------------------------------------------------------------ */
typedef struct gprx_exact gprx_exact;

/* Validates and uploads X (n×d, column-major) and y; sizes the n×n device
 * buffers.  Replaces FittedGpr::prepare + FitBuffers::new
 * (src/gpr/fitted.rs:210-290, src/workspace.rs:100-119).  No factor yet. */
gprx_status gprx_exact_create(const double* x, uint64_t n, uint64_t d, const double* y,
                              const gprx_kernel_node* nodes, int32_t n_nodes,
                              const double* theta, int32_t n_theta,
                              const gprx_options* options, gprx_exact** out);
gprx_status gprx_exact_destroy(gprx_exact* h);
/* Re-uploads X and y of the same shape (the handle keeps its buffers). */
gprx_status gprx_exact_set_data(gprx_exact* h, const double* x, const double* y);
uint64_t gprx_exact_num_params(const gprx_exact* h);
/* log θ of the kernel then log σn² (Gpr::get_params). */
gprx_status gprx_exact_get_params(gprx_exact* h, double* out, uint64_t p);
/* The training points in buffer order: x (n×d, column-major, n rows) and y
 * (n), host memory (FittedGpr::x / y, src/gpr/fitted.rs:1091,324; an online
 * model's current points, in the order of gprx_online_point_ids). */
gprx_status gprx_exact_data(gprx_exact* h, double* x_out, double* y_out);
/* Writes θ and factors A = K + σn² I (+ jitter retries) at it; on failure
 * the previous θ and its factor are restored (src/gpr/exact_fit.rs:196-206).
 * On an online model this, gprx_exact_eval, gprx_exact_hessian and
 * gprx_exact_value_gradient_hessian run through an LLT of the current points
 * and leave the model online at the new θ; a failure leaves its LDLT, α and θ
 * unchanged (OnlineGpr::set_params / value_and_gradient_into / hessian_into,
 * src/gpr/online.rs:659-697, with_llt_view :1151-1185). */
gprx_status gprx_exact_set_params(gprx_exact* h, const double* params, uint64_t p);
/* Factors at the stored θ (Gpr<Fixed>::factor → factor_written_k_with_policy,
 * src/gpr/factor.rs:515-542). */
gprx_status gprx_exact_factor(gprx_exact* h);
/* One NLML + gradient evaluation at `params` (ExactFit::value_and_gradient_into_fit,
 * src/gpr/exact_fit.rs:319-341).  `grad` may be NULL (value only). */
gprx_status gprx_exact_eval(gprx_exact* h, const double* params, uint64_t p,
                            double* nlml, double* grad);
/* Hessian of the NLML at `params`, row-major p × p into `out`
 * (FittedGpr::hessian_into, src/gpr/fitted.rs:665; ExactFit::hessian_into_fit,
 * src/gpr/exact_fit.rs:443-637).  Leaves the model at `params` as
 * gprx_exact_eval with a gradient does. */
gprx_status gprx_exact_hessian(gprx_exact* h, const double* params, uint64_t p, double* out);
/* NLML, gradient and Hessian of one evaluation at `params`
 * (TwiceDifferentiable::value_gradient_hessian_into, src/objective.rs:427;
 * ExactFit::value_gradient_hessian_into_fit, src/gpr/exact_fit.rs:468-482). */
gprx_status gprx_exact_value_gradient_hessian(gprx_exact* h, const double* params, uint64_t p, double* nlml,
                                              double* grad, double* hess);
/* NLML of the current factor (GprCore::neg_log_marginal_likelihood, src/gpr/shared.rs:245-260). */
gprx_status gprx_exact_nlml(gprx_exact* h, double* nlml);
/* jitter j the current factor took (ExactFit factor_jitter). */
gprx_status gprx_exact_factor_jitter(gprx_exact* h, double* jitter);
/* Predictive mean and diagonal variance at q query points (column-major q×d)
 * (GprCore::write_moments, src/gpr/shared.rs:754-820). */
gprx_status gprx_exact_predict(gprx_exact* h, const double* xs, uint64_t q, int32_t variance_kind,
                               double* mean, double* var);
/* Predictive mean and diagonal variance for k requests against k fitted
 * exact models in one launch (no counterpart in the reference: each request
 * is one GprCore::write_moments, src/gpr/shared.rs:754-820; the serving loop
 * batches small predictions of different models with it).  Request i asks
 * handles[i] at q[i] points xs[i] (column-major q[i]×d) and receives mean[i]
 * and var[i] (q[i] values each); a handle may appear several times.  Every
 * model has at most 1024 points and 16 features, is not online, and all share
 * one device, d and the kernel's ARD width (else GPRX_CAPACITY /
 * GPRX_INVALID_CONFIG).  One CTA computes each 16-query tile of a request in
 * a fixed order, so a request's results do not depend on the others; they
 * agree with gprx_exact_predict to rounding (a different summation order).
 * The work runs on handles[0]'s stream; the call returns when it is done. */
gprx_status gprx_exact_predict_group(gprx_exact* const* handles, uint64_t k, const double* const* xs,
                                     const uint64_t* q, int32_t variance_kind, double* const* mean,
                                     double* const* var);

/* Saved models (gprx's format_version 1: <dir>/config.json and
 * <dir>/model.safetensors, docs/persist-format.md; src/persist/mod.rs).
 * gprx_exact_save writes x, y, the kernel tree, noise and jitter policy
 * (FittedGpr::save, OnlineGpr::save); with_factor also writes l and α
 * (save_with_factor: l is L of an LLT model, or the unit-lower L with D on
 * the diagonal of an online LDLT model with its point ids).  gprx_exact_load
 * reads such a directory into a resident handle on `device` (LoadedGpr::load):
 * a stored factor is copied to the device straight from the mapped file and
 * the model predicts without refactoring; without one the first use factors.
 * This backend reads and writes rbf / rbf_ard / constant / periodic leaves
 * under sum / product, identity input and target maps and double precision;
 * other files are refused with GPRX_PERSIST_FAILED naming what is missing. */
gprx_status gprx_exact_save(gprx_exact* h, const char* dir, int32_t with_factor);
gprx_status gprx_exact_load(const char* dir, int32_t device, gprx_exact** out);
/* Host-side access to a saved directory (no GPU needed). */
typedef struct {
  uint64_t n, d;
  int32_t n_nodes, n_theta;   /* n_theta = kernel parameters + 1 */
  int32_t has_factor;         /* 1: l and alpha are stored */
  int32_t factor_kind;        /* 0 llt, 1 ldlt */
  double factor_jitter;
  gprx_options jitter;        /* the stored jitter policy (other fields default) */
  uint64_t next_point_id;     /* ldlt only */
} gprx_persist_info;
gprx_status gprx_persist_inspect(const char* dir, gprx_persist_info* out);
/* nodes[n_nodes], theta[n_theta] (log), x[n·d] column-major, y[n]; l[n·n]
 * and alpha[n] when has_factor (nullable), point_ids[n] when ldlt (nullable). */
gprx_status gprx_persist_read(const char* dir, gprx_kernel_node* nodes, double* theta, double* x, double* y,
                              double* l, double* alpha, uint64_t* point_ids);
/* Writes a model directory from host arrays (factor_kind 0 llt / 1 ldlt;
 * l and alpha nullable = no factor; point_ids required for ldlt). */
gprx_status gprx_persist_write(const char* dir, const double* x, uint64_t n, uint64_t d, const double* y,
                               const gprx_kernel_node* nodes, int32_t n_nodes, const double* theta, int32_t n_theta,
                               const gprx_options* jitter, const double* l, const double* alpha, int32_t factor_kind,
                               double factor_jitter, const uint64_t* point_ids, uint64_t next_point_id);

/* Leave-one-out mean and variance at every training point (GPML §5.4.2):
 * mean_i = y_i − α_i / Q_ii, observation variance 1 / Q_ii, latent
 * max(0, 1 / Q_ii − σn²), Q = (K + σn² I)⁻¹ (FittedGpr::loo_predict_with,
 * src/gpr/fitted.rs:712; GprCore::loo_predict_with, src/gpr/shared.rs:522-567;
 * OnlineGpr::loo_predict_with, src/gpr/online.rs:716).  mean, var: n values
 * in training (index) order.  Q_ii ≤ 0 → GPRX_NOT_POSITIVE_DEFINITE. */
gprx_status gprx_exact_loo(gprx_exact* h, int32_t variance_kind, double* mean, double* var);
/* Predictive mean and the q×q query covariance K** − VᵀV, V = L⁻¹K(X, X*)
 * (D-weighted for an online LDLT model); latent diagonal clipped at 0,
 * observation adds σn² on the diagonal (FittedGpr::predict_covariance_with,
 * src/gpr/fitted.rs:992; GprCore::write_covariance, src/gpr/shared.rs:425-520).
 * cov: column-major q×q. */
gprx_status gprx_exact_predict_covariance(gprx_exact* h, const double* xs, uint64_t q, int32_t variance_kind,
                                          double* mean, double* cov);
/* n_draws posterior draws at the queries, column-major q × n_draws: column k
 * is μ + L z_k with L the Cholesky factor of the predictive covariance
 * (retried with the model's jitter policy, stage PREDICT) and z_k the next q
 * unit normals of the seeded generator at `seed` (FittedGpr::sample_with,
 * src/gpr/fitted.rs:1056; PredictiveCovariance::draw, src/prediction.rs:206-243).
 * Zero draws form the covariance and write nothing. */
gprx_status gprx_exact_sample(gprx_exact* h, const double* xs, uint64_t q, int32_t variance_kind, uint64_t n_draws,
                              uint64_t seed, double* out);
/* α = A⁻¹ y of the current factor (n values). */
gprx_status gprx_exact_alpha(gprx_exact* h, double* out, uint64_t n);
/* Gpr::fit with the default Lbfgs (src/gpr/trainer.rs:533-613, src/optimizer/lbfgs.rs:126-172):
 * optimizes θ, then refactors at the best θ and publishes α for predict. */
gprx_status gprx_exact_fit(gprx_exact* h, const gprx_lbfgs_options* opt, gprx_fit_report* report);
/* Gpr::fit with the TrustRegion optimizer (src/optimizer/trust_region.rs:143-258):
 * trust region with the Steihaug subproblem over gprx_exact_value_gradient_hessian
 * in logit coordinates, then the factor at the best θ.  NULL opt = defaults. */
gprx_status gprx_exact_fit_trust_region(gprx_exact* h, const gprx_trust_region_options* opt,
                                        gprx_fit_report* report);
/* Per-stage device time of the last eval in milliseconds:
 * [fill, factor, inverse, gradient, total] (the reference's insert-stages idea). */
gprx_status gprx_exact_stage_times(gprx_exact* h, double* out5);

/* The CUDA stream (a cudaStream_t) the handle enqueues its work on, so a
 * caller can time the handle's kernels with events on that stream. */
gprx_status gprx_exact_stream(gprx_exact* h, void** stream);

/* ---- online exact GPR (src/gpr/online.rs) ---- */
/* FittedGpr::into_online: LLT → LDLT (src/gpr/fitted.rs:757-765,
 * src/gpr/factor_store.rs:157-179); assigns PointIds 0..n-1. */
gprx_status gprx_online_begin(gprx_exact* h);
/* OnlineGpr::insert (src/gpr/online.rs:794-906): bordered LDLT append. */
gprx_status gprx_online_insert(gprx_exact* h, const double* x_new, double y_new, uint64_t* id);
/* OnlineGpr::delete (src/gpr/online.rs:564-611): LDLT row/column delete. */
gprx_status gprx_online_delete(gprx_exact* h, uint64_t id);
uint64_t gprx_online_n(const gprx_exact* h);
/* PointIds in buffer order (src/points.rs:76). */
gprx_status gprx_online_point_ids(gprx_exact* h, uint64_t* out, uint64_t n);

/* ------------------------------------------------------------------ */
/* VFE sparse GPR (src/sgpr/)                                           */
/* ------------------------------------------------------------------ */
typedef struct gprx_sgpr gprx_sgpr;

/* Uploads X (n×d), y and the inducing points Z (m×d); SparseCore::prepare
 * (src/sparse/core.rs:314).  No assembly yet. */
gprx_status gprx_sgpr_create(const double* x, uint64_t n, uint64_t d, const double* y,
                             const double* z, uint64_t m,
                             const gprx_kernel_node* nodes, int32_t n_nodes,
                             const double* theta, int32_t n_theta,
                             const gprx_options* options, gprx_sgpr** out);
gprx_status gprx_sgpr_destroy(gprx_sgpr* h);
uint64_t gprx_sgpr_num_params(const gprx_sgpr* h);
gprx_status gprx_sgpr_get_params(gprx_sgpr* h, double* out, uint64_t p);
/* assemble_vfe at the stored θ (src/sgpr/factor/vfe.rs:191-277). */
gprx_status gprx_sgpr_factor(gprx_sgpr* h);
/* Writes θ and reassembles at it; on failure the previous θ and its
 * assembly are restored (FittedSgpr::set_params, src/sgpr/fitted.rs). */
gprx_status gprx_sgpr_set_params(gprx_sgpr* h, const double* params, uint64_t p);
/* FittedSgpr::value_and_gradient_into (src/sgpr/fitted.rs:306-326):
 * reassembly, vfe_neg_log_marginal_likelihood (vfe.rs:338-369) and
 * analytic_gradient (derivatives.rs:283-366).  `grad` may be NULL. */
gprx_status gprx_sgpr_eval(gprx_sgpr* h, const double* params, uint64_t p, double* nlml, double* grad);
gprx_status gprx_sgpr_nlml(gprx_sgpr* h, double* nlml);
/* vfe_predict_into / vfe_latent (src/sgpr/factor/predict.rs:102-262). */
gprx_status gprx_sgpr_predict(gprx_sgpr* h, const double* xs, uint64_t q, int32_t variance_kind,
                              double* mean, double* var);
/* Mean and the q×q query covariance of the VFE posterior, column-major:
 * off the diagonal K** − A*ᵀA* + σn² S*ᵀS* (A* = L_mm⁻¹ K_m*, S* = L_B⁻¹ A*),
 * on it the predictive variance of gprx_sgpr_predict
 * (FittedSgpr::predict_covariance_with, src/sgpr/fitted.rs:818-850;
 * src/sgpr/factor/predict.rs:263-345, src/sparse/core.rs:641-667). */
gprx_status gprx_sgpr_predict_covariance(gprx_sgpr* h, const double* xs, uint64_t q, int32_t variance_kind,
                                         double* mean, double* cov);
/* Posterior draws from that covariance, as gprx_exact_sample (the model's
 * jitter retries; FittedSgpr::sample_with, src/sgpr/fitted.rs:855-900). */
gprx_status gprx_sgpr_sample(gprx_sgpr* h, const double* xs, uint64_t q, int32_t variance_kind, uint64_t n_draws,
                             uint64_t seed, double* out);
gprx_status gprx_sgpr_fit(gprx_sgpr* h, const gprx_lbfgs_options* opt, gprx_fit_report* report);
/* OnlineSgpr::insert → append_point (src/sgpr/online/mod.rs:1695-1810). */
gprx_status gprx_sgpr_insert(gprx_sgpr* h, const double* x_new, double y_new, uint64_t* id);
/* OnlineSgpr::delete (src/sgpr/online/mod.rs:903-1000): rank-1 downdate of L_B,
 * reassembly when the downdate fails or the pivot gate does not hold. */
gprx_status gprx_sgpr_delete(gprx_sgpr* h, uint64_t id);
uint64_t gprx_sgpr_n(const gprx_sgpr* h);
/* 1 when the last insert/delete (of a point or of an inducing point)
 * updated in place, 0 when it reassembled. */
int32_t gprx_sgpr_last_step_in_place(const gprx_sgpr* h);
/* PointIds in registry order (src/points.rs:76). */
gprx_status gprx_sgpr_point_ids(gprx_sgpr* h, uint64_t* out, uint64_t n);
/* Replaces the inducing set Z (m×d) and reassembles: an inducing insert or
 * delete (OnlineSgpr::insert_inducing / delete_inducing, src/sgpr/online/mod.rs:1301,1943)
 * taken by reassembly. */
gprx_status gprx_sgpr_set_inducing(gprx_sgpr* h, const double* z, uint64_t m);
/* OnlineSgpr::insert_inducing / delete_inducing / inducing_ids
 * (src/sgpr/online/mod.rs:1943,1301,694): append one inducing point (its id
 * is returned; ids are never reused) or remove one by id (m ≤ 1 →
 * GPRX_INSUFFICIENT_DATA, unknown id → GPRX_INVALID_POINT_ID).  An insert
 * takes the bordered update of the factors and one new row of A (O(n m);
 * inducing_append, src/sgpr/factor/updates.rs:296-390) when K_mm's factor
 * took no jitter, its pivots hold (min L_ii² / K_ii > 1e-5) and both bordered
 * pivots exceed 1e-5 of their diagonal, and room for the row exists;
 * otherwise, and for a delete, the VFE system of the new set is assembled
 * (O(n m²), the reference's own fallback), so the model equals Sgpr::factor
 * at the same θ, X and Z (within 1e-10 after a bordered insert).
 * gprx_sgpr_last_step_in_place tells which.  On an error the model keeps its
 * inducing set. */
gprx_status gprx_sgpr_insert_inducing(gprx_sgpr* h, const double* z_new, uint64_t* id);
gprx_status gprx_sgpr_delete_inducing(gprx_sgpr* h, uint64_t id);
uint64_t gprx_sgpr_m(const gprx_sgpr* h);
gprx_status gprx_sgpr_inducing_ids(const gprx_sgpr* h, uint64_t* out, uint64_t m);

/* Sharded VFE evaluation: n split over processes (one GPU each), each
 * process holding a handle created with ITS points and the SAME inducing
 * inputs Z; K_mm and its factor are replicated.  The sums over n that the
 * assembly and the gradient need (assemble_vfe, src/sgpr/factor/vfe.rs:191-277;
 * analytic_gradient, src/sgpr/factor/derivatives.rs:283-366) travel in two
 * device exchange buffers owned by the caller (doubles, sizes from
 * gprx_sgpr_shard_sizes), which the caller sums over the processes (an
 * all-reduce) between the calls:
 *   gprx_sgpr_shard_assemble(h, θ, exchange1)   -> this shard's sums
 *   all-reduce(exchange1)
 *   gprx_sgpr_shard_nlml(h, exchange1, &nlml, exchange2 or NULL)
 *   all-reduce(exchange2)
 *   gprx_sgpr_shard_gradient(h, exchange2, grad)
 * Every process gets the same NLML and gradient, equal to the unsharded
 * evaluation's; afterwards the handle predicts with the global posterior.
 * Each call returns after its work has finished on the handle's stream. */
gprx_status gprx_sgpr_shard_sizes(const gprx_sgpr* h, uint64_t* exchange1, uint64_t* exchange2);
gprx_status gprx_sgpr_shard_assemble(gprx_sgpr* h, const double* params, uint64_t p, double* exchange1);
gprx_status gprx_sgpr_shard_nlml(gprx_sgpr* h, const double* exchange1, double* nlml, double* exchange2);
gprx_status gprx_sgpr_shard_gradient(gprx_sgpr* h, const double* exchange2, double* grad);
/* jitter j the K_mm factor took. */
gprx_status gprx_sgpr_kmm_jitter(gprx_sgpr* h, double* jitter);
/* The CUDA stream (a cudaStream_t) of the handle, for event timing. */
gprx_status gprx_sgpr_stream(gprx_sgpr* h, void** stream);
/* Device time of the last assembly / gradient in ms: [K_mm + A, B + sums, gradient]. */
gprx_status gprx_sgpr_stage_times(gprx_sgpr* h, double* out3);



/* ------------------------------------------------------------------ */
/* batched exact GPR: many independent problems, one kernel tree        */
/* (no single reference counterpart: each problem is what Gpr::fit /    */
/* ExactFit::value_and_gradient_into_fit does for one model,            */
/* src/gpr/exact_fit.rs:319-341, src/optimizer/lbfgs.rs:28-172)         */
/* ------------------------------------------------------------------ */
typedef struct gprx_batch gprx_batch;

/* Largest n of one batched problem. */
#define GPRX_BATCH_MAX_N 2048

/* Uploads n_problems problems that share the kernel tree and d.  Problem i
 * has n[i] points; x holds the problems' n[i]×d column-major blocks one after
 * another and y their targets likewise.  n_theta = kernel parameters + 1. */
gprx_status gprx_batch_create(const double* x, const double* y, const uint64_t* n, uint64_t n_problems,
                              uint64_t d, const gprx_kernel_node* nodes, int32_t n_nodes, int32_t n_theta,
                              const gprx_options* options, gprx_batch** out);
gprx_status gprx_batch_destroy(gprx_batch* h);
uint64_t gprx_batch_num_params(const gprx_batch* h);
/* NLML and gradient of every problem at its own θ (row i of params,
 * n_problems × p, log space) in one launch.  status[i] is GPRX_OK or why
 * problem i could not be evaluated (its nlml / grad are then unset); the
 * call itself fails only for invalid arguments or a device error. */
gprx_status gprx_batch_eval(gprx_batch* h, const double* params, uint64_t p, double* nlml, double* grad,
                            int32_t* status);
/* Fits every problem as gprx_exact_fit fits one (L-BFGS over the logit map,
 * barrier on failed evaluations, restarts from the same seeded draws), with
 * all optimizers on the device and the evaluation rounds replayed from one
 * CUDA graph.  Writes the best θ (n_problems × p), one report and one status
 * per problem. */
gprx_status gprx_batch_fit(gprx_batch* h, const double* params0, uint64_t p, const gprx_lbfgs_options* opt,
                           double* params_out, gprx_fit_report* reports, int32_t* status);
/* The CUDA stream (a cudaStream_t) of the handle, for event timing. */
gprx_status gprx_batch_stream(gprx_batch* h, void** stream);

/* Schedule of the batched evaluation (no counterpart in the reference).
 * Problems fall into GPRX_BATCH_SIZE_CLASSES size classes (n ≤ 64, ≤ 128,
 * …, ≤ 4096, larger); each class runs its in-CTA FP64 GEMMs with one of
 * GPRX_BATCH_TILE_SHAPES tile shapes (0: 64×128×64, 1: 64×64×32,
 * 2: 32×64×32, 3: 32×32×16).  The first gprx_batch_eval / gprx_batch_fit
 * autotunes it: every class present is timed with every shape on a sample of
 * its problems and the fastest is kept (cached per device and kernel tree
 * for the life of the process).  Every shape gives the same results bit for
 * bit.  gprx_batch_autotune re-tunes at the given θ (n_problems × p);
 * gprx_batch_set_schedule fixes the shapes and turns tuning off;
 * gprx_batch_schedule reads the shapes, the tuning times (ms per launch,
 * classes × shapes, nullable) and whether tuning ran. */
#define GPRX_BATCH_SIZE_CLASSES 8
#define GPRX_BATCH_TILE_SHAPES 4
gprx_status gprx_batch_autotune(gprx_batch* h, const double* params, uint64_t p);
gprx_status gprx_batch_set_schedule(gprx_batch* h, const int32_t* tile_of_class);
gprx_status gprx_batch_schedule(const gprx_batch* h, int32_t* tile_of_class, float* tune_ms, int32_t* tuned);

/* ------------------------------------------------------------------ */
/* serving: a request loop over resident exact models on one GPU (no    */
/* counterpart in the reference; each request is the work of Gpr::fit, */
/* FittedGpr::predict_with, OnlineGpr::insert / delete)                 */
/* ------------------------------------------------------------------ */
typedef struct gprx_server gprx_server;

typedef struct {
  int32_t device;
  int32_t workers;            /* host worker threads = requests in flight */
  uint64_t hbm_budget_bytes;  /* device memory the resident models may take */
} gprx_server_options;

typedef struct {
  gprx_status status;
  uint64_t model;
  int32_t kind;               /* 0 fit, 1 predict, 2 add, 3 remove */
  int64_t submit_ns, start_ns, end_ns;  /* steady-clock times */
  int32_t merged;             /* requests that shared this request's launch */
  char message[256];
} gprx_request_info;

typedef struct {
  uint64_t completed;
  uint64_t merged_launches;      /* predict launches that served several requests */
  uint64_t used_bytes;
  uint64_t resident_models;
  uint64_t merged_fit_launches;  /* batched fit launches that served several models */
} gprx_server_stats_t;

void gprx_server_options_default(gprx_server_options* opt);
/* Starts the worker threads. */
gprx_status gprx_server_create(const gprx_server_options* opt, gprx_server** out);
/* Stops the workers (requests still queued are dropped) and frees every model. */
gprx_status gprx_server_destroy(gprx_server* s);
/* Queues a fit (optimize = 1: L-BFGS; 0: factor at θ) of a new model; the
 * request id is also the model id.  Inputs are copied at submission. */
gprx_status gprx_server_fit(gprx_server* s, const double* x, uint64_t n, uint64_t d, const double* y,
                            const gprx_kernel_node* nodes, int32_t n_nodes, const double* theta, int32_t n_theta,
                            const gprx_options* options, const gprx_lbfgs_options* lbfgs, int32_t optimize,
                            uint64_t* request_id);
/* Queues a prediction at q points (column-major q×d, copied); mean and var
 * (q values each) are written when the request completes and must stay
 * valid until gprx_server_wait returns for it. */
gprx_status gprx_server_predict(gprx_server* s, uint64_t model, const double* xs, uint64_t q, uint64_t d,
                                int32_t variance_kind, double* mean, double* var, uint64_t* request_id);
/* Queues an online insert of k points (x column-major k×d, copied); ids_out
 * (k values, may be NULL) receives their PointIds on completion. */
gprx_status gprx_server_add(gprx_server* s, uint64_t model, const double* x, const double* y, uint64_t k, uint64_t d,
                            uint64_t* ids_out, uint64_t* request_id);
/* Queues an online delete of k PointIds (copied). */
gprx_status gprx_server_remove(gprx_server* s, uint64_t model, const uint64_t* ids, uint64_t k,
                               uint64_t* request_id);
/* Blocks until the request completes; returns its status.  A completed
 * predict / add / remove request is forgotten after this call. */
gprx_status gprx_server_wait(gprx_server* s, uint64_t request_id, gprx_request_info* info);
gprx_status gprx_server_stats(gprx_server* s, gprx_server_stats_t* out);

/* Allocation-free NLML + gradient of ONE exact problem (no counterpart in the
 * reference).  For callers that cannot allocate device memory when they need
 * an evaluation: work issued while a CUDA graph is being captured, code inside
 * a framework or server that owns every byte of the device, or a loop that
 * cannot take the device-wide synchronisation of cudaMalloc/cudaFree.
 *  - x (n×d column-major), y, nlml, grad (p values, may be NULL) and status
 *    are DEVICE pointers owned by the caller; params (log θ, p values) and the
 *    kernel tree are host memory read during the call.
 *  - n ≤ 512 and p ≤ 16; larger requests return GPRX_CAPACITY / INVALID_CONFIG.
 *  - The work is enqueued on `stream` (a cudaStream_t; NULL = the current
 *    device's default stream) and runs on the device that owns the stream.
 *    The call returns without waiting: *status (a gprx_status) and the
 *    results are valid once the stream reaches them.  On a failed evaluation
 *    *status says why and nlml / grad are written as 0; a NaN or infinity in
 *    x or y gives GPRX_NONFINITE_INPUT.
 *  - Of `options` (NULL = gprx_options_default) the jitter fields and
 *    `device` are read; `device` must be the stream's device, else the call
 *    returns GPRX_INVALID_CONFIG without enqueuing work.
 *  - The scratch is one fixed 5.3 MB array in device memory per GPU, shared by
 *    every call: calls whose work overlaps on the GPU (other streams, other
 *    threads) race and must be ordered by the caller.  Each call starts from
 *    a fresh header, so the previous call's leftovers (another n, a failed
 *    factor) do not reach its result.
 *  - Set-up: the first call on a device looks up the array's device address
 *    and sets the kernel's shared-memory limit.  A call with n = 0 does only
 *    that (x, y, the kernel tree and the outputs are not read, nothing is
 *    enqueued) and returns GPRX_OK; make it, or any first call, before a
 *    stream capture begins.
 *  - Same result as gprx_batch_eval / gprx_exact_eval of the same problem
 *    (one CTA evaluates it in a fixed order). */
gprx_status gprx_exact_eval_noalloc(const double* x, const double* y, uint64_t n, uint64_t d,
                                    const gprx_kernel_node* nodes, int32_t n_nodes, const double* params, uint64_t p,
                                    const gprx_options* options, double* nlml, double* grad, int32_t* status,
                                    void* stream);

/* ------------------------------------------------------------------ */
/* device microbenchmarks (diagnostics; no gprx counterpart)            */
/* ------------------------------------------------------------------ */
/* ms per launch of the FP64 DMMA GEMM C(m×n) = op(A)·op(B), k deep. */
gprx_status gprx_probe_dgemm(int32_t m, int32_t n, int32_t k, int32_t trans_a, int32_t trans_b, int32_t reps,
                             double* ms_per_launch);
/* ms per blocked Cholesky factor of an n×n SPD matrix. */
gprx_status gprx_probe_potrf(int32_t n, int32_t reps, double* ms_per_factor);
/* int8-sliced FP64 product A·Bᵀ (S slices, 4..8) against the DMMA product on
 * random operands: out[0] ms per emulated GEMM, out[1] ms slicing both
 * operands, out[2] ms per DMMA GEMM, out[3] max |C − C_ref| / (|A|·|B|ᵀ),
 * out[4] ms per emulated update C −= A·Bᵀ (C read and written).  out holds
 * 5 doubles. */
gprx_status gprx_probe_emu_gemm(int32_t m, int32_t n, int32_t k, int32_t S, int32_t reps, double* out);

/* ------------------------------------------------------------------ */
/* seeded random numbers (src/rng.rs): Xoshiro256++ seeded by SplitMix64 */
/* ------------------------------------------------------------------ */
typedef struct { uint64_t s[4]; } gprx_rng;
void gprx_rng_seed(gprx_rng* rng, uint64_t seed);
uint64_t gprx_rng_next_u64(gprx_rng* rng);
double gprx_rng_unit(gprx_rng* rng);
uint64_t gprx_rng_up_to(gprx_rng* rng, uint64_t max);
double gprx_rng_normal(gprx_rng* rng);
void gprx_rng_fill_unit(gprx_rng* rng, double* out, uint64_t count);
void gprx_rng_fill_normal(gprx_rng* rng, double* out, uint64_t count);
/* `count` distinct indices of 0..n-1 by a partial Fisher–Yates shuffle
 * driven by up_to (the seeded inducing subset). */
gprx_status gprx_rng_subset(gprx_rng* rng, uint64_t n, uint64_t count, uint64_t* out);

#ifdef __cplusplus
}
#endif
#endif /* GPRX_CUDA_H */
