// capi.cu — the extern "C" boundary (include/gprx_cuda.h): argument checks,
// error records, the exact-GPR entry points, Gpr::fit over L-BFGS, and the
// seeded RNG (gprx src/rng.rs).

#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <new>
#include <string>

#include "exact.cuh"
#include "persist.h"
#include "lbfgs.h"
#include "trust_region.h"

namespace gprx {

static std::atomic<uint64_t> g_launches{0};
void count_launch(int k) { g_launches.fetch_add((uint64_t)k, std::memory_order_relaxed); }
uint64_t launches() { return g_launches.load(std::memory_order_relaxed); }

gprx_error_info& last_error() {
  static thread_local gprx_error_info info{};
  return info;
}

gprx_status set_error(gprx_status st, const std::string& msg) {
  gprx_error_info& e = last_error();
  std::memset(&e, 0, sizeof(e));
  e.status = st;
  std::snprintf(e.message, sizeof(e.message), "%s", msg.c_str());
  return st;
}

gprx_status set_cuda_error(cudaError_t err, const char* where) {
  gprx_status st = (err == cudaErrorMemoryAllocation) ? GPRX_OUT_OF_MEMORY : GPRX_CUDA_ERROR;
  set_error(st, std::string(cudaGetErrorString(err)) + " at " + where);
  last_error().cuda_error = (int)err;
  return st;
}

gprx_status set_cholesky_error(double jitter, uint64_t size, int stage) {
  set_error(GPRX_CHOLESKY_FAILED, "Cholesky factorization failed (non-positive pivot)");
  gprx_error_info& e = last_error();
  e.jitter = jitter;
  e.matrix_size = size;
  e.stage = stage;
  return GPRX_CHOLESKY_FAILED;
}

gprx_status status_to_error(const DevStatus& st, double jitter, uint64_t size, int stage) {
  switch (st.code) {
    case GPRX_OK: return GPRX_OK;
    case GPRX_CHOLESKY_FAILED: return set_cholesky_error(jitter, size, stage);
    case GPRX_NONFINITE_KERNEL: return set_error(GPRX_NONFINITE_KERNEL, "non-finite kernel value");
    case GPRX_TIMEOUT: return set_error(GPRX_TIMEOUT, "bounded device wait ran out");
    default: return set_error(st.code, "device status " + std::to_string(st.code));
  }
}

bool all_finite(const double* v, size_t n) {
  for (size_t i = 0; i < n; ++i)
    if (!std::isfinite(v[i])) return false;
  return true;
}

// ---------------------------------------------------------------------------
// fit: L-BFGS (host, reverse communication) over device evaluations
// ---------------------------------------------------------------------------
using EvalFn = gprx_status (*)(void* ctx, const double* log_theta, double* f, double* g);

gprx_status fit_lbfgs(void* ctx, EvalFn eval, int p, const double* theta0, const gprx_lbfgs_options* o,
                      gprx_fit_report* rep, std::vector<double>& best_theta) {
  gprx_lbfgs_options opt;
  if (o) opt = *o;
  else gprx_lbfgs_options_default(&opt);
  if (!(opt.interval_lo > 0.0) || !(opt.interval_hi > opt.interval_lo) || !std::isfinite(opt.interval_hi))
    return set_error(GPRX_INVALID_CONFIG, "parameter interval must be 0 < lo < hi");
  if (!(opt.tolerance >= 0.0) || !std::isfinite(opt.tolerance))
    return set_error(GPRX_INVALID_CONFIG, "L-BFGS gradient tolerance must be finite and >= 0");
  if (p > LBFGS_HOST_VARS) return set_error(GPRX_INVALID_CONFIG, "too many parameters for the optimizer");
  if (opt.history_size > LBFGS_HOST_HISTORY)
    return set_error(GPRX_INVALID_CONFIG, "L-BFGS history must be at most " + std::to_string(LBFGS_HOST_HISTORY));
  LogitMap map;
  map.init(opt.interval_lo, opt.interval_hi);
  LbfgsConfig cfg;
  cfg.history = opt.history_size > 0 ? opt.history_size : 10;
  cfg.max_iterations = opt.max_iterations;
  cfg.tol_grad = opt.tolerance;
  std::vector<double> z0(p);
  if (!map.from_log(theta0, p, z0.data())) return set_error(GPRX_INVALID_HYPERPARAMETER, "initial θ outside the interval");
  std::vector<double> logt(p), jac(p), g(p);
  double best_f = BARRIER_COST;
  std::vector<double> best_z;
  uint64_t total_evals = 0, iters = 0;
  double gnorm = 0.0;
  bool conv = false;
  gprx_rng rng;
  gprx_rng_seed(&rng, opt.seed);
  gprx_status first_err = GPRX_OK;
  for (int run = 0; run <= opt.restarts; ++run) {
    std::vector<double> zs(p);
    if (run == 0) {
      zs = z0;
    } else {
      // log-uniform start in each interval (optimizer/logit.rs sample_log_uniform_z)
      for (int i = 0; i < p; ++i) {
        double u = gprx_rng_unit(&rng);
        const double eps = 1.0 / 9007199254740992.0;
        u = std::min(std::max(u, eps), 1.0 - eps);
        double lt = map.ln_lo + u * (map.ln_hi - map.ln_lo);
        map.from_log(&lt, 1, &zs[i]);
      }
    }
    std::unique_ptr<HostLbfgs> lbp(new HostLbfgs());
    HostLbfgs& lb = *lbp;
    lb.start(cfg, zs.data(), p);
    gprx_status last = GPRX_OK;
    while (lb.task() == HostLbfgs::EVALUATE) {
      map.to_log(lb.point(), p, logt.data(), jac.data());
      double f;
      gprx_status st = eval(ctx, logt.data(), &f, g.data());
      if (st == GPRX_CUDA_ERROR || st == GPRX_OUT_OF_MEMORY || st == GPRX_TIMEOUT) return st;
      if (st != GPRX_OK || !std::isfinite(f)) {
        last = st;
        f = BARRIER_COST;
        std::fill(g.begin(), g.end(), 0.0);
      } else {
        for (int i = 0; i < p; ++i) g[i] *= jac[i];
      }
      lb.resume(f, g.data());
    }
    total_evals += lb.evaluations();
    if (lb.best_value() < best_f) {
      best_f = lb.best_value();
      best_z.assign(lb.best(), lb.best() + p);
      iters = lb.iterations();
      gnorm = lb.grad_norm();
      conv = lb.converged();
    }
    if (run == 0 && !(lb.best_value() < BARRIER_COST)) first_err = last != GPRX_OK ? last : GPRX_NOT_CONVERGED;
  }
  if (best_z.empty() || !(best_f < BARRIER_COST)) {
    if (first_err == GPRX_OK) first_err = GPRX_NOT_CONVERGED;
    gprx_status st = set_error(first_err, "no evaluable point was found");
    last_error().iterations = iters;
    return st;
  }
  best_theta.resize(p);
  map.to_log(best_z.data(), p, best_theta.data(), nullptr);
  if (rep) {
    rep->nlml = best_f;
    rep->iterations = iters;
    rep->evaluations = total_evals;
    rep->grad_norm = gnorm;
    rep->converged = conv ? 1 : 0;
  }
  return GPRX_OK;
}

// fit: trust region (host) over the joint value / gradient / Hessian
gprx_status fit_trust_region(ExactState& s, int p, const double* theta0, const gprx_trust_region_options* o,
                             gprx_fit_report* rep, std::vector<double>& best_theta) {
  gprx_trust_region_options opt;
  if (o) opt = *o;
  else gprx_trust_region_options_default(&opt);
  if (!(opt.interval_lo > 0.0) || !(opt.interval_hi > opt.interval_lo) || !std::isfinite(opt.interval_hi))
    return set_error(GPRX_INVALID_CONFIG, "parameter interval must be 0 < lo < hi");
  if (!(opt.tolerance >= 0.0) || !std::isfinite(opt.tolerance))
    return set_error(GPRX_INVALID_CONFIG, "trust-region gradient tolerance must be finite and >= 0");
  if (!(std::isfinite(opt.initial_radius) && std::isfinite(opt.max_radius) && opt.initial_radius > 0.0 &&
        opt.initial_radius <= opt.max_radius))
    return set_error(GPRX_INVALID_CONFIG, "trust radii must satisfy 0 < initial <= max and be finite");
  LogitMap map;
  map.init(opt.interval_lo, opt.interval_hi);
  TrustRegionConfig cfg;
  cfg.max_iterations = opt.max_iterations;
  cfg.tol_grad = opt.tolerance;
  cfg.initial_radius = opt.initial_radius;
  cfg.max_radius = opt.max_radius;
  std::vector<double> z0(p);
  if (!map.from_log(theta0, p, z0.data())) return set_error(GPRX_INVALID_HYPERPARAMETER, "initial θ outside the interval");
  std::vector<double> logt(p), jac(p), jac2(p), gl(p), hl((size_t)p * p);
  gprx_status fatal = GPRX_OK, last = GPRX_OK;
  // joint evaluation in z: g_z = J g, H_z = J H J + diag(g ∘ d²logθ/dz²)
  // (chain_logit_hess, src/optimizer/logit.rs:139-157)
  TrJointFn joint = [&](const double* z, double* f, double* g, double* h) -> bool {
    if (fatal != GPRX_OK) return false;
    map.to_log(z, p, logt.data(), jac.data());
    map.second(z, p, jac2.data());
    gprx_status st = s.hessian(logt.data(), hl.data(), f, gl.data());
    if (st == GPRX_CUDA_ERROR || st == GPRX_OUT_OF_MEMORY || st == GPRX_TIMEOUT) {
      fatal = st;
      return false;
    }
    if (st != GPRX_OK || !std::isfinite(*f)) {
      last = st != GPRX_OK ? st : GPRX_NOT_CONVERGED;
      return false;
    }
    for (int i = 0; i < p; ++i) {
      for (int j = 0; j < p; ++j) h[(size_t)i * p + j] = hl[(size_t)i * p + j] * jac[i] * jac[j];
      h[(size_t)i * p + i] += gl[i] * jac2[i];
      g[i] = gl[i] * jac[i];
    }
    return true;
  };
  gprx_rng rng;
  gprx_rng_seed(&rng, opt.seed);
  TrustRegionResult best;
  bool have = false;
  uint64_t total_evals = 0;
  for (int run = 0; run <= opt.restarts; ++run) {
    std::vector<double> zs(p);
    if (run == 0) {
      zs = z0;
    } else {
      for (int i = 0; i < p; ++i) {
        double u = gprx_rng_unit(&rng);
        const double eps = 1.0 / 9007199254740992.0;
        u = std::min(std::max(u, eps), 1.0 - eps);
        double lt = map.ln_lo + u * (map.ln_hi - map.ln_lo);
        map.from_log(&lt, 1, &zs[i]);
      }
    }
    TrustRegionResult r;
    const bool ok = trust_region_run(cfg, zs, joint, r);
    total_evals += r.evaluations;
    if (fatal != GPRX_OK) return fatal;
    if (!ok) {
      // the first start must be evaluable (its error is the caller's); a
      // restart that cannot start is skipped (src/optimizer/mod.rs:218-224)
      if (run == 0) return set_error(last != GPRX_OK ? last : GPRX_NOT_CONVERGED, "the initial θ cannot be evaluated");
      continue;
    }
    if (!have || r.best_value < best.best_value) {
      best = r;
      have = true;
    }
  }
  if (!have || !(best.best_value < BARRIER_COST))
    return set_error(GPRX_NOT_CONVERGED, "no evaluable point was found");
  best_theta.resize(p);
  map.to_log(best.best.data(), p, best_theta.data(), nullptr);
  if (rep) {
    rep->nlml = best.best_value;
    rep->iterations = best.iterations;
    rep->evaluations = total_evals;
    rep->grad_norm = best.grad_norm;
    rep->converged = best.converged ? 1 : 0;
  }
  return GPRX_OK;
}

static gprx_status exact_eval_cb(void* ctx, const double* lt, double* f, double* g) {
  return ((ExactState*)ctx)->eval(lt, f, g);
}

}  // namespace gprx

using namespace gprx;

#define CHECK_HANDLE(h) \
  if (!(h)) return set_error(GPRX_INVALID_ARGUMENT, "null handle")

extern "C" {

int32_t gprx_abi_version(void) { return GPRX_CUDA_ABI_VERSION; }

void gprx_options_default(gprx_options* o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->precision = GPRX_PRECISION_FP64;
  o->jitter_kind = GPRX_JITTER_FIXED;
  o->jitter_initial = 0.0;
  o->jitter_multiplier = 1.0;
  o->jitter_max_retries = 0;
  o->jitter_max = 0.0;
  o->device = 0;
  o->block_size = 0;
}

void gprx_options_default_sparse(gprx_options* o) {
  gprx_options_default(o);
  if (!o) return;
  o->jitter_kind = GPRX_JITTER_ADAPTIVE;
  o->jitter_initial = 1e-8;
  o->jitter_multiplier = 10.0;
  o->jitter_max_retries = 5;
  o->jitter_max = 1e-3;
}

void gprx_lbfgs_options_default(gprx_lbfgs_options* o) {
  if (!o) return;
  o->max_iterations = 100;
  o->tolerance = 1.4901161193847656e-08;
  o->history_size = 10;
  o->restarts = 0;
  o->seed = 0;
  o->interval_lo = 1e-5;
  o->interval_hi = 1e5;
}

void gprx_trust_region_options_default(gprx_trust_region_options* o) {
  if (!o) return;
  o->max_iterations = 100;
  o->tolerance = 1.4901161193847656e-08;
  o->initial_radius = 1.0;
  o->max_radius = 100.0;
  o->restarts = 0;
  o->seed = 0;
  o->interval_lo = 1e-5;
  o->interval_hi = 1e5;
}

gprx_status gprx_last_error(gprx_error_info* out) {
  if (!out) return GPRX_INVALID_ARGUMENT;
  *out = last_error();
  return GPRX_OK;
}

uint64_t gprx_launch_count(void) { return launches(); }

gprx_status gprx_exact_create(const double* x, uint64_t n, uint64_t d, const double* y, const gprx_kernel_node* nodes,
                              int32_t n_nodes, const double* theta, int32_t n_theta, const gprx_options* options,
                              gprx_exact** out) {
  if (!out) return set_error(GPRX_INVALID_ARGUMENT, "null output handle");
  *out = nullptr;
  gprx_exact* h = new (std::nothrow) gprx_exact;
  if (!h) return set_error(GPRX_OUT_OF_MEMORY, "host allocation");
  gprx_status st = h->s.create(x, n, d, y, nodes, n_nodes, theta, n_theta, options);
  if (st != GPRX_OK) {
    delete h;
    return st;
  }
  *out = h;
  return GPRX_OK;
}

gprx_status gprx_exact_destroy(gprx_exact* h) {
  if (h) delete h;
  return GPRX_OK;
}

gprx_status gprx_exact_set_data(gprx_exact* h, const double* x, const double* y) {
  CHECK_HANDLE(h);
  ExactState& s = h->s;
  if (!x || !y) return set_error(GPRX_INVALID_ARGUMENT, "null pointer");
  if (s.online) return set_error(GPRX_INVALID_CONFIG, "an online model changes points by insert/delete");
  if (!all_finite(x, (size_t)s.n * s.d) || !all_finite(y, s.n)) return set_error(GPRX_NONFINITE_INPUT, "non-finite input");
  GPRX_CUDA_TRY(cudaMemcpy2DAsync(s.x.p, sizeof(double) * s.cap, x, sizeof(double) * s.n, sizeof(double) * s.n, s.d,
                                  cudaMemcpyHostToDevice, s.stream));
  GPRX_CUDA_TRY(cudaMemcpyAsync(s.y.p, y, sizeof(double) * s.n, cudaMemcpyHostToDevice, s.stream));
  s.y_host.assign(y, y + s.n);
  s.factor_ok = s.alpha_ok = false;
  return GPRX_OK;
}

uint64_t gprx_exact_num_params(const gprx_exact* h) { return h ? (uint64_t)h->s.num_params() : 0; }

gprx_status gprx_exact_get_params(gprx_exact* h, double* out, uint64_t p) {
  CHECK_HANDLE(h);
  if (!out || p != (uint64_t)h->s.num_params()) return set_error(GPRX_SHAPE_MISMATCH, "parameter count");
  h->s.get_params(out);
  return GPRX_OK;
}

gprx_status gprx_exact_data(gprx_exact* h, double* x_out, double* y_out) {
  CHECK_HANDLE(h);
  ExactState& s = h->s;
  if (!x_out || !y_out) return set_error(GPRX_INVALID_ARGUMENT, "null pointer");
  GPRX_CUDA_TRY(cudaMemcpy2DAsync(x_out, sizeof(double) * s.n, s.x.p, sizeof(double) * s.cap, sizeof(double) * s.n, s.d,
                                  cudaMemcpyDeviceToHost, s.stream));
  GPRX_CUDA_TRY(cudaMemcpyAsync(y_out, s.y.p, sizeof(double) * s.n, cudaMemcpyDeviceToHost, s.stream));
  GPRX_CUDA_TRY(cudaStreamSynchronize(s.stream));
  return GPRX_OK;
}

gprx_status gprx_exact_set_params(gprx_exact* h, const double* params, uint64_t p) {
  CHECK_HANDLE(h);
  ExactState& s = h->s;
  if (!params || p != (uint64_t)s.num_params()) return set_error(GPRX_SHAPE_MISMATCH, "parameter count");
  // an online model goes through an LLT view (OnlineGpr::set_params, src/gpr/online.rs:659)
  std::vector<double> prev(p);
  s.get_params(prev.data());
  return s.with_llt_view([&]() -> gprx_status {
    gprx_status st = s.write_params(params);
    if (st != GPRX_OK) return st;
    st = s.factor_current();
    if (st != GPRX_OK) {
      gprx_error_info saved = last_error();
      s.write_params(prev.data());
      s.factor_current();
      last_error() = saved;
    }
    return st;
  });
}

gprx_status gprx_exact_factor(gprx_exact* h) {
  CHECK_HANDLE(h);
  if (h->s.online) return GPRX_OK;
  return h->s.factor_current();
}

gprx_status gprx_exact_eval(gprx_exact* h, const double* params, uint64_t p, double* nlml, double* grad) {
  CHECK_HANDLE(h);
  if (!params || !nlml) return set_error(GPRX_INVALID_ARGUMENT, "null pointer");
  if (p != (uint64_t)h->s.num_params()) return set_error(GPRX_SHAPE_MISMATCH, "parameter count");
  return h->s.with_llt_view([&] { return h->s.eval(params, nlml, grad); });
}

gprx_status gprx_exact_hessian(gprx_exact* h, const double* params, uint64_t p, double* out) {
  CHECK_HANDLE(h);
  if (!params || !out) return set_error(GPRX_INVALID_ARGUMENT, "null pointer");
  if (p != (uint64_t)h->s.num_params()) return set_error(GPRX_SHAPE_MISMATCH, "parameter count");
  return h->s.with_llt_view([&] { return h->s.hessian(params, out); });
}

gprx_status gprx_exact_value_gradient_hessian(gprx_exact* h, const double* params, uint64_t p, double* nlml,
                                              double* grad, double* hess) {
  CHECK_HANDLE(h);
  if (!params || !nlml || !grad || !hess) return set_error(GPRX_INVALID_ARGUMENT, "null pointer");
  if (p != (uint64_t)h->s.num_params()) return set_error(GPRX_SHAPE_MISMATCH, "parameter count");
  return h->s.with_llt_view([&] { return h->s.hessian(params, hess, nlml, grad); });
}

gprx_status gprx_exact_nlml(gprx_exact* h, double* nlml) {
  CHECK_HANDLE(h);
  if (!nlml) return set_error(GPRX_INVALID_ARGUMENT, "null pointer");
  return h->s.nlml(nlml);
}

gprx_status gprx_exact_factor_jitter(gprx_exact* h, double* jitter) {
  CHECK_HANDLE(h);
  if (!jitter) return set_error(GPRX_INVALID_ARGUMENT, "null pointer");
  *jitter = h->s.jitter;
  return GPRX_OK;
}

gprx_status gprx_exact_predict(gprx_exact* h, const double* xs, uint64_t q, int32_t kind, double* mean, double* var) {
  CHECK_HANDLE(h);
  return h->s.predict(xs, q, kind, mean, var);
}

gprx_status gprx_exact_save(gprx_exact* h, const char* dir, int32_t with_factor) {
  CHECK_HANDLE(h);
  return h->s.save(dir, with_factor != 0);
}

gprx_status gprx_exact_load(const char* dir, int32_t device, gprx_exact** out) {
  if (!dir || !out) return set_error(GPRX_INVALID_ARGUMENT, "null pointer");
  *out = nullptr;
  PersistModel m;
  gprx_status st = persist_read(dir, m, true);
  if (st != GPRX_OK) return st;
  gprx_options o;
  gprx_options_default(&o);
  o.jitter_kind = m.jitter.jitter_kind;
  o.jitter_initial = m.jitter.jitter_initial;
  o.jitter_multiplier = m.jitter.jitter_multiplier;
  o.jitter_max_retries = m.jitter.jitter_max_retries;
  o.jitter_max = m.jitter.jitter_max;
  o.device = device;
  std::vector<double> theta(m.theta);
  theta.push_back(m.log_noise);
  std::unique_ptr<gprx_exact> h(new (std::nothrow) gprx_exact());
  if (!h) return set_error(GPRX_OUT_OF_MEMORY, "host allocation");
  st = h->s.create(m.x.data(), (uint64_t)m.n, (uint64_t)m.d, m.y.data(), m.nodes.data(), (int)m.nodes.size(),
                   theta.data(), (int)theta.size(), &o);
  if (st != GPRX_OK) return st;
  if (m.has_factor) {
    st = h->s.adopt_factor(m.l_map, m.alpha.data(), m.ldlt, m.factor_jitter, m.ids, m.next_id);
    if (st != GPRX_OK) return st;
  } else if (m.ldlt) {
    // an online model saved without its factor: factor, go online, keep the ids
    if ((st = h->s.online_begin()) != GPRX_OK) return st;
    h->s.ids = m.ids;
    h->s.next_id = m.next_id;
  }
  *out = h.release();
  return GPRX_OK;
}

gprx_status gprx_exact_loo(gprx_exact* h, int32_t kind, double* mean, double* var) {
  CHECK_HANDLE(h);
  return h->s.loo(kind, mean, var);
}

gprx_status gprx_exact_predict_covariance(gprx_exact* h, const double* xs, uint64_t q, int32_t kind, double* mean,
                                          double* cov) {
  CHECK_HANDLE(h);
  return h->s.predict_covariance(xs, q, kind, mean, cov);
}

gprx_status gprx_exact_sample(gprx_exact* h, const double* xs, uint64_t q, int32_t kind, uint64_t n_draws,
                              uint64_t seed, double* out) {
  CHECK_HANDLE(h);
  return h->s.sample(xs, q, kind, n_draws, seed, out);
}

gprx_status gprx_exact_alpha(gprx_exact* h, double* out, uint64_t n) {
  CHECK_HANDLE(h);
  ExactState& s = h->s;
  if (!out || n != (uint64_t)s.n) return set_error(GPRX_SHAPE_MISMATCH, "alpha length");
  gprx_status st;
  if (s.online) {
    if (!s.alpha_ok && (st = s.online_alpha()) != GPRX_OK) return st;
  } else if (!s.alpha_ok) {
    if ((st = s.factor_current()) != GPRX_OK) return st;
  }
  GPRX_CUDA_TRY(cudaMemcpyAsync(out, s.alpha.p, sizeof(double) * s.n, cudaMemcpyDeviceToHost, s.stream));
  GPRX_CUDA_TRY(cudaStreamSynchronize(s.stream));
  return GPRX_OK;
}

gprx_status gprx_exact_fit(gprx_exact* h, const gprx_lbfgs_options* opt, gprx_fit_report* report) {
  CHECK_HANDLE(h);
  ExactState& s = h->s;
  if (s.online) return set_error(GPRX_INVALID_CONFIG, "an online model is not refitted");
  int p = s.num_params();
  std::vector<double> theta0(p), best;
  s.get_params(theta0.data());
  gprx_status st = fit_lbfgs(&s, exact_eval_cb, p, theta0.data(), opt, report, best);
  if (st != GPRX_OK) {
    gprx_error_info saved = last_error();
    s.write_params(theta0.data());
    s.factor_current();
    last_error() = saved;
    return st;
  }
  // commit at the optimizer's best θ and publish α (exact_fit.rs:743-773, shared.rs:203)
  st = s.write_params(best.data());
  if (st == GPRX_OK) st = s.factor_current();
  if (st == GPRX_OK && report) st = s.nlml(&report->nlml);
  return st;
}

gprx_status gprx_exact_fit_trust_region(gprx_exact* h, const gprx_trust_region_options* opt,
                                        gprx_fit_report* report) {
  CHECK_HANDLE(h);
  ExactState& s = h->s;
  if (s.online) return set_error(GPRX_INVALID_CONFIG, "an online model is not refitted");
  int p = s.num_params();
  std::vector<double> theta0(p), best;
  s.get_params(theta0.data());
  gprx_status st = fit_trust_region(s, p, theta0.data(), opt, report, best);
  if (st != GPRX_OK) {
    gprx_error_info saved = last_error();
    s.write_params(theta0.data());
    s.factor_current();
    last_error() = saved;
    return st;
  }
  st = s.write_params(best.data());
  if (st == GPRX_OK) st = s.factor_current();
  if (st == GPRX_OK && report) st = s.nlml(&report->nlml);
  return st;
}

gprx_status gprx_exact_stage_times(gprx_exact* h, double* out5) {
  CHECK_HANDLE(h);
  if (!out5) return set_error(GPRX_INVALID_ARGUMENT, "null pointer");
  return h->s.stage_times(out5);
}

gprx_status gprx_exact_stream(gprx_exact* h, void** stream) {
  CHECK_HANDLE(h);
  if (!stream) return set_error(GPRX_INVALID_ARGUMENT, "null pointer");
  *stream = (void*)h->s.stream;
  return GPRX_OK;
}

gprx_status gprx_online_begin(gprx_exact* h) {
  CHECK_HANDLE(h);
  return h->s.online_begin();
}

gprx_status gprx_online_insert(gprx_exact* h, const double* x_new, double y_new, uint64_t* id) {
  CHECK_HANDLE(h);
  return h->s.online_insert(x_new, y_new, id);
}

gprx_status gprx_online_delete(gprx_exact* h, uint64_t id) {
  CHECK_HANDLE(h);
  return h->s.online_delete(id);
}

uint64_t gprx_online_n(const gprx_exact* h) { return h ? (uint64_t)h->s.n : 0; }

gprx_status gprx_online_point_ids(gprx_exact* h, uint64_t* out, uint64_t n) {
  CHECK_HANDLE(h);
  if (!out || n != (uint64_t)h->s.n) return set_error(GPRX_SHAPE_MISMATCH, "id count");
  std::copy(h->s.ids.begin(), h->s.ids.end(), out);
  return GPRX_OK;
}

// ---------------------------------------------------------------------------
// Xoshiro256++ seeded by SplitMix64 (src/rng.rs:10-87)
// ---------------------------------------------------------------------------
static inline uint64_t rotl64(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }

void gprx_rng_seed(gprx_rng* r, uint64_t seed) {
  uint64_t x = seed;
  for (int i = 0; i < 4; ++i) {
    x += 0x9e3779b97f4a7c15ULL;
    uint64_t z = x;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    r->s[i] = z ^ (z >> 31);
  }
}

uint64_t gprx_rng_next_u64(gprx_rng* r) {
  uint64_t* s = r->s;
  uint64_t result = rotl64(s[0] + s[3], 23) + s[0];
  uint64_t t = s[1] << 17;
  s[2] ^= s[0];
  s[3] ^= s[1];
  s[1] ^= s[2];
  s[0] ^= s[3];
  s[2] ^= t;
  s[3] = rotl64(s[3], 45);
  return result;
}

double gprx_rng_unit(gprx_rng* r) { return (double)(gprx_rng_next_u64(r) >> 11) * (1.0 / 9007199254740992.0); }

uint64_t gprx_rng_up_to(gprx_rng* r, uint64_t max) {
  // Lemire's widened-product rejection (src/rng.rs:52-64)
  uint64_t range = max + 1;
  if (range == 0) return gprx_rng_next_u64(r);
  uint64_t threshold = (0 - range) % range;
  for (;;) {
    unsigned __int128 wide = (unsigned __int128)gprx_rng_next_u64(r) * range;
    if ((uint64_t)wide >= threshold) return (uint64_t)(wide >> 64);
  }
}

static double open_unit(gprx_rng* r) {
  double u = gprx_rng_unit(r);
  const double eps = 1.0 / 9007199254740992.0;
  if (u <= eps) return eps;
  if (u >= 1.0 - eps) return 1.0 - eps;
  return u;
}

double gprx_rng_normal(gprx_rng* r) {
  // Box–Muller (src/rng.rs:83-87)
  double u1 = std::max(open_unit(r), 2.2250738585072014e-308);
  double u2 = open_unit(r);
  return std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * M_PI * u2);
}

void gprx_rng_fill_unit(gprx_rng* r, double* out, uint64_t count) {
  for (uint64_t i = 0; i < count; ++i) out[i] = gprx_rng_unit(r);
}

void gprx_rng_fill_normal(gprx_rng* r, double* out, uint64_t count) {
  for (uint64_t i = 0; i < count; ++i) out[i] = gprx_rng_normal(r);
}

gprx_status gprx_rng_subset(gprx_rng* r, uint64_t n, uint64_t count, uint64_t* out) {
  if (!r || !out) return set_error(GPRX_INVALID_ARGUMENT, "null pointer");
  if (count > n) return set_error(GPRX_SHAPE_MISMATCH, "subset larger than the population");
  // partial Fisher–Yates over a sparse swap map
  std::vector<std::pair<uint64_t, uint64_t>> swaps;
  auto get = [&](uint64_t i) {
    for (auto& p : swaps)
      if (p.first == i) return p.second;
    return i;
  };
  auto set = [&](uint64_t i, uint64_t v) {
    for (auto& p : swaps)
      if (p.first == i) {
        p.second = v;
        return;
      }
    swaps.emplace_back(i, v);
  };
  for (uint64_t k = 0; k < count; ++k) {
    uint64_t j = k + gprx_rng_up_to(r, n - 1 - k);
    uint64_t vk = get(k), vj = get(j);
    set(k, vj);
    set(j, vk);
    out[k] = vj;
  }
  return GPRX_OK;
}

}  // extern "C"
