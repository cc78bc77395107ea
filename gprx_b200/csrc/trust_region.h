// trust_region.h — the trust-region method with the Steihaug conjugate-
// gradient subproblem, over an objective that returns value, gradient and
// Hessian in one call.
//
// Reference: gprx's TrustRegion (src/optimizer/trust_region.rs:19-258) is
// argmin 0.11's TrustRegion with the Steihaug subproblem (at most 4p + 10 CG
// iterations), initial radius 1, maximum radius 100, ≤ 100 iterations and a
// stop when ‖g‖ ≤ √ε, run in the logit coordinates of the parameter
// intervals with the Hessian chained through the map
// (src/optimizer/logit.rs:52-157).  Every candidate is evaluated through the
// joint value/gradient/Hessian call; a point that cannot be evaluated costs
// the barrier 1e300 with a zero gradient and Hessian
// (src/optimizer/adapter.rs:26,118-160).
//
// argmin is not vendored with the reference; this restates the published
// algorithms (Nocedal & Wright, Numerical Optimization, 2nd ed., Algorithm
// 4.1 for the radius update with η = 1/8: ρ < 1/4 shrinks the radius to
// ‖s‖/4, ρ > 3/4 with the step on the boundary (to 10 ulp of the radius)
// doubles it up to the maximum; Algorithm 7.2 for Steihaug's CG).
// Its trajectory is not claimed to be bit-identical to argmin's; the checks
// are the reference's own optimizer tests and the NLML it reaches.
//
// Host only.  The caller supplies the joint evaluation as a callable.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <functional>
#include <vector>

namespace gprx {

struct TrustRegionConfig {
  uint64_t max_iterations = 100;
  double tol_grad = 1.4901161193847656e-08;  // √ε
  double initial_radius = 1.0;
  double max_radius = 100.0;
  double eta = 0.125;                        // accept when ρ > η
  double cg_epsilon = 1e-10;                 // Steihaug: stop when ‖r‖ < ε
};

struct TrustRegionResult {
  std::vector<double> best;   // lowest-cost accepted point
  double best_value = 0.0;
  double grad_norm = 0.0;     // at the best point
  uint64_t iterations = 0;
  uint64_t evaluations = 0;
  bool converged = false;     // stopped on the gradient test
};

// Joint evaluation at z: returns false when the point cannot be evaluated
// (the caller's own error reporting happens outside).
using TrJointFn = std::function<bool(const double* z, double* f, double* g, double* h)>;

namespace tr_detail {

inline double dot(const std::vector<double>& a, const std::vector<double>& b) {
  double s = 0.0;
  for (size_t i = 0; i < a.size(); ++i) s += a[i] * b[i];
  return s;
}

inline void matvec(const std::vector<double>& h, const std::vector<double>& v, std::vector<double>& out) {
  const size_t p = v.size();
  for (size_t i = 0; i < p; ++i) {
    double s = 0.0;
    for (size_t j = 0; j < p; ++j) s += h[i * p + j] * v[j];
    out[i] = s;
  }
}

// Model value m(s) − f = gᵀs + ½ sᵀHs.
inline double model(const std::vector<double>& g, const std::vector<double>& h, const std::vector<double>& s) {
  std::vector<double> hs(s.size());
  matvec(h, s, hs);
  return dot(g, s) + 0.5 * dot(s, hs);
}

// The two τ with ‖z + τ d‖ = Δ (τ_neg ≤ 0 ≤ τ_pos when ‖z‖ ≤ Δ).
inline void boundary_taus(const std::vector<double>& z, const std::vector<double>& d, double radius, double* tneg,
                          double* tpos) {
  const double a = dot(d, d), b = 2.0 * dot(z, d), c = dot(z, z) - radius * radius;
  const double disc = std::sqrt(std::max(b * b - 4.0 * a * c, 0.0));
  *tneg = (-b - disc) / (2.0 * a);
  *tpos = (-b + disc) / (2.0 * a);
}

}  // namespace tr_detail

// Steihaug's truncated CG for min gᵀs + ½ sᵀHs subject to ‖s‖ ≤ Δ.
inline std::vector<double> steihaug(const std::vector<double>& g, const std::vector<double>& h, double radius,
                                    double epsilon, uint64_t max_iters) {
  using namespace tr_detail;
  const size_t p = g.size();
  std::vector<double> z(p, 0.0), r = g, d(p), bd(p);
  for (size_t i = 0; i < p; ++i) d[i] = -r[i];
  if (std::sqrt(dot(r, r)) < epsilon) return z;
  auto on_boundary = [&](bool pick_model_min) {
    double tn, tp;
    boundary_taus(z, d, radius, &tn, &tp);
    std::vector<double> sp(p), sn(p);
    for (size_t i = 0; i < p; ++i) {
      sp[i] = z[i] + tp * d[i];
      sn[i] = z[i] + tn * d[i];
    }
    if (pick_model_min && model(g, h, sn) < model(g, h, sp)) return sn;
    return sp;
  };
  for (uint64_t it = 0; it < max_iters; ++it) {
    matvec(h, d, bd);
    const double dbd = dot(d, bd);
    if (dbd <= 0.0) return on_boundary(true);   // negative curvature: to the boundary
    const double rr = dot(r, r);
    const double alpha = rr / dbd;
    std::vector<double> zn(p);
    for (size_t i = 0; i < p; ++i) zn[i] = z[i] + alpha * d[i];
    if (std::sqrt(dot(zn, zn)) >= radius) return on_boundary(false);
    std::vector<double> rn(p);
    for (size_t i = 0; i < p; ++i) rn[i] = r[i] + alpha * bd[i];
    if (std::sqrt(dot(rn, rn)) < epsilon) return zn;
    const double beta = dot(rn, rn) / rr;
    for (size_t i = 0; i < p; ++i) d[i] = -rn[i] + beta * d[i];
    z.swap(zn);
    r.swap(rn);
  }
  return z;
}

// Runs the method from z0.  The start must be evaluable: returns false (and
// evaluates nothing else) when it is not.
inline bool trust_region_run(const TrustRegionConfig& cfg, const std::vector<double>& z0, const TrJointFn& eval,
                             TrustRegionResult& out) {
  using namespace tr_detail;
  const size_t p = z0.size();
  std::vector<double> z = z0, g(p), h(p * p);
  double f = 0.0;
  out = TrustRegionResult();
  out.evaluations = 1;
  if (!eval(z.data(), &f, g.data(), h.data()) || !std::isfinite(f)) return false;
  out.best = z;
  out.best_value = f;
  out.grad_norm = std::sqrt(dot(g, g));
  double radius = cfg.initial_radius;
  std::vector<double> zc(p), gc(p), hc(p * p);
  for (uint64_t it = 0; it < cfg.max_iterations; ++it) {
    if (std::sqrt(dot(g, g)) <= cfg.tol_grad) {
      out.converged = true;
      break;
    }
    const std::vector<double> s = steihaug(g, h, radius, cfg.cg_epsilon, 4 * (uint64_t)p + 10);
    for (size_t i = 0; i < p; ++i) zc[i] = z[i] + s[i];
    double fc = 0.0;
    ++out.evaluations;
    if (!eval(zc.data(), &fc, gc.data(), hc.data()) || !std::isfinite(fc)) {
      fc = 1.0e300;
      std::fill(gc.begin(), gc.end(), 0.0);
      std::fill(hc.begin(), hc.end(), 0.0);
    }
    const double predicted = -model(g, h, s);
    const double rho = (f - fc) / predicted;
    if (rho > cfg.eta) {
      z = zc;
      f = fc;
      g = gc;
      h = hc;
    }
    const double sn = std::sqrt(dot(s, s));
    if (rho < 0.25)
      radius = 0.25 * sn;
    else if (rho > 0.75 && std::fabs(sn - radius) <= 10.0 * 2.220446049250313e-16 * std::max(radius, 1.0))
      radius = std::min(2.0 * radius, cfg.max_radius);
    out.iterations = it + 1;
    if (f < out.best_value) {
      out.best = z;
      out.best_value = f;
      out.grad_norm = std::sqrt(dot(g, g));
    }
  }
  if (!out.converged && std::sqrt(dot(g, g)) <= cfg.tol_grad) out.converged = true;
  return true;
}

}  // namespace gprx
