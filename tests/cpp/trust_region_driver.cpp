// Test driver for the trust-region method (gprx_b200/csrc/trust_region.h,
// compiled for the host) on the reference's own optimizer test objectives
// (src/optimizer/trust_region.rs:260-531): a quadratic bowl, √(1 + x²) whose
// plain Newton step diverges and which cannot be evaluated beyond |x| = 50,
// −cos x from a point of negative curvature, and a shifted bowl.  Plus the
// logit chain rule of the Hessian against finite differences.  Prints one
// JSON object per case.
#include <cmath>
#include <cstdio>
#include <vector>

#include "../../gprx_b200/csrc/lbfgs.h"
#include "../../gprx_b200/csrc/trust_region.h"

using namespace gprx;

static void report(const char* name, bool ok, const TrustRegionResult& r) {
  std::printf("{\"case\": \"%s\", \"ok\": %d, \"f\": %.17g, \"x\": [", name, ok ? 1 : 0, r.best_value);
  for (size_t i = 0; i < r.best.size(); ++i) std::printf("%s%.17g", i ? ", " : "", r.best[i]);
  std::printf("], \"iters\": %llu, \"evals\": %llu, \"converged\": %d}\n", (unsigned long long)r.iterations,
              (unsigned long long)r.evaluations, r.converged ? 1 : 0);
}

int main() {
  {
    TrustRegionConfig cfg;
    cfg.max_iterations = 50;
    TrustRegionResult r;
    bool ok = trust_region_run(cfg, {1.0, -0.5}, [](const double* x, double* f, double* g, double* h) {
      g[0] = x[0];
      g[1] = x[1];
      h[0] = 1.0; h[1] = 0.0; h[2] = 0.0; h[3] = 1.0;
      *f = 0.5 * (x[0] * x[0] + x[1] * x[1]);
      return true;
    }, r);
    report("bowl", ok, r);
  }
  for (double start : {1.5, 2.0, 4.0, -3.0}) {
    TrustRegionConfig cfg;
    cfg.max_iterations = 200;
    TrustRegionResult r;
    bool ok = trust_region_run(cfg, {start}, [](const double* x, double* f, double* g, double* h) {
      if (std::fabs(x[0]) > 50.0) return false;
      const double root = std::sqrt(1.0 + x[0] * x[0]);
      *f = root;
      g[0] = x[0] / root;
      h[0] = std::pow(1.0 + x[0] * x[0], -1.5);
      return true;
    }, r);
    char name[64];
    std::snprintf(name, sizeof(name), "sqrt1p_%g", start);
    report(name, ok, r);
  }
  {
    TrustRegionConfig cfg;
    cfg.max_iterations = 200;
    TrustRegionResult r;
    bool ok = trust_region_run(cfg, {2.0}, [](const double* x, double* f, double* g, double* h) {
      *f = -std::cos(x[0]);
      g[0] = std::sin(x[0]);
      h[0] = std::cos(x[0]);
      return true;
    }, r);
    report("negative_curvature", ok, r);
  }
  {
    TrustRegionConfig cfg;
    TrustRegionResult r;
    bool ok = trust_region_run(cfg, {2.0, 1.0}, [](const double* x, double* f, double* g, double* h) {
      g[0] = 2.0 * (x[0] - 0.3);
      g[1] = 4.0 * (x[1] + 0.2);
      h[0] = 2.0; h[1] = 0.0; h[2] = 0.0; h[3] = 4.0;
      *f = (x[0] - 0.3) * (x[0] - 0.3) + 2.0 * (x[1] + 0.2) * (x[1] + 0.2);
      return true;
    }, r);
    report("shifted_bowl", ok, r);
  }
  {
    // a start that cannot be evaluated is the caller's error
    TrustRegionConfig cfg;
    TrustRegionResult r;
    bool ok = trust_region_run(cfg, {100.0}, [](const double* x, double*, double*, double*) {
      return std::fabs(x[0]) <= 50.0;
    }, r);
    std::printf("{\"case\": \"bad_start\", \"ok\": %d, \"evals\": %llu}\n", ok ? 1 : 0,
                (unsigned long long)r.evaluations);
  }
  {
    // Hessian through the logit map: d²/dz² of F(logθ(z)) against central
    // differences of the chained gradient, F(t) = Σ t_i⁴ + t_0 t_1
    LogitMap map;
    map.init(1e-6, 1e6);
    const double z[2] = {0.3, -1.1};
    auto grad_z = [&](const double* zz, double* gz) {
      double t[2], jac[2];
      map.to_log(zz, 2, t, jac);
      gz[0] = (4.0 * t[0] * t[0] * t[0] + t[1]) * jac[0];
      gz[1] = (4.0 * t[1] * t[1] * t[1] + t[0]) * jac[1];
    };
    double t[2], jac[2], jac2[2];
    map.to_log(z, 2, t, jac);
    map.second(z, 2, jac2);
    const double gt[2] = {4.0 * t[0] * t[0] * t[0] + t[1], 4.0 * t[1] * t[1] * t[1] + t[0]};
    const double ht[4] = {12.0 * t[0] * t[0], 1.0, 1.0, 12.0 * t[1] * t[1]};
    double hz[4];
    for (int i = 0; i < 2; ++i)
      for (int j = 0; j < 2; ++j) hz[i * 2 + j] = ht[i * 2 + j] * jac[i] * jac[j] + (i == j ? gt[i] * jac2[i] : 0.0);
    double err = 0.0;
    const double e = 1e-6;
    for (int j = 0; j < 2; ++j) {
      double zp[2] = {z[0], z[1]}, zm[2] = {z[0], z[1]}, gp[2], gm[2];
      zp[j] += e;
      zm[j] -= e;
      grad_z(zp, gp);
      grad_z(zm, gm);
      for (int i = 0; i < 2; ++i) {
        const double fd = (gp[i] - gm[i]) / (2.0 * e);
        err = std::max(err, std::fabs(fd - hz[i * 2 + j]) / std::max(std::fabs(fd), 1.0));
      }
    }
    std::printf("{\"case\": \"logit_hessian\", \"err\": %.3g}\n", err);
  }
  return 0;
}
