// Test driver for the L-BFGS (gprx_b200/csrc/lbfgs.h, compiled for the host) on analytic
// objectives: Rosenbrock, a quadratic with a barrier region (a point that
// cannot be evaluated costs 1e300 with a zero gradient, as gprx's EvalCache
// does), and the logit map round trip.  Prints one JSON object per case.
#include <cmath>
#include <cstdio>
#include <vector>

#include "../../gprx_b200/csrc/lbfgs.h"

using namespace gprx;

template <class F>
static void run(const char* name, F f, std::vector<double> x0, double tol) {
  LbfgsConfig cfg;
  cfg.tol_grad = tol;
  cfg.max_iterations = 500;
  static HostLbfgs lb;
  lb.start(cfg, x0.data(), (int)x0.size());
  std::vector<double> g(x0.size());
  while (lb.task() == HostLbfgs::EVALUATE) {
    std::vector<double> pt(lb.point(), lb.point() + x0.size());
    double v = f(pt, g);
    lb.resume(v, g.data());
  }
  std::printf("{\"case\": \"%s\", \"f\": %.17g, \"x\": [", name, lb.best_value());
  for (size_t i = 0; i < x0.size(); ++i) std::printf("%s%.17g", i ? ", " : "", lb.best()[i]);
  std::printf("], \"iters\": %llu, \"evals\": %llu, \"converged\": %d}\n", (unsigned long long)lb.iterations(),
              (unsigned long long)lb.evaluations(), lb.converged() ? 1 : 0);
}

int main() {
  run("rosenbrock",
      [](const std::vector<double>& x, std::vector<double>& g) {
        double a = 1.0 - x[0], b = x[1] - x[0] * x[0];
        g[0] = -2.0 * a - 400.0 * x[0] * b;
        g[1] = 200.0 * b;
        return a * a + 100.0 * b * b;
      },
      {-1.2, 1.0}, 1e-8);
  run("barrier_quadratic",
      [](const std::vector<double>& x, std::vector<double>& g) {
        if (x[0] > 3.0) {  // cannot be evaluated
          g[0] = g[1] = 0.0;
          return BARRIER_COST;
        }
        g[0] = 2.0 * (x[0] - 2.5);
        g[1] = 8.0 * (x[1] + 1.0);
        return (x[0] - 2.5) * (x[0] - 2.5) + 4.0 * (x[1] + 1.0) * (x[1] + 1.0);
      },
      {-20.0, 5.0}, 1e-8);
  LogitMap map;
  map.init(1e-5, 1e5);
  double lt[3] = {std::log(0.3), std::log(2.0), std::log(1e-3)}, z[3], back[3], jac[3];
  bool ok = map.from_log(lt, 3, z);
  map.to_log(z, 3, back, jac);
  double err = 0.0;
  for (int i = 0; i < 3; ++i) err = std::fmax(err, std::fabs(back[i] - lt[i]));
  // dlogθ/dz against a central difference
  double fd_err = 0.0;
  for (int i = 0; i < 3; ++i) {
    double zp[3] = {z[0], z[1], z[2]}, zm[3] = {z[0], z[1], z[2]}, lp[3], lm[3];
    zp[i] += 1e-6;
    zm[i] -= 1e-6;
    map.to_log(zp, 3, lp, nullptr);
    map.to_log(zm, 3, lm, nullptr);
    fd_err = std::fmax(fd_err, std::fabs((lp[i] - lm[i]) / 2e-6 - jac[i]));
  }
  std::printf("{\"case\": \"logit\", \"ok\": %d, \"roundtrip\": %.3g, \"jac\": %.3g}\n", ok ? 1 : 0, err, fd_err);
  return 0;
}
