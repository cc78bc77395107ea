// lbfgs.h — L-BFGS with the Moré–Thuente line search, in reverse
// communication, over the logit map of gprx's parameter intervals.
//
// Reference: gprx's default optimizer Lbfgs (src/optimizer/lbfgs.rs:28-172) is
// argmin 0.11's LBFGS (history 10, gradient tolerance √ε, ≤100 iterations)
// with MoreThuenteLineSearch, run in z space of the logit map
// (src/optimizer/logit.rs:10-242): log θ = ln lo + σ(z/s)·ln(hi/lo),
// s = ln(hi/lo)/4.  A point that cannot be evaluated costs the barrier 1e300
// with a zero gradient (src/optimizer/adapter.rs:26,118-160).
//
// argmin is not vendored with the reference; this is a restatement of the
// published algorithms (Nocedal 1980 two-loop recursion; Moré & Thuente 1994
// as in MINPACK-2 dcsrch/dcstep).  Its trajectory is not bit-identical to
// argmin's; results are checked against the reference's fit goldens.
//
// Reverse communication lets one driver advance many independent problems
// and evaluate all their pending points in one batched device launch.
#pragma once

#include <cstdint>
#include <vector>

namespace gprx {

constexpr double BARRIER_COST = 1.0e300;

struct LogitMap {
  std::vector<double> ln_lo, ln_hi;
  void init(int n, double lo, double hi);
  double scale(int i) const { return (ln_hi[i] - ln_lo[i]) / 4.0; }
  // z → log θ and dlogθ/dz
  void to_log(const double* z, double* log_theta, double* jac) const;
  // log θ → z (fails when θ is outside the open interval)
  bool from_log(const double* log_theta, double* z) const;
};

class MoreThuente {
 public:
  double ftol = 1e-4, gtol = 0.9, xtol = 1e-10, stpmin = 1e-20, stpmax = 1e20;
  int max_evals = 20;
  // Starts a search from f0, g0 (directional derivative, < 0), first step stp.
  // Returns false when g0 ≥ 0 (not a descent direction).
  bool start(double f0, double g0, double stp);
  enum Result { CONTINUE, CONVERGED, STOP };
  // Consumes f, g at the current step; sets the next step (CONTINUE) or ends.
  Result step(double f, double g);
  double stp() const { return stp_; }
  int evals() const { return nfev_; }

 private:
  bool brackt_ = false;
  int stage_ = 1, nfev_ = 0;
  double finit_ = 0, ginit_ = 0, gtest_ = 0, width_ = 0, width1_ = 0;
  double stx_ = 0, fx_ = 0, gx_ = 0, sty_ = 0, fy_ = 0, gy_ = 0, stmin_ = 0, stmax_ = 0, stp_ = 0;
};

struct LbfgsConfig {
  int history = 10;
  uint64_t max_iterations = 100;
  double tol_grad = 1.4901161193847656e-08;  // √ε
  double tol_cost = 2.220446049250313e-16;   // ε
};

class LbfgsRC {
 public:
  enum Task { EVALUATE, DONE };
  void start(const LbfgsConfig& cfg, const double* z0, int n);
  // Point to evaluate (z space) while task() == EVALUATE.
  const std::vector<double>& point() const { return xt_; }
  // Feeds f, ∇f (z space) at point(); f = BARRIER_COST with a zero gradient
  // for a point that could not be evaluated.
  void resume(double f, const double* g);
  Task task() const { return task_; }
  const std::vector<double>& best() const { return best_x_; }
  double best_value() const { return best_f_; }
  uint64_t iterations() const { return iter_; }
  uint64_t evaluations() const { return nev_; }
  double grad_norm() const { return gnorm_; }
  bool converged() const { return converged_; }

 private:
  void begin_iteration();
  void finish(bool conv);
  LbfgsConfig cfg_{};
  int n_ = 0;
  Task task_ = DONE;
  int phase_ = 0;  // 0 initial evaluation, 1 line search
  std::vector<double> x_, g_, d_, xt_, gt_;
  double f_ = 0, ft_ = 0;
  std::vector<std::vector<double>> S_, Y_;
  std::vector<double> rho_;
  MoreThuente ls_;
  std::vector<double> best_x_;
  double best_f_ = BARRIER_COST;
  uint64_t iter_ = 0, nev_ = 0;
  double gnorm_ = 0;
  bool converged_ = false;
  // best point seen inside the current line search
  std::vector<double> ls_best_x_, ls_best_g_;
  double ls_best_f_ = BARRIER_COST;
};

}  // namespace gprx
