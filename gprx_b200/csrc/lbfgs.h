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
// Header-only, fixed-capacity and __host__ __device__: the single-model fit
// drives one state on the host, the batched fit keeps one state per problem
// in device memory and advances them all in one kernel between evaluation
// launches.  Reverse communication: the caller evaluates point() and feeds the
// value and gradient back through resume().
#pragma once

#include <math.h>
#include <stdint.h>

#if defined(__CUDACC__)
#define GPRX_HD __host__ __device__
#else
#define GPRX_HD
#endif

namespace gprx {

constexpr double BARRIER_COST = 1.0e300;

// Logit map of one open interval (lo, hi) shared by every parameter.
struct LogitMap {
  double ln_lo = 0.0, ln_hi = 0.0;
  GPRX_HD void init(double lo, double hi) {
    ln_lo = log(lo);
    ln_hi = log(hi);
  }
  GPRX_HD double scale() const { return (ln_hi - ln_lo) / 4.0; }
  GPRX_HD static double sigmoid(double z) {
    if (z >= 0.0) {
      double e = exp(-z);
      return 1.0 / (1.0 + e);
    }
    double e = exp(z);
    return e / (1.0 + e);
  }
  // z → log θ and dlogθ/dz (jac may be null)
  GPRX_HD void to_log(const double* z, int n, double* log_theta, double* jac) const {
    const double s = scale(), span = ln_hi - ln_lo;
    for (int i = 0; i < n; ++i) {
      double u = sigmoid(z[i] / s);
      log_theta[i] = ln_lo + u * span;
      if (jac) jac[i] = span * u * (1.0 - u) / s;
    }
  }
  // d²logθ/dz² (the chain rule's second-order term of the Hessian,
  // src/optimizer/logit.rs:139-157)
  GPRX_HD void second(const double* z, int n, double* d2) const {
    const double s = scale(), span = ln_hi - ln_lo;
    for (int i = 0; i < n; ++i) {
      double u = sigmoid(z[i] / s);
      d2[i] = span * u * (1.0 - u) * (1.0 - 2.0 * u) / (s * s);
    }
  }
  // log θ → z (fails when θ is outside the open interval)
  GPRX_HD bool from_log(const double* log_theta, int n, double* z) const {
    const double eps = 2.220446049250313e-16;
    const double lo = exp(ln_lo), hi = exp(ln_hi);
    for (int i = 0; i < n; ++i) {
      double v = exp(log_theta[i]);
      if (!(isfinite(v) && v > lo && v < hi)) return false;
      double u = (log(v) - ln_lo) / (ln_hi - ln_lo);
      u = fmin(fmax(u, eps), 1.0 - eps);
      z[i] = log(u / (1.0 - u)) * scale();
    }
    return true;
  }
};

// MINPACK-2 dcstep: safeguarded cubic / quadratic step of the Moré–Thuente
// search.
GPRX_HD inline double lb_max3(double a, double b, double c) { return fmax(fmax(a, b), c); }

GPRX_HD inline void dcstep(double& stx, double& fx, double& dx, double& sty, double& fy, double& dy, double& stp,
                           double fp, double dp, bool& brackt, double stpmin, double stpmax) {
  double sgnd = dp * (dx / fabs(dx));
  double stpf;
  if (fp > fx) {
    double theta = 3.0 * (fx - fp) / (stp - stx) + dx + dp;
    double s = lb_max3(fabs(theta), fabs(dx), fabs(dp));
    double gamma = s * sqrt(fmax(0.0, (theta / s) * (theta / s) - (dx / s) * (dp / s)));
    if (stp < stx) gamma = -gamma;
    double p = (gamma - dx) + theta;
    double q = ((gamma - dx) + gamma) + dp;
    double r = p / q;
    double stpc = stx + r * (stp - stx);
    double stpq = stx + ((dx / ((fx - fp) / (stp - stx) + dx)) / 2.0) * (stp - stx);
    if (fabs(stpc - stx) < fabs(stpq - stx)) stpf = stpc;
    else stpf = stpc + (stpq - stpc) / 2.0;
    brackt = true;
  } else if (sgnd < 0.0) {
    double theta = 3.0 * (fx - fp) / (stp - stx) + dx + dp;
    double s = lb_max3(fabs(theta), fabs(dx), fabs(dp));
    double gamma = s * sqrt(fmax(0.0, (theta / s) * (theta / s) - (dx / s) * (dp / s)));
    if (stp > stx) gamma = -gamma;
    double p = (gamma - dp) + theta;
    double q = ((gamma - dp) + gamma) + dx;
    double r = p / q;
    double stpc = stp + r * (stx - stp);
    double stpq = stp + (dp / (dp - dx)) * (stx - stp);
    stpf = fabs(stpc - stp) > fabs(stpq - stp) ? stpc : stpq;
    brackt = true;
  } else if (fabs(dp) < fabs(dx)) {
    double theta = 3.0 * (fx - fp) / (stp - stx) + dx + dp;
    double s = lb_max3(fabs(theta), fabs(dx), fabs(dp));
    double gamma = s * sqrt(fmax(0.0, (theta / s) * (theta / s) - (dx / s) * (dp / s)));
    if (stp > stx) gamma = -gamma;
    double p = (gamma - dp) + theta;
    double q = (gamma + (dx - dp)) + gamma;
    double r = p / q;
    double stpc;
    if (r < 0.0 && gamma != 0.0) stpc = stp + r * (stx - stp);
    else if (stp > stx) stpc = stpmax;
    else stpc = stpmin;
    double stpq = stp + (dp / (dp - dx)) * (stx - stp);
    if (brackt) {
      stpf = fabs(stpc - stp) < fabs(stpq - stp) ? stpc : stpq;
      if (stp > stx) stpf = fmin(stp + 0.66 * (sty - stp), stpf);
      else stpf = fmax(stp + 0.66 * (sty - stp), stpf);
    } else {
      stpf = fabs(stpc - stp) > fabs(stpq - stp) ? stpc : stpq;
      stpf = fmin(stpmax, stpf);
      stpf = fmax(stpmin, stpf);
    }
  } else {
    if (brackt) {
      double theta = 3.0 * (fp - fy) / (sty - stp) + dy + dp;
      double s = lb_max3(fabs(theta), fabs(dy), fabs(dp));
      double gamma = s * sqrt(fmax(0.0, (theta / s) * (theta / s) - (dy / s) * (dp / s)));
      if (stp > sty) gamma = -gamma;
      double p = (gamma - dp) + theta;
      double q = ((gamma - dp) + gamma) + dy;
      double r = p / q;
      stpf = stp + r * (sty - stp);
    } else if (stp > stx) {
      stpf = stpmax;
    } else {
      stpf = stpmin;
    }
  }
  if (fp > fx) {
    sty = stp;
    fy = fp;
    dy = dp;
  } else {
    if (sgnd < 0.0) {
      sty = stx;
      fy = fx;
      dy = dx;
    }
    stx = stp;
    fx = fp;
    dx = dp;
  }
  stp = stpf;
}

struct MoreThuente {
  double ftol = 1e-4, gtol = 0.9, xtol = 1e-10, stpmin = 1e-20, stpmax = 1e20;
  int max_evals = 20;
  enum Result { CONTINUE, CONVERGED, STOP };

  bool brackt_ = false;
  int stage_ = 1, nfev_ = 0;
  double finit_ = 0, ginit_ = 0, gtest_ = 0, width_ = 0, width1_ = 0;
  double stx_ = 0, fx_ = 0, gx_ = 0, sty_ = 0, fy_ = 0, gy_ = 0, stmin_ = 0, stmax_ = 0, stp_ = 0;

  GPRX_HD double stp() const { return stp_; }
  GPRX_HD int evals() const { return nfev_; }

  // Starts a search from f0, g0 (directional derivative, < 0), first step stp.
  // Returns false when g0 ≥ 0 (not a descent direction).
  GPRX_HD bool start(double f0, double g0, double stp) {
    if (!(g0 < 0.0)) return false;
    brackt_ = false;
    stage_ = 1;
    nfev_ = 0;
    finit_ = f0;
    ginit_ = g0;
    gtest_ = ftol * ginit_;
    width_ = stpmax - stpmin;
    width1_ = 2.0 * width_;
    stx_ = 0.0;
    fx_ = finit_;
    gx_ = ginit_;
    sty_ = 0.0;
    fy_ = finit_;
    gy_ = ginit_;
    stmin_ = 0.0;
    stmax_ = stp + 4.0 * stp;
    stp_ = fmin(fmax(stp, stpmin), stpmax);
    return true;
  }

  // Consumes f, g at the current step; sets the next step (CONTINUE) or ends.
  GPRX_HD Result step(double f, double g) {
    ++nfev_;
    if (!(f < 0.5 * BARRIER_COST)) {
      // A point that cannot be evaluated: its cost carries no slope to
      // interpolate (the cubic step cancels to zero), so the interval closes
      // on it and the next trial moves a quarter of the way back toward the
      // best point so far.
      if (nfev_ >= max_evals) return STOP;
      brackt_ = true;
      sty_ = stp_;
      fy_ = f;
      gy_ = 0.0;
      stmin_ = fmin(stx_, sty_);
      stmax_ = fmax(stx_, sty_);
      stp_ = stx_ + 0.25 * (stp_ - stx_);
      if (fabs(stp_ - stx_) <= xtol * fmax(fabs(stx_), 1e-300)) return STOP;
      return CONTINUE;
    }
    double ftest = finit_ + stp_ * gtest_;
    if (stage_ == 1 && f <= ftest && g >= 0.0) stage_ = 2;
    if (brackt_ && (stp_ <= stmin_ || stp_ >= stmax_)) return STOP;
    if (brackt_ && stmax_ - stmin_ <= xtol * stmax_) return STOP;
    if (stp_ == stpmax && f <= ftest && g <= gtest_) return STOP;
    if (stp_ == stpmin && (f > ftest || g >= gtest_)) return STOP;
    if (f <= ftest && fabs(g) <= gtol * (-ginit_)) return CONVERGED;
    if (nfev_ >= max_evals) return STOP;
    if (stage_ == 1 && f <= fx_ && f > ftest) {
      double fm = f - stp_ * gtest_, fxm = fx_ - stx_ * gtest_, fym = fy_ - sty_ * gtest_;
      double gm = g - gtest_, gxm = gx_ - gtest_, gym = gy_ - gtest_;
      dcstep(stx_, fxm, gxm, sty_, fym, gym, stp_, fm, gm, brackt_, stmin_, stmax_);
      fx_ = fxm + stx_ * gtest_;
      fy_ = fym + sty_ * gtest_;
      gx_ = gxm + gtest_;
      gy_ = gym + gtest_;
    } else {
      dcstep(stx_, fx_, gx_, sty_, fy_, gy_, stp_, f, g, brackt_, stmin_, stmax_);
    }
    if (brackt_) {
      if (fabs(sty_ - stx_) >= 0.66 * width1_) stp_ = stx_ + 0.5 * (sty_ - stx_);
      width1_ = width_;
      width_ = fabs(sty_ - stx_);
    }
    if (brackt_) {
      stmin_ = fmin(stx_, sty_);
      stmax_ = fmax(stx_, sty_);
    } else {
      stmin_ = stp_ + 1.1 * (stp_ - stx_);
      stmax_ = stp_ + 4.0 * (stp_ - stx_);
    }
    stp_ = fmin(fmax(stp_, stpmin), stpmax);
    if ((brackt_ && (stp_ <= stmin_ || stp_ >= stmax_)) || (brackt_ && stmax_ - stmin_ <= xtol * stmax_)) stp_ = stx_;
    return CONTINUE;
  }
};

struct LbfgsConfig {
  int history = 10;
  uint64_t max_iterations = 100;
  double tol_grad = 1.4901161193847656e-08;  // √ε
  double tol_cost = 2.220446049250313e-16;   // ε
};

// One L-BFGS run over at most MP variables with at most MH stored pairs.
// The pair history is a ring: the two-loop recursion visits it newest to
// oldest and back, as a list with the oldest pair dropped first.
template <int MP, int MH>
struct LbfgsRC {
  enum Task { EVALUATE = 0, DONE = 1 };

  LbfgsConfig cfg_{};
  int n_ = 0;
  int task_ = DONE;
  int phase_ = 0;  // 0 initial evaluation, 1 line search
  int hlen_ = 0, hhead_ = 0;  // pairs stored, slot of the oldest
  double x_[MP], g_[MP], d_[MP], xt_[MP];
  double f_ = 0;
  double S_[MH][MP], Y_[MH][MP], rho_[MH];
  MoreThuente ls_;
  double best_x_[MP];
  double best_f_ = BARRIER_COST;
  uint64_t iter_ = 0, nev_ = 0;
  double gnorm_ = 0;
  bool converged_ = false;
  // best point seen inside the current line search
  bool ls_has_best_ = false;
  double ls_best_x_[MP], ls_best_g_[MP];
  double ls_best_f_ = BARRIER_COST;

  static constexpr int max_vars = MP;
  static constexpr int max_history = MH;

  // Point to evaluate (z space) while task() == EVALUATE.
  GPRX_HD const double* point() const { return xt_; }
  GPRX_HD int task() const { return task_; }
  GPRX_HD const double* best() const { return best_x_; }
  GPRX_HD double best_value() const { return best_f_; }
  GPRX_HD uint64_t iterations() const { return iter_; }
  GPRX_HD uint64_t evaluations() const { return nev_; }
  GPRX_HD double grad_norm() const { return gnorm_; }
  GPRX_HD bool converged() const { return converged_; }
  GPRX_HD int size() const { return n_; }

  // n ≤ MP and cfg.history ≤ MH (the caller checks).
  GPRX_HD void start(const LbfgsConfig& cfg, const double* z0, int n) {
    cfg_ = cfg;
    n_ = n;
    for (int j = 0; j < n; ++j) {
      x_[j] = z0[j];
      xt_[j] = z0[j];
      g_[j] = 0.0;
      d_[j] = 0.0;
      best_x_[j] = z0[j];
    }
    hlen_ = hhead_ = 0;
    ls_ = MoreThuente();  // device states start as raw memory
    ls_has_best_ = false;
    ls_best_f_ = BARRIER_COST;
    f_ = 0.0;
    gnorm_ = 0.0;
    best_f_ = BARRIER_COST;
    iter_ = nev_ = 0;
    converged_ = false;
    phase_ = 0;
    task_ = EVALUATE;
  }

  // Feeds f, ∇f (z space) at point(); f = BARRIER_COST with a zero gradient
  // for a point that could not be evaluated.
  GPRX_HD void resume(double f, const double* g) {
    ++nev_;
    if (!isfinite(f)) f = BARRIER_COST;
    if (f < best_f_) {
      best_f_ = f;
      for (int j = 0; j < n_; ++j) best_x_[j] = xt_[j];
    }
    if (phase_ == 0) {
      f_ = f;
      for (int j = 0; j < n_; ++j) g_[j] = g[j];
      gnorm_ = norm(g_);
      if (f >= BARRIER_COST) {
        finish(false);
        return;
      }
      if (gnorm_ < cfg_.tol_grad) {
        finish(true);
        return;
      }
      begin_iteration();
      return;
    }
    // line-search trial at xt_
    double gd = 0.0;
    for (int j = 0; j < n_; ++j) gd += g[j] * d_[j];
    if (f < ls_best_f_) {
      ls_best_f_ = f;
      ls_has_best_ = true;
      for (int j = 0; j < n_; ++j) {
        ls_best_x_[j] = xt_[j];
        ls_best_g_[j] = g[j];
      }
    }
    MoreThuente::Result r = ls_.step(f, gd);
    if (r == MoreThuente::CONTINUE) {
      for (int j = 0; j < n_; ++j) xt_[j] = x_[j] + ls_.stp() * d_[j];
      return;
    }
    // accept the line search's best point
    if (!ls_has_best_ || !(ls_best_f_ < f_)) {
      // no decrease along d: stop (argmin ends the run when the search fails)
      finish(gnorm_ < cfg_.tol_grad);
      return;
    }
    double s[MP], y[MP];
    double sy = 0.0;
    for (int j = 0; j < n_; ++j) {
      s[j] = ls_best_x_[j] - x_[j];
      y[j] = ls_best_g_[j] - g_[j];
      sy += s[j] * y[j];
    }
    double fprev = f_;
    for (int j = 0; j < n_; ++j) {
      x_[j] = ls_best_x_[j];
      g_[j] = ls_best_g_[j];
    }
    f_ = ls_best_f_;
    ++iter_;
    if (sy > 0.0) push_pair(s, y, 1.0 / sy);
    gnorm_ = norm(g_);
    if (gnorm_ < cfg_.tol_grad) {
      finish(true);
      return;
    }
    if (fabs(fprev - f_) < cfg_.tol_cost) {
      finish(true);
      return;
    }
    begin_iteration();
  }

 private:
  GPRX_HD double norm(const double* v) const {
    double s = 0.0;
    for (int j = 0; j < n_; ++j) s += v[j] * v[j];
    return sqrt(s);
  }
  // i-th stored pair, oldest first
  GPRX_HD int slot(int i) const { return (hhead_ + i) % MH; }
  GPRX_HD void push_pair(const double* s, const double* y, double rho) {
    int hist = cfg_.history < MH ? cfg_.history : MH;
    int at;
    if (hlen_ < hist) {
      at = slot(hlen_);
      ++hlen_;
    } else {
      at = hhead_;  // overwrite the oldest
      hhead_ = (hhead_ + 1) % MH;
    }
    for (int j = 0; j < n_; ++j) {
      S_[at][j] = s[j];
      Y_[at][j] = y[j];
    }
    rho_[at] = rho;
  }
  GPRX_HD void finish(bool conv) {
    converged_ = conv;
    task_ = DONE;
  }
  GPRX_HD void begin_iteration() {
    if (iter_ >= cfg_.max_iterations) {
      finish(false);
      return;
    }
    // two-loop recursion: d = −H g
    double q[MP], a[MH];
    for (int j = 0; j < n_; ++j) q[j] = g_[j];
    const int k = hlen_;
    for (int i = k - 1; i >= 0; --i) {
      const int sl = slot(i);
      double s = 0.0;
      for (int j = 0; j < n_; ++j) s += S_[sl][j] * q[j];
      a[i] = rho_[sl] * s;
      for (int j = 0; j < n_; ++j) q[j] -= a[i] * Y_[sl][j];
    }
    double gamma = 1.0;
    if (k > 0) {
      const int sl = slot(k - 1);
      double sy = 0.0, yy = 0.0;
      for (int j = 0; j < n_; ++j) {
        sy += S_[sl][j] * Y_[sl][j];
        yy += Y_[sl][j] * Y_[sl][j];
      }
      gamma = sy / yy;
    }
    for (int j = 0; j < n_; ++j) q[j] *= gamma;
    for (int i = 0; i < k; ++i) {
      const int sl = slot(i);
      double s = 0.0;
      for (int j = 0; j < n_; ++j) s += Y_[sl][j] * q[j];
      double b = rho_[sl] * s;
      for (int j = 0; j < n_; ++j) q[j] += S_[sl][j] * (a[i] - b);
    }
    double gd = 0.0;
    for (int j = 0; j < n_; ++j) {
      d_[j] = -q[j];
      gd += g_[j] * d_[j];
    }
    if (!(gd < 0.0)) {
      // not a descent direction: restart from steepest descent
      hlen_ = hhead_ = 0;
      gd = 0.0;
      for (int j = 0; j < n_; ++j) {
        d_[j] = -g_[j];
        gd -= g_[j] * g_[j];
      }
      if (!(gd < 0.0)) {
        finish(true);
        return;
      }
    }
    if (!ls_.start(f_, gd, 1.0)) {
      finish(false);
      return;
    }
    ls_best_f_ = BARRIER_COST;
    ls_has_best_ = false;
    phase_ = 1;
    for (int j = 0; j < n_; ++j) xt_[j] = x_[j] + ls_.stp() * d_[j];
    task_ = EVALUATE;
  }
};

// The single-model fit's state: every parameter of a kernel tree plus noise.
constexpr int LBFGS_HOST_VARS = 48;
constexpr int LBFGS_HOST_HISTORY = 32;
using HostLbfgs = LbfgsRC<LBFGS_HOST_VARS, LBFGS_HOST_HISTORY>;

}  // namespace gprx
