// lbfgs.cpp — see lbfgs.h.
#include "lbfgs.h"

#include <algorithm>
#include <cmath>

namespace gprx {

// ---------------------------------------------------------------------------
// logit map (src/optimizer/logit.rs:116-242)
// ---------------------------------------------------------------------------
void LogitMap::init(int n, double lo, double hi) {
  ln_lo.assign(n, std::log(lo));
  ln_hi.assign(n, std::log(hi));
}

static double sigmoid(double z) {
  if (z >= 0.0) {
    double e = std::exp(-z);
    return 1.0 / (1.0 + e);
  }
  double e = std::exp(z);
  return e / (1.0 + e);
}

void LogitMap::to_log(const double* z, double* log_theta, double* jac) const {
  for (size_t i = 0; i < ln_lo.size(); ++i) {
    double s = scale((int)i);
    double u = sigmoid(z[i] / s);
    double span = ln_hi[i] - ln_lo[i];
    log_theta[i] = ln_lo[i] + u * span;
    if (jac) jac[i] = span * u * (1.0 - u) / s;
  }
}

bool LogitMap::from_log(const double* log_theta, double* z) const {
  const double eps = 2.220446049250313e-16;
  for (size_t i = 0; i < ln_lo.size(); ++i) {
    double v = std::exp(log_theta[i]);
    double lo = std::exp(ln_lo[i]), hi = std::exp(ln_hi[i]);
    if (!(std::isfinite(v) && v > lo && v < hi)) return false;
    double u = (std::log(v) - ln_lo[i]) / (ln_hi[i] - ln_lo[i]);
    u = std::min(std::max(u, eps), 1.0 - eps);
    z[i] = std::log(u / (1.0 - u)) * scale((int)i);
  }
  return true;
}

// ---------------------------------------------------------------------------
// Moré–Thuente (MINPACK-2 dcsrch / dcstep)
// ---------------------------------------------------------------------------
static void dcstep(double& stx, double& fx, double& dx, double& sty, double& fy, double& dy, double& stp, double fp,
                   double dp, bool& brackt, double stpmin, double stpmax) {
  double sgnd = dp * (dx / std::fabs(dx));
  double stpf;
  if (fp > fx) {
    double theta = 3.0 * (fx - fp) / (stp - stx) + dx + dp;
    double s = std::max({std::fabs(theta), std::fabs(dx), std::fabs(dp)});
    double gamma = s * std::sqrt(std::max(0.0, (theta / s) * (theta / s) - (dx / s) * (dp / s)));
    if (stp < stx) gamma = -gamma;
    double p = (gamma - dx) + theta;
    double q = ((gamma - dx) + gamma) + dp;
    double r = p / q;
    double stpc = stx + r * (stp - stx);
    double stpq = stx + ((dx / ((fx - fp) / (stp - stx) + dx)) / 2.0) * (stp - stx);
    if (std::fabs(stpc - stx) < std::fabs(stpq - stx)) stpf = stpc;
    else stpf = stpc + (stpq - stpc) / 2.0;
    brackt = true;
  } else if (sgnd < 0.0) {
    double theta = 3.0 * (fx - fp) / (stp - stx) + dx + dp;
    double s = std::max({std::fabs(theta), std::fabs(dx), std::fabs(dp)});
    double gamma = s * std::sqrt(std::max(0.0, (theta / s) * (theta / s) - (dx / s) * (dp / s)));
    if (stp > stx) gamma = -gamma;
    double p = (gamma - dp) + theta;
    double q = ((gamma - dp) + gamma) + dx;
    double r = p / q;
    double stpc = stp + r * (stx - stp);
    double stpq = stp + (dp / (dp - dx)) * (stx - stp);
    stpf = std::fabs(stpc - stp) > std::fabs(stpq - stp) ? stpc : stpq;
    brackt = true;
  } else if (std::fabs(dp) < std::fabs(dx)) {
    double theta = 3.0 * (fx - fp) / (stp - stx) + dx + dp;
    double s = std::max({std::fabs(theta), std::fabs(dx), std::fabs(dp)});
    double gamma = s * std::sqrt(std::max(0.0, (theta / s) * (theta / s) - (dx / s) * (dp / s)));
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
      stpf = std::fabs(stpc - stp) < std::fabs(stpq - stp) ? stpc : stpq;
      if (stp > stx) stpf = std::min(stp + 0.66 * (sty - stp), stpf);
      else stpf = std::max(stp + 0.66 * (sty - stp), stpf);
    } else {
      stpf = std::fabs(stpc - stp) > std::fabs(stpq - stp) ? stpc : stpq;
      stpf = std::min(stpmax, stpf);
      stpf = std::max(stpmin, stpf);
    }
  } else {
    if (brackt) {
      double theta = 3.0 * (fp - fy) / (sty - stp) + dy + dp;
      double s = std::max({std::fabs(theta), std::fabs(dy), std::fabs(dp)});
      double gamma = s * std::sqrt(std::max(0.0, (theta / s) * (theta / s) - (dy / s) * (dp / s)));
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

bool MoreThuente::start(double f0, double g0, double stp) {
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
  stp_ = std::min(std::max(stp, stpmin), stpmax);
  return true;
}

MoreThuente::Result MoreThuente::step(double f, double g) {
  ++nfev_;
  if (!(f < 0.5 * BARRIER_COST)) {
    // A point that cannot be evaluated: its cost carries no slope to
    // interpolate (the cubic step cancels to zero), so the interval closes on
    // it and the next trial moves a quarter of the way back toward the best
    // point so far.
    if (nfev_ >= max_evals) return STOP;
    brackt_ = true;
    sty_ = stp_;
    fy_ = f;
    gy_ = 0.0;
    stmin_ = std::min(stx_, sty_);
    stmax_ = std::max(stx_, sty_);
    stp_ = stx_ + 0.25 * (stp_ - stx_);
    if (std::fabs(stp_ - stx_) <= xtol * std::max(std::fabs(stx_), 1e-300)) return STOP;
    return CONTINUE;
  }
  double ftest = finit_ + stp_ * gtest_;
  if (stage_ == 1 && f <= ftest && g >= 0.0) stage_ = 2;
  if (brackt_ && (stp_ <= stmin_ || stp_ >= stmax_)) return STOP;
  if (brackt_ && stmax_ - stmin_ <= xtol * stmax_) return STOP;
  if (stp_ == stpmax && f <= ftest && g <= gtest_) return STOP;
  if (stp_ == stpmin && (f > ftest || g >= gtest_)) return STOP;
  if (f <= ftest && std::fabs(g) <= gtol * (-ginit_)) return CONVERGED;
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
    if (std::fabs(sty_ - stx_) >= 0.66 * width1_) stp_ = stx_ + 0.5 * (sty_ - stx_);
    width1_ = width_;
    width_ = std::fabs(sty_ - stx_);
  }
  if (brackt_) {
    stmin_ = std::min(stx_, sty_);
    stmax_ = std::max(stx_, sty_);
  } else {
    stmin_ = stp_ + 1.1 * (stp_ - stx_);
    stmax_ = stp_ + 4.0 * (stp_ - stx_);
  }
  stp_ = std::min(std::max(stp_, stpmin), stpmax);
  if ((brackt_ && (stp_ <= stmin_ || stp_ >= stmax_)) || (brackt_ && stmax_ - stmin_ <= xtol * stmax_)) stp_ = stx_;
  return CONTINUE;
}

// ---------------------------------------------------------------------------
// L-BFGS in reverse communication
// ---------------------------------------------------------------------------
static double norm2(const std::vector<double>& v) {
  double s = 0.0;
  for (double a : v) s += a * a;
  return std::sqrt(s);
}

void LbfgsRC::start(const LbfgsConfig& cfg, const double* z0, int n) {
  cfg_ = cfg;
  n_ = n;
  x_.assign(z0, z0 + n);
  xt_ = x_;
  g_.assign(n, 0.0);
  gt_.assign(n, 0.0);
  d_.assign(n, 0.0);
  S_.clear();
  Y_.clear();
  rho_.clear();
  best_x_ = x_;
  best_f_ = BARRIER_COST;
  iter_ = nev_ = 0;
  converged_ = false;
  phase_ = 0;
  task_ = EVALUATE;
}

void LbfgsRC::finish(bool conv) {
  converged_ = conv;
  task_ = DONE;
}

void LbfgsRC::begin_iteration() {
  if (iter_ >= cfg_.max_iterations) {
    finish(false);
    return;
  }
  // two-loop recursion: d = −H g
  std::vector<double> q = g_;
  int k = (int)S_.size();
  std::vector<double> a(k);
  for (int i = k - 1; i >= 0; --i) {
    double s = 0.0;
    for (int j = 0; j < n_; ++j) s += S_[i][j] * q[j];
    a[i] = rho_[i] * s;
    for (int j = 0; j < n_; ++j) q[j] -= a[i] * Y_[i][j];
  }
  double gamma = 1.0;
  if (k > 0) {
    double sy = 0.0, yy = 0.0;
    for (int j = 0; j < n_; ++j) {
      sy += S_[k - 1][j] * Y_[k - 1][j];
      yy += Y_[k - 1][j] * Y_[k - 1][j];
    }
    gamma = sy / yy;
  }
  for (int j = 0; j < n_; ++j) q[j] *= gamma;
  for (int i = 0; i < k; ++i) {
    double s = 0.0;
    for (int j = 0; j < n_; ++j) s += Y_[i][j] * q[j];
    double b = rho_[i] * s;
    for (int j = 0; j < n_; ++j) q[j] += S_[i][j] * (a[i] - b);
  }
  double gd = 0.0;
  for (int j = 0; j < n_; ++j) {
    d_[j] = -q[j];
    gd += g_[j] * d_[j];
  }
  if (!(gd < 0.0)) {
    // not a descent direction: restart from steepest descent
    S_.clear();
    Y_.clear();
    rho_.clear();
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
  ls_best_x_.clear();
  phase_ = 1;
  for (int j = 0; j < n_; ++j) xt_[j] = x_[j] + ls_.stp() * d_[j];
  task_ = EVALUATE;
}

void LbfgsRC::resume(double f, const double* g) {
  ++nev_;
  if (!std::isfinite(f)) f = BARRIER_COST;
  if (f < best_f_) {
    best_f_ = f;
    best_x_ = xt_;
  }
  if (phase_ == 0) {
    f_ = f;
    g_.assign(g, g + n_);
    gnorm_ = norm2(g_);
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
    ls_best_x_ = xt_;
    ls_best_g_.assign(g, g + n_);
  }
  MoreThuente::Result r = ls_.step(f, gd);
  if (r == MoreThuente::CONTINUE) {
    for (int j = 0; j < n_; ++j) xt_[j] = x_[j] + ls_.stp() * d_[j];
    return;
  }
  // accept the line search's best point
  if (ls_best_x_.empty() || !(ls_best_f_ < f_)) {
    // no decrease along d: stop (argmin ends the run when the search fails)
    finish(gnorm_ < cfg_.tol_grad);
    return;
  }
  std::vector<double> s(n_), y(n_);
  double sy = 0.0;
  for (int j = 0; j < n_; ++j) {
    s[j] = ls_best_x_[j] - x_[j];
    y[j] = ls_best_g_[j] - g_[j];
    sy += s[j] * y[j];
  }
  double fprev = f_;
  x_ = ls_best_x_;
  g_ = ls_best_g_;
  f_ = ls_best_f_;
  ++iter_;
  if (sy > 0.0) {
    S_.push_back(s);
    Y_.push_back(y);
    rho_.push_back(1.0 / sy);
    if ((int)S_.size() > cfg_.history) {
      S_.erase(S_.begin());
      Y_.erase(Y_.begin());
      rho_.erase(rho_.begin());
    }
  }
  gnorm_ = norm2(g_);
  if (gnorm_ < cfg_.tol_grad) {
    finish(true);
    return;
  }
  if (std::fabs(fprev - f_) < cfg_.tol_cost) {
    finish(true);
    return;
  }
  begin_iteration();
}

}  // namespace gprx
