// gprx_oracle.cpp — TEST INFRASTRUCTURE ONLY.
//
// A plain FP64 CPU restatement of gprx 0.2.0's exact-GPR and VFE-SGPR
// objective-and-prediction path.  It is the parity reference for the CUDA
// backend (tests, __graft_entry__.smoke) and the timed CPU baseline of
// bench.py (kind "port"); nothing in the product links or calls it.
//
// The reference is Rust and cannot be built here (no cargo/rustc; faer 0.24.4,
// argmin 0.11.0 and wide 0.7.33 are not vendored), so this file restates the
// published algorithms.  Each function cites the reference file:line it
// follows.  Linear algebra that gprx delegates to faer 0.24.4 (LLT, triangular
// solves, LDLT row/column delete) is restated from the textbook algorithms:
// right-looking blocked Cholesky, forward/back substitution, and the rank-1
// LDLT update of Gill, Golub, Murray and Saunders (1974, method C1).
//
// Pinned by tests/test_oracle_golden.py against the reference's committed
// goldens (compare/goldens/*.json via tests/golden/make_fixtures.py) and the
// Xoshiro256++ sequence pinned in src/rng.rs.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// ---------------------------------------------------------------------------
// Kernel tree (src/kernel/spec.rs:106, flattened Sum/Product, docs/design.md:288-294)
// ---------------------------------------------------------------------------
enum { SUM = 1, PRODUCT = 2, RBF = 10, RBF_ARD = 11, CONSTANT = 12, PERIODIC = 13 };

struct Node {
  int kind = 0;
  int arg = 0;
  int param = 0;             // first θ index of a leaf
  std::vector<int> children; // for SUM / PRODUCT
};

struct Tree {
  std::vector<Node> nodes;
  std::vector<double> theta; // log params, depth-first
  int n_params = 0;
  bool ok = true;

  int parse(const int32_t* flat, int n_flat, int at) {
    if (at >= n_flat) { ok = false; return at; }
    int idx = (int)nodes.size();
    nodes.push_back(Node{});
    nodes[idx].kind = flat[2 * at];
    nodes[idx].arg = flat[2 * at + 1];
    int next = at + 1;
    int kind = nodes[idx].kind;
    if (kind == SUM || kind == PRODUCT) {
      for (int c = 0; c < nodes[idx].arg; ++c) {
        int child = (int)nodes.size();
        nodes[idx].children.push_back(child);
        next = parse(flat, n_flat, next);
      }
    } else {
      nodes[idx].param = n_params;
      if (kind == RBF || kind == CONSTANT) n_params += 1;
      else if (kind == PERIODIC) n_params += 2;
      else if (kind == RBF_ARD) n_params += nodes[idx].arg;
      else ok = false;
    }
    return next;
  }
};

bool build_tree(Tree& t, const int32_t* flat, int n_flat, const double* theta, int n_theta) {
  t.nodes.clear();
  t.n_params = 0;
  t.ok = true;
  int end = t.parse(flat, n_flat, 0);
  if (!t.ok || end != n_flat || t.n_params != n_theta) return false;
  t.theta.assign(theta, theta + n_theta);
  return true;
}

// Leaf value at one pair (src/kernel/rbf.rs:18, rbf_ard.rs:16, constant.rs:12,
// periodic.rs:598-611).  x1/x2 point at feature 0 with strides s1/s2.
double leaf_value(const Tree& t, const Node& nd, const double* x1, int64_t s1, const double* x2,
                  int64_t s2, int d) {
  const double* th = t.theta.data() + nd.param;
  switch (nd.kind) {
    case CONSTANT:
      return std::exp(th[0]);
    case RBF: {
      double r2 = 0.0;
      for (int f = 0; f < d; ++f) { double df = x1[f * s1] - x2[f * s2]; r2 += df * df; }
      double ell = std::exp(th[0]);
      return std::exp(-0.5 * r2 / (ell * ell));
    }
    case RBF_ARD: {
      double q = 0.0;
      for (int f = 0; f < d; ++f) {
        double ell = std::exp(th[f]);
        double df = (x1[f * s1] - x2[f * s2]) / ell;
        q += df * df;
      }
      return std::exp(-0.5 * q);
    }
    case PERIODIC: {
      double r2 = 0.0;
      for (int f = 0; f < d; ++f) { double df = x1[f * s1] - x2[f * s2]; r2 += df * df; }
      double r = std::sqrt(std::max(r2, 0.0));
      double ell = std::exp(th[0]), p = std::exp(th[1]);
      double s = std::sin(M_PI * r / p);
      return std::exp(-2.0 * s * s / (ell * ell));
    }
  }
  return NAN;
}

// ∂leaf/∂(its log params) (src/kernel/rbf.rs:470, rbf_ard.rs grad, constant.rs,
// periodic.rs:613-638).  Writes nd's parameters into g (indexed globally).
void leaf_grad(const Tree& t, const Node& nd, const double* x1, int64_t s1, const double* x2,
               int64_t s2, int d, double scale, double* g) {
  const double* th = t.theta.data() + nd.param;
  switch (nd.kind) {
    case CONSTANT:
      g[nd.param] += scale * std::exp(th[0]);
      return;
    case RBF: {
      double r2 = 0.0;
      for (int f = 0; f < d; ++f) { double df = x1[f * s1] - x2[f * s2]; r2 += df * df; }
      double ell = std::exp(th[0]);
      double inv = 1.0 / (ell * ell);
      double k = std::exp(-0.5 * r2 * inv);
      g[nd.param] += scale * k * r2 * inv;
      return;
    }
    case RBF_ARD: {
      double q = 0.0;
      double sq[64];
      for (int f = 0; f < d; ++f) {
        double ell = std::exp(th[f]);
        double df = (x1[f * s1] - x2[f * s2]) / ell;
        sq[f] = df * df;
        q += sq[f];
      }
      double k = std::exp(-0.5 * q);
      for (int f = 0; f < d; ++f) g[nd.param + f] += scale * k * sq[f];
      return;
    }
    case PERIODIC: {
      double r2 = 0.0;
      for (int f = 0; f < d; ++f) { double df = x1[f * s1] - x2[f * s2]; r2 += df * df; }
      double r = std::sqrt(std::max(r2, 0.0));
      double ell = std::exp(th[0]), p = std::exp(th[1]);
      double a = M_PI * r / p;
      double s = std::sin(a), c = std::cos(a);
      double inv = 1.0 / (ell * ell);
      double k = std::exp(-2.0 * s * s * inv);
      g[nd.param] += scale * k * 4.0 * s * s * inv;
      g[nd.param + 1] += scale * k * 4.0 * s * c * a * inv;
      return;
    }
  }
}

double node_value(const Tree& t, int idx, const double* x1, int64_t s1, const double* x2, int64_t s2,
                  int d) {
  const Node& nd = t.nodes[idx];
  if (nd.kind == SUM) {
    double v = 0.0;
    for (int c : nd.children) v += node_value(t, c, x1, s1, x2, s2, d);
    return v;
  }
  if (nd.kind == PRODUCT) {
    double v = 1.0;
    for (int c : nd.children) v *= node_value(t, c, x1, s1, x2, s2, d);
    return v;
  }
  return leaf_value(t, nd, x1, s1, x2, s2, d);
}

// Reverse walk: a Sum gives every term the same weight, a Product gives a
// factor the weight times the other factors (src/kernel/compiled/weighted.rs:274-345).
void node_grad(const Tree& t, int idx, const double* x1, int64_t s1, const double* x2, int64_t s2,
               int d, double scale, double* g) {
  const Node& nd = t.nodes[idx];
  if (nd.kind == SUM) {
    for (int c : nd.children) node_grad(t, c, x1, s1, x2, s2, d, scale, g);
    return;
  }
  if (nd.kind == PRODUCT) {
    std::vector<double> vals;
    for (int c : nd.children) vals.push_back(node_value(t, c, x1, s1, x2, s2, d));
    for (size_t a = 0; a < nd.children.size(); ++a) {
      double others = 1.0;
      for (size_t b = 0; b < vals.size(); ++b)
        if (b != a) others *= vals[b];
      node_grad(t, nd.children[a], x1, s1, x2, s2, d, scale * others, g);
    }
    return;
  }
  leaf_grad(t, nd, x1, s1, x2, s2, d, scale, g);
}

inline double kval(const Tree& t, const double* x1, int64_t s1, const double* x2, int64_t s2, int d) {
  return node_value(t, 0, x1, s1, x2, s2, d);
}

// ---------------------------------------------------------------------------
// Dense FP64 linear algebra, column-major (faer restated)
// ---------------------------------------------------------------------------
using Mat = std::vector<double>;
#define AT(a, ld, i, j) (a)[(size_t)(i) + (size_t)(j) * (size_t)(ld)]

// C[i][j] -= Σ_t A[i][t] B[j][t] for i in [0,mi), j in [0,mj), packed row-major
// A (mi×kt) and B (mj×kt); only (i,j) with row0+i >= col0+j when lower.
void packed_update(double* c, int64_t ldc, const double* a, int mi, const double* b, int mj, int kt,
                   int64_t row0, int64_t col0, bool lower) {
  const int BI = 4, BJ = 4;
#pragma omp parallel for schedule(dynamic, 1)
  for (int jb = 0; jb < mj; jb += BJ) {
    for (int ib = 0; ib < mi; ib += BI) {
      if (lower && row0 + ib + BI - 1 < col0 + jb) continue;
      double acc[BI][BJ] = {{0}};
      int ni = std::min(BI, mi - ib), nj = std::min(BJ, mj - jb);
      if (ni == BI && nj == BJ) {
        const double* a0 = a + (size_t)(ib + 0) * kt;
        const double* a1 = a + (size_t)(ib + 1) * kt;
        const double* a2 = a + (size_t)(ib + 2) * kt;
        const double* a3 = a + (size_t)(ib + 3) * kt;
        const double* b0 = b + (size_t)(jb + 0) * kt;
        const double* b1 = b + (size_t)(jb + 1) * kt;
        const double* b2 = b + (size_t)(jb + 2) * kt;
        const double* b3 = b + (size_t)(jb + 3) * kt;
        for (int q = 0; q < kt; ++q) {
          double x0 = a0[q], x1 = a1[q], x2 = a2[q], x3 = a3[q];
          double y0 = b0[q], y1 = b1[q], y2 = b2[q], y3 = b3[q];
          acc[0][0] += x0 * y0; acc[0][1] += x0 * y1; acc[0][2] += x0 * y2; acc[0][3] += x0 * y3;
          acc[1][0] += x1 * y0; acc[1][1] += x1 * y1; acc[1][2] += x1 * y2; acc[1][3] += x1 * y3;
          acc[2][0] += x2 * y0; acc[2][1] += x2 * y1; acc[2][2] += x2 * y2; acc[2][3] += x2 * y3;
          acc[3][0] += x3 * y0; acc[3][1] += x3 * y1; acc[3][2] += x3 * y2; acc[3][3] += x3 * y3;
        }
      } else {
        for (int i = 0; i < ni; ++i)
          for (int j = 0; j < nj; ++j) {
            double s = 0.0;
            for (int q = 0; q < kt; ++q) s += a[(size_t)(ib + i) * kt + q] * b[(size_t)(jb + j) * kt + q];
            acc[i][j] = s;
          }
      }
      for (int j = 0; j < nj; ++j)
        for (int i = 0; i < ni; ++i) {
          if (lower && row0 + ib + i < col0 + jb + j) continue;
          c[(size_t)(ib + i) + (size_t)(jb + j) * ldc] -= acc[i][j];
        }
    }
  }
}

// Unblocked lower Cholesky of the nb×nb block at (k,k); false on a pivot that is
// not positive (faer NonPositivePivot → CholeskyFailed, src/linalg/chol.rs:141-167).
bool potf2(double* a, int64_t ld, int64_t k, int nb) {
  for (int j = 0; j < nb; ++j) {
    double* cj = &AT(a, ld, k, k + j);
    double d = cj[j];
    for (int q = 0; q < j; ++q) { double l = AT(a, ld, k + j, k + q); d -= l * l; }
    if (!(d > 0.0)) return false;
    double ljj = std::sqrt(d);
    cj[j] = ljj;
    for (int i = j + 1; i < nb; ++i) {
      double s = cj[i];
      for (int q = 0; q < j; ++q) s -= AT(a, ld, k + i, k + q) * AT(a, ld, k + j, k + q);
      cj[i] = s / ljj;
    }
  }
  return true;
}

// Right-looking blocked LLT in place (lower).  Upper triangle is not read.
bool potrf(double* a, int64_t n, int64_t ld) {
  const int NB = 64;
  std::vector<double> panel;
  for (int64_t k = 0; k < n; k += NB) {
    int nb = (int)std::min<int64_t>(NB, n - k);
    if (!potf2(a, ld, k, nb)) return false;
    int64_t rest = n - k - nb;
    if (rest <= 0) break;
    // panel: rows below solve X L_kkᵀ = A  (row-wise substitution)
#pragma omp parallel for schedule(static)
    for (int64_t i = k + nb; i < n; ++i) {
      for (int j = 0; j < nb; ++j) {
        double s = AT(a, ld, i, k + j);
        for (int q = 0; q < j; ++q) s -= AT(a, ld, i, k + q) * AT(a, ld, k + j, k + q);
        AT(a, ld, i, k + j) = s / AT(a, ld, k + j, k + j);
      }
    }
    panel.assign((size_t)rest * nb, 0.0);
    for (int64_t i = 0; i < rest; ++i)
      for (int j = 0; j < nb; ++j) panel[(size_t)i * nb + j] = AT(a, ld, k + nb + i, k + j);
    packed_update(&AT(a, ld, k + nb, k + nb), ld, panel.data(), (int)rest, panel.data(), (int)rest, nb,
                  0, 0, true);
  }
  return true;
}

// L z = b then Lᵀ x = z, in place (faer llt::solve, src/linalg/chol.rs:334-339).
void llt_solve(const double* l, int64_t n, int64_t ld, double* b) {
  for (int64_t i = 0; i < n; ++i) {
    double s = b[i];
    for (int64_t q = 0; q < i; ++q) s -= AT(l, ld, i, q) * b[q];
    b[i] = s / AT(l, ld, i, i);
  }
  for (int64_t i = n - 1; i >= 0; --i) {
    double s = b[i];
    for (int64_t q = i + 1; q < n; ++q) s -= AT(l, ld, q, i) * b[q];
    b[i] = s / AT(l, ld, i, i);
  }
}

// Overwrites each column of B (n×q) with L⁻¹ B (faer solve_lower_triangular_in_place),
// column-oriented: x_t = b_t / L_tt, then b_i −= L_it x_t down column t of L
// (contiguous in memory).
void trsm_lower(const double* l, int64_t n, int64_t ld, double* b, int64_t q, int64_t ldb) {
#pragma omp parallel for schedule(static)
  for (int64_t c = 0; c < q; ++c) {
    double* col = b + c * ldb;
    for (int64_t t = 0; t < n; ++t) {
      const double xt = col[t] / AT(l, ld, t, t);
      col[t] = xt;
      const double* lt = &AT(l, ld, 0, t);
      for (int64_t i = t + 1; i < n; ++i) col[i] -= lt[i] * xt;
    }
  }
}

// C (m×m, ldc) = A Bᵀ over the n columns of the column-major m×n matrices A and
// B (lower triangle only when `lower`), in chunks of columns packed row-wise
// for packed_update; sums over n accumulate chunk by chunk.
void gemm_abt_cols(const double* a, const double* b, int64_t m, int64_t n, double* c, int64_t ldc, bool lower) {
  const int64_t KC = 1024;
  for (int64_t j = 0; j < m; ++j)
    for (int64_t i = 0; i < m; ++i) AT(c, ldc, i, j) = 0.0;
  std::vector<double> pa((size_t)m * KC), pb;
  if (a != b) pb.resize((size_t)m * KC);
  for (int64_t c0 = 0; c0 < n; c0 += KC) {
    int kt = (int)std::min<int64_t>(KC, n - c0);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < m; ++i)
      for (int t = 0; t < kt; ++t) {
        pa[(size_t)i * kt + t] = AT(a, m, i, c0 + t);
        if (a != b) pb[(size_t)i * kt + t] = AT(b, m, i, c0 + t);
      }
    // packed_update subtracts: accumulate −A Bᵀ and flip the sign at the end
    packed_update(c, ldc, pa.data(), (int)m, a != b ? pb.data() : pa.data(), (int)m, kt, 0, 0, lower);
  }
  for (int64_t j = 0; j < m; ++j)
    for (int64_t i = lower ? j : 0; i < m; ++i) AT(c, ldc, i, j) = -AT(c, ldc, i, j);
}

// Overwrites each column of B (n×q) with L⁻ᵀ B.
void trsm_lower_t(const double* l, int64_t n, int64_t ld, double* b, int64_t q, int64_t ldb) {
#pragma omp parallel for schedule(static)
  for (int64_t c = 0; c < q; ++c) {
    double* col = b + c * ldb;
    for (int64_t i = n - 1; i >= 0; --i) {
      double s = col[i];
      for (int64_t t = i + 1; t < n; ++t) s -= AT(l, ld, t, i) * col[t];
      col[i] = s / AT(l, ld, i, i);
    }
  }
}

// K⁻¹ (lower) from L: the identity-RHS solve of FitBuffers::form_gradient_w
// (src/workspace.rs:395-425), written as X = L⁻¹ then K⁻¹ = Xᵀ X.
void llt_inverse(const double* l, int64_t n, int64_t ld, double* kinv, int64_t ldk) {
  Mat x((size_t)n * n, 0.0);
  // X = L⁻¹ by block rows: X_k = L_kk⁻¹ B_k (forward substitution), then
  // B_{>k, ≤k} −= L_{>k,k} X_{k, ≤k}; B starts as the identity.
  for (int64_t i = 0; i < n; ++i) x[(size_t)i * n + i] = 1.0;
  const int NB = 64;
  std::vector<double> pa, pb;
  for (int64_t k = 0; k < n; k += NB) {
    int nb = (int)std::min<int64_t>(NB, n - k);
    int64_t cols = k + nb;
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < cols; ++c) {
      double* col = &x[(size_t)c * n];
      for (int i = 0; i < nb; ++i) {
        double s = col[k + i];
        for (int t = 0; t < i; ++t) s -= AT(l, ld, k + i, k + t) * col[k + t];
        col[k + i] = s / AT(l, ld, k + i, k + i);
      }
    }
    int64_t rest = n - cols;
    if (rest <= 0) break;
    pa.assign((size_t)rest * nb, 0.0);
    for (int64_t i = 0; i < rest; ++i)
      for (int t = 0; t < nb; ++t) pa[(size_t)i * nb + t] = AT(l, ld, cols + i, k + t);
    pb.assign((size_t)cols * nb, 0.0);
    for (int64_t c = 0; c < cols; ++c)
      for (int t = 0; t < nb; ++t) pb[(size_t)c * nb + t] = x[(size_t)c * n + k + t];
    packed_update(&x[(size_t)cols], n, pa.data(), (int)rest, pb.data(), (int)cols, nb, 0, 0, false);
  }
  // K⁻¹_ij = Σ_{t ≥ i} X_ti X_tj for i ≥ j (columns of X are contiguous).
#pragma omp parallel for schedule(dynamic, 8)
  for (int64_t j = 0; j < n; ++j) {
    const double* cj = &x[(size_t)j * n];
    for (int64_t i = j; i < n; ++i) {
      const double* ci = &x[(size_t)i * n];
      double s = 0.0;
      for (int64_t t = i; t < n; ++t) s += ci[t] * cj[t];
      AT(kinv, ldk, i, j) = s;
    }
  }
}

// Lower training Gram (CompiledKernel::eval_gram, Triangle::Lower; src/kernel/compiled/gram.rs:103)
bool gram_lower(const Tree& t, const double* x, int64_t n, int d, double* k, int64_t ld) {
  bool finite = true;
#pragma omp parallel for schedule(dynamic, 16) reduction(&& : finite)
  for (int64_t j = 0; j < n; ++j)
    for (int64_t i = j; i < n; ++i) {
      double v = kval(t, x + i, n, x + j, n, d);
      if (!std::isfinite(v)) finite = false;
      AT(k, ld, i, j) = v;
    }
  return finite;
}

// JitterPolicy retry list (src/policy.rs:306-397): the sequence after j = 0.
std::vector<double> retry_jitters(int kind, double initial, double mult, int max_retries, double max_j) {
  std::vector<double> out;
  if (kind == 0) {
    if (initial > 0.0) out.push_back(initial);
    return out;
  }
  double j = initial;
  for (int r = 0; r < max_retries; ++r) {
    if (!(j <= max_j)) break;
    out.push_back(j);
    double g = j * mult;
    if (!std::isfinite(g)) break;
    j = g;
  }
  return out;
}

struct Factor {
  int64_t n = 0;
  Mat l;        // n×n, lower
  std::vector<double> alpha;
  double jitter = 0.0;
};

// factor_written_k_with_policy (src/gpr/factor.rs:515-542): clear, fill, add
// σn² + j, Cholesky, solve α; retried with the jitter list.
int factor_exact(const Tree& t, const double* x, int64_t n, int d, const double* y, double noise,
                 const std::vector<double>& jitters, Factor& f, double* last_j) {
  f.n = n;
  f.l.assign((size_t)n * n, 0.0);
  std::vector<double> js;
  js.push_back(0.0);
  js.insert(js.end(), jitters.begin(), jitters.end());
  for (double j : js) {
    *last_j = j;
    std::fill(f.l.begin(), f.l.end(), 0.0);
    if (!gram_lower(t, x, n, d, f.l.data(), n)) return 2;  // NonFiniteKernelValue
    for (int64_t i = 0; i < n; ++i) AT(f.l, n, i, i) += noise + j;
    if (potrf(f.l.data(), n, n)) {
      f.alpha.assign(y, y + n);
      llt_solve(f.l.data(), n, n, f.alpha.data());
      f.jitter = j;
      return 0;
    }
  }
  return 1;  // CholeskyFailed
}

// neg_mll_from_factor (src/gpr/factor.rs:555-568)
double nlml_from_factor(const Factor& f, const double* y) {
  double quad = 0.0, logdet = 0.0;
  for (int64_t i = 0; i < f.n; ++i) quad += y[i] * f.alpha[i];
  for (int64_t i = 0; i < f.n; ++i) logdet += std::log(AT(f.l, f.n, i, i));
  return 0.5 * (quad + 2.0 * logdet + (double)f.n * std::log(2.0 * M_PI));
}

// ---------------------------------------------------------------------------
// Xoshiro256++ / SplitMix64 (src/rng.rs:10-87)
// ---------------------------------------------------------------------------
struct Rng {
  uint64_t s[4];
};
inline uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
void rng_seed(Rng& r, uint64_t seed) {
  uint64_t x = seed;
  for (int i = 0; i < 4; ++i) {
    x += 0x9e3779b97f4a7c15ULL;
    uint64_t z = x;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    r.s[i] = z ^ (z >> 31);
  }
}
uint64_t rng_next(Rng& r) {
  uint64_t* s = r.s;
  uint64_t result = rotl(s[0] + s[3], 23) + s[0];
  uint64_t t = s[1] << 17;
  s[2] ^= s[0];
  s[3] ^= s[1];
  s[1] ^= s[2];
  s[0] ^= s[3];
  s[2] ^= t;
  s[3] = rotl(s[3], 45);
  return result;
}

// Value, gradient and Hessian (in the log parameters, dense over all np
// kernel parameters) of node idx at one pair.  A Sum adds its children's
// triples; a Product folds them with (f, g, H)·(c, gc, Hc) = (f c,
// f gc + c g, f Hc + c H + g gcᵀ + gc gᵀ).  Leaf second derivatives
// (u = r²/ℓ², u_f = Δ_f²/ℓ_f², φ = π r / p, s = sin φ, c = cos φ):
//   constant k = e^θ: ∂ = ∂² = k;  rbf: ∂ = k u, ∂² = k (u² − 2u);
//   rbf_ard: ∂_f = k u_f, ∂_fg = k u_f u_g − 2 δ_fg k u_f;
//   periodic (a = 4 s²/ℓ², b = 4 s c φ/ℓ²): ∂_ℓ = k a, ∂_p = k b,
//   ∂_ℓℓ = k (a² − 2a), ∂_ℓp = k b (a − 2),
//   ∂_pp = k (b² + 4 (φ² (s² − c²) − s c φ)/ℓ²).
// These are the second-order kernel walks of CompiledKernel::hess_gram
// (src/kernel/compiled/, used by src/gpr/exact_fit.rs:583-610).
void node_vgh(const Tree& t, int idx, const double* x1, int64_t s1, const double* x2, int64_t s2, int d,
              double& f, std::vector<double>& g, std::vector<double>& h) {
  const int np = t.n_params;
  const Node& nd = t.nodes[idx];
  g.assign(np, 0.0);
  h.assign((size_t)np * np, 0.0);
  if (nd.kind == SUM || nd.kind == PRODUCT) {
    f = nd.kind == SUM ? 0.0 : 1.0;
    double c;
    std::vector<double> gc, hc;
    for (int ch : nd.children) {
      node_vgh(t, ch, x1, s1, x2, s2, d, c, gc, hc);
      if (nd.kind == SUM) {
        f += c;
        for (int a = 0; a < np; ++a) g[a] += gc[a];
        for (size_t e = 0; e < h.size(); ++e) h[e] += hc[e];
      } else {
        for (int a = 0; a < np; ++a)
          for (int b = 0; b < np; ++b)
            h[(size_t)a * np + b] = f * hc[(size_t)a * np + b] + c * h[(size_t)a * np + b] + g[a] * gc[b] +
                                    gc[a] * g[b];
        for (int a = 0; a < np; ++a) g[a] = f * gc[a] + c * g[a];
        f *= c;
      }
    }
    return;
  }
  const double* th = t.theta.data() + nd.param;
  const int p0 = nd.param;
  double r2 = 0.0;
  for (int q = 0; q < d; ++q) { double df = x1[q * s1] - x2[q * s2]; r2 += df * df; }
  switch (nd.kind) {
    case CONSTANT:
      f = std::exp(th[0]);
      g[p0] = f;
      h[(size_t)p0 * np + p0] = f;
      return;
    case RBF: {
      double ell = std::exp(th[0]);
      double u = r2 / (ell * ell);
      f = std::exp(-0.5 * u);
      g[p0] = f * u;
      h[(size_t)p0 * np + p0] = f * (u * u - 2.0 * u);
      return;
    }
    case RBF_ARD: {
      std::vector<double> u(d);
      double q = 0.0;
      for (int a = 0; a < d; ++a) {
        double ell = std::exp(th[a]);
        double df = (x1[a * s1] - x2[a * s2]) / ell;
        u[a] = df * df;
        q += u[a];
      }
      f = std::exp(-0.5 * q);
      for (int a = 0; a < d; ++a) {
        g[p0 + a] = f * u[a];
        for (int b = 0; b < d; ++b)
          h[(size_t)(p0 + a) * np + p0 + b] = f * u[a] * u[b] - (a == b ? 2.0 * f * u[a] : 0.0);
      }
      return;
    }
    case PERIODIC: {
      double r = std::sqrt(std::max(r2, 0.0));
      double ell = std::exp(th[0]), per = std::exp(th[1]);
      double inv = 1.0 / (ell * ell);
      double phi = M_PI * r / per;
      double sn = std::sin(phi), cs = std::cos(phi);
      f = std::exp(-2.0 * sn * sn * inv);
      double a = 4.0 * sn * sn * inv, b = 4.0 * sn * cs * phi * inv;
      g[p0] = f * a;
      g[p0 + 1] = f * b;
      h[(size_t)p0 * np + p0] = f * (a * a - 2.0 * a);
      h[(size_t)p0 * np + p0 + 1] = h[(size_t)(p0 + 1) * np + p0] = f * b * (a - 2.0);
      h[(size_t)(p0 + 1) * np + p0 + 1] = f * (b * b + 4.0 * inv * (phi * phi * (sn * sn - cs * cs) - sn * cs * phi));
      return;
    }
  }
  f = NAN;
}

}  // namespace

// ===========================================================================
// C API (ctypes)
// ===========================================================================
extern "C" {

int orc_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

void orc_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

int orc_num_params(const int32_t* nodes, int n_nodes) {
  Tree t;
  int end = t.parse(nodes, n_nodes, 0);
  if (!t.ok || end != n_nodes) return -1;
  return t.n_params;
}

// Lower Gram K(X,X) (no noise) into k (n×n col-major; upper untouched).
int orc_gram_lower(const int32_t* nodes, int n_nodes, const double* theta, int n_theta, const double* x,
                   int64_t n, int d, double* k) {
  Tree t;
  if (!build_tree(t, nodes, n_nodes, theta, n_theta)) return 3;
  return gram_lower(t, x, n, d, k, n) ? 0 : 2;
}

// K(X1, X2) n1×n2 (eval_cross_slots, src/kernel/compiled/gram.rs:203).
int orc_cross(const int32_t* nodes, int n_nodes, const double* theta, int n_theta, const double* x1,
              int64_t n1, const double* x2, int64_t n2, int d, double* out) {
  Tree t;
  if (!build_tree(t, nodes, n_nodes, theta, n_theta)) return 3;
#pragma omp parallel for schedule(static)
  for (int64_t j = 0; j < n2; ++j)
    for (int64_t i = 0; i < n1; ++i) AT(out, n1, i, j) = kval(t, x1 + i, n1, x2 + j, n2, d);
  return 0;
}

// In-place lower Cholesky; returns 1 on a non-positive pivot.
int orc_potrf(double* a, int64_t n) { return potrf(a, n, n) ? 0 : 1; }

// K⁻¹ lower from L.
void orc_llt_inverse(const double* l, int64_t n, double* kinv) { llt_inverse(l, n, n, kinv, n); }

// One exact NLML + gradient evaluation (ExactFit::value_and_gradient_into_fit,
// src/gpr/exact_fit.rs:319-341 and :665-729; src/workspace.rs:395-425).
// params = [kernel log θ..., log σn²].  grad may be NULL.  alpha (n) may be NULL.
int orc_exact_eval(const int32_t* nodes, int n_nodes, const double* params, int n_params,
                   const double* x, int64_t n, int d, const double* y, int jitter_kind,
                   double jitter_initial, double jitter_mult, int jitter_retries, double jitter_max,
                   double* nlml, double* grad, double* alpha, double* jitter_used) {
  Tree t;
  int nk = n_params - 1;
  if (!build_tree(t, nodes, n_nodes, params, nk)) return 3;
  double noise = std::exp(params[nk]);
  Factor f;
  double last_j = 0.0;
  int st = factor_exact(t, x, n, d, y, noise,
                        retry_jitters(jitter_kind, jitter_initial, jitter_mult, jitter_retries, jitter_max),
                        f, &last_j);
  if (jitter_used) *jitter_used = last_j;
  if (st != 0) return st;
  *nlml = nlml_from_factor(f, y);
  if (alpha) std::copy(f.alpha.begin(), f.alpha.end(), alpha);
  if (!grad) return 0;
  Mat kinv((size_t)n * n, 0.0);
  llt_inverse(f.l.data(), n, n, kinv.data(), n);
  // W = ααᵀ − K⁻¹ (form_w_lower, src/workspace.rs:351-360); lower-triangle
  // Frobenius with weight 1 on the diagonal and 2 off it (src/linalg/dense.rs:20-34).
  // Each column's sum is formed on its own, then the columns are folded in
  // column order (par_lower_fold, src/kernel/dist.rs:187-233), so the result
  // does not depend on the thread count.
  int np = n_params;
  std::vector<double> cols((size_t)n * np, 0.0);
#pragma omp parallel for schedule(dynamic, 16)
  for (int64_t j = 0; j < n; ++j) {
    double* g = &cols[(size_t)j * np];
    for (int64_t i = j; i < n; ++i) {
      double w = f.alpha[i] * f.alpha[j] - AT(kinv, n, i, j);
      double scale = (i == j) ? w : 2.0 * w;
      node_grad(t, 0, x + i, n, x + j, n, d, scale, g);
    }
  }
  std::vector<double> g(np, 0.0);
  for (int64_t j = 0; j < n; ++j)
    for (int p = 0; p < np; ++p) g[p] += cols[(size_t)j * np + p];
  for (int p = 0; p < nk; ++p) grad[p] = -0.5 * g[p];
  // noise: −½ σn² Σ W_ii (src/gpr/exact_fit.rs:676-682)
  double wdiag = 0.0;
  for (int64_t i = 0; i < n; ++i) wdiag += f.alpha[i] * f.alpha[i] - AT(kinv, n, i, i);
  grad[nk] = -0.5 * noise * wdiag;
  return 0;
}

// Predictive moments at q points (GprCore::write_moments, src/gpr/shared.rs:754-820).
// kind 0 = latent, 1 = observation.
int orc_exact_predict(const int32_t* nodes, int n_nodes, const double* params, int n_params,
                      const double* x, int64_t n, int d, const double* y, int jitter_kind,
                      double jitter_initial, double jitter_mult, int jitter_retries, double jitter_max,
                      const double* xs, int64_t q, int kind, double* mean, double* var) {
  Tree t;
  int nk = n_params - 1;
  if (!build_tree(t, nodes, n_nodes, params, nk)) return 3;
  double noise = std::exp(params[nk]);
  Factor f;
  double last_j = 0.0;
  int st = factor_exact(t, x, n, d, y, noise,
                        retry_jitters(jitter_kind, jitter_initial, jitter_mult, jitter_retries, jitter_max),
                        f, &last_j);
  if (st != 0) return st;
  Mat ks((size_t)n * q);
#pragma omp parallel for schedule(static)
  for (int64_t c = 0; c < q; ++c)
    for (int64_t i = 0; i < n; ++i) AT(ks, n, i, c) = kval(t, x + i, n, xs + c, q, d);
  for (int64_t c = 0; c < q; ++c) {
    double m = 0.0;
    for (int64_t i = 0; i < n; ++i) m += AT(ks, n, i, c) * f.alpha[i];
    mean[c] = m;
  }
  trsm_lower(f.l.data(), n, n, ks.data(), q, n);
  for (int64_t c = 0; c < q; ++c) {
    double quad = 0.0;
    for (int64_t i = 0; i < n; ++i) quad += AT(ks, n, i, c) * AT(ks, n, i, c);
    double kss = kval(t, xs + c, q, xs + c, q, d);
    double lat = kss - quad;
    if (lat < 0.0) lat = 0.0;
    var[c] = kind == 1 ? lat + noise : lat;
  }
  return 0;
}

// Leave-one-out at every training point (GprCore::loo_predict_with,
// src/gpr/shared.rs:522-567; GPML §5.4.2): Q = (K + σn² I)⁻¹,
// mean_i = y_i − α_i / Q_ii, observation variance 1 / Q_ii, latent
// max(0, 1 / Q_ii − σn²).  Returns 17 when a Q_ii is not positive.
int orc_exact_loo(const int32_t* nodes, int n_nodes, const double* params, int n_params, const double* x, int64_t n,
                  int d, const double* y, int jitter_kind, double jitter_initial, double jitter_mult,
                  int jitter_retries, double jitter_max, int kind, double* mean, double* var) {
  Tree t;
  int nk = n_params - 1;
  if (!build_tree(t, nodes, n_nodes, params, nk)) return 3;
  double noise = std::exp(params[nk]);
  Factor f;
  double last_j = 0.0;
  int st = factor_exact(t, x, n, d, y, noise,
                        retry_jitters(jitter_kind, jitter_initial, jitter_mult, jitter_retries, jitter_max),
                        f, &last_j);
  if (st != 0) return st;
  Mat kinv((size_t)n * n, 0.0);
  llt_inverse(f.l.data(), n, n, kinv.data(), n);
  for (int64_t i = 0; i < n; ++i) {
    double q = AT(kinv, n, i, i);
    if (!(q > 0.0) || !std::isfinite(q)) return 17;
    mean[i] = y[i] - f.alpha[i] / q;
    double obs = 1.0 / q;
    var[i] = kind == 1 ? obs : std::max(obs - noise, 0.0);
  }
  return 0;
}

// Hessian of the NLML at params, row-major p × p (ExactFit::fill_hessian_from_factor
// and add_first_order, src/gpr/exact_fit.rs:483-579):
//   H_ij = −½ Σ_{a≥b} c_ab W_ab ∂²A_ab/∂θ_i∂θ_j − ½ ⟨S_i, S_j⟩_F + v_iᵀ v_j,
// W = ααᵀ − A⁻¹, c = 1 on the diagonal and 2 off it, S_i = L⁻¹ A_i L⁻ᵀ,
// v_i = L⁻¹ A_i α, A_i = ∂K/∂θ_i or σn² I for the noise (whose second
// derivative is σn² I, and 0 mixed with a kernel parameter).
int orc_exact_hessian(const int32_t* nodes, int n_nodes, const double* params, int n_params, const double* x,
                      int64_t n, int d, const double* y, int jitter_kind, double jitter_initial, double jitter_mult,
                      int jitter_retries, double jitter_max, double* hess) {
  Tree t;
  const int nk = n_params - 1, np = n_params;
  if (!build_tree(t, nodes, n_nodes, params, nk)) return 3;
  const double noise = std::exp(params[nk]);
  Factor f;
  double last_j = 0.0;
  int st = factor_exact(t, x, n, d, y, noise,
                        retry_jitters(jitter_kind, jitter_initial, jitter_mult, jitter_retries, jitter_max),
                        f, &last_j);
  if (st != 0) return st;
  Mat kinv((size_t)n * n, 0.0);
  llt_inverse(f.l.data(), n, n, kinv.data(), n);
  // dK/dθ_i (full, one n×n per kernel parameter) and the second-order sum
  std::vector<Mat> da(np, Mat((size_t)n * n, 0.0));
  std::vector<double> sec((size_t)np * np, 0.0);
  std::vector<double> g, h;
  double kv;
  for (int64_t b = 0; b < n; ++b)
    for (int64_t a = b; a < n; ++a) {
      node_vgh(t, 0, x + a, n, x + b, n, d, kv, g, h);
      const double w = f.alpha[a] * f.alpha[b] - AT(kinv, n, a, b);
      const double cw = a == b ? w : 2.0 * w;
      for (int i = 0; i < nk; ++i) {
        AT(da[i], n, a, b) = AT(da[i], n, b, a) = g[i];
        for (int j = 0; j < nk; ++j) sec[(size_t)i * np + j] += cw * h[(size_t)i * nk + j];
      }
    }
  double trw = 0.0;
  for (int64_t a = 0; a < n; ++a) trw += f.alpha[a] * f.alpha[a] - AT(kinv, n, a, a);
  sec[(size_t)nk * np + nk] = noise * trw;
  for (int64_t a = 0; a < n; ++a) AT(da[nk], n, a, a) = noise;
  // S_i = L⁻¹ A_i L⁻ᵀ (two triangular solves) and v_i = L⁻¹ A_i α
  std::vector<Mat> sm(np);
  std::vector<std::vector<double>> vv(np, std::vector<double>(n, 0.0));
  for (int i = 0; i < np; ++i) {
    for (int64_t a = 0; a < n; ++a) {
      double acc = 0.0;
      for (int64_t b = 0; b < n; ++b) acc += AT(da[i], n, a, b) * f.alpha[b];
      vv[i][a] = acc;
    }
    trsm_lower(f.l.data(), n, n, vv[i].data(), 1, n);
    Mat m = da[i];
    trsm_lower(f.l.data(), n, n, m.data(), n, n);
    Mat mt((size_t)n * n);
    for (int64_t a = 0; a < n; ++a)
      for (int64_t b = 0; b < n; ++b) AT(mt, n, a, b) = AT(m, n, b, a);
    trsm_lower(f.l.data(), n, n, mt.data(), n, n);
    sm[i] = std::move(mt);
  }
  // upper triangle (i ≤ j), mirrored
  for (int i = 0; i < np; ++i)
    for (int j = i; j < np; ++j) {
      double fro = 0.0, vd = 0.0;
      for (size_t e = 0; e < (size_t)n * n; ++e) fro += sm[i][e] * sm[j][e];
      for (int64_t a = 0; a < n; ++a) vd += vv[i][a] * vv[j][a];
      hess[(size_t)i * np + j] = hess[(size_t)j * np + i] = -0.5 * sec[(size_t)i * np + j] - 0.5 * fro + vd;
    }
  return 0;
}

// Mean and the q×q query covariance K** − VᵀV, V = L⁻¹K* (GprCore::write_covariance,
// src/gpr/shared.rs:425-520): latent diagonal clipped at 0, observation adds σn².
static int exact_covariance(const Tree& t, double noise, const Factor& f, const double* x, int64_t n, int d,
                            const double* xs, int64_t q, int kind, double* mean, double* cov) {
  Mat ks((size_t)n * q);
#pragma omp parallel for schedule(static)
  for (int64_t c = 0; c < q; ++c)
    for (int64_t i = 0; i < n; ++i) AT(ks, n, i, c) = kval(t, x + i, n, xs + c, q, d);
  for (int64_t c = 0; c < q; ++c) {
    double m = 0.0;
    for (int64_t i = 0; i < n; ++i) m += AT(ks, n, i, c) * f.alpha[i];
    mean[c] = m;
  }
  trsm_lower(f.l.data(), n, n, ks.data(), q, n);
#pragma omp parallel for schedule(static)
  for (int64_t c = 0; c < q; ++c)
    for (int64_t r = 0; r < q; ++r) {
      double dot = 0.0;
      for (int64_t k = 0; k < n; ++k) dot += AT(ks, n, k, r) * AT(ks, n, k, c);
      cov[r + c * q] = kval(t, xs + r, q, xs + c, q, d) - dot;
    }
  for (int64_t i = 0; i < q; ++i) {
    double v = cov[i + i * q];
    if (v < 0.0) v = 0.0;
    cov[i + i * q] = kind == 1 ? v + noise : v;
  }
  return 0;
}

int orc_exact_covariance(const int32_t* nodes, int n_nodes, const double* params, int n_params, const double* x,
                         int64_t n, int d, const double* y, int jitter_kind, double jitter_initial,
                         double jitter_mult, int jitter_retries, double jitter_max, const double* xs, int64_t q,
                         int kind, double* mean, double* cov) {
  Tree t;
  int nk = n_params - 1;
  if (!build_tree(t, nodes, n_nodes, params, nk)) return 3;
  double noise = std::exp(params[nk]);
  Factor f;
  double last_j = 0.0;
  int st = factor_exact(t, x, n, d, y, noise,
                        retry_jitters(jitter_kind, jitter_initial, jitter_mult, jitter_retries, jitter_max),
                        f, &last_j);
  if (st != 0) return st;
  return exact_covariance(t, noise, f, x, n, d, xs, q, kind, mean, cov);
}

// μ + L z_k for n_draws seeded standard-normal vectors, L the LLT of cov
// with the jitter retries (FittedGpr::sample_with, src/prediction.rs:206-243;
// Box–Muller on the open-unit draws of the seeded Xoshiro256++, src/rng.rs:83-87).
static int draw_samples(const std::vector<double>& cov, const std::vector<double>& mean, int64_t q,
                        const std::vector<double>& jl, int64_t n_draws, uint64_t seed, double* out) {
  if (n_draws == 0) return 0;
  std::vector<double> js{0.0};
  js.insert(js.end(), jl.begin(), jl.end());
  Mat l((size_t)q * q);
  bool ok = false;
  for (double j : js) {
    l.assign(cov.begin(), cov.end());
    for (int64_t i = 0; i < q; ++i) AT(l, q, i, i) += j;
    if (potrf(l.data(), q, q)) {
      ok = true;
      break;
    }
  }
  if (!ok) return 1;
  Rng r;
  rng_seed(r, seed);
  auto unit = [&]() { return (double)(rng_next(r) >> 11) * (1.0 / 9007199254740992.0); };
  auto open_unit = [&]() {
    double u = unit();
    const double eps = 1.0 / 9007199254740992.0;
    return u <= eps ? eps : (u >= 1.0 - eps ? 1.0 - eps : u);
  };
  std::vector<double> z(q), lz(q);
  for (int64_t k = 0; k < n_draws; ++k) {
    for (int64_t i = 0; i < q; ++i) {
      double u1 = std::max(open_unit(), 2.2250738585072014e-308);
      double u2 = open_unit();
      z[i] = std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * M_PI * u2);
    }
    std::fill(lz.begin(), lz.end(), 0.0);
    for (int64_t j = 0; j < q; ++j)
      for (int64_t i = j; i < q; ++i) lz[i] += AT(l, q, i, j) * z[j];
    for (int64_t i = 0; i < q; ++i) out[k * q + i] = mean[i] + lz[i];
  }
  return 0;
}

// Posterior draws (PredictiveCovariance::draw, src/prediction.rs:206-243):
// LLT of the covariance retried with the jitter list (src/linalg/chol.rs:20-43),
// then column k = μ + L z_k, z_k the next q unit normals (src/rng.rs:72-87),
// L z summed column by column as mul_lower_vec (src/linalg/dense.rs:409-422).
int orc_exact_sample(const int32_t* nodes, int n_nodes, const double* params, int n_params, const double* x,
                     int64_t n, int d, const double* y, int jitter_kind, double jitter_initial, double jitter_mult,
                     int jitter_retries, double jitter_max, const double* xs, int64_t q, int kind, int64_t n_draws,
                     uint64_t seed, double* out) {
  Tree t;
  int nk = n_params - 1;
  if (!build_tree(t, nodes, n_nodes, params, nk)) return 3;
  double noise = std::exp(params[nk]);
  auto jl = retry_jitters(jitter_kind, jitter_initial, jitter_mult, jitter_retries, jitter_max);
  Factor f;
  double last_j = 0.0;
  int st = factor_exact(t, x, n, d, y, noise, jl, f, &last_j);
  if (st != 0) return st;
  std::vector<double> mean(q), cov((size_t)q * q);
  exact_covariance(t, noise, f, x, n, d, xs, q, kind, mean.data(), cov.data());
  return draw_samples(cov, mean, q, jl, n_draws, seed, out);
}

// ---------------------------------------------------------------------------
// Online exact GPR: LDLT store (src/gpr/factor_store.rs:100-260, src/linalg/ldlt.rs)
// ---------------------------------------------------------------------------
struct OrcOnline {
  Tree t;
  int d = 0;
  int64_t n = 0;
  double noise = 0.0, jitter = 0.0;
  std::vector<double> x;  // column-major n×d, rebuilt on each change
  std::vector<double> y;
  std::vector<std::vector<double>> rows;  // rows[i] = row i of unit L (length i) ; D separately
  std::vector<double> dg;
  std::vector<uint64_t> ids;
  uint64_t next_id = 0;
};

void* orc_online_create(const int32_t* nodes, int n_nodes, const double* params, int n_params,
                        const double* x, int64_t n, int d, const double* y) {
  OrcOnline* h = new OrcOnline;
  int nk = n_params - 1;
  if (!build_tree(h->t, nodes, n_nodes, params, nk)) { delete h; return nullptr; }
  h->noise = std::exp(params[nk]);
  h->d = d;
  Factor f;
  double lj = 0.0;
  if (factor_exact(h->t, x, n, d, y, h->noise, {}, f, &lj) != 0) { delete h; return nullptr; }
  h->n = n;
  h->x.assign(x, x + n * d);
  h->y.assign(y, y + n);
  // FittedGpr::into_online: D_j = L_jj², L_ij / L_jj (factor_store.rs:157-179)
  h->rows.resize(n);
  h->dg.resize(n);
  for (int64_t i = 0; i < n; ++i) {
    h->rows[i].resize(i);
    double lii = AT(f.l, n, i, i);
    h->dg[i] = lii * lii;
    for (int64_t j = 0; j < i; ++j) h->rows[i][j] = AT(f.l, n, i, j) / AT(f.l, n, j, j);
  }
  for (int64_t i = 0; i < n; ++i) h->ids.push_back(h->next_id++);
  return h;
}

void orc_online_destroy(void* p) { delete (OrcOnline*)p; }
int64_t orc_online_n(void* p) { return ((OrcOnline*)p)->n; }

// append_border (factor_store.rs:210-237): L w = k; v = D⁻¹ w; δ = k_new − Σ v² D.
int orc_online_insert(void* p, const double* xnew, double ynew, uint64_t* id) {
  OrcOnline* h = (OrcOnline*)p;
  int64_t n = h->n;
  int d = h->d;
  std::vector<double> k(n);
  for (int64_t i = 0; i < n; ++i) k[i] = kval(h->t, h->x.data() + i, n, xnew, 1, d);
  double knew = kval(h->t, xnew, 1, xnew, 1, d) + h->noise + h->jitter;
  for (int64_t i = 0; i < n; ++i) {
    double s = k[i];
    for (int64_t j = 0; j < i; ++j) s -= h->rows[i][j] * k[j];
    k[i] = s;
  }
  std::vector<double> v(n);
  double vtdv = 0.0;
  for (int64_t i = 0; i < n; ++i) {
    v[i] = k[i] / h->dg[i];
    vtdv += v[i] * v[i] * h->dg[i];
  }
  double delta = knew - vtdv;
  if (!(delta > 0.0) || !std::isfinite(delta)) return 1;
  h->rows.push_back(v);
  h->dg.push_back(delta);
  std::vector<double> nx((size_t)(n + 1) * d);
  for (int f = 0; f < d; ++f) {
    for (int64_t i = 0; i < n; ++i) nx[(size_t)f * (n + 1) + i] = h->x[(size_t)f * n + i];
    nx[(size_t)f * (n + 1) + n] = xnew[f];
  }
  h->x.swap(nx);
  h->y.push_back(ynew);
  h->n = n + 1;
  *id = h->next_id++;
  h->ids.push_back(*id);
  return 0;
}

// OnlineGpr::delete (online.rs:564-611); the LDLT row/column delete is the
// rank-1 update of the trailing block by D_k l_k l_kᵀ (Gill–Golub–Murray–
// Saunders C1), then the row/column is dropped.  Ids are compacted in order.
int orc_online_delete(void* p, uint64_t id) {
  OrcOnline* h = (OrcOnline*)p;
  int64_t n = h->n;
  if (n <= 1) return 5;
  int64_t idx = -1;
  for (int64_t i = 0; i < n; ++i)
    if (h->ids[i] == id) { idx = i; break; }
  if (idx < 0) return 4;
  int64_t m = n - idx - 1;
  std::vector<double> w(m);
  for (int64_t r = 0; r < m; ++r) w[r] = h->rows[idx + 1 + r][idx];
  double a = h->dg[idx];
  for (int64_t j = 0; j < m; ++j) {
    int64_t jj = idx + 1 + j;
    double pj = w[j];
    double dj = h->dg[jj];
    double dnew = dj + a * pj * pj;
    double beta = pj * a / dnew;
    a = dj * a / dnew;
    h->dg[jj] = dnew;
    for (int64_t r = j + 1; r < m; ++r) {
      int64_t rr = idx + 1 + r;
      w[r] -= pj * h->rows[rr][jj];
      h->rows[rr][jj] += beta * w[r];
    }
  }
  for (int64_t r = idx + 1; r < n; ++r) h->rows[r].erase(h->rows[r].begin() + idx);
  h->rows.erase(h->rows.begin() + idx);
  h->dg.erase(h->dg.begin() + idx);
  std::vector<double> nx((size_t)(n - 1) * h->d);
  for (int f = 0; f < h->d; ++f) {
    int64_t o = 0;
    for (int64_t i = 0; i < n; ++i)
      if (i != idx) nx[(size_t)f * (n - 1) + o++] = h->x[(size_t)f * n + i];
  }
  h->x.swap(nx);
  h->y.erase(h->y.begin() + idx);
  h->ids.erase(h->ids.begin() + idx);
  h->n = n - 1;
  return 0;
}

void orc_online_ids(void* p, uint64_t* out) {
  OrcOnline* h = (OrcOnline*)p;
  for (int64_t i = 0; i < h->n; ++i) out[i] = h->ids[i];
}

static void online_alpha(OrcOnline* h, std::vector<double>& a) {
  int64_t n = h->n;
  a = h->y;
  for (int64_t i = 0; i < n; ++i)
    for (int64_t j = 0; j < i; ++j) a[i] -= h->rows[i][j] * a[j];
  for (int64_t i = 0; i < n; ++i) a[i] /= h->dg[i];
  for (int64_t i = n - 1; i >= 0; --i)
    for (int64_t r = i + 1; r < n; ++r) a[i] -= h->rows[r][i] * a[r];
}

// NLML from LDLT: ½(yᵀα + Σ ln D + n ln 2π) (StoredFactor::log_det, shared.rs).
double orc_online_nlml(void* p) {
  OrcOnline* h = (OrcOnline*)p;
  std::vector<double> a;
  online_alpha(h, a);
  double quad = 0.0, ld = 0.0;
  for (int64_t i = 0; i < h->n; ++i) {
    quad += h->y[i] * a[i];
    ld += std::log(h->dg[i]);
  }
  return 0.5 * (quad + ld + (double)h->n * std::log(2.0 * M_PI));
}

void orc_online_predict(void* p, const double* xs, int64_t q, int kind, double* mean, double* var) {
  OrcOnline* h = (OrcOnline*)p;
  int64_t n = h->n;
  std::vector<double> a;
  online_alpha(h, a);
  std::vector<double> k(n);
  for (int64_t c = 0; c < q; ++c) {
    for (int64_t i = 0; i < n; ++i) k[i] = kval(h->t, h->x.data() + i, n, xs + c, q, h->d);
    double m = 0.0;
    for (int64_t i = 0; i < n; ++i) m += k[i] * a[i];
    mean[c] = m;
    for (int64_t i = 0; i < n; ++i)
      for (int64_t j = 0; j < i; ++j) k[i] -= h->rows[i][j] * k[j];
    double quad = 0.0;
    for (int64_t i = 0; i < n; ++i) quad += k[i] * k[i] / h->dg[i];
    double lat = kval(h->t, xs + c, q, xs + c, q, h->d) - quad;
    if (lat < 0.0) lat = 0.0;
    var[c] = kind == 1 ? lat + h->noise : lat;
  }
}

// D and unit-lower L as a dense n×n (L below the diagonal, D on it).
void orc_online_ld(void* p, double* out) {
  OrcOnline* h = (OrcOnline*)p;
  int64_t n = h->n;
  for (int64_t j = 0; j < n; ++j)
    for (int64_t i = 0; i < n; ++i)
      AT(out, n, i, j) = i == j ? h->dg[i] : (i > j ? h->rows[i][j] : 0.0);
}

// ---------------------------------------------------------------------------
// VFE sparse GPR (src/sgpr/factor/vfe.rs, derivatives.rs, predict.rs)
// ---------------------------------------------------------------------------
struct OrcSgpr {
  Tree t;
  int d = 0;
  int64_t n = 0, m = 0;
  double noise = 0.0;
  int jk = 1;
  double ji = 1e-8, jm = 10.0, jx = 1e-3;
  int jr = 5;
  std::vector<double> x, y, z;  // column-major
  std::vector<uint64_t> ids;
  uint64_t next_id = 0;
  // assembled state
  Mat lmm, a, bl;  // L (m×m), A (m×n), L_B (m×m)
  std::vector<double> w, ay;
  // Σ_c (k(x_c, x_c) − ‖a_c‖²), the trace term's numerator summed per point
  // (each term is the point's Nyström residual, ≥ 0); the reference computes
  // it as Σ k_ii − ‖A‖²_F (vfe.rs:338-369), the same sum in another
  // association, which loses digits to cancellation at large n.
  double trace_sum = 0.0, kmm_jitter = 0.0, pivot_ratio = 1.0;
  int last_in_place = 0;
};

static double sumsq_ld(const double* v, int64_t n) {
  long double s = 0.0L;
  for (int64_t i = 0; i < n; ++i) s += (long double)v[i] * v[i];
  return (double)s;
}

static double dot_ld(const double* a, const double* b, int64_t n) {
  long double s = 0.0L;
  for (int64_t i = 0; i < n; ++i) s += (long double)a[i] * b[i];
  return (double)s;
}

static double min_pivot_ratio(const Mat& l, int64_t m) {
  // min_pivot_ratio (src/sgpr/factor/updates.rs:414-427)
  double r = 1.0;
  for (int64_t i = 0; i < m; ++i) {
    double row2 = 0.0;
    for (int64_t k = 0; k <= i; ++k) row2 += AT(l, m, i, k) * AT(l, m, i, k);
    double piv = AT(l, m, i, i);
    double ratio = piv * piv / row2;
    if (!std::isfinite(ratio)) ratio = 0.0;
    r = std::min(r, ratio);
  }
  return r;
}

// assemble_vfe (vfe.rs:191-277)
static int sgpr_assemble(OrcSgpr* h) {
  int64_t n = h->n, m = h->m;
  int d = h->d;
  h->lmm.assign((size_t)m * m, 0.0);
  std::vector<double> jit;
  jit.push_back(0.0);
  auto rj = retry_jitters(h->jk, h->ji, h->jm, h->jr, h->jx);
  jit.insert(jit.end(), rj.begin(), rj.end());
  bool ok = false;
  for (double j : jit) {
    std::fill(h->lmm.begin(), h->lmm.end(), 0.0);
    if (!gram_lower(h->t, h->z.data(), m, d, h->lmm.data(), m)) return 2;
    if (j != 0.0)
      for (int64_t i = 0; i < m; ++i) AT(h->lmm, m, i, i) += j;
    if (potrf(h->lmm.data(), m, m)) { ok = true; h->kmm_jitter = j; break; }
  }
  if (!ok) return 1;
  h->pivot_ratio = min_pivot_ratio(h->lmm, m);
  h->a.assign((size_t)m * n, 0.0);
#pragma omp parallel for schedule(static)
  for (int64_t c = 0; c < n; ++c)
    for (int64_t i = 0; i < m; ++i) AT(h->a, m, i, c) = kval(h->t, h->z.data() + i, m, h->x.data() + c, n, d);
  trsm_lower(h->lmm.data(), m, m, h->a.data(), n, m);
  // B = A Aᵀ + σ² I (gram_aat_plus_noise, src/linalg/dense.rs:231-239)
  h->bl.assign((size_t)m * m, 0.0);
  gemm_abt_cols(h->a.data(), h->a.data(), m, n, h->bl.data(), m, true);
  for (int64_t i = 0; i < m; ++i) AT(h->bl, m, i, i) += h->noise;
  if (!potrf(h->bl.data(), m, m)) return 1;
  // Σ_c (k_cc − ‖a_c‖²) and A y, the long sums over n in long double
  long double tr = 0.0L;
  std::vector<long double> ay(m, 0.0L);
#pragma omp parallel
  {
    long double tr_t = 0.0L;
    std::vector<long double> ay_t(m, 0.0L);
#pragma omp for schedule(static)
    for (int64_t c = 0; c < n; ++c) {
      const double* ac = &AT(h->a, m, 0, c);
      long double ss = 0.0L;
      for (int64_t i = 0; i < m; ++i) {
        ss += (long double)ac[i] * ac[i];
        ay_t[i] += (long double)ac[i] * h->y[c];
      }
      tr_t += (long double)kval(h->t, h->x.data() + c, n, h->x.data() + c, n, d) - ss;
    }
#pragma omp critical
    {
      tr += tr_t;
      for (int64_t i = 0; i < m; ++i) ay[i] += ay_t[i];
    }
  }
  h->trace_sum = (double)tr;
  h->ay.assign(m, 0.0);
  for (int64_t i = 0; i < m; ++i) h->ay[i] = (double)ay[i];
  h->w = h->ay;
  llt_solve(h->bl.data(), m, m, h->w.data());
  return 0;
}

void* orc_sgpr_create(const int32_t* nodes, int n_nodes, const double* params, int n_params,
                      const double* x, int64_t n, int d, const double* y, const double* z, int64_t m,
                      int jitter_kind, double ji, double jm, int jr, double jx, int* status) {
  OrcSgpr* h = new OrcSgpr;
  int nk = n_params - 1;
  if (!build_tree(h->t, nodes, n_nodes, params, nk)) { *status = 3; delete h; return nullptr; }
  h->noise = std::exp(params[nk]);
  h->d = d;
  h->n = n;
  h->m = m;
  h->x.assign(x, x + n * d);
  h->y.assign(y, y + n);
  h->z.assign(z, z + m * d);
  h->jk = jitter_kind; h->ji = ji; h->jm = jm; h->jr = jr; h->jx = jx;
  for (int64_t i = 0; i < n; ++i) h->ids.push_back(h->next_id++);
  *status = sgpr_assemble(h);
  if (*status != 0) { delete h; return nullptr; }
  return h;
}

void orc_sgpr_destroy(void* p) { delete (OrcSgpr*)p; }
int64_t orc_sgpr_n(void* p) { return ((OrcSgpr*)p)->n; }
double orc_sgpr_kmm_jitter(void* p) { return ((OrcSgpr*)p)->kmm_jitter; }
int orc_sgpr_last_in_place(void* p) { return ((OrcSgpr*)p)->last_in_place; }

// vfe_neg_log_marginal_likelihood (vfe.rs:338-369)
double orc_sgpr_nlml(void* p) {
  OrcSgpr* h = (OrcSgpr*)p;
  int64_t n = h->n, m = h->m;
  double ldb = 0.0;
  for (int64_t i = 0; i < m; ++i) ldb += std::log(AT(h->bl, m, i, i));
  ldb *= 2.0;
  double logdet = ((double)n - (double)m) * std::log(h->noise) + ldb;
  double y2 = sumsq_ld(h->y.data(), n);
  double ayw = dot_ld(h->ay.data(), h->w.data(), m);
  double quad = (y2 - ayw) / h->noise;
  double trace = h->trace_sum / (2.0 * h->noise);
  return 0.5 * ((double)n * std::log(2.0 * M_PI) + logdet + quad) + trace;
}

// analytic_gradient with VfeEngine::adjoint (derivatives.rs:102-144, 186-202, 283-366).
void orc_sgpr_grad(void* p, double* grad) {
  OrcSgpr* h = (OrcSgpr*)p;
  int64_t n = h->n, m = h->m;
  int d = h->d;
  double noise = h->noise;
  // G = B⁻¹ A − (w rᵀ + A)/σ², r = y − Aᵀ w
  Mat g = h->a;
  trsm_lower(h->bl.data(), m, m, g.data(), n, m);
  trsm_lower_t(h->bl.data(), m, m, g.data(), n, m);
  std::vector<double> r(n);
#pragma omp parallel for schedule(static)
  for (int64_t c = 0; c < n; ++c) r[c] = h->y[c] - dot_ld(&AT(h->a, m, 0, c), h->w.data(), m);
  double inv = 1.0 / noise;
#pragma omp parallel for schedule(static)
  for (int64_t c = 0; c < n; ++c)
    for (int64_t i = 0; i < m; ++i) AT(g, m, i, c) -= (h->w[i] * r[c] + AT(h->a, m, i, c)) * inv;
  // H = G Aᵀ (m×m)
  Mat hh((size_t)m * m, 0.0);
  gemm_abt_cols(g.data(), h->a.data(), m, n, hh.data(), m, false);
  // w_mn = L⁻ᵀ G
  trsm_lower_t(h->lmm.data(), m, m, g.data(), n, m);
  // X = tril½(H); X ← L⁻ᵀ X; Xt = Xᵀ; Xt ← L⁻ᵀ Xt; w_mm = −½(Xt + Xtᵀ)
  Mat xm((size_t)m * m, 0.0);
  for (int64_t j = 0; j < m; ++j)
    for (int64_t i = j; i < m; ++i) AT(xm, m, i, j) = (i == j ? 0.5 : 1.0) * AT(hh, m, i, j);
  trsm_lower_t(h->lmm.data(), m, m, xm.data(), m, m);
  Mat xt((size_t)m * m);
  for (int64_t j = 0; j < m; ++j)
    for (int64_t i = 0; i < m; ++i) AT(xt, m, i, j) = AT(xm, m, j, i);
  trsm_lower_t(h->lmm.data(), m, m, xt.data(), m, m);
  Mat wmm((size_t)m * m);
  for (int64_t j = 0; j < m; ++j)
    for (int64_t i = 0; i < m; ++i) AT(wmm, m, i, j) = -0.5 * (AT(xt, m, j, i) + AT(xt, m, i, j));
  double wdiag = 0.5 * inv;
  int nk = h->t.n_params;
  std::vector<double> gk(nk, 0.0);
  // ⟨w_mm, ∂K_mm⟩ over the lower triangle with weights 1 / 2 (write_square_contraction)
  for (int64_t j = 0; j < m; ++j)
    for (int64_t i = j; i < m; ++i) {
      double s = (i == j ? 1.0 : 2.0) * AT(wmm, m, i, j);
      node_grad(h->t, 0, h->z.data() + i, m, h->z.data() + j, m, d, s, gk.data());
    }
  // ⟨w_mn, ∂K(Z, X)⟩ over the full rectangle (add_cross_contraction_mn) and
  // w_diag Σ ∂k(x_c, x_c) (add_diag_contraction): one column of sums per
  // point, the columns summed in long double
  std::vector<long double> gl(nk, 0.0L);
#pragma omp parallel
  {
    std::vector<long double> gt(nk, 0.0L);
    std::vector<double> gc(nk);
#pragma omp for schedule(static)
    for (int64_t c = 0; c < n; ++c) {
      std::fill(gc.begin(), gc.end(), 0.0);
      for (int64_t i = 0; i < m; ++i)
        node_grad(h->t, 0, h->z.data() + i, m, h->x.data() + c, n, d, AT(g, m, i, c), gc.data());
      node_grad(h->t, 0, h->x.data() + c, n, h->x.data() + c, n, d, wdiag, gc.data());
      for (int q = 0; q < nk; ++q) gt[q] += gc[q];
    }
#pragma omp critical
    for (int q = 0; q < nk; ++q) gl[q] += gt[q];
  }
  for (int q = 0; q < nk; ++q) grad[q] = (double)((long double)gk[q] + gl[q]);
  // directional_noise (derivatives.rs:186-202) with d_noise = σ²
  double y2 = sumsq_ld(h->y.data(), n);
  double ayw = dot_ld(h->ay.data(), h->w.data(), m);
  double quad = (y2 - ayw) / noise;
  double trace = h->trace_sum / (2.0 * noise);
  // trace_solve(L_B, σ² I) = σ² tr(B⁻¹)
  Mat binv((size_t)m * m, 0.0);
  llt_inverse(h->bl.data(), m, m, binv.data(), m);
  double trb = 0.0;
  for (int64_t i = 0; i < m; ++i) trb += AT(binv, m, i, i);
  double dn = noise;
  double d_logdet_b = dn * trb;
  double ww = sumsq_ld(h->w.data(), m);
  double d_q = -dn * ww;
  double d_quad = -d_q / noise - quad * dn / noise;
  double d_trace = -trace * dn / noise;
  double nm = (double)n - (double)m;
  grad[nk] = 0.5 * (nm * dn / noise + d_logdet_b + d_quad) + d_trace;
}

// vfe_latent (predict.rs:197-262)
void orc_sgpr_predict(void* p, const double* xs, int64_t q, int kind, double* mean, double* var) {
  OrcSgpr* h = (OrcSgpr*)p;
  int64_t m = h->m;
  int d = h->d;
  Mat as((size_t)m * q);
  for (int64_t c = 0; c < q; ++c)
    for (int64_t i = 0; i < m; ++i) AT(as, m, i, c) = kval(h->t, h->z.data() + i, m, xs + c, q, d);
  trsm_lower(h->lmm.data(), m, m, as.data(), q, m);
  Mat bs = as;
  trsm_lower(h->bl.data(), m, m, bs.data(), q, m);
  for (int64_t c = 0; c < q; ++c) {
    double an = 0.0, bn = 0.0, mu = 0.0;
    for (int64_t i = 0; i < m; ++i) {
      an += AT(as, m, i, c) * AT(as, m, i, c);
      bn += AT(bs, m, i, c) * AT(bs, m, i, c);
      mu += AT(as, m, i, c) * h->w[i];
    }
    double lat = kval(h->t, xs + c, q, xs + c, q, d) - an + h->noise * bn;
    if (lat < 0.0) lat = 0.0;
    mean[c] = mu;
    var[c] = kind == 1 ? lat + h->noise : lat;
  }
}

// Query covariance of the VFE posterior (predict_vfe_covariance,
// src/sgpr/factor/predict.rs:263-345; SparseCore::finish_covariance,
// src/sparse/core.rs:641-667): off the diagonal K** − A*ᵀA* + σn² S*ᵀS*
// with A* = L_mm⁻¹ K_m*, S* = L_B⁻¹ A*; on it the predictive variance.
static void sgpr_covariance(OrcSgpr* h, const double* xs, int64_t q, int kind, double* mean, double* cov) {
  int64_t m = h->m;
  int d = h->d;
  std::vector<double> var(q);
  orc_sgpr_predict(h, xs, q, kind, mean, var.data());
  Mat as((size_t)m * q);
  for (int64_t c = 0; c < q; ++c)
    for (int64_t i = 0; i < m; ++i) AT(as, m, i, c) = kval(h->t, h->z.data() + i, m, xs + c, q, d);
  trsm_lower(h->lmm.data(), m, m, as.data(), q, m);
  Mat bs = as;
  trsm_lower(h->bl.data(), m, m, bs.data(), q, m);
  for (int64_t c = 0; c < q; ++c)
    for (int64_t r = 0; r < q; ++r) {
      if (r == c) {
        cov[r + c * q] = var[r];
        continue;
      }
      double ad = 0.0, sd = 0.0;
      for (int64_t k = 0; k < m; ++k) {
        ad += AT(as, m, k, r) * AT(as, m, k, c);
        sd += AT(bs, m, k, r) * AT(bs, m, k, c);
      }
      cov[r + c * q] = kval(h->t, xs + r, q, xs + c, q, d) - ad + h->noise * sd;
    }
}

void orc_sgpr_covariance(void* p, const double* xs, int64_t q, int kind, double* mean, double* cov) {
  sgpr_covariance((OrcSgpr*)p, xs, q, kind, mean, cov);
}

// FittedSgpr::sample_with (src/sgpr/fitted.rs:855-900): the exact model's
// draw from the VFE covariance, with the model's jitter retries.
int orc_sgpr_sample(void* p, const double* xs, int64_t q, int kind, int64_t n_draws, uint64_t seed, double* out) {
  OrcSgpr* h = (OrcSgpr*)p;
  std::vector<double> mean(q), cov((size_t)q * q);
  sgpr_covariance(h, xs, q, kind, mean.data(), cov.data());
  return draw_samples(cov, mean, q, retry_jitters(h->jk, h->ji, h->jm, h->jr, h->jx), n_draws, seed, out);
}

static void sgpr_set_points(OrcSgpr* h, std::vector<double>& nx, std::vector<double>& ny, int64_t n) {
  h->x.swap(nx);
  h->y.swap(ny);
  h->n = n;
}

// OnlineSgpr::insert → append_point (online/mod.rs:1695-1810); chol_rank1_update (chol.rs:450-466)
int orc_sgpr_insert(void* p, const double* xnew, double ynew, uint64_t* id) {
  OrcSgpr* h = (OrcSgpr*)p;
  int64_t n = h->n, m = h->m;
  int d = h->d;
  std::vector<double> nx((size_t)(n + 1) * d);
  for (int f = 0; f < d; ++f) {
    for (int64_t i = 0; i < n; ++i) nx[(size_t)f * (n + 1) + i] = h->x[(size_t)f * n + i];
    nx[(size_t)f * (n + 1) + n] = xnew[f];
  }
  std::vector<double> ny = h->y;
  ny.push_back(ynew);
  *id = h->next_id++;
  h->ids.push_back(*id);
  if (!(h->pivot_ratio > 8.0 * 2.220446049250313e-16)) {
    sgpr_set_points(h, nx, ny, n + 1);
    h->last_in_place = 0;
    return sgpr_assemble(h);
  }
  std::vector<double> v(m);
  for (int64_t i = 0; i < m; ++i) v[i] = kval(h->t, h->z.data() + i, m, xnew, 1, d);
  trsm_lower(h->lmm.data(), m, m, v.data(), 1, m);
  double kd = kval(h->t, xnew, 1, xnew, 1, d);
  h->trace_sum += (double)((long double)kd - (long double)sumsq_ld(v.data(), m));
  for (int64_t i = 0; i < m; ++i) h->ay[i] += v[i] * ynew;
  Mat na((size_t)m * (n + 1));
  std::copy(h->a.begin(), h->a.end(), na.begin());
  for (int64_t i = 0; i < m; ++i) AT(na, m, i, n) = v[i];
  h->a.swap(na);
  // rank-1 update of L_B
  for (int64_t k = 0; k < m; ++k) {
    double lkk = AT(h->bl, m, k, k), vk = v[k];
    double r = std::sqrt(lkk * lkk + vk * vk);
    double c = r / lkk, s = vk / lkk;
    AT(h->bl, m, k, k) = r;
    for (int64_t i = k + 1; i < m; ++i) {
      double li = AT(h->bl, m, i, k), vi = v[i];
      AT(h->bl, m, i, k) = (li + s * vi) / c;
      v[i] = c * vi - s * AT(h->bl, m, i, k);
    }
  }
  sgpr_set_points(h, nx, ny, n + 1);
  h->w = h->ay;
  llt_solve(h->bl.data(), m, m, h->w.data());
  h->last_in_place = 1;
  return 0;
}

// OnlineSgpr::delete (online/mod.rs:903-1000); chol_rank1_downdate (chol.rs:468-493)
int orc_sgpr_delete(void* p, uint64_t id) {
  OrcSgpr* h = (OrcSgpr*)p;
  int64_t n = h->n, m = h->m;
  int d = h->d;
  if (n <= 1) return 5;
  int64_t idx = -1;
  for (int64_t i = 0; i < n; ++i)
    if (h->ids[i] == id) { idx = i; break; }
  if (idx < 0) return 4;
  std::vector<double> v(m);
  for (int64_t i = 0; i < m; ++i) v[i] = AT(h->a, m, i, idx);
  const double* xp_base = h->x.data() + idx;
  double kd = kval(h->t, xp_base, n, xp_base, n, d);
  double coln = sumsq_ld(v.data(), m);
  std::vector<double> nx((size_t)(n - 1) * d);
  for (int f = 0; f < d; ++f) {
    int64_t o = 0;
    for (int64_t i = 0; i < n; ++i)
      if (i != idx) nx[(size_t)f * (n - 1) + o++] = h->x[(size_t)f * n + i];
  }
  std::vector<double> ny = h->y;
  ny.erase(ny.begin() + idx);
  Mat trial = h->bl;
  std::vector<double> vt = v;
  bool ok = h->pivot_ratio > 8.0 * 2.220446049250313e-16;
  if (ok) {
    for (int64_t k = 0; k < m && ok; ++k) {
      double lkk = AT(trial, m, k, k), vk = vt[k];
      double r2 = lkk * lkk - vk * vk;
      if (r2 <= 0.0 || !std::isfinite(r2)) { ok = false; break; }
      double r = std::sqrt(r2);
      double c = r / lkk, s = vk / lkk;
      AT(trial, m, k, k) = r;
      for (int64_t i = k + 1; i < m; ++i) {
        double li = AT(trial, m, i, k), vi = vt[i];
        AT(trial, m, i, k) = (li - s * vi) / c;
        vt[i] = c * vi - s * AT(trial, m, i, k);
      }
    }
  }
  double yi = h->y[idx];
  h->ids.erase(h->ids.begin() + idx);
  if (ok) {
    h->trace_sum -= (double)((long double)kd - (long double)coln);
    for (int64_t i = 0; i < m; ++i) h->ay[i] -= v[i] * yi;
    Mat na((size_t)m * (n - 1));
    int64_t o = 0;
    for (int64_t c = 0; c < n; ++c) {
      if (c == idx) continue;
      for (int64_t i = 0; i < m; ++i) AT(na, m, i, o) = AT(h->a, m, i, c);
      ++o;
    }
    h->a.swap(na);
    h->bl.swap(trial);
    sgpr_set_points(h, nx, ny, n - 1);
    h->w = h->ay;
    llt_solve(h->bl.data(), m, m, h->w.data());
    h->last_in_place = 1;
    return 0;
  }
  sgpr_set_points(h, nx, ny, n - 1);
  h->last_in_place = 0;
  return sgpr_assemble(h);
}

// OnlineSgpr::insert_inducing (src/sgpr/online/mod.rs:1943-1992,1154-1220;
// inducing_append, src/sgpr/factor/updates.rs:296-390): from a factor of
// K_mm without jitter whose pivots hold (min L_ii²/K_ii > 1e-5), the bordered
// LLT of K_mm and B and the new row of A, a_new = (k(z, X) − lᵀA)/ℓ; when a
// bordered pivot is at most 1e-5 of its diagonal, or the factor's gate does
// not hold, the VFE system of the new set is assembled.  last_in_place
// tells which.
int orc_sgpr_insert_inducing(void* p, const double* znew) {
  OrcSgpr* h = (OrcSgpr*)p;
  const int64_t n = h->n, m = h->m;
  const int d = h->d;
  const double tau = 1e-5;
  std::vector<double> nz((size_t)(m + 1) * d);
  for (int f = 0; f < d; ++f) {
    for (int64_t i = 0; i < m; ++i) nz[(size_t)f * (m + 1) + i] = h->z[(size_t)f * m + i];
    nz[(size_t)f * (m + 1) + m] = znew[f];
  }
  bool ok = h->kmm_jitter <= 0.0 && h->pivot_ratio > tau;
  std::vector<double> l(m), a_new(n), b(m);
  double ell = 0.0, beta = 0.0;
  long double an2 = 0.0L;
  if (ok) {
    for (int64_t i = 0; i < m; ++i) l[i] = kval(h->t, h->z.data() + i, m, znew, 1, d);
    trsm_lower(h->lmm.data(), m, m, l.data(), 1, m);
    const double kdiag = kval(h->t, znew, 1, znew, 1, d) + h->kmm_jitter;
    double ell2 = kdiag - sumsq_ld(l.data(), m);
    ok = std::isfinite(ell2) && ell2 > tau * kdiag;
    if (ok) {
      ell = std::sqrt(ell2);
#pragma omp parallel for schedule(static)
      for (int64_t c = 0; c < n; ++c)
        a_new[c] = (kval(h->t, znew, 1, h->x.data() + c, n, d) - dot_ld(l.data(), &AT(h->a, m, 0, c), m)) / ell;
      for (int64_t c = 0; c < n; ++c) an2 += (long double)a_new[c] * a_new[c];
      std::vector<long double> v(m, 0.0L);
#pragma omp parallel
      {
        std::vector<long double> vt(m, 0.0L);
#pragma omp for schedule(static)
        for (int64_t c = 0; c < n; ++c)
          for (int64_t i = 0; i < m; ++i) vt[i] += (long double)AT(h->a, m, i, c) * a_new[c];
#pragma omp critical
        for (int64_t i = 0; i < m; ++i) v[i] += vt[i];
      }
      for (int64_t i = 0; i < m; ++i) b[i] = (double)v[i];
      trsm_lower(h->bl.data(), m, m, b.data(), 1, m);
      const double bdiag = h->noise + (double)an2;
      const double beta2 = bdiag - sumsq_ld(b.data(), m);
      ok = std::isfinite(beta2) && beta2 > tau * bdiag;
      beta = ok ? std::sqrt(beta2) : 0.0;
    }
  }
  if (!ok) {
    h->z.swap(nz);
    h->m = m + 1;
    h->last_in_place = 0;
    return sgpr_assemble(h);
  }
  const int64_t m1 = m + 1;
  Mat nl((size_t)m1 * m1, 0.0), nb((size_t)m1 * m1, 0.0), na((size_t)m1 * n);
  for (int64_t j = 0; j < m; ++j)
    for (int64_t i = j; i < m; ++i) {
      AT(nl, m1, i, j) = AT(h->lmm, m, i, j);
      AT(nb, m1, i, j) = AT(h->bl, m, i, j);
    }
  for (int64_t j = 0; j < m; ++j) {
    AT(nl, m1, m, j) = l[j];
    AT(nb, m1, m, j) = b[j];
  }
  AT(nl, m1, m, m) = ell;
  AT(nb, m1, m, m) = beta;
  for (int64_t c = 0; c < n; ++c) {
    for (int64_t i = 0; i < m; ++i) AT(na, m1, i, c) = AT(h->a, m, i, c);
    AT(na, m1, m, c) = a_new[c];
  }
  h->lmm.swap(nl);
  h->bl.swap(nb);
  h->a.swap(na);
  h->z.swap(nz);
  h->m = m1;
  h->trace_sum -= (double)an2;
  // A y and w from the new A and L_B (refresh_w)
  std::vector<long double> ay(m1, 0.0L);
  for (int64_t c = 0; c < n; ++c)
    for (int64_t i = 0; i < m1; ++i) ay[i] += (long double)AT(h->a, m1, i, c) * h->y[c];
  h->ay.assign(m1, 0.0);
  for (int64_t i = 0; i < m1; ++i) h->ay[i] = (double)ay[i];
  h->w = h->ay;
  llt_solve(h->bl.data(), m1, m1, h->w.data());
  h->pivot_ratio = min_pivot_ratio(h->lmm, m1);
  h->last_in_place = 1;
  return 0;
}

// Replaces the inducing set (an inducing insert/delete taken by reassembly).
int orc_sgpr_set_inducing(void* p, const double* z, int64_t m) {
  OrcSgpr* h = (OrcSgpr*)p;
  h->last_in_place = 0;
  h->z.assign(z, z + m * h->d);
  h->m = m;
  return sgpr_assemble(h);
}

// ---------------------------------------------------------------------------
// RNG (src/rng.rs)
// ---------------------------------------------------------------------------
void orc_rng_seed(uint64_t* state, uint64_t seed) {
  Rng r;
  rng_seed(r, seed);
  std::memcpy(state, r.s, sizeof r.s);
}
uint64_t orc_rng_next(uint64_t* state) {
  Rng r;
  std::memcpy(r.s, state, sizeof r.s);
  uint64_t v = rng_next(r);
  std::memcpy(state, r.s, sizeof r.s);
  return v;
}

}  // extern "C"
