// kernels.cu — KernelSpec trees on the device: lower Gram fill, cross fill
// and the fused W = ααᵀ − K⁻¹ gradient contraction.
//
// Reference: CompiledKernel::eval_gram / eval_cross_slots (gprx
// src/kernel/compiled/gram.rs:103,203), the leaf formulas of
// src/kernel/{rbf.rs:18, rbf_ard.rs:16, constant.rs:12, periodic.rs:598-638},
// and the weighted-gradient walk (src/kernel/compiled/weighted.rs:274-345,
// src/gpr/exact_fit.rs:665-729).  The tree is expanded on the host into a sum
// of products of leaves so that the device code indexes registers statically.

#include <cmath>
#include <string>

#include "kernels.cuh"

namespace gprx {

// ---------------------------------------------------------------------------
// host: tree parsing and expansion
// ---------------------------------------------------------------------------
namespace {
struct Parsed {
  std::vector<std::vector<int>> terms;  // each term: leaf indices
};

bool expand(const std::vector<gprx_kernel_node>& nodes, int& at, std::vector<int>& leaf_kind,
            std::vector<int>& leaf_arg, std::vector<int>& leaf_param, int& n_params, Parsed& out,
            std::string* why) {
  if (at >= (int)nodes.size()) {
    if (why) *why = "kernel node list ends inside a SUM/PRODUCT";
    return false;
  }
  gprx_kernel_node nd = nodes[at++];
  if (nd.kind == GPRX_NODE_SUM || nd.kind == GPRX_NODE_PRODUCT) {
    if (nd.arg < 1) {
      if (why) *why = "SUM/PRODUCT node needs at least one child";
      return false;
    }
    std::vector<std::vector<int>> acc;
    for (int c = 0; c < nd.arg; ++c) {
      Parsed child;
      if (!expand(nodes, at, leaf_kind, leaf_arg, leaf_param, n_params, child, why)) return false;
      if (nd.kind == GPRX_NODE_SUM) {
        acc.insert(acc.end(), child.terms.begin(), child.terms.end());
      } else if (c == 0) {
        acc = child.terms;
      } else {
        std::vector<std::vector<int>> prod;
        for (auto& a : acc)
          for (auto& b : child.terms) {
            std::vector<int> t = a;
            t.insert(t.end(), b.begin(), b.end());
            prod.push_back(t);
          }
        acc.swap(prod);
      }
    }
    out.terms = acc;
    return true;
  }
  int np;
  switch (nd.kind) {
    case GPRX_LEAF_RBF: np = 1; break;
    case GPRX_LEAF_CONSTANT: np = 1; break;
    case GPRX_LEAF_PERIODIC: np = 2; break;
    case GPRX_LEAF_RBF_ARD: np = nd.arg; break;
    default:
      if (why) *why = "unknown kernel node kind " + std::to_string(nd.kind);
      return false;
  }
  int idx = (int)leaf_kind.size();
  leaf_kind.push_back(nd.kind);
  leaf_arg.push_back(nd.arg);
  leaf_param.push_back(n_params);
  n_params += np;
  out.terms = {{idx}};
  return true;
}
}  // namespace

gprx_status HostKernel::init(const gprx_kernel_node* ns, int n_nodes, const double* th, int n_theta, int dim,
                             std::string* why) {
  if (!ns || n_nodes <= 0 || n_nodes > GPRX_MAX_NODES) {
    if (why) *why = "kernel must have 1.." + std::to_string(GPRX_MAX_NODES) + " nodes";
    return GPRX_INVALID_CONFIG;
  }
  nodes.assign(ns, ns + n_nodes);
  std::vector<int> kind, arg, param;
  int np = 0, at = 0;
  Parsed p;
  if (!expand(nodes, at, kind, arg, param, np, p, why)) return GPRX_INVALID_CONFIG;
  if (at != n_nodes) {
    if (why) *why = "kernel node list has trailing nodes";
    return GPRX_INVALID_CONFIG;
  }
  if (np != n_theta) {
    if (why) *why = "kernel has " + std::to_string(np) + " parameters, got " + std::to_string(n_theta);
    return GPRX_SHAPE_MISMATCH;
  }
  if ((int)kind.size() > KT_MAX_LEAVES || (int)p.terms.size() > KT_MAX_TERMS || np > GPRX_MAX_PARAMS) {
    if (why) *why = "kernel tree too large for the device evaluator";
    return GPRX_INVALID_CONFIG;
  }
  if (dim < 1 || dim > GPRX_MAX_DIM) {
    if (why) *why = "d must be in 1.." + std::to_string(GPRX_MAX_DIM);
    return GPRX_SHAPE_MISMATCH;
  }
  d = dim;
  n_params = np;
  tree = KTree{};
  tree.n_leaves = (int)kind.size();
  tree.n_terms = (int)p.terms.size();
  tree.n_params = np;
  tree.d = dim;
  tree.ard_leaf = -1;
  tree.ard_param = -1;
  for (size_t t = 0; t < p.terms.size(); ++t) {
    unsigned mask = 0;
    for (int l : p.terms[t]) {
      if (mask & (1u << l)) {
        if (why) *why = "a product repeats a leaf";
        return GPRX_INVALID_CONFIG;
      }
      mask |= 1u << l;
    }
    tree.term_mask[t] = mask;
  }
  for (size_t l = 0; l < kind.size(); ++l) {
    tree.leaf[l].kind = kind[l];
    tree.leaf[l].param = param[l];
    if (kind[l] == GPRX_LEAF_RBF_ARD) {
      if (tree.ard_leaf >= 0) {
        if (why) *why = "at most one RBF_ARD leaf is supported";
        return GPRX_INVALID_CONFIG;
      }
      if (arg[l] != dim) {
        if (why) *why = "RBF_ARD dimension does not match d";
        return GPRX_SHAPE_MISMATCH;
      }
      tree.ard_leaf = (int)l;
      tree.ard_param = param[l];
    }
  }
  ard_d = 0;
  if (tree.ard_leaf >= 0) ard_d = dim <= 4 ? 4 : dim <= 8 ? 8 : dim <= 16 ? 16 : 32;
  int ns_total = grad_slots(ard_d);
  slot_param.assign(ns_total, -1);
  for (int l = 0; l < tree.n_leaves; ++l) {
    int k = tree.leaf[l].kind;
    if (k == GPRX_LEAF_RBF || k == GPRX_LEAF_CONSTANT) slot_param[2 * l] = tree.leaf[l].param;
    if (k == GPRX_LEAF_PERIODIC) {
      slot_param[2 * l] = tree.leaf[l].param;
      slot_param[2 * l + 1] = tree.leaf[l].param + 1;
    }
  }
  if (tree.ard_leaf >= 0)
    for (int f = 0; f < dim; ++f) slot_param[GRAD_SLOTS_LEAF + f] = tree.ard_param + f;
  theta.assign(th, th + n_theta);
  return set_theta(th);
}

gprx_status HostKernel::set_theta(const double* th) {
  for (int i = 0; i < n_params; ++i)
    if (!std::isfinite(th[i])) return GPRX_INVALID_HYPERPARAMETER;
  theta.assign(th, th + n_params);
  return (gprx_status)kt_set_theta(tree, theta.data());
}

// ---------------------------------------------------------------------------
// device: fills
// ---------------------------------------------------------------------------
constexpr int FT = 64;           // fill / contraction tile
constexpr int FILL_THREADS = 256;

__device__ __forceinline__ void lower_tile_of(long long idx, int& ti, int& tj) {
  // idx enumerates (ti, tj) with tj ≤ ti row by row: idx = ti(ti+1)/2 + tj
  double r = floor((sqrt(8.0 * (double)idx + 1.0) - 1.0) * 0.5);
  long long t = (long long)r;
  while ((t + 1) * (t + 2) / 2 <= idx) ++t;
  while (t * (t + 1) / 2 > idx) --t;
  ti = (int)t;
  tj = (int)(idx - t * (t + 1) / 2);
}

template <int ARD_D>
__device__ __forceinline__ double pair_value(const KTree& t, const double* xi, const double* xj, int d) {
  double dx[ARD_D > 0 ? ARD_D : 1];
  double r2 = 0.0;
  for (int f = 0; f < d; ++f) {
    double v = xi[f * FT] - xj[f * FT];
    r2 = fma(v, v, r2);
    if (ARD_D > 0) {
#pragma unroll
      for (int g = 0; g < (ARD_D > 0 ? ARD_D : 1); ++g)
        if (g == f) dx[g] = v;
    }
  }
  return kt_value<ARD_D>(t, dx, r2);
}

template <int ARD_D>
__global__ void __launch_bounds__(FILL_THREADS) fill_lower_kernel(KTree t, const double* x, long long ldx, int n,
                                                                  double* K, long long ld, double diag_add,
                                                                  DevStatus* st) {
  __shared__ double xi[GPRX_MAX_DIM * FT];
  __shared__ double xj[GPRX_MAX_DIM * FT];
  if (dev_failed(st)) return;
  const int d = t.d;
  const int nt = (n + FT - 1) / FT;
  const long long ntiles = (long long)nt * (nt + 1) / 2;
  bool bad = false;
  for (long long idx = blockIdx.x; idx < ntiles; idx += gridDim.x) {
    int ti, tj;
    lower_tile_of(idx, ti, tj);
    const int i0 = ti * FT, j0 = tj * FT;
    __syncthreads();
    for (int e = threadIdx.x; e < d * FT; e += blockDim.x) {
      int r = e % FT, f = e / FT;
      xi[f * FT + r] = (i0 + r < n) ? x[(i0 + r) + (long long)f * ldx] : 0.0;
      xj[f * FT + r] = (j0 + r < n) ? x[(j0 + r) + (long long)f * ldx] : 0.0;
    }
    __syncthreads();
    const int r = threadIdx.x % FT;
    const int i = i0 + r;
    for (int c = threadIdx.x / FT; c < FT; c += FILL_THREADS / FT) {
      int j = j0 + c;
      if (i >= n || j >= n || i < j) continue;
      double v = pair_value<ARD_D>(t, xi + r, xj + c, d);
      if (i == j) v += diag_add;
      if (!isfinite(v)) bad = true;
      K[i + (long long)j * ld] = v;
    }
  }
  if (bad) dev_fail(st, GPRX_NONFINITE_KERNEL, 0);
}

// The lower fill for trees of at most NL leaves, PW pairs per thread
// (independent FP64 chains); every value is computed as in fill_lower_kernel.
template <int ARD_D, int NL, int PW>
__global__ void __launch_bounds__(FILL_THREADS) fill_lower_w_kernel(KTree t, const double* x, long long ldx, int n,
                                                                    double* K, long long ld, double diag_add,
                                                                    DevStatus* st) {
  constexpr int AD = ARD_D > 0 ? ARD_D : 1;
  constexpr int CS = FILL_THREADS / FT;
  static_assert((FT / CS) % PW == 0, "pairs per thread");
  __shared__ double xi[GPRX_MAX_DIM * FT];
  __shared__ double xj[GPRX_MAX_DIM * FT];
  if (dev_failed(st)) return;
  const int d = t.d;
  const int nt = (n + FT - 1) / FT;
  const long long ntiles = (long long)nt * (nt + 1) / 2;
  bool bad = false;
  for (long long idx = blockIdx.x; idx < ntiles; idx += gridDim.x) {
    int ti, tj;
    lower_tile_of(idx, ti, tj);
    const int i0 = ti * FT, j0 = tj * FT;
    __syncthreads();
    for (int e = threadIdx.x; e < d * FT; e += blockDim.x) {
      int r = e % FT, f = e / FT;
      xi[f * FT + r] = (i0 + r < n) ? x[(i0 + r) + (long long)f * ldx] : 0.0;
      xj[f * FT + r] = (j0 + r < n) ? x[(j0 + r) + (long long)f * ldx] : 0.0;
    }
    __syncthreads();
    const int r = threadIdx.x % FT;
    const int i = i0 + r;
    if (i >= n) continue;
#pragma unroll 1
    for (int c0 = threadIdx.x / FT; c0 < FT; c0 += CS * PW) {
      if (j0 + c0 > i) break;  // every later pair of this thread lies above the diagonal
      double dx[PW][AD], r2[PW], kv[PW];
#pragma unroll
      for (int w = 0; w < PW; ++w) {
        const int c = c0 + w * CS;
        double rr = 0.0;
        for (int f = 0; f < d; ++f) {
          const double v = xi[f * FT + r] - xj[f * FT + c];
          rr = fma(v, v, rr);
          if (ARD_D > 0) {
#pragma unroll
            for (int g = 0; g < AD; ++g)
              if (g == f) dx[w][g] = v;
          }
        }
        r2[w] = rr;
      }
      kt_value_w<ARD_D, PW, NL>(t, dx, r2, kv);
#pragma unroll
      for (int w = 0; w < PW; ++w) {
        const int j = j0 + c0 + w * CS;
        if (j >= n || i < j) continue;
        double v = kv[w];
        if (i == j) v += diag_add;
        if (!isfinite(v)) bad = true;
        K[i + (long long)j * ld] = v;
      }
    }
  }
  if (bad) dev_fail(st, GPRX_NONFINITE_KERNEL, 0);
}

template <int ARD_D>
__global__ void __launch_bounds__(FILL_THREADS) fill_cross_kernel(KTree t, const double* x1, long long ldx1, int n1,
                                                                  const double* x2, long long ldx2, int n2,
                                                                  double* out, long long ld, DevStatus* st) {
  __shared__ double xi[GPRX_MAX_DIM * FT];
  __shared__ double xj[GPRX_MAX_DIM * FT];
  if (dev_failed(st)) return;
  const int d = t.d;
  const int tm = (n1 + FT - 1) / FT, tn = (n2 + FT - 1) / FT;
  const long long ntiles = (long long)tm * tn;
  bool bad = false;
  for (long long idx = blockIdx.x; idx < ntiles; idx += gridDim.x) {
    const int i0 = (int)(idx % tm) * FT, j0 = (int)(idx / tm) * FT;
    __syncthreads();
    for (int e = threadIdx.x; e < d * FT; e += blockDim.x) {
      int r = e % FT, f = e / FT;
      xi[f * FT + r] = (i0 + r < n1) ? x1[(i0 + r) + (long long)f * ldx1] : 0.0;
      xj[f * FT + r] = (j0 + r < n2) ? x2[(j0 + r) + (long long)f * ldx2] : 0.0;
    }
    __syncthreads();
    const int r = threadIdx.x % FT;
    const int i = i0 + r;
    for (int c = threadIdx.x / FT; c < FT; c += FILL_THREADS / FT) {
      int j = j0 + c;
      if (i >= n1 || j >= n2) continue;
      double v = pair_value<ARD_D>(t, xi + r, xj + c, d);
      if (!isfinite(v)) bad = true;
      out[i + (long long)j * ld] = v;
    }
  }
  if (bad) dev_fail(st, GPRX_NONFINITE_KERNEL, 0);
}

// The cross fill for trees of at most NL leaves, PW pairs per thread; every
// value is computed as in fill_cross_kernel.
template <int ARD_D, int NL, int PW>
__global__ void __launch_bounds__(FILL_THREADS) fill_cross_w_kernel(KTree t, const double* x1, long long ldx1,
                                                                    int n1, const double* x2, long long ldx2, int n2,
                                                                    double* out, long long ld, DevStatus* st) {
  constexpr int AD = ARD_D > 0 ? ARD_D : 1;
  constexpr int CS = FILL_THREADS / FT;
  static_assert((FT / CS) % PW == 0, "pairs per thread");
  __shared__ double xi[GPRX_MAX_DIM * FT];
  __shared__ double xj[GPRX_MAX_DIM * FT];
  if (dev_failed(st)) return;
  const int d = t.d;
  const int tm = (n1 + FT - 1) / FT, tn = (n2 + FT - 1) / FT;
  const long long ntiles = (long long)tm * tn;
  bool bad = false;
  for (long long idx = blockIdx.x; idx < ntiles; idx += gridDim.x) {
    const int i0 = (int)(idx % tm) * FT, j0 = (int)(idx / tm) * FT;
    __syncthreads();
    for (int e = threadIdx.x; e < d * FT; e += blockDim.x) {
      int r = e % FT, f = e / FT;
      xi[f * FT + r] = (i0 + r < n1) ? x1[(i0 + r) + (long long)f * ldx1] : 0.0;
      xj[f * FT + r] = (j0 + r < n2) ? x2[(j0 + r) + (long long)f * ldx2] : 0.0;
    }
    __syncthreads();
    const int r = threadIdx.x % FT;
    const int i = i0 + r;
    if (i >= n1) continue;
#pragma unroll 1
    for (int c0 = threadIdx.x / FT; c0 < FT; c0 += CS * PW) {
      if (j0 + c0 >= n2) break;
      double dx[PW][AD], r2[PW], kv[PW];
#pragma unroll
      for (int w = 0; w < PW; ++w) {
        const int c = c0 + w * CS;
        double rr = 0.0;
        for (int f = 0; f < d; ++f) {
          const double v = xi[f * FT + r] - xj[f * FT + c];
          rr = fma(v, v, rr);
          if (ARD_D > 0) {
#pragma unroll
            for (int g = 0; g < AD; ++g)
              if (g == f) dx[w][g] = v;
          }
        }
        r2[w] = rr;
      }
      kt_value_w<ARD_D, PW, NL>(t, dx, r2, kv);
#pragma unroll
      for (int w = 0; w < PW; ++w) {
        const int j = j0 + c0 + w * CS;
        if (j >= n2) continue;
        if (!isfinite(kv[w])) bad = true;
        out[i + (long long)j * ld] = kv[w];
      }
    }
  }
  if (bad) dev_fail(st, GPRX_NONFINITE_KERNEL, 0);
}

static int fill_grid(long long ntiles) {
  long long cap = 148LL * 8;
  return (int)std::max<long long>(1, std::min(ntiles, cap));
}

cudaError_t fill_lower(const HostKernel& k, const double* x, long long ldx, int n, double* K, long long ld,
                       double diag_add, DevStatus* st, cudaStream_t s) {
  int nt = (n + FT - 1) / FT;
  int grid = fill_grid((long long)nt * (nt + 1) / 2);
  // trees of at most two leaves: four pairs per thread
  if (k.tree.n_leaves <= 2 && (k.ard_d == 0 || k.ard_d == 4 || k.ard_d == 8)) {
    switch (k.ard_d) {
      case 0: GPRX_LAUNCH((fill_lower_w_kernel<0, 2, 4>), grid, FILL_THREADS, 0, s, k.tree, x, ldx, n, K, ld, diag_add, st); break;
      case 4: GPRX_LAUNCH((fill_lower_w_kernel<4, 2, 4>), grid, FILL_THREADS, 0, s, k.tree, x, ldx, n, K, ld, diag_add, st); break;
      default: GPRX_LAUNCH((fill_lower_w_kernel<8, 2, 4>), grid, FILL_THREADS, 0, s, k.tree, x, ldx, n, K, ld, diag_add, st); break;
    }
    return cudaGetLastError();
  }
  switch (k.ard_d) {
    case 0: GPRX_LAUNCH(fill_lower_kernel<0>, grid, FILL_THREADS, 0, s, k.tree, x, ldx, n, K, ld, diag_add, st); break;
    case 4: GPRX_LAUNCH(fill_lower_kernel<4>, grid, FILL_THREADS, 0, s, k.tree, x, ldx, n, K, ld, diag_add, st); break;
    case 8: GPRX_LAUNCH(fill_lower_kernel<8>, grid, FILL_THREADS, 0, s, k.tree, x, ldx, n, K, ld, diag_add, st); break;
    case 16: GPRX_LAUNCH(fill_lower_kernel<16>, grid, FILL_THREADS, 0, s, k.tree, x, ldx, n, K, ld, diag_add, st); break;
    default: GPRX_LAUNCH(fill_lower_kernel<32>, grid, FILL_THREADS, 0, s, k.tree, x, ldx, n, K, ld, diag_add, st); break;
  }
  return cudaGetLastError();
}

cudaError_t fill_cross(const HostKernel& k, const double* x1, long long ldx1, int n1, const double* x2,
                       long long ldx2, int n2, double* out, long long ld, DevStatus* st, cudaStream_t s) {
  if (n1 <= 0 || n2 <= 0) return cudaSuccess;
  long long ntiles = (long long)((n1 + FT - 1) / FT) * ((n2 + FT - 1) / FT);
  int grid = fill_grid(ntiles);
#define GPRX_CROSS(D) \
  GPRX_LAUNCH(fill_cross_kernel<D>, grid, FILL_THREADS, 0, s, k.tree, x1, ldx1, n1, x2, ldx2, n2, out, ld, st)
#define GPRX_CROSS_W(D)                                                                                         \
  GPRX_LAUNCH((fill_cross_w_kernel<D, 2, 4>), grid, FILL_THREADS, 0, s, k.tree, x1, ldx1, n1, x2, ldx2, n2, out, \
              ld, st)
  // trees of at most two leaves: four pairs per thread
  if (k.tree.n_leaves <= 2 && (k.ard_d == 0 || k.ard_d == 4 || k.ard_d == 8)) {
    switch (k.ard_d) {
      case 0: GPRX_CROSS_W(0); break;
      case 4: GPRX_CROSS_W(4); break;
      default: GPRX_CROSS_W(8); break;
    }
    return cudaGetLastError();
  }
#undef GPRX_CROSS_W
  switch (k.ard_d) {
    case 0: GPRX_CROSS(0); break;
    case 4: GPRX_CROSS(4); break;
    case 8: GPRX_CROSS(8); break;
    case 16: GPRX_CROSS(16); break;
    default: GPRX_CROSS(32); break;
  }
#undef GPRX_CROSS
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// device: gradient contraction
// ---------------------------------------------------------------------------
constexpr int GRAD_THREADS = 256;  // two blocks per SM for trees of ARD width ≤ 8 (128 registers, no spills)
constexpr int GRAD_MAX_BLOCKS = 148 * 4;

int grad_max_blocks() { return GRAD_MAX_BLOCKS; }

// Writes one block's slot sums (warp shuffles, then warps in a fixed order).
template <int NS>
__device__ __forceinline__ void store_slots(double (&vals)[NS], double (*red)[NS], double* out) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    double v = warp_sum(vals[s]);
    if (lane == 0) red[warp][s] = v;
  }
  __syncthreads();
  for (int s = threadIdx.x; s < NS; s += blockDim.x) {
    double v = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) v += red[w][s];
    out[s] = v;
  }
}

// Lower-triangle contraction Σ_{i≥j} c_ij W_ij ∂K_ij/∂θ (c = 1 diagonal, 2 off).
// With alpha: W_ij = α_i α_j − M_ij (the exact-GPR weight, M = K⁻¹) and the
// last slot collects Σ W_ii; without: W_ij = M_ij.
template <int ARD_D>
__global__ void __launch_bounds__(GRAD_THREADS, ARD_D <= 8 ? 2 : 1) grad_contract_kernel(KTree t, const double* x, long long ldx, int n,
                                                                     const double* kinv, long long ld,
                                                                     const double* alpha, double* partials,
                                                                     const DevStatus* st) {
  constexpr int AD = ARD_D > 0 ? ARD_D : 1;
  constexpr int NS = GRAD_SLOTS_LEAF + AD + 1;
  __shared__ double xi[GPRX_MAX_DIM * FT];
  __shared__ double xj[GPRX_MAX_DIM * FT];
  __shared__ double ai[FT], aj[FT];
  __shared__ double red[GRAD_THREADS / 32][NS];
  if (dev_failed(st)) return;
  const int d = t.d;
  const bool amode = alpha != nullptr;
  double acc_leaf[KT_MAX_LEAVES][KT_ACC_PER_LEAF];
  double acc_ard[AD];
  double acc_noise = 0.0;
#pragma unroll
  for (int l = 0; l < KT_MAX_LEAVES; ++l) acc_leaf[l][0] = acc_leaf[l][1] = 0.0;
#pragma unroll
  for (int f = 0; f < AD; ++f) acc_ard[f] = 0.0;

  const int nt = (n + FT - 1) / FT;
  const long long ntiles = (long long)nt * (nt + 1) / 2;
  for (long long idx = blockIdx.x; idx < ntiles; idx += gridDim.x) {
    int ti, tj;
    lower_tile_of(idx, ti, tj);
    const int i0 = ti * FT, j0 = tj * FT;
    __syncthreads();
    for (int e = threadIdx.x; e < d * FT; e += blockDim.x) {
      int r = e % FT, f = e / FT;
      xi[f * FT + r] = (i0 + r < n) ? x[(i0 + r) + (long long)f * ldx] : 0.0;
      xj[f * FT + r] = (j0 + r < n) ? x[(j0 + r) + (long long)f * ldx] : 0.0;
    }
    if (amode && threadIdx.x < FT) {
      int r = threadIdx.x;
      ai[r] = (i0 + r < n) ? alpha[i0 + r] : 0.0;
      aj[r] = (j0 + r < n) ? alpha[j0 + r] : 0.0;
    }
    __syncthreads();
    const int r = threadIdx.x % FT;
    const int i = i0 + r;
    for (int c = threadIdx.x / FT; c < FT; c += GRAD_THREADS / FT) {
      int j = j0 + c;
      if (i >= n || j >= n || i < j) continue;
      double m = kinv[i + (long long)j * ld];
      double w = amode ? fma(ai[r], aj[c], -m) : m;
      double cw = (i == j) ? w : 2.0 * w;
      if (i == j) acc_noise += w;
      double dx[AD];
      double r2 = 0.0;
      for (int f = 0; f < d; ++f) {
        double v = xi[f * FT + r] - xj[f * FT + c];
        r2 = fma(v, v, r2);
        if (ARD_D > 0) {
#pragma unroll
          for (int g = 0; g < AD; ++g)
            if (g == f) dx[g] = v;
        }
      }
      kt_accumulate_grad<ARD_D>(t, dx, r2, cw, acc_leaf, acc_ard);
    }
  }
  double vals[NS];
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    if (s < GRAD_SLOTS_LEAF) vals[s] = acc_leaf[s / 2][s % 2];
    else if (s < GRAD_SLOTS_LEAF + AD) vals[s] = acc_ard[s - GRAD_SLOTS_LEAF];
    else vals[s] = acc_noise;
  }
  store_slots<NS>(vals, red, partials + (long long)blockIdx.x * NS);
}

// The same contraction for trees of at most NL leaves, PW pairs per thread
// (independent FP64 chains the scheduler interleaves).  A thread takes the
// same pairs in the same order as grad_contract_kernel and pairs outside the
// lower triangle add exact zeros, so every accumulator receives the same
// terms in the same order: the same bits (a tree has at most one ARD leaf,
// so no two leaves share an accumulator).
template <int ARD_D, int NL, int PW>
__global__ void __launch_bounds__(GRAD_THREADS, 2) grad_contract_w_kernel(KTree t, const double* x, long long ldx,
                                                                          int n, const double* kinv, long long ld,
                                                                          const double* alpha, double* partials,
                                                                          const DevStatus* st) {
  constexpr int AD = ARD_D > 0 ? ARD_D : 1;
  constexpr int NS = GRAD_SLOTS_LEAF + AD + 1;
  constexpr int CS = GRAD_THREADS / FT;  // column stride of one thread
  static_assert((FT / CS) % PW == 0, "pairs per thread");
  __shared__ double xi[GPRX_MAX_DIM * FT];
  __shared__ double xj[GPRX_MAX_DIM * FT];
  __shared__ double ai[FT], aj[FT];
  __shared__ double red[GRAD_THREADS / 32][NS];
  if (dev_failed(st)) return;
  const int d = t.d;
  const bool amode = alpha != nullptr;
  double acc_leaf[NL][KT_ACC_PER_LEAF];
  double acc_ard[AD];
  double acc_noise = 0.0;
#pragma unroll
  for (int l = 0; l < NL; ++l) acc_leaf[l][0] = acc_leaf[l][1] = 0.0;
#pragma unroll
  for (int f = 0; f < AD; ++f) acc_ard[f] = 0.0;

  const int nt = (n + FT - 1) / FT;
  const long long ntiles = (long long)nt * (nt + 1) / 2;
  for (long long idx = blockIdx.x; idx < ntiles; idx += gridDim.x) {
    int ti, tj;
    lower_tile_of(idx, ti, tj);
    const int i0 = ti * FT, j0 = tj * FT;
    __syncthreads();
    for (int e = threadIdx.x; e < d * FT; e += blockDim.x) {
      int r = e % FT, f = e / FT;
      xi[f * FT + r] = (i0 + r < n) ? x[(i0 + r) + (long long)f * ldx] : 0.0;
      xj[f * FT + r] = (j0 + r < n) ? x[(j0 + r) + (long long)f * ldx] : 0.0;
    }
    if (amode && threadIdx.x < FT) {
      int r = threadIdx.x;
      ai[r] = (i0 + r < n) ? alpha[i0 + r] : 0.0;
      aj[r] = (j0 + r < n) ? alpha[j0 + r] : 0.0;
    }
    __syncthreads();
    const int r = threadIdx.x % FT;
    const int i = i0 + r;
    if (i >= n) continue;
#pragma unroll 1
    for (int c0 = threadIdx.x / FT; c0 < FT; c0 += CS * PW) {
      if (j0 + c0 > i) break;  // every later pair of this thread lies above the diagonal
      double dx[PW][AD], r2[PW], wt[PW];
#pragma unroll
      for (int w = 0; w < PW; ++w) {
        const int c = c0 + w * CS, j = j0 + c;
        const bool in = j < n && i >= j;
        double cw = 0.0;
        if (in) {
          const double m = kinv[i + (long long)j * ld];
          const double wv = amode ? fma(ai[r], aj[c], -m) : m;
          cw = (i == j) ? wv : 2.0 * wv;
          if (i == j) acc_noise += wv;
        }
        wt[w] = cw;
        double rr = 0.0;
        for (int f = 0; f < d; ++f) {
          const double v = xi[f * FT + r] - xj[f * FT + c];
          rr = fma(v, v, rr);
          if (ARD_D > 0) {
#pragma unroll
            for (int g = 0; g < AD; ++g)
              if (g == f) dx[w][g] = v;
          }
        }
        r2[w] = rr;
      }
      kt_accumulate_grad_w<ARD_D, PW, NL>(t, dx, r2, wt, acc_leaf, acc_ard);
    }
  }
  double vals[NS];
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    if (s < GRAD_SLOTS_LEAF) vals[s] = (s / 2 < NL) ? acc_leaf[s / 2][s % 2] : 0.0;
    else if (s < GRAD_SLOTS_LEAF + AD) vals[s] = acc_ard[s - GRAD_SLOTS_LEAF];
    else vals[s] = acc_noise;
  }
  store_slots<NS>(vals, red, partials + (long long)blockIdx.x * NS);
}

// Rectangle contraction Σ_{i,c} W_ic ∂k(z_i, x_c)/∂θ (W is m×n, ldw).
template <int ARD_D>
__global__ void __launch_bounds__(GRAD_THREADS, ARD_D <= 8 ? 2 : 1) cross_contract_kernel(KTree t, const double* z, long long ldz, int m,
                                                                      const double* x, long long ldx, int n,
                                                                      const double* W, long long ldw, double* partials,
                                                                      const DevStatus* st) {
  constexpr int AD = ARD_D > 0 ? ARD_D : 1;
  constexpr int NS = GRAD_SLOTS_LEAF + AD + 1;
  __shared__ double xi[GPRX_MAX_DIM * FT];
  __shared__ double xj[GPRX_MAX_DIM * FT];
  __shared__ double red[GRAD_THREADS / 32][NS];
  if (dev_failed(st)) return;
  const int d = t.d;
  double acc_leaf[KT_MAX_LEAVES][KT_ACC_PER_LEAF];
  double acc_ard[AD];
#pragma unroll
  for (int l = 0; l < KT_MAX_LEAVES; ++l) acc_leaf[l][0] = acc_leaf[l][1] = 0.0;
#pragma unroll
  for (int f = 0; f < AD; ++f) acc_ard[f] = 0.0;
  const int tm = (m + FT - 1) / FT, tn = (n + FT - 1) / FT;
  const long long ntiles = (long long)tm * tn;
  for (long long idx = blockIdx.x; idx < ntiles; idx += gridDim.x) {
    const int i0 = (int)(idx % tm) * FT, j0 = (int)(idx / tm) * FT;
    __syncthreads();
    for (int e = threadIdx.x; e < d * FT; e += blockDim.x) {
      int r = e % FT, f = e / FT;
      xi[f * FT + r] = (i0 + r < m) ? z[(i0 + r) + (long long)f * ldz] : 0.0;
      xj[f * FT + r] = (j0 + r < n) ? x[(j0 + r) + (long long)f * ldx] : 0.0;
    }
    __syncthreads();
    const int r = threadIdx.x % FT;
    const int i = i0 + r;
    for (int c = threadIdx.x / FT; c < FT; c += GRAD_THREADS / FT) {
      int j = j0 + c;
      if (i >= m || j >= n) continue;
      double w = W[i + (long long)j * ldw];
      double dx[AD];
      double r2 = 0.0;
      for (int f = 0; f < d; ++f) {
        double v = xi[f * FT + r] - xj[f * FT + c];
        r2 = fma(v, v, r2);
        if (ARD_D > 0) {
#pragma unroll
          for (int g = 0; g < AD; ++g)
            if (g == f) dx[g] = v;
        }
      }
      kt_accumulate_grad<ARD_D>(t, dx, r2, w, acc_leaf, acc_ard);
    }
  }
  double vals[NS];
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    if (s < GRAD_SLOTS_LEAF) vals[s] = acc_leaf[s / 2][s % 2];
    else if (s < GRAD_SLOTS_LEAF + AD) vals[s] = acc_ard[s - GRAD_SLOTS_LEAF];
    else vals[s] = 0.0;
  }
  store_slots<NS>(vals, red, partials + (long long)blockIdx.x * NS);
}

// The cross contraction for trees of at most NL leaves, PW pairs per thread;
// every accumulator receives the terms of cross_contract_kernel in the same
// order (pairs past the matrix add exact zeros): the same bits.
template <int ARD_D, int NL, int PW>
__global__ void __launch_bounds__(GRAD_THREADS, 2) cross_contract_w_kernel(KTree t, const double* z, long long ldz,
                                                                           int m, const double* x, long long ldx,
                                                                           int n, const double* W, long long ldw,
                                                                           double* partials, const DevStatus* st) {
  constexpr int AD = ARD_D > 0 ? ARD_D : 1;
  constexpr int NS = GRAD_SLOTS_LEAF + AD + 1;
  constexpr int CS = GRAD_THREADS / FT;
  static_assert((FT / CS) % PW == 0, "pairs per thread");
  __shared__ double xi[GPRX_MAX_DIM * FT];
  __shared__ double xj[GPRX_MAX_DIM * FT];
  __shared__ double red[GRAD_THREADS / 32][NS];
  if (dev_failed(st)) return;
  const int d = t.d;
  double acc_leaf[NL][KT_ACC_PER_LEAF];
  double acc_ard[AD];
#pragma unroll
  for (int l = 0; l < NL; ++l) acc_leaf[l][0] = acc_leaf[l][1] = 0.0;
#pragma unroll
  for (int f = 0; f < AD; ++f) acc_ard[f] = 0.0;
  const int tm = (m + FT - 1) / FT, tn = (n + FT - 1) / FT;
  const long long ntiles = (long long)tm * tn;
  for (long long idx = blockIdx.x; idx < ntiles; idx += gridDim.x) {
    const int i0 = (int)(idx % tm) * FT, j0 = (int)(idx / tm) * FT;
    __syncthreads();
    for (int e = threadIdx.x; e < d * FT; e += blockDim.x) {
      int r = e % FT, f = e / FT;
      xi[f * FT + r] = (i0 + r < m) ? z[(i0 + r) + (long long)f * ldz] : 0.0;
      xj[f * FT + r] = (j0 + r < n) ? x[(j0 + r) + (long long)f * ldx] : 0.0;
    }
    __syncthreads();
    const int r = threadIdx.x % FT;
    const int i = i0 + r;
    if (i >= m) continue;
#pragma unroll 1
    for (int c0 = threadIdx.x / FT; c0 < FT; c0 += CS * PW) {
      if (j0 + c0 >= n) break;
      double dx[PW][AD], r2[PW], wt[PW];
#pragma unroll
      for (int w = 0; w < PW; ++w) {
        const int c = c0 + w * CS, j = j0 + c;
        wt[w] = j < n ? W[i + (long long)j * ldw] : 0.0;
        double rr = 0.0;
        for (int f = 0; f < d; ++f) {
          const double v = xi[f * FT + r] - xj[f * FT + c];
          rr = fma(v, v, rr);
          if (ARD_D > 0) {
#pragma unroll
            for (int g = 0; g < AD; ++g)
              if (g == f) dx[w][g] = v;
          }
        }
        r2[w] = rr;
      }
      kt_accumulate_grad_w<ARD_D, PW, NL>(t, dx, r2, wt, acc_leaf, acc_ard);
    }
  }
  double vals[NS];
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    if (s < GRAD_SLOTS_LEAF) vals[s] = (s / 2 < NL) ? acc_leaf[s / 2][s % 2] : 0.0;
    else if (s < GRAD_SLOTS_LEAF + AD) vals[s] = acc_ard[s - GRAD_SLOTS_LEAF];
    else vals[s] = 0.0;
  }
  store_slots<NS>(vals, red, partials + (long long)blockIdx.x * NS);
}

cudaError_t grad_contract(const HostKernel& k, const double* x, long long ldx, int n, const double* kinv, long long ld,
                          const double* alpha, double* partials, int* blocks_out, DevStatus* st, cudaStream_t s) {
  int nt = (n + FT - 1) / FT;
  long long ntiles = (long long)nt * (nt + 1) / 2;
  int grid = (int)std::max<long long>(1, std::min<long long>(ntiles, GRAD_MAX_BLOCKS));
  *blocks_out = grid;
#define GPRX_GRAD(D) \
  GPRX_LAUNCH(grad_contract_kernel<D>, grid, GRAD_THREADS, 0, s, k.tree, x, ldx, n, kinv, ld, alpha, partials, st)
#define GPRX_GRAD_W(D)                                                                                         \
  GPRX_LAUNCH((grad_contract_w_kernel<D, 2, 2>), grid, GRAD_THREADS, 0, s, k.tree, x, ldx, n, kinv, ld, alpha, \
              partials, st)
  // trees of at most two leaves: two pairs per thread
  if (k.tree.n_leaves <= 2 && (k.ard_d == 0 || k.ard_d == 4 || k.ard_d == 8)) {
    switch (k.ard_d) {
      case 0: GPRX_GRAD_W(0); break;
      case 4: GPRX_GRAD_W(4); break;
      default: GPRX_GRAD_W(8); break;
    }
    return cudaGetLastError();
  }
#undef GPRX_GRAD_W
  switch (k.ard_d) {
    case 0: GPRX_GRAD(0); break;
    case 4: GPRX_GRAD(4); break;
    case 8: GPRX_GRAD(8); break;
    case 16: GPRX_GRAD(16); break;
    default: GPRX_GRAD(32); break;
  }
#undef GPRX_GRAD
  return cudaGetLastError();
}

cudaError_t cross_contract(const HostKernel& k, const double* z, long long ldz, int m, const double* x, long long ldx,
                           int n, const double* W, long long ldw, double* partials, int* blocks_out, DevStatus* st,
                           cudaStream_t s) {
  long long ntiles = (long long)((m + FT - 1) / FT) * ((n + FT - 1) / FT);
  int grid = (int)std::max<long long>(1, std::min<long long>(ntiles, GRAD_MAX_BLOCKS));
  *blocks_out = grid;
#define GPRX_CC(D)                                                                                                  \
  GPRX_LAUNCH(cross_contract_kernel<D>, grid, GRAD_THREADS, 0, s, k.tree, z, ldz, m, x, ldx, n, W, ldw, partials, \
              st)
#define GPRX_CC_W(D)                                                                                             \
  GPRX_LAUNCH((cross_contract_w_kernel<D, 2, 2>), grid, GRAD_THREADS, 0, s, k.tree, z, ldz, m, x, ldx, n, W, ldw, \
              partials, st)
  // trees of at most two leaves: two pairs per thread
  if (k.tree.n_leaves <= 2 && (k.ard_d == 0 || k.ard_d == 4 || k.ard_d == 8)) {
    switch (k.ard_d) {
      case 0: GPRX_CC_W(0); break;
      case 4: GPRX_CC_W(4); break;
      default: GPRX_CC_W(8); break;
    }
    return cudaGetLastError();
  }
#undef GPRX_CC_W
  switch (k.ard_d) {
    case 0: GPRX_CC(0); break;
    case 4: GPRX_CC(4); break;
    case 8: GPRX_CC(8); break;
    case 16: GPRX_CC(16); break;
    default: GPRX_CC(32); break;
  }
#undef GPRX_CC
  return cudaGetLastError();
}

// grad[p] = scale · Σ_slots(p); grad[n_kernel] = noise_coef · Σ (last slot).
__global__ void grad_finalize_kernel(const double* partials, int blocks, int ns, const int* slot_param, int n_kernel,
                                     double scale, double noise_coef, double* grad, const DevStatus* st) {
  __shared__ double tot[64];
  if (dev_failed(st)) return;
  for (int s = threadIdx.x; s < ns; s += blockDim.x) {
    double v = 0.0;
    for (int b = 0; b < blocks; ++b) v += partials[(long long)b * ns + s];
    tot[s] = v;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int p = 0; p <= n_kernel; ++p) grad[p] = 0.0;
    for (int s = 0; s < ns - 1; ++s) {
      int p = slot_param[s];
      if (p >= 0) grad[p] += tot[s];
    }
    for (int p = 0; p < n_kernel; ++p) grad[p] *= scale;
    grad[n_kernel] = noise_coef * tot[ns - 1];
  }
}

cudaError_t grad_finalize(const HostKernel& k, const double* partials, int blocks, const int* slot_param_dev,
                          double scale, double noise_coef, double* grad, DevStatus* st, cudaStream_t s) {
  int ns = grad_slots(k.ard_d);
  GPRX_LAUNCH(grad_finalize_kernel, 1, 64, 0, s, partials, blocks, ns, slot_param_dev, k.n_params, scale,
              noise_coef, grad, st);
  return cudaGetLastError();
}

}  // namespace gprx
