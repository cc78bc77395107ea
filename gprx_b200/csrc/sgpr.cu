// sgpr.cu — VFE sparse GPR on the device: assembly, NLML, adjoint gradient,
// prediction and the online X insert / delete.
//
// Reference: assemble_vfe (gprx src/sgpr/factor/vfe.rs:191-277),
// vfe_neg_log_marginal_likelihood (vfe.rs:338-369), VfeEngine::adjoint and
// analytic_gradient (src/sgpr/factor/derivatives.rs:102-144,186-202,283-366),
// vfe_latent (src/sgpr/factor/predict.rs:197-262), OnlineSgpr::insert /
// append_point and delete (src/sgpr/online/mod.rs:1695-1810, 903-1000) with
// chol_rank1_update / downdate (src/linalg/chol.rs:450-493) and the X-step
// pivot gate (src/sgpr/factor/updates.rs:217-290, min_pivot_ratio :414).
//
// Layout: Z is m×d, X is n×d (column-major, leading dimension = capacity);
// A = L⁻¹K(Z, X) is m×n with leading dimension ldm (≥ m).  A's columns, X and
// y are kept in slot order; a host-side table maps the reference's point
// order (the PointId registry) onto slots, so a delete moves one column.

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "dense_f64.cuh"
#include "emu_gemm.cuh"
#include "exact.cuh"
#include "kernels.cuh"
#include "lbfgs.h"
#include "runtime.cuh"

namespace gprx {

gprx_status fit_lbfgs(void* ctx, gprx_status (*eval)(void*, const double*, double*, double*), int p,
                      const double* theta0, const gprx_lbfgs_options* o, gprx_fit_report* rep,
                      std::vector<double>& best_theta);

constexpr double X_STEP_PIVOT_RTOL = 8.0 * 2.220446049250313e-16;  // updates.rs:252

// ---------------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------------
// B[i, j] = Σ_s P_s[i, j] + σ² δ_ij for the lower (or full) m×m matrix.
__global__ void split_reduce_kernel(const double* P, int S, long long stride, int m, long long ld, double diag,
                                    bool lower, double* B, const DevStatus* st) {
  if (dev_failed(st)) return;
  long long total = (long long)m * m;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    int i = (int)(e % m), j = (int)(e / m);
    if (lower && i < j) continue;
    double v = 0.0;
    for (int s = 0; s < S; ++s) v += P[s * stride + i + (long long)j * ld];
    if (i == j) v += diag;
    B[i + (long long)j * ld] = v;
  }
}

// Σ over an m×n column-major matrix of squares: one partial per block.
__global__ void sumsq_kernel(const double* A, long long ld, int m, long long n, double* partial,
                             const DevStatus* st) {
  __shared__ double red[32];
  if (dev_failed(st)) return;
  double acc = 0.0;
  long long total = (long long)m * n;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    int i = (int)(e % m);
    long long c = e / m;
    double v = A[i + c * ld];
    acc = fma(v, v, acc);
  }
  double s = block_sum(acc, red);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

// Σ_c (kdiag − ‖A[:, c]‖²) over the n columns of the m×n matrix A: each term
// is point c's Nyström residual k(x_c, x_c) − k_cᵀ K_mm⁻¹ k_c ≥ 0, so the sum
// keeps its digits where Σ k_ii − ‖A‖²_F (vfe.rs:338-369) cancels.  One warp
// per column; one partial per block.
__global__ void trace_residual_kernel(const double* A, long long ld, int m, long long n, double kdiag,
                                      double* partial, const DevStatus* st) {
  __shared__ double red[32];
  if (dev_failed(st)) return;
  const int lane = threadIdx.x & 31;
  const long long warp = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
  double acc = 0.0;
  for (long long c = warp; c < n; c += nw) {
    const double* a = A + c * ld;
    double ss = 0.0;
    for (int i = lane; i < m; i += 32) ss = fma(a[i], a[i], ss);
    ss = warp_sum(ss);
    if (lane == 0) acc += kdiag - ss;
  }
  double s = block_sum(acc, red);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

// Σ y² in extended precision (the host's long double).
static double sumsq_host(const std::vector<double>& v) {
  long double s = 0.0L;
  for (double e : v) s += (long double)e * e;
  return (double)s;
}

__global__ void sum_partials_kernel(const double* partial, int count, double* out, const DevStatus* st) {
  __shared__ double red[32];
  if (dev_failed(st)) return;
  double acc = 0.0;
  for (int i = threadIdx.x; i < count; i += blockDim.x) acc += partial[i];
  double s = block_sum(acc, red);
  if (threadIdx.x == 0) *out = s;
}

// G[:, c] −= (w r_c + A[:, c]) / σ² with r_c = y_c − A[:, c]ᵀ w (one warp per column).
__global__ void adjoint_update_kernel(const double* A, double* G, long long ld, int m, long long n, const double* w,
                                      const double* y, double inv_noise, const DevStatus* st) {
  if (dev_failed(st)) return;
  long long warp = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long c = warp; c < n; c += nw) {
    const double* a = A + c * ld;
    double acc = 0.0;
    for (int i = lane; i < m; i += 32) acc = fma(a[i], w[i], acc);
    acc = warp_sum(acc);
    double rc = y[c] - acc;
    double* g = G + c * ld;
    for (int i = lane; i < m; i += 32) g[i] -= fma(w[i], rc, a[i]) * inv_noise;
  }
}

// X = tril½(H) (lower, diagonal halved, zero above)
__global__ void tril_half_kernel(const double* H, long long ld, int m, double* X) {
  long long total = (long long)m * m;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    int i = (int)(e % m), j = (int)(e / m);
    double v = H[i + (long long)j * ld];
    X[i + (long long)j * ld] = i > j ? v : (i == j ? 0.5 * v : 0.0);
  }
}

__global__ void transpose_kernel(const double* X, long long ld, int m, double* Y) {
  __shared__ double tile[32][33];
  int bi = blockIdx.x * 32, bj = blockIdx.y * 32;
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    int i = bi + threadIdx.x, j = bj + r;
    tile[r][threadIdx.x] = (i < m && j < m) ? X[i + (long long)j * ld] : 0.0;
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    int i = bj + threadIdx.x, j = bi + r;
    if (i < m && j < m) Y[i + (long long)j * ld] = tile[threadIdx.x][r];
  }
}

// W = −½ (Yᵀ + Y)
__global__ void neg_sym_half_kernel(const double* Y, long long ld, int m, double* W) {
  long long total = (long long)m * m;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    int i = (int)(e % m), j = (int)(e / m);
    W[i + (long long)j * ld] = -0.5 * (Y[j + (long long)i * ld] + Y[i + (long long)j * ld]);
  }
}

// min over rows of L_ii² / Σ_k L_ik² (min_pivot_ratio, updates.rs:414-427)
__global__ void pivot_ratio_kernel(const double* L, long long ld, int m, double* out) {
  __shared__ double red[32];
  double mn = 1.0;
  for (int i = threadIdx.x; i < m; i += blockDim.x) {
    double row2 = 0.0;
    for (int k = 0; k <= i; ++k) {
      double v = L[i + (long long)k * ld];
      row2 = fma(v, v, row2);
    }
    double piv = L[i + (long long)i * ld];
    double r = piv * piv / row2;
    if (!isfinite(r)) r = 0.0;
    mn = fmin(mn, r);
  }
  // block min
  for (int o = 16; o > 0; o >>= 1) mn = fmin(mn, __shfl_xor_sync(0xffffffffu, mn, o));
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) red[warp] = mn;
  __syncthreads();
  if (threadIdx.x == 0) {
    double r = 1.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) r = fmin(r, red[w]);
    *out = r;
  }
}

// Rank-1 update (sign = +1) or downdate (−1) of the lower m×m factor L with v
// (destroyed), chol_rank1_update / chol_rank1_downdate (chol.rs:450-493),
// 32 columns per step: warp 0 runs the step's rotations on its own rows,
// then all threads apply them to the rows below.  A downdate whose r² is not
// positive and finite sets the status (CHOLESKY_FAILED) and stops.
constexpr int R1C_THREADS = 256;
__global__ void __launch_bounds__(R1C_THREADS) chol_rank1_kernel(double* L, long long ld, int m, double* v,
                                                                  double sign, DevStatus* st) {
  __shared__ double Cc[32], Ss[32];
  __shared__ int bad;
  if (dev_failed(st)) return;
  if (threadIdx.x == 0) bad = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int kb = 0; kb < m; kb += 32) {
    const int nbk = min(32, m - kb);
    if (warp == 0) {
      const int r = kb + lane;
      const bool live = lane < nbk;
      double vr = live ? v[r] : 0.0;
      double l[32];
#pragma unroll
      for (int c = 0; c < 32; ++c) l[c] = (live && c <= lane) ? L[r + (long long)(kb + c) * ld] : 0.0;
      int fail = 0;
#pragma unroll
      for (int c = 0; c < 32; ++c) {
        if (c < nbk) {
          double lkk = __shfl_sync(0xffffffffu, l[c], c);
          double vk = __shfl_sync(0xffffffffu, vr, c);
          double r2 = fma(sign * vk, vk, lkk * lkk);
          if (!(r2 > 0.0) || !isfinite(r2)) fail = 1;
          double rr = sqrt(fmax(r2, 0.0));
          double cc = rr / lkk, ss = vk / lkk;
          if (lane == 0) {
            Cc[c] = cc;
            Ss[c] = ss;
          }
          if (lane == c) l[c] = rr;
          else if (live && lane > c) {
            l[c] = fma(sign * ss, vr, l[c]) / cc;
            vr = fma(cc, vr, -ss * l[c]);
          }
        }
      }
      if (live) {
#pragma unroll
        for (int c = 0; c < 32; ++c)
          if (c <= lane) L[r + (long long)(kb + c) * ld] = l[c];
        v[r] = vr;
      }
      if (fail && lane == 0) bad = 1;
    }
    __syncthreads();
    if (bad) {
      if (threadIdx.x == 0) dev_fail(st, GPRX_CHOLESKY_FAILED, kb);
      return;
    }
    for (int r = kb + nbk + threadIdx.x; r < m; r += blockDim.x) {
      double vr = v[r];
      for (int c = 0; c < nbk; ++c) {
        double* lp = L + r + (long long)(kb + c) * ld;
        double lv = fma(sign * Ss[c], vr, *lp) / Cc[c];
        *lp = lv;
        vr = fma(Cc[c], vr, -Ss[c] * lv);
      }
      v[r] = vr;
    }
    __syncthreads();
  }
}

// Row m of a lower factor L (ld): L[m, 0..m-1] = v, L[m, m] = diag, and zeros
// above the diagonal of column m.
__global__ void border_row_kernel(double* L, long long ld, int m, const double* v, double diag) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < m) {
    L[m + (long long)i * ld] = v[i];
    L[i + (long long)m * ld] = 0.0;
  } else if (i == m) {
    L[m + (long long)m * ld] = diag;
  }
}

// The new row of A: a_c = (k(z, x_c) − (Aᵀ l)_c) / ℓ, into row m of A (ld)
// and into a contiguous copy.
__global__ void border_a_row_kernel(const double* krow, const double* atl, double inv_ell, double* A, long long ld,
                                    int m, long long n, double* copy) {
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
    const double v = (krow[c] - atl[c]) * inv_ell;
    A[m + c * ld] = v;
    copy[c] = v;
  }
}

__global__ void axpy_kernel(double* y, const double* x, double a, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] = fma(a, x[i], y[i]);
}

__global__ void sgpr_finish_var_kernel(const double* an, const double* bn, int q, double kss, double noise, int kind,
                                       double* var, const DevStatus* st) {
  if (dev_failed(st)) return;
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= q) return;
  double lat = kss - an[j] + noise * bn[j];
  if (lat < 0.0) lat = 0.0;
  var[j] = kind == GPRX_VARIANCE_OBSERVATION ? lat + noise : lat;
}

static int grid_for(long long work, int per) {
  return (int)std::max<long long>(1, std::min<long long>((work + per - 1) / per, 148LL * 16));
}

// ---------------------------------------------------------------------------
// state
// ---------------------------------------------------------------------------
struct SgprState {
  int device = 0;
  cudaStream_t stream = nullptr;
  gprx_options opt{};
  HostKernel kern;
  double log_noise = 0.0;
  long long n = 0, cap = 0;
  int m = 0, d = 0;
  long long ldm = 0;
  DevBuf<double> x, y, z, Lmm, linv_mm, Amat, Bl, linv_B, w, ay, G, H, Wm, Xb, Xt, splitbuf, partials, res, vtmp,
      qbuf, qbuf2, qx, Btrial, covbuf, covl, covlinv, zbuf, border;
  DevBuf<int> slot_param;
  DevBuf<DevStatus> status;
  // mixed precision: the two m×m Gram products over n (B = A Aᵀ and H = G Aᵀ)
  // emulated on the int8 tensor cores, split over K across CTAs
  DevBuf<int8_t> emu_sa, emu_sb;
  DevBuf<double> emu_part;
  DevBuf<int> emu_ea, emu_eb, emu_err;
  DevBuf<unsigned long long> emu_ma, emu_mb;
  HostPinned<int> emu_err_h;
  static constexpr long long EMU_MIN_N = 16384;  // smallest n that uses the emulated products
  static constexpr int EMU_S = 7;                // int8 digits per entry
  static constexpr int EMU_PART_K = 32768;       // K of one split-K part: K·S·2^12 < 2^31 keeps its int32 sums exact
  static constexpr int EMU_GROUP = 8 * EMU_PART_K;  // columns of n sliced at a time (8 parts in flight)
  static constexpr int TRSM_LEAF = 256;          // rows of the blocked solves under the recursive m×n solves
  bool use_emu() const { return opt.precision == GPRX_PRECISION_MIXED && n >= EMU_MIN_N; }
  gprx_status ensure_emu(EmuWork& w);
  HostPinned<double> res_h;
  HostPinned<DevStatus> status_h;
  FactorCtx fctx;
  // host scalars of the assembly
  // trace_sum = Σ_c (k(x_c, x_c) − ‖a_c‖²), the numerator of the VFE trace term
  double trace_sum = 0.0, y2 = 0.0, kmm_jitter = 0.0, pivot_ratio = 1.0;
  bool assembled = false;
  std::vector<double> y_host;     // slot order
  std::vector<long long> order;   // registry index → slot
  std::vector<uint64_t> ids;      // registry order
  uint64_t next_id = 0;
  int last_in_place = 0;
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};

  ~SgprState() {
    if (stream) cudaStreamSynchronize(stream);
    for (auto& e : ev)
      if (e) cudaEventDestroy(e);
    if (stream) cudaStreamDestroy(stream);
  }

  double noise() const { return std::exp(log_noise); }
  int num_params() const { return kern.n_params + 1; }

  gprx_status reset_status() {
    GPRX_CUDA_TRY(cudaMemsetAsync(status.p, 0, sizeof(DevStatus), stream));
    return GPRX_OK;
  }
  gprx_status read_status(DevStatus* out) {
    GPRX_CUDA_TRY(cudaMemcpyAsync(status_h.p, status.p, sizeof(DevStatus), cudaMemcpyDeviceToHost, stream));
    GPRX_CUDA_TRY(cudaStreamSynchronize(stream));
    *out = *status_h.p;
    return GPRX_OK;
  }
  gprx_status sync_check(int stage) {
    DevStatus ds;
    gprx_status st = read_status(&ds);
    if (st != GPRX_OK) return st;
    if (ds.code != GPRX_OK) return status_to_error(ds, kmm_jitter, m, stage);
    return GPRX_OK;
  }

  gprx_status create(const double* xh, uint64_t nn, uint64_t dd, const double* yh, const double* zh, uint64_t mm,
                     const gprx_kernel_node* nodes, int n_nodes, const double* theta, int n_theta,
                     const gprx_options* o);
  gprx_status ensure_points(long long needed);
  gprx_status assemble();
  gprx_status write_params(const double* params);
  gprx_status nlml(double* out);
  gprx_status gradient(double* grad);
  gprx_status eval(const double* params, double* nlml_out, double* grad);
  gprx_status predict(const double* xs, uint64_t q, int kind, double* mean, double* var);
  gprx_status covariance_dev(const double* xs, uint64_t q, int kind, double* mean_host);
  gprx_status predict_covariance(const double* xs, uint64_t q, int kind, double* mean, double* cov);
  gprx_status sample(const double* xs, uint64_t q, int kind, uint64_t n_draws, uint64_t seed, double* out);
  gprx_status solve_w();
  gprx_status insert(const double* xnew, double ynew, uint64_t* id);
  gprx_status remove(uint64_t id);
  gprx_status set_inducing(const double* zh, uint64_t mm);
  // OnlineSgpr::insert_inducing / delete_inducing (src/sgpr/online/mod.rs:1301,1943)
  std::vector<uint64_t> inducing_ids;
  uint64_t next_inducing_id = 0;
  gprx_status insert_inducing(const double* znew, uint64_t* id);
  gprx_status delete_inducing(uint64_t id);
  gprx_status replace_inducing(const std::vector<double>& znew, int mm);
  // the bordered insert of one inducing point; *applied = false when a gate
  // sends the change to the assembly instead (nothing changed then)
  gprx_status insert_inducing_bordered(const double* znew, bool* applied);
  // out (m) = A v for a device vector v over the n points (split-K product)
  gprx_status a_times(const double* v, double* out);
  // one shard of a VFE evaluation over n split across processes (the sums
  // over n travel in two exchange buffers that the caller sums over shards)
  gprx_status factor_kmm_and_a(EmuWork& ew, bool& emu);
  gprx_status shard_assemble(const double* params, double* e1);
  gprx_status shard_nlml(const double* e1, double* nlml_out, double* e2);
  gprx_status shard_gradient(const double* e2, double* grad);
  uint64_t shard_e1() const { return (uint64_t)m * m + m + 3; }
  uint64_t shard_e2() const { return (uint64_t)m * m + kern.n_params + 1; }
  double n_total = 0.0, shard_y2 = 0.0;  // Σ n and Σ y² over the shards of the last shard evaluation
  bool shard_ready = false;
  // the device state is a sharded evaluation's global posterior: predictions
  // use it; the NLML and online steps of this handle reassemble its own points
  bool sharded = false;
  void drop_shard_state() {
    if (sharded) assembled = false;
    sharded = false;
  }
  void get_params(double* out) const {
    for (int i = 0; i < kern.n_params; ++i) out[i] = kern.theta[i];
    out[kern.n_params] = log_noise;
  }
};

static bool in_default_interval(double log_v) {
  double v = std::exp(log_v);
  return std::isfinite(v) && v > 1e-5 && v < 1e5;
}

// ∂k(x, x)/∂θ for a stationary tree: only Constant leaves move the diagonal
// (RBF, RBF_ARD and Periodic are 1 at r = 0 for every θ).
static void diag_grad(const HostKernel& k, std::vector<double>& out) {
  out.assign(k.n_params, 0.0);
  const KTree& t = k.tree;
  double v0[KT_MAX_LEAVES];
  for (int l = 0; l < t.n_leaves; ++l) v0[l] = t.leaf[l].kind == GPRX_LEAF_CONSTANT ? t.leaf[l].c0 : 1.0;
  for (int tt = 0; tt < t.n_terms; ++tt)
    for (int l = 0; l < t.n_leaves; ++l) {
      if (!((t.term_mask[tt] >> l) & 1u) || t.leaf[l].kind != GPRX_LEAF_CONSTANT) continue;
      double others = 1.0;
      for (int o = 0; o < t.n_leaves; ++o)
        if (o != l && ((t.term_mask[tt] >> o) & 1u)) others *= v0[o];
      out[t.leaf[l].param] += others * t.leaf[l].c0;
    }
}

gprx_status SgprState::create(const double* xh, uint64_t nn, uint64_t dd, const double* yh, const double* zh,
                              uint64_t mm, const gprx_kernel_node* nodes, int n_nodes, const double* theta,
                              int n_theta, const gprx_options* o) {
  if (!xh || !yh || !zh || !nodes || !theta) return set_error(GPRX_INVALID_ARGUMENT, "null pointer");
  if (nn == 0 || mm == 0) return set_error(GPRX_EMPTY_INPUT, "no points or no inducing points");
  if (dd == 0) return set_error(GPRX_EMPTY_INPUT, "no features (d = 0)");
  if (mm > 65536) return set_error(GPRX_CAPACITY, "m too large");
  if (!all_finite(xh, nn * dd) || !all_finite(yh, nn) || !all_finite(zh, mm * dd))
    return set_error(GPRX_NONFINITE_INPUT, "non-finite input");
  if (o) opt = *o;
  else gprx_options_default_sparse(&opt);
  if (n_theta < 1) return set_error(GPRX_SHAPE_MISMATCH, "theta must hold the kernel parameters and log noise");
  std::string why;
  gprx_status st = kern.init(nodes, n_nodes, theta, n_theta - 1, (int)dd, &why);
  if (st != GPRX_OK) return set_error(st, why);
  for (int i = 0; i < n_theta; ++i)
    if (!in_default_interval(theta[i])) return set_error(GPRX_INVALID_HYPERPARAMETER, "hyperparameter outside (1e-5, 1e5)");
  log_noise = theta[n_theta - 1];
  n = (long long)nn;
  m = (int)mm;
  d = (int)dd;
  ldm = round_ld(m);
  device = opt.device;
  GPRX_CUDA_TRY(cudaSetDevice(device));
  GPRX_CUDA_TRY(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
  for (auto& e : ev) GPRX_CUDA_TRY(cudaEventCreate(&e));
  int nblk = ceil_div(m, NB);
  // the m×m factors keep ld columns, the room a bordered inducing insert grows into
  if (z.alloc((size_t)m * d) || Lmm.alloc((size_t)ldm * ldm) || linv_mm.alloc((size_t)nblk * NB * NB) ||
      Bl.alloc((size_t)ldm * ldm) || linv_B.alloc((size_t)nblk * NB * NB) || w.alloc(ldm) || ay.alloc(ldm) ||
      vtmp.alloc(ldm) || partials.alloc((size_t)grad_max_blocks() * 2 * 64 + 4096) || res.alloc(128) ||
      slot_param.alloc(64) || status.alloc(1))
    return set_error(GPRX_OUT_OF_MEMORY, "device allocation failed");
  GPRX_CUDA_TRY(res_h.ensure(128));
  GPRX_CUDA_TRY(status_h.ensure(1));
  if ((st = ensure_points(n)) != GPRX_OK) return st;
  GPRX_CUDA_TRY(cudaMemcpy2DAsync(x.p, sizeof(double) * cap, xh, sizeof(double) * n, sizeof(double) * n, d,
                                  cudaMemcpyHostToDevice, stream));
  GPRX_CUDA_TRY(cudaMemcpyAsync(y.p, yh, sizeof(double) * n, cudaMemcpyHostToDevice, stream));
  GPRX_CUDA_TRY(cudaMemcpyAsync(z.p, zh, sizeof(double) * m * d, cudaMemcpyHostToDevice, stream));
  std::vector<int> sp(64, -1);
  std::copy(kern.slot_param.begin(), kern.slot_param.end(), sp.begin());
  GPRX_CUDA_TRY(cudaMemcpyAsync(slot_param.p, sp.data(), sizeof(int) * 64, cudaMemcpyHostToDevice, stream));
  GPRX_CUDA_TRY(cudaStreamSynchronize(stream));
  y_host.assign(yh, yh + n);
  y2 = sumsq_host(y_host);
  for (long long i = 0; i < n; ++i) {
    order.push_back(i);
    ids.push_back(next_id++);
  }
  for (int i = 0; i < m; ++i) inducing_ids.push_back(next_inducing_id++);
  return GPRX_OK;
}

// Capacity of the point buffers (x, y, A): grows ×2 and keeps the contents.
gprx_status SgprState::ensure_points(long long needed) {
  if (needed <= cap && x.p) return GPRX_OK;
  long long new_cap = std::max(needed, std::max(cap, 1LL) * 2);
  if (!x.p) new_cap = needed;
  DevBuf<double> nx, ny, nA;
  if (nx.alloc((size_t)new_cap * d) || ny.alloc(new_cap) || nA.alloc((size_t)ldm * new_cap))
    return set_error(GPRX_OUT_OF_MEMORY, "point buffers");
  if (x.p && n > 0) {
    GPRX_CUDA_TRY(cudaMemcpy2DAsync(nx.p, sizeof(double) * new_cap, x.p, sizeof(double) * cap, sizeof(double) * n,
                                    d, cudaMemcpyDeviceToDevice, stream));
    GPRX_CUDA_TRY(cudaMemcpyAsync(ny.p, y.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, stream));
    if (assembled)
      GPRX_CUDA_TRY(cudaMemcpyAsync(nA.p, Amat.p, sizeof(double) * ldm * n, cudaMemcpyDeviceToDevice, stream));
    GPRX_CUDA_TRY(cudaStreamSynchronize(stream));
  }
  std::swap(x.p, nx.p);
  std::swap(x.n, nx.n);
  std::swap(y.p, ny.p);
  std::swap(y.n, ny.n);
  std::swap(Amat.p, nA.p);
  std::swap(Amat.n, nA.n);
  cap = new_cap;
  G.reset();
  return GPRX_OK;
}

gprx_status SgprState::write_params(const double* params) {
  int p = num_params();
  for (int i = 0; i < p; ++i)
    if (!in_default_interval(params[i])) return set_error(GPRX_INVALID_HYPERPARAMETER, "hyperparameter outside (1e-5, 1e5)");
  gprx_status st = kern.set_theta(params);
  if (st != GPRX_OK) return set_error(st, "invalid kernel hyperparameter");
  log_noise = params[p - 1];
  assembled = false;
  return GPRX_OK;
}


// B = Σ_slices A_s A_sᵀ (+ σ² I on the diagonal), lower or full, by split-K.
static cudaError_t syrk_splitk(const double* A, long long lda, int m, long long n, const double* B, long long ldb,
                               bool lower, double diag, DevBuf<double>& split, double* out, long long ldo,
                               DevStatus* st, cudaStream_t s) {
  int S = (int)std::min<long long>(32, std::max<long long>(1, n / 2048));
  size_t need = (size_t)S * ldo * m;
  if (split.ensure(need) != cudaSuccess) return cudaErrorMemoryAllocation;
  GemmParams p = gemm_params(m, m, (int)std::min<long long>(n, INT32_MAX), A, lda, B, ldb, split.p, ldo, 1.0, 0.0, st);
  p.mode = GEMM_SPLIT_K | (lower ? GEMM_LOWER_TILES : 0);
  p.splits = S;
  p.split_stride = (long long)ldo * m;
  cudaError_t e = dgemm(false, true, p, s);
  if (e != cudaSuccess) return e;
  split_reduce_kernel<<<grid_for((long long)m * m, 256), 256, 0, s>>>(split.p, S, (long long)ldo * m, m, ldo, diag,
                                                                       lower, out, st);
  count_launch();
  return cudaGetLastError();
}

gprx_status SgprState::ensure_emu(EmuWork& w) {
  const int kmax = (int)std::min<long long>(EMU_GROUP, n);
  const size_t bytes = emu_slice_bytes(m, kmax, EMU_S);
  const size_t rows = (size_t)emu_pad_rows(m);
  const int parts = emu_splitk_parts(emu_pad_k(kmax), EMU_PART_K / EMU_KC);
  if (emu_sa.ensure(bytes) || emu_sb.ensure(bytes) || emu_ea.ensure(rows) || emu_eb.ensure(rows) ||
      emu_ma.ensure(rows) || emu_mb.ensure(rows) || emu_err.ensure(1) || emu_part.ensure((size_t)parts * ldm * m))
    return set_error(GPRX_OUT_OF_MEMORY, "device allocation of the emulated-product scratch failed");
  GPRX_CUDA_TRY(emu_err_h.ensure(1));
  w.sa = emu_sa.p; w.sb = emu_sb.p; w.ea = emu_ea.p; w.eb = emu_eb.p; w.ma = emu_ma.p; w.mb = emu_mb.p;
  w.err = emu_err.p;
  w.S = EMU_S;
  return GPRX_OK;
}

// C (m×m, lower part only when lower) = (accumulate ? C : 0) + Σ_z part_z,
// the parts summed in order z = 0, 1, … (deterministic)
__global__ void gram_parts_kernel(const double* part, long long ldp, long long pstride, int nz, int m, bool lower,
                                  bool accumulate, double* C, long long ldc) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < (long long)m * m;
       e += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(e % m), j = (int)(e / m);
    if (lower && i < j) continue;
    double acc = accumulate ? C[i + (long long)j * ldc] : 0.0;
    for (int z = 0; z < nz; ++z) acc += part[z * pstride + i + (long long)j * ldp];
    C[i + (long long)j * ldc] = acc;
  }
}

// C (m×m) = X Yᵀ for X, Y m×nn (rows of length nn), lower or full: n sliced in
// groups of EMU_GROUP columns, each group's product split over K into parts
// of EMU_PART_K computed side by side and summed in FP64.
static cudaError_t emu_gram(const double* X, const double* Y, long long ld, int m, long long nn, bool lower, double* C,
                            long long ldc, const EmuWork& w, double* part, long long ldp, int group, int part_k,
                            cudaStream_t s) {
  cudaError_t e = cudaSuccess;
  const long long pstride = ldp * m;
  for (long long k0 = 0; k0 < nn && e == cudaSuccess; k0 += group) {
    const int kc = (int)std::min<long long>(group, nn - k0);
    EmuOperand a = w.op_a(m, kc);
    e = emu_slice(X + k0 * ld, ld, false, a, s);
    EmuOperand b = a;
    if (e == cudaSuccess && Y != X) {
      b = w.op_b(m, kc);
      e = emu_slice(Y + k0 * ld, ld, false, b, s);
    }
    const int kz = part_k / EMU_KC;
    if (e == cudaSuccess) e = emu_gemm_splitk(a, b, part, ldp, pstride, kz, lower, w.err, s);
    if (e == cudaSuccess) {
      GPRX_LAUNCH(gram_parts_kernel, grid_for((long long)m * m, 256), 256, 0, s, part, ldp, pstride,
                  emu_splitk_parts(a.Kpad, kz), m, lower, k0 > 0, C, ldc);
      e = cudaGetLastError();
    }
  }
  return e;
}

__global__ void add_diag_kernel(double* C, long long ld, int m, double v) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < m) C[i + (long long)i * ld] += v;
}

gprx_status SgprState::assemble() {
  if (n > INT32_MAX) return set_error(GPRX_CAPACITY, "n too large for one assembly");
  const int nn = (int)n;
  std::vector<double> js{0.0};
  auto r = retry_list(opt);
  js.insert(js.end(), r.begin(), r.end());
  bool ok = false;
  gprx_status st;
  GPRX_CUDA_TRY(cudaEventRecord(ev[0], stream));
  for (double j : js) {
    if ((st = reset_status()) != GPRX_OK) return st;
    GPRX_CUDA_TRY(fill_lower(kern, z.p, m, m, Lmm.p, ldm, j, status.p, stream));
    GPRX_CUDA_TRY(potrf_blocked(Lmm.p, ldm, m, linv_mm.p, status.p, stream, &fctx));
    DevStatus ds;
    if ((st = read_status(&ds)) != GPRX_OK) return st;
    if (ds.code == GPRX_OK) {
      ok = true;
      kmm_jitter = j;
      break;
    }
    if (ds.code != GPRX_CHOLESKY_FAILED) return status_to_error(ds, j, m, GPRX_STAGE_FIT);
  }
  if (!ok) return set_cholesky_error(js.back(), m, GPRX_STAGE_FIT);
  pivot_ratio_kernel<<<1, 1024, 0, stream>>>(Lmm.p, ldm, m, res.p + 10);
  count_launch();
  // A = L⁻¹ K(Z, X)
  GPRX_CUDA_TRY(fill_cross(kern, z.p, m, m, x.p, cap, nn, Amat.p, ldm, status.p, stream));
  EmuWork ew;
  const bool emu = use_emu();
  if (emu) {
    if ((st = ensure_emu(ew)) != GPRX_OK) return st;
    GPRX_CUDA_TRY(cudaMemsetAsync(emu_err.p, 0, sizeof(int), stream));
  }
  GPRX_CUDA_TRY(trsm_lower_rec(Lmm.p, ldm, m, linv_mm.p, Amat.p, ldm, nn, TRSM_LEAF, status.p, stream));
  GPRX_CUDA_TRY(cudaEventRecord(ev[1], stream));
  // B = A Aᵀ + σ² I, L_B
  if (emu) {
    GPRX_CUDA_TRY(emu_gram(Amat.p, Amat.p, ldm, m, nn, true, Bl.p, ldm, ew, emu_part.p, ldm, EMU_GROUP, EMU_PART_K,
                           stream));
    add_diag_kernel<<<ceil_div(m, 256), 256, 0, stream>>>(Bl.p, ldm, m, noise());
    count_launch();
  } else {
    GPRX_CUDA_TRY(syrk_splitk(Amat.p, ldm, m, nn, Amat.p, ldm, true, noise(), splitbuf, Bl.p, ldm, status.p, stream));
  }
  GPRX_CUDA_TRY(potrf_blocked(Bl.p, ldm, m, linv_B.p, status.p, stream, &fctx));
  // Σ_c (k_cc − ‖a_c‖²) and A y
  int blocks = grid_for((long long)nn * 32, 1024);
  trace_residual_kernel<<<blocks, 256, 0, stream>>>(Amat.p, ldm, m, nn, kern.diag_value(), partials.p, status.p);
  sum_partials_kernel<<<1, 1024, 0, stream>>>(partials.p, blocks, res.p + 11, status.p);
  count_launch(2);
  {
    int S = (int)std::min<long long>(32, std::max<long long>(1, nn / 4096));
    if (splitbuf.ensure((size_t)S * ldm) != cudaSuccess) return set_error(GPRX_OUT_OF_MEMORY, "split buffer");
    GemmParams p = gemm_params(m, 1, nn, Amat.p, ldm, y.p, nn, splitbuf.p, ldm, 1.0, 0.0, status.p);
    p.mode = GEMM_SPLIT_K;
    p.splits = S;
    p.split_stride = ldm;
    GPRX_CUDA_TRY(dgemm(false, false, p, stream));
    split_reduce_kernel<<<grid_for(m, 256), 256, 0, stream>>>(splitbuf.p, S, ldm, m, 0, 0.0, false, ay.p, status.p);
    count_launch();
  }
  GPRX_CUDA_TRY(cudaMemcpyAsync(res_h.p, res.p + 10, sizeof(double) * 2, cudaMemcpyDeviceToHost, stream));
  if (emu) GPRX_CUDA_TRY(cudaMemcpyAsync(emu_err_h.p, emu_err.p, sizeof(int), cudaMemcpyDeviceToHost, stream));
  if ((st = sync_check(GPRX_STAGE_FIT)) != GPRX_OK) return st;
  if (emu && *emu_err_h.p) return set_error(GPRX_TIMEOUT, "an emulated product's bounded wait ran out");
  pivot_ratio = res_h.p[0];
  trace_sum = res_h.p[1];
  assembled = true;
  sharded = false;
  st = solve_w();
  GPRX_CUDA_TRY(cudaEventRecord(ev[2], stream));
  return st;
}

gprx_status SgprState::solve_w() {
  GPRX_CUDA_TRY(cudaMemcpyAsync(w.p, ay.p, sizeof(double) * m, cudaMemcpyDeviceToDevice, stream));
  GPRX_CUDA_TRY(trsm_lower(Bl.p, ldm, m, linv_B.p, w.p, ldm, 1, status.p, stream));
  GPRX_CUDA_TRY(trsm_lower_t(Bl.p, ldm, m, linv_B.p, w.p, ldm, 1, status.p, stream));
  return sync_check(GPRX_STAGE_FIT);
}

gprx_status SgprState::nlml(double* out) {
  gprx_status st;
  drop_shard_state();
  if (!assembled && (st = assemble()) != GPRX_OK) return st;
  if ((st = reset_status()) != GPRX_OK) return st;
  GPRX_CUDA_TRY(logdet_diag(Bl.p, ldm, m, false, res.p + 0, status.p, stream));
  GPRX_CUDA_TRY(dot_dev(ay.p, w.p, m, res.p + 1, status.p, stream));
  GPRX_CUDA_TRY(cudaMemcpyAsync(res_h.p, res.p, sizeof(double) * 2, cudaMemcpyDeviceToHost, stream));
  if ((st = sync_check(GPRX_STAGE_FIT)) != GPRX_OK) return st;
  const double noise_v = noise();
  const double logdet = ((double)n - (double)m) * std::log(noise_v) + res_h.p[0];
  const double quad = (y2 - res_h.p[1]) / noise_v;
  const double trace = trace_sum / (2.0 * noise_v);
  *out = 0.5 * ((double)n * std::log(2.0 * M_PI) + logdet + quad) + trace;
  return GPRX_OK;
}

gprx_status SgprState::gradient(double* grad) {
  const int nn = (int)n;
  const double noise_v = noise();
  gprx_status st;
  if (G.ensure((size_t)ldm * std::max(cap, 1LL)) != cudaSuccess || H.ensure((size_t)ldm * m) != cudaSuccess ||
      Wm.ensure((size_t)ldm * m) != cudaSuccess || Xb.ensure((size_t)ldm * m) != cudaSuccess ||
      Xt.ensure((size_t)ldm * m) != cudaSuccess)
    return set_error(GPRX_OUT_OF_MEMORY, "gradient buffers");
  if ((st = reset_status()) != GPRX_OK) return st;
  // G = B⁻¹ A − (w rᵀ + A)/σ²: B⁻¹ A by the two triangular solves (an
  // explicit B⁻¹ would carry cond(B)·ε into the small residual G)
  const bool emu = use_emu();
  EmuWork ew;
  if (emu) {
    if ((st = ensure_emu(ew)) != GPRX_OK) return st;
    GPRX_CUDA_TRY(cudaMemsetAsync(emu_err.p, 0, sizeof(int), stream));
  }
  GPRX_CUDA_TRY(cudaMemcpyAsync(G.p, Amat.p, sizeof(double) * ldm * nn, cudaMemcpyDeviceToDevice, stream));
  GPRX_CUDA_TRY(trsm_lower_rec(Bl.p, ldm, m, linv_B.p, G.p, ldm, nn, TRSM_LEAF, status.p, stream));
  GPRX_CUDA_TRY(trsm_lower_t_rec(Bl.p, ldm, m, linv_B.p, G.p, ldm, nn, TRSM_LEAF, status.p, stream));
  adjoint_update_kernel<<<grid_for((long long)nn * 32, 256), 256, 0, stream>>>(Amat.p, G.p, ldm, m, nn, w.p, y.p,
                                                                                1.0 / noise_v, status.p);
  count_launch();
  // H = G Aᵀ; w_mn = L⁻ᵀ G
  if (emu) {
    GPRX_CUDA_TRY(emu_gram(G.p, Amat.p, ldm, m, nn, false, H.p, ldm, ew, emu_part.p, ldm, EMU_GROUP, EMU_PART_K,
                           stream));
  } else {
    GPRX_CUDA_TRY(syrk_splitk(G.p, ldm, m, nn, Amat.p, ldm, false, 0.0, splitbuf, H.p, ldm, status.p, stream));
  }
  GPRX_CUDA_TRY(trsm_lower_t_rec(Lmm.p, ldm, m, linv_mm.p, G.p, ldm, nn, TRSM_LEAF, status.p, stream));
  // w_mm = −sym(L⁻ᵀ tril½(H) L⁻¹)
  tril_half_kernel<<<grid_for((long long)m * m, 256), 256, 0, stream>>>(H.p, ldm, m, Xb.p);
  count_launch();
  GPRX_CUDA_TRY(trsm_lower_t(Lmm.p, ldm, m, linv_mm.p, Xb.p, ldm, m, status.p, stream));
  {
    dim3 tb(32, 8), tg(ceil_div(m, 32), ceil_div(m, 32));
    transpose_kernel<<<tg, tb, 0, stream>>>(Xb.p, ldm, m, Xt.p);
    count_launch();
  }
  GPRX_CUDA_TRY(trsm_lower_t(Lmm.p, ldm, m, linv_mm.p, Xt.p, ldm, m, status.p, stream));
  neg_sym_half_kernel<<<grid_for((long long)m * m, 256), 256, 0, stream>>>(Xt.p, ldm, m, Wm.p);
  count_launch();
  // contractions: ⟨w_mm, ∂K_mm⟩ (lower, weights 1 / 2) and ⟨w_mn, ∂K(Z, X)⟩
  int b1 = 0, b2 = 0;
  const int ns = grad_slots(kern.ard_d);
  GPRX_CUDA_TRY(grad_contract(kern, z.p, m, m, Wm.p, ldm, nullptr, partials.p, &b1, status.p, stream));
  GPRX_CUDA_TRY(cross_contract(kern, z.p, m, m, x.p, cap, nn, G.p, ldm, partials.p + (long long)b1 * ns, &b2,
                               status.p, stream));
  GPRX_CUDA_TRY(grad_finalize(kern, partials.p, b1 + b2, slot_param.p, 1.0, 0.0, res.p + 20, status.p, stream));
  // tr(B⁻¹) = ‖L_B⁻¹‖²_F and ‖w‖²
  GPRX_CUDA_TRY(cudaMemsetAsync(Xt.p, 0, sizeof(double) * ldm * m, stream));
  if (H.ensure((size_t)((m + 1) / 2) * ((m + 1) / 2) + 1) != cudaSuccess) return set_error(GPRX_OUT_OF_MEMORY, "scratch");
  GPRX_CUDA_TRY(trtri_blocked(Bl.p, ldm, m, linv_B.p, Xt.p, ldm, H.p, status.p, stream));
  int blocks = grid_for((long long)m * m, 1024);
  sumsq_kernel<<<blocks, 256, 0, stream>>>(Xt.p, ldm, m, m, partials.p + 8192, status.p);
  sum_partials_kernel<<<1, 1024, 0, stream>>>(partials.p + 8192, blocks, res.p + 2, status.p);
  count_launch(2);
  GPRX_CUDA_TRY(dot_dev(w.p, w.p, m, res.p + 3, status.p, stream));
  GPRX_CUDA_TRY(dot_dev(ay.p, w.p, m, res.p + 4, status.p, stream));
  GPRX_CUDA_TRY(cudaMemcpyAsync(res_h.p, res.p, sizeof(double) * 128, cudaMemcpyDeviceToHost, stream));
  if (emu) GPRX_CUDA_TRY(cudaMemcpyAsync(emu_err_h.p, emu_err.p, sizeof(int), cudaMemcpyDeviceToHost, stream));
  if ((st = sync_check(GPRX_STAGE_FIT)) != GPRX_OK) return st;
  if (emu && *emu_err_h.p) return set_error(GPRX_TIMEOUT, "an emulated product's bounded wait ran out");
  const int nk = kern.n_params;
  std::vector<double> dg;
  diag_grad(kern, dg);
  const double wdiag = 0.5 / noise_v;
  for (int i = 0; i < nk; ++i) grad[i] = res_h.p[20 + i] + wdiag * (double)n * dg[i];
  // directional_noise (derivatives.rs:186-202) with ∂σ² = σ²
  const double trb = res_h.p[2], ww = res_h.p[3], ayw = res_h.p[4];
  const double quad = (y2 - ayw) / noise_v;
  const double trace = trace_sum / (2.0 * noise_v);
  const double dn = noise_v;
  const double d_logdet_b = dn * trb;
  const double d_q = -dn * ww;
  const double d_quad = -d_q / noise_v - quad * dn / noise_v;
  const double d_trace = -trace * dn / noise_v;
  grad[nk] = 0.5 * (((double)n - (double)m) * dn / noise_v + d_logdet_b + d_quad) + d_trace;
  GPRX_CUDA_TRY(cudaEventRecord(ev[3], stream));
  return GPRX_OK;
}

gprx_status SgprState::eval(const double* params, double* nlml_out, double* grad) {
  const int p = num_params();
  std::vector<double> prev(p);
  get_params(prev.data());
  gprx_status st = write_params(params);
  if (st != GPRX_OK) return st;
  st = assemble();
  if (st == GPRX_OK) st = nlml(nlml_out);
  if (st == GPRX_OK && grad) st = gradient(grad);
  if (st != GPRX_OK) {
    gprx_error_info saved = last_error();
    write_params(prev.data());
    assemble();
    last_error() = saved;
    return st;
  }
  if (!std::isfinite(*nlml_out)) return set_error(GPRX_NOT_CONVERGED, "non-finite NLML");
  return GPRX_OK;
}

gprx_status SgprState::predict(const double* xs, uint64_t q, int kind, double* mean, double* var) {
  if (!xs || !mean || !var) return set_error(GPRX_INVALID_ARGUMENT, "null pointer");
  if (kind != GPRX_VARIANCE_LATENT && kind != GPRX_VARIANCE_OBSERVATION)
    return set_error(GPRX_INVALID_ARGUMENT, "variance kind");
  if (q == 0) return GPRX_OK;
  if (!all_finite(xs, q * d)) return set_error(GPRX_NONFINITE_INPUT, "non-finite query");
  gprx_status st;
  if (!assembled && (st = assemble()) != GPRX_OK) return st;
  const int qc_max = (int)std::max<long long>(1, std::min<long long>((long long)q, (1LL << 26) / std::max(m, 1)));
  if (qbuf.ensure((size_t)ldm * qc_max) || qbuf2.ensure((size_t)ldm * qc_max) ||
      qx.ensure((size_t)qc_max * (d + 4)))
    return set_error(GPRX_OUT_OF_MEMORY, "predict scratch");
  HostPinned<double> hm;
  GPRX_CUDA_TRY(hm.ensure(2 * (size_t)qc_max));
  const double kss = kern.diag_value();
  if ((st = reset_status()) != GPRX_OK) return st;
  for (uint64_t c0 = 0; c0 < q; c0 += qc_max) {
    int qc = (int)std::min<uint64_t>(qc_max, q - c0);
    double* xq = qx.p;
    double* mdev = qx.p + (size_t)qc_max * d;
    double* vdev = mdev + qc_max;
    double* an = vdev + qc_max;
    double* bn = an + qc_max;
    GPRX_CUDA_TRY(cudaMemcpy2DAsync(xq, sizeof(double) * qc, xs + c0, sizeof(double) * q, sizeof(double) * qc, d,
                                    cudaMemcpyHostToDevice, stream));
    GPRX_CUDA_TRY(fill_cross(kern, z.p, m, m, xq, qc, qc, qbuf.p, ldm, status.p, stream));
    GPRX_CUDA_TRY(trsm_lower(Lmm.p, ldm, m, linv_mm.p, qbuf.p, ldm, qc, status.p, stream));
    GPRX_CUDA_TRY(gemv_t(qbuf.p, ldm, m, qc, false, w.p, mdev, status.p, stream));
    GPRX_CUDA_TRY(col_sumsq(qbuf.p, ldm, m, qc, nullptr, an, status.p, stream));
    GPRX_CUDA_TRY(cudaMemcpyAsync(qbuf2.p, qbuf.p, sizeof(double) * ldm * qc, cudaMemcpyDeviceToDevice, stream));
    GPRX_CUDA_TRY(trsm_lower(Bl.p, ldm, m, linv_B.p, qbuf2.p, ldm, qc, status.p, stream));
    GPRX_CUDA_TRY(col_sumsq(qbuf2.p, ldm, m, qc, nullptr, bn, status.p, stream));
    sgpr_finish_var_kernel<<<ceil_div(qc, 256), 256, 0, stream>>>(an, bn, qc, kss, noise(), kind, vdev, status.p);
    count_launch();
    GPRX_CUDA_TRY(cudaMemcpyAsync(hm.p, mdev, sizeof(double) * qc, cudaMemcpyDeviceToHost, stream));
    GPRX_CUDA_TRY(cudaMemcpyAsync(hm.p + qc_max, vdev, sizeof(double) * qc, cudaMemcpyDeviceToHost, stream));
    if ((st = sync_check(GPRX_STAGE_PREDICT)) != GPRX_OK) return st;
    std::copy(hm.p, hm.p + qc, mean + c0);
    std::copy(hm.p + qc_max, hm.p + qc_max + qc, var + c0);
  }
  return GPRX_OK;
}

// covariance: lower triangle K** − A*ᵀA* + σn² S*ᵀS* mirrored off the
// diagonal, the predictive variance on it
__global__ void sgpr_cov_finish_kernel(double* C, int q, const double* var) {
  const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (e >= (long long)q * q) return;
  const int i = (int)(e % q), j = (int)(e / q);
  if (i == j) C[e] = var[i];
  else if (i < j) C[e] = C[j + (long long)i * q];
}

// The VFE query covariance on the device (predict_vfe_covariance,
// src/sgpr/factor/predict.rs:263-345; SparseCore::finish_covariance,
// src/sparse/core.rs:641-667) into covbuf (q×q, both triangles).
gprx_status SgprState::covariance_dev(const double* xs, uint64_t q, int kind, double* mean_host) {
  if (kind != GPRX_VARIANCE_LATENT && kind != GPRX_VARIANCE_OBSERVATION)
    return set_error(GPRX_INVALID_ARGUMENT, "variance kind");
  if (q > (uint64_t)INT32_MAX) return set_error(GPRX_CAPACITY, "too many query points");
  if (!all_finite(xs, q * d)) return set_error(GPRX_NONFINITE_INPUT, "non-finite query");
  gprx_status st;
  if (!assembled && (st = assemble()) != GPRX_OK) return st;
  const int qi = (int)q;
  if (qbuf.ensure((size_t)ldm * q) || qbuf2.ensure((size_t)ldm * q) || qx.ensure((size_t)q * (d + 4)) ||
      covbuf.ensure((size_t)q * q))
    return set_error(GPRX_OUT_OF_MEMORY, "covariance buffers");
  double* xq = qx.p;
  double* mdev = qx.p + (size_t)q * d;
  double* vdev = mdev + q;
  double* an = vdev + q;
  double* bn = an + q;
  if ((st = reset_status()) != GPRX_OK) return st;
  GPRX_CUDA_TRY(cudaMemcpyAsync(xq, xs, sizeof(double) * q * d, cudaMemcpyHostToDevice, stream));
  GPRX_CUDA_TRY(fill_cross(kern, z.p, m, m, xq, qi, qi, qbuf.p, ldm, status.p, stream));
  GPRX_CUDA_TRY(trsm_lower(Lmm.p, ldm, m, linv_mm.p, qbuf.p, ldm, qi, status.p, stream));
  GPRX_CUDA_TRY(gemv_t(qbuf.p, ldm, m, qi, false, w.p, mdev, status.p, stream));
  GPRX_CUDA_TRY(col_sumsq(qbuf.p, ldm, m, qi, nullptr, an, status.p, stream));
  GPRX_CUDA_TRY(cudaMemcpyAsync(qbuf2.p, qbuf.p, sizeof(double) * ldm * q, cudaMemcpyDeviceToDevice, stream));
  GPRX_CUDA_TRY(trsm_lower(Bl.p, ldm, m, linv_B.p, qbuf2.p, ldm, qi, status.p, stream));
  GPRX_CUDA_TRY(col_sumsq(qbuf2.p, ldm, m, qi, nullptr, bn, status.p, stream));
  sgpr_finish_var_kernel<<<ceil_div(qi, 256), 256, 0, stream>>>(an, bn, qi, kern.diag_value(), noise(), kind, vdev,
                                                                   status.p);
  count_launch();
  GPRX_CUDA_TRY(fill_lower(kern, xq, qi, qi, covbuf.p, qi, 0.0, status.p, stream));
  GemmParams pa = gemm_params(qi, qi, m, qbuf.p, ldm, qbuf.p, ldm, covbuf.p, qi, -1.0, 1.0, status.p);
  pa.mode = GEMM_LOWER_TILES;
  GPRX_CUDA_TRY(dgemm(true, false, pa, stream));
  GemmParams pb = gemm_params(qi, qi, m, qbuf2.p, ldm, qbuf2.p, ldm, covbuf.p, qi, noise(), 1.0, status.p);
  pb.mode = GEMM_LOWER_TILES;
  GPRX_CUDA_TRY(dgemm(true, false, pb, stream));
  sgpr_cov_finish_kernel<<<(int)(((long long)qi * qi + 255) / 256), 256, 0, stream>>>(covbuf.p, qi, vdev);
  count_launch();
  GPRX_CUDA_TRY(cudaGetLastError());
  GPRX_CUDA_TRY(cudaMemcpyAsync(mean_host, mdev, sizeof(double) * q, cudaMemcpyDeviceToHost, stream));
  return sync_check(GPRX_STAGE_PREDICT);
}

gprx_status SgprState::predict_covariance(const double* xs, uint64_t q, int kind, double* mean, double* cov) {
  if (!xs || !mean || !cov) return set_error(GPRX_INVALID_ARGUMENT, "null pointer");
  if (q == 0) return GPRX_OK;
  gprx_status st = covariance_dev(xs, q, kind, mean);
  if (st != GPRX_OK) return st;
  GPRX_CUDA_TRY(cudaMemcpyAsync(cov, covbuf.p, sizeof(double) * q * q, cudaMemcpyDeviceToHost, stream));
  GPRX_CUDA_TRY(cudaStreamSynchronize(stream));
  return GPRX_OK;
}

// FittedSgpr::sample_with (src/sgpr/fitted.rs:855-900): the exact model's
// draw from the VFE covariance, with this model's jitter retries.
gprx_status SgprState::sample(const double* xs, uint64_t q, int kind, uint64_t n_draws, uint64_t seed,
                              double* out) {
  if (!xs || (n_draws > 0 && !out)) return set_error(GPRX_INVALID_ARGUMENT, "null pointer");
  if (q == 0) return GPRX_OK;
  if (n_draws > (uint64_t)INT32_MAX) return set_error(GPRX_CAPACITY, "too many draws");
  std::vector<double> mean(q);
  gprx_status st = covariance_dev(xs, q, kind, mean.data());
  if (st != GPRX_OK || n_draws == 0) return st;
  return draw_posterior(covbuf.p, (int)q, mean.data(), n_draws, seed, jitter_attempts(opt), covl, covlinv, zbuf,
                        status.p, stream, [&] { return reset_status(); },
                        [&](DevStatus* ds) { return read_status(ds); }, out);
}

gprx_status SgprState::insert(const double* xnew, double ynew, uint64_t* id) {
  if (!xnew || !id) return set_error(GPRX_INVALID_ARGUMENT, "null pointer");
  if (!all_finite(xnew, d) || !std::isfinite(ynew)) return set_error(GPRX_NONFINITE_INPUT, "non-finite point");
  gprx_status st;
  drop_shard_state();
  if (!assembled && (st = assemble()) != GPRX_OK) return st;
  if ((st = ensure_points(n + 1)) != GPRX_OK) return st;
  const long long slot = n;
  GPRX_CUDA_TRY(cudaMemcpy2DAsync(x.p + slot, sizeof(double) * cap, xnew, sizeof(double), sizeof(double), d,
                                  cudaMemcpyHostToDevice, stream));
  GPRX_CUDA_TRY(cudaMemcpyAsync(y.p + slot, &ynew, sizeof(double), cudaMemcpyHostToDevice, stream));
  GPRX_CUDA_TRY(cudaStreamSynchronize(stream));
  const bool in_place = pivot_ratio > X_STEP_PIVOT_RTOL;
  n += 1;
  y_host.push_back(ynew);
  y2 += ynew * ynew;
  order.push_back(slot);
  *id = next_id++;
  ids.push_back(*id);
  if (!in_place) {
    last_in_place = 0;
    return assemble();
  }
  if ((st = reset_status()) != GPRX_OK) return st;
  // a = L⁻¹ k(Z, x) into A's new column; sums; L_B rank-1 update; w again
  double* col = Amat.p + slot * ldm;
  GPRX_CUDA_TRY(fill_cross(kern, z.p, m, m, x.p + slot, cap, 1, col, ldm, status.p, stream));
  GPRX_CUDA_TRY(trsm_lower(Lmm.p, ldm, m, linv_mm.p, col, ldm, 1, status.p, stream));
  GPRX_CUDA_TRY(dot_dev(col, col, m, res.p + 12, status.p, stream));
  axpy_kernel<<<ceil_div(m, 256), 256, 0, stream>>>(ay.p, col, ynew, m);
  count_launch();
  GPRX_CUDA_TRY(cudaMemcpyAsync(vtmp.p, col, sizeof(double) * m, cudaMemcpyDeviceToDevice, stream));
  chol_rank1_kernel<<<1, R1C_THREADS, 0, stream>>>(Bl.p, ldm, m, vtmp.p, 1.0, status.p);
  count_launch();
  GPRX_CUDA_TRY(tri_inv_blocks(Bl.p, ldm, m, false, linv_B.p, status.p, stream));
  GPRX_CUDA_TRY(cudaMemcpyAsync(res_h.p, res.p + 12, sizeof(double), cudaMemcpyDeviceToHost, stream));
  if ((st = sync_check(GPRX_STAGE_ONLINE_INSERT)) != GPRX_OK) return st;
  trace_sum += kern.diag_value() - res_h.p[0];
  last_in_place = 1;
  return solve_w();
}

gprx_status SgprState::remove(uint64_t id) {
  if (n <= 1) return set_error(GPRX_INSUFFICIENT_DATA, "an online model keeps at least one point");
  auto it = std::lower_bound(ids.begin(), ids.end(), id);
  if (it == ids.end() || *it != id) return set_error(GPRX_INVALID_POINT_ID, "unknown point id");
  const long long idx = it - ids.begin();
  gprx_status st;
  drop_shard_state();
  if (!assembled && (st = assemble()) != GPRX_OK) return st;
  const long long slot = order[idx], last = n - 1;
  const double ydel = y_host[slot];
  bool ok = pivot_ratio > X_STEP_PIVOT_RTOL;
  if (ok) {
    // trial downdate of L_B with the point's column of A
    // the trial factor becomes L_B on success: it keeps L_B's ld columns
    if (Btrial.ensure((size_t)ldm * ldm) != cudaSuccess) return set_error(GPRX_OUT_OF_MEMORY, "trial factor");
    if ((st = reset_status()) != GPRX_OK) return st;
    const double* col = Amat.p + slot * ldm;
    GPRX_CUDA_TRY(cudaMemcpyAsync(Btrial.p, Bl.p, sizeof(double) * ldm * m, cudaMemcpyDeviceToDevice, stream));
    GPRX_CUDA_TRY(cudaMemcpyAsync(vtmp.p, col, sizeof(double) * m, cudaMemcpyDeviceToDevice, stream));
    GPRX_CUDA_TRY(dot_dev(col, col, m, res.p + 12, status.p, stream));
    chol_rank1_kernel<<<1, R1C_THREADS, 0, stream>>>(Btrial.p, ldm, m, vtmp.p, -1.0, status.p);
    count_launch();
    DevStatus ds;
    GPRX_CUDA_TRY(cudaMemcpyAsync(res_h.p, res.p + 12, sizeof(double), cudaMemcpyDeviceToHost, stream));
    if ((st = read_status(&ds)) != GPRX_OK) return st;
    if (ds.code == GPRX_CHOLESKY_FAILED) ok = false;
    else if (ds.code != GPRX_OK) return status_to_error(ds, 0.0, m, GPRX_STAGE_ONLINE_DELETE);
    if (ok) {
      trace_sum -= kern.diag_value() - res_h.p[0];
      axpy_kernel<<<ceil_div(m, 256), 256, 0, stream>>>(ay.p, col, -ydel, m);
      count_launch();
      std::swap(Bl.p, Btrial.p);
      std::swap(Bl.n, Btrial.n);
      GPRX_CUDA_TRY(tri_inv_blocks(Bl.p, ldm, m, false, linv_B.p, status.p, stream));
    }
  }
  // the last slot moves into the freed one (A column, x row, y)
  if (slot != last) {
    if (assembled)
      GPRX_CUDA_TRY(cudaMemcpyAsync(Amat.p + slot * ldm, Amat.p + last * ldm, sizeof(double) * m,
                                    cudaMemcpyDeviceToDevice, stream));
    GPRX_CUDA_TRY(cudaMemcpy2DAsync(x.p + slot, sizeof(double) * cap, x.p + last, sizeof(double) * cap,
                                    sizeof(double), d, cudaMemcpyDeviceToDevice, stream));
    GPRX_CUDA_TRY(cudaMemcpyAsync(y.p + slot, y.p + last, sizeof(double), cudaMemcpyDeviceToDevice, stream));
    y_host[slot] = y_host[last];
    for (auto& o : order)
      if (o == last) o = slot;
  }
  y_host.pop_back();
  y2 -= ydel * ydel;
  order.erase(order.begin() + idx);
  ids.erase(it);
  n -= 1;
  if (!ok) {
    last_in_place = 0;
    y2 = sumsq_host(y_host);
    return assemble();
  }
  last_in_place = 1;
  return solve_w();
}

// The inducing points as the host sees them (m×d column-major).
static gprx_status download_z(SgprState& s, std::vector<double>& out) {
  out.resize((size_t)s.m * s.d);
  GPRX_CUDA_TRY(cudaMemcpyAsync(out.data(), s.z.p, sizeof(double) * out.size(), cudaMemcpyDeviceToHost, s.stream));
  GPRX_CUDA_TRY(cudaStreamSynchronize(s.stream));
  return GPRX_OK;
}

// Assembles the VFE system of a changed inducing set; on failure the model
// goes back to the set it had (OnlineSgpr::atomically).  An insert takes the
// bordered update below when its gates hold; a delete, and an insert whose
// gates do not hold, assemble the new set (the reference's own fallback,
// O(n m²)), so their results are those of Sgpr::factor at the same θ, X and
// Z.  The reference's trailing delete (a rank-1 update of L_mm, then A solved
// against it from K(Z, X) = L A and B formed again) keeps the assembly's
// O(n m²) solve and Gram product and saves only the kernel evaluations of
// K(Z, X), which on the GPU cost a small part of the assembly; the delete
// takes the assembly.
gprx_status SgprState::replace_inducing(const std::vector<double>& znew, int mm) {
  std::vector<double> old;
  gprx_status st = download_z(*this, old);
  if (st != GPRX_OK) return st;
  const int m_old = m;
  st = set_inducing(znew.data(), (uint64_t)mm);
  if (st != GPRX_OK) {
    gprx_error_info saved = last_error();
    set_inducing(old.data(), (uint64_t)m_old);
    last_error() = saved;
  }
  return st;
}

gprx_status SgprState::a_times(const double* v, double* out) {
  const int nn = (int)n;
  const int S = (int)std::min<long long>(32, std::max<long long>(1, nn / 4096));
  if (splitbuf.ensure((size_t)S * ldm) != cudaSuccess) return set_error(GPRX_OUT_OF_MEMORY, "split buffer");
  GemmParams p = gemm_params(m, 1, nn, Amat.p, ldm, v, nn, splitbuf.p, ldm, 1.0, 0.0, status.p);
  p.mode = GEMM_SPLIT_K;
  p.splits = S;
  p.split_stride = ldm;
  GPRX_CUDA_TRY(dgemm(false, false, p, stream));
  split_reduce_kernel<<<grid_for(m, 256), 256, 0, stream>>>(splitbuf.p, S, ldm, m, 0, 0.0, false, out, status.p);
  count_launch();
  return GPRX_OK;
}

// OnlineSgpr::insert_inducing by the bordered update (inducing_append,
// src/sgpr/factor/updates.rs:296-390; ADR 0005): from a factor of K_mm without
// jitter whose pivots hold (min L_ii² / K_ii > 1e-5), l = L⁻¹ k(Z, z),
// ℓ² = k(z, z) − ‖l‖², the new row of A a = (k(z, X) − Aᵀ l) / ℓ (O(n m)),
// b = L_B⁻¹ (A a), β² = σ² + ‖a‖² − ‖b‖²; both bordered pivots must exceed
// 1e-5 of the diagonal they cancel from.  Needs room for row m in the
// buffers (m + 1 ≤ ld and the same number of diagonal blocks); otherwise,
// or when a gate does not hold, *applied is false and nothing changed.
gprx_status SgprState::insert_inducing_bordered(const double* znew, bool* applied) {
  *applied = false;
  constexpr double TAU = 1e-5;
  if (kmm_jitter > 0.0 || !(pivot_ratio > TAU)) return GPRX_OK;
  if (m + 1 > ldm || ceil_div(m + 1, NB) != ceil_div(m, NB) || n > INT32_MAX) return GPRX_OK;
  const size_t need = (size_t)ldm * (size_t)(m + 1);
  if (Lmm.n < need || Bl.n < need || linv_mm.n < (size_t)ceil_div(m + 1, NB) * NB * NB ||
      linv_B.n < (size_t)ceil_div(m + 1, NB) * NB * NB || Amat.n < (size_t)ldm * (size_t)std::max(cap, 1LL))
    return GPRX_OK;
  gprx_status st;
  if (!assembled && (st = assemble()) != GPRX_OK) return st;
  const int nn = (int)n;
  if (border.ensure((size_t)3 * std::max(cap, 1LL) + 2 * ldm + d) != cudaSuccess)
    return set_error(GPRX_OUT_OF_MEMORY, "border buffers");
  double* krow = border.p;               // k(z, X) (n)
  double* atl = krow + cap;              // Aᵀ l (n)
  double* arow = atl + cap;              // the new row of A (n)
  double* lvec = arow + cap;             // l (m)
  double* bvec = lvec + ldm;             // b (m)
  double* zdev = bvec + ldm;             // z (d)
  if ((st = reset_status()) != GPRX_OK) return st;
  GPRX_CUDA_TRY(cudaMemcpyAsync(zdev, znew, sizeof(double) * d, cudaMemcpyHostToDevice, stream));
  GPRX_CUDA_TRY(fill_cross(kern, z.p, m, m, zdev, 1, 1, lvec, ldm, status.p, stream));
  GPRX_CUDA_TRY(trsm_lower(Lmm.p, ldm, m, linv_mm.p, lvec, ldm, 1, status.p, stream));
  GPRX_CUDA_TRY(dot_dev(lvec, lvec, m, res.p + 30, status.p, stream));
  GPRX_CUDA_TRY(cudaMemcpyAsync(res_h.p + 30, res.p + 30, sizeof(double), cudaMemcpyDeviceToHost, stream));
  if ((st = sync_check(GPRX_STAGE_ONLINE_INSERT)) != GPRX_OK) return st;
  const double kdiag = kern.diag_value() + kmm_jitter;
  const double ell2 = kdiag - res_h.p[30];
  if (!(std::isfinite(ell2) && ell2 > TAU * kdiag)) return GPRX_OK;
  const double ell = std::sqrt(ell2);
  // a = (k(z, X) − Aᵀ l) / ℓ; ‖a‖², a·y; b = L_B⁻¹ (A a)
  GPRX_CUDA_TRY(fill_cross(kern, zdev, 1, 1, x.p, cap, nn, krow, 1, status.p, stream));
  GPRX_CUDA_TRY(gemv_t(Amat.p, ldm, m, nn, false, lvec, atl, status.p, stream));
  border_a_row_kernel<<<grid_for(nn, 256), 256, 0, stream>>>(krow, atl, 1.0 / ell, Amat.p, ldm, m, nn, arow);
  count_launch();
  if ((st = a_times(arow, bvec)) != GPRX_OK) return st;
  GPRX_CUDA_TRY(trsm_lower(Bl.p, ldm, m, linv_B.p, bvec, ldm, 1, status.p, stream));
  GPRX_CUDA_TRY(dot_dev(arow, arow, nn, res.p + 31, status.p, stream));
  GPRX_CUDA_TRY(dot_dev(bvec, bvec, m, res.p + 32, status.p, stream));
  GPRX_CUDA_TRY(cudaMemcpyAsync(res_h.p + 31, res.p + 31, sizeof(double) * 2, cudaMemcpyDeviceToHost, stream));
  if ((st = sync_check(GPRX_STAGE_ONLINE_INSERT)) != GPRX_OK) return st;
  const double an2 = res_h.p[31];
  const double bdiag = noise() + an2;
  const double beta2 = bdiag - res_h.p[32];
  if (!(std::isfinite(beta2) && beta2 > TAU * bdiag)) return GPRX_OK;  // row m of A is scratch beyond m
  // commit: Z, the bordered L and L_B and their diagonal-block inverses, A y, w
  std::vector<double> zo, zn((size_t)(m + 1) * d);
  if ((st = download_z(*this, zo)) != GPRX_OK) return st;
  for (int f = 0; f < d; ++f) {
    std::copy(zo.begin() + (size_t)f * m, zo.begin() + (size_t)(f + 1) * m, zn.begin() + (size_t)f * (m + 1));
    zn[(size_t)f * (m + 1) + m] = znew[f];
  }
  if (z.alloc(zn.size()) != cudaSuccess) return set_error(GPRX_OUT_OF_MEMORY, "inducing points");
  GPRX_CUDA_TRY(cudaMemcpyAsync(z.p, zn.data(), sizeof(double) * zn.size(), cudaMemcpyHostToDevice, stream));
  border_row_kernel<<<ceil_div(m + 1, 256), 256, 0, stream>>>(Lmm.p, ldm, m, lvec, ell);
  border_row_kernel<<<ceil_div(m + 1, 256), 256, 0, stream>>>(Bl.p, ldm, m, bvec, std::sqrt(beta2));
  count_launch(2);
  m += 1;
  GPRX_CUDA_TRY(tri_inv_blocks(Lmm.p, ldm, m, false, linv_mm.p, status.p, stream));
  GPRX_CUDA_TRY(tri_inv_blocks(Bl.p, ldm, m, false, linv_B.p, status.p, stream));
  if ((st = a_times(y.p, ay.p)) != GPRX_OK) return st;
  pivot_ratio_kernel<<<1, 1024, 0, stream>>>(Lmm.p, ldm, m, res.p + 10);
  count_launch();
  GPRX_CUDA_TRY(cudaMemcpyAsync(res_h.p + 10, res.p + 10, sizeof(double), cudaMemcpyDeviceToHost, stream));
  if ((st = sync_check(GPRX_STAGE_ONLINE_INSERT)) != GPRX_OK) return st;
  pivot_ratio = res_h.p[10];
  trace_sum -= an2;
  *applied = true;
  last_in_place = 1;
  return solve_w();
}

gprx_status SgprState::insert_inducing(const double* znew, uint64_t* id) {
  if (!znew || !id) return set_error(GPRX_INVALID_ARGUMENT, "null pointer");
  if (!all_finite(znew, d)) return set_error(GPRX_NONFINITE_INPUT, "non-finite inducing point");
  drop_shard_state();
  bool applied = false;
  gprx_status st = insert_inducing_bordered(znew, &applied);
  if (st != GPRX_OK) {
    // a device failure part way: go back to the current set by assembly
    gprx_error_info saved = last_error();
    std::vector<double> zo;
    if (download_z(*this, zo) == GPRX_OK) set_inducing(zo.data(), (uint64_t)m);
    last_error() = saved;
    return st;
  }
  if (applied) {
    *id = next_inducing_id++;
    inducing_ids.push_back(*id);
    return GPRX_OK;
  }
  last_in_place = 0;
  std::vector<double> zo, zn((size_t)(m + 1) * d);
  st = download_z(*this, zo);
  if (st != GPRX_OK) return st;
  for (int f = 0; f < d; ++f) {  // append a row (column-major)
    std::copy(zo.begin() + (size_t)f * m, zo.begin() + (size_t)(f + 1) * m, zn.begin() + (size_t)f * (m + 1));
    zn[(size_t)f * (m + 1) + m] = znew[f];
  }
  if ((st = replace_inducing(zn, m + 1)) != GPRX_OK) return st;
  *id = next_inducing_id++;
  inducing_ids.push_back(*id);
  return GPRX_OK;
}

gprx_status SgprState::delete_inducing(uint64_t id) {
  if (m <= 1) return set_error(GPRX_INSUFFICIENT_DATA, "an inducing delete needs at least 2 inducing points");
  auto it = std::find(inducing_ids.begin(), inducing_ids.end(), id);
  if (it == inducing_ids.end()) return set_error(GPRX_INVALID_POINT_ID, "unknown inducing id " + std::to_string(id));
  const int idx = (int)(it - inducing_ids.begin());
  std::vector<double> zo, zn;
  gprx_status st = download_z(*this, zo);
  if (st != GPRX_OK) return st;
  zn.reserve((size_t)(m - 1) * d);
  for (int f = 0; f < d; ++f)
    for (int i = 0; i < m; ++i)
      if (i != idx) zn.push_back(zo[(size_t)f * m + i]);
  drop_shard_state();
  last_in_place = 0;
  if ((st = replace_inducing(zn, m - 1)) != GPRX_OK) return st;
  inducing_ids.erase(inducing_ids.begin() + idx);
  return GPRX_OK;
}

gprx_status SgprState::set_inducing(const double* zh, uint64_t mm) {
  if (!zh) return set_error(GPRX_INVALID_ARGUMENT, "null pointer");
  if (mm == 0) return set_error(GPRX_EMPTY_INPUT, "no inducing points");
  if (!all_finite(zh, mm * d)) return set_error(GPRX_NONFINITE_INPUT, "non-finite inducing point");
  int new_ldm = (int)round_ld((long long)mm);
  if ((int)mm != m) {
    int nblk = ceil_div((int)mm, NB);
    // A is re-laid out for the new m (its contents are recomputed below)
    DevBuf<double> nA;
    if (z.alloc((size_t)mm * d) || Lmm.alloc((size_t)new_ldm * new_ldm) || linv_mm.alloc((size_t)nblk * NB * NB) ||
        Bl.alloc((size_t)new_ldm * new_ldm) || linv_B.alloc((size_t)nblk * NB * NB) || w.alloc(new_ldm) ||
        ay.alloc(new_ldm) || vtmp.alloc(new_ldm) || nA.alloc((size_t)new_ldm * std::max(cap, 1LL)))
      return set_error(GPRX_OUT_OF_MEMORY, "inducing buffers");
    std::swap(Amat.p, nA.p);
    std::swap(Amat.n, nA.n);
    G.reset();
    Btrial.reset();
    m = (int)mm;
    ldm = new_ldm;
  }
  GPRX_CUDA_TRY(cudaMemcpyAsync(z.p, zh, sizeof(double) * m * d, cudaMemcpyHostToDevice, stream));
  assembled = false;
  return assemble();
}

// ---------------------------------------------------------------------------
// sharded evaluation (one shard = the points this handle holds; Z, K_mm and
// L are replicated).  Exchange buffer 1 (m² + m + 3): B_s = A_s A_sᵀ (lower,
// ld m, upper zero), A_s y_s, Σ_c (k_cc − ‖a_c‖²) over the shard's points,
// Σ y_s², n_s.  Exchange buffer 2 (m² + p): H_s = G_s A_sᵀ (ld m) and the
// θ-gradient of the cross term
// ⟨L⁻ᵀ G_s, ∂K(Z, X_s)⟩.  Both are sums over n, so their sum over the shards
// is the unsharded value (assemble_vfe, src/sgpr/factor/vfe.rs:191-277;
// analytic_gradient, src/sgpr/factor/derivatives.rs:283-366).
// ---------------------------------------------------------------------------
gprx_status SgprState::factor_kmm_and_a(EmuWork& ew, bool& emu) {
  const int nn = (int)n;
  std::vector<double> js{0.0};
  auto r = retry_list(opt);
  js.insert(js.end(), r.begin(), r.end());
  bool ok = false;
  gprx_status st;
  for (double j : js) {
    if ((st = reset_status()) != GPRX_OK) return st;
    GPRX_CUDA_TRY(fill_lower(kern, z.p, m, m, Lmm.p, ldm, j, status.p, stream));
    GPRX_CUDA_TRY(potrf_blocked(Lmm.p, ldm, m, linv_mm.p, status.p, stream, &fctx));
    DevStatus ds;
    if ((st = read_status(&ds)) != GPRX_OK) return st;
    if (ds.code == GPRX_OK) {
      ok = true;
      kmm_jitter = j;
      break;
    }
    if (ds.code != GPRX_CHOLESKY_FAILED) return status_to_error(ds, j, m, GPRX_STAGE_FIT);
  }
  if (!ok) return set_cholesky_error(js.back(), m, GPRX_STAGE_FIT);
  pivot_ratio_kernel<<<1, 1024, 0, stream>>>(Lmm.p, ldm, m, res.p + 10);
  count_launch();
  GPRX_CUDA_TRY(fill_cross(kern, z.p, m, m, x.p, cap, nn, Amat.p, ldm, status.p, stream));
  emu = use_emu();
  if (emu) {
    if ((st = ensure_emu(ew)) != GPRX_OK) return st;
    GPRX_CUDA_TRY(cudaMemsetAsync(emu_err.p, 0, sizeof(int), stream));
  }
  GPRX_CUDA_TRY(trsm_lower_rec(Lmm.p, ldm, m, linv_mm.p, Amat.p, ldm, nn, TRSM_LEAF, status.p, stream));
  return GPRX_OK;
}

gprx_status SgprState::shard_assemble(const double* params, double* e1) {
  if (!params || !e1) return set_error(GPRX_INVALID_ARGUMENT, "null pointer");
  if (n > INT32_MAX) return set_error(GPRX_CAPACITY, "n too large for one assembly");
  shard_ready = false;
  gprx_status st = write_params(params);
  if (st != GPRX_OK) return st;
  const int nn = (int)n;
  EmuWork ew;
  bool emu = false;
  if ((st = factor_kmm_and_a(ew, emu)) != GPRX_OK) return st;
  const long long mm2 = (long long)m * m;
  GPRX_CUDA_TRY(cudaMemsetAsync(e1, 0, sizeof(double) * mm2, stream));
  if (emu) {
    GPRX_CUDA_TRY(emu_gram(Amat.p, Amat.p, ldm, m, nn, true, e1, m, ew, emu_part.p, ldm, EMU_GROUP, EMU_PART_K,
                           stream));
  } else {
    GPRX_CUDA_TRY(syrk_splitk(Amat.p, ldm, m, nn, Amat.p, ldm, true, 0.0, splitbuf, e1, m, status.p, stream));
  }
  int blocks = grid_for((long long)nn * 32, 1024);
  trace_residual_kernel<<<blocks, 256, 0, stream>>>(Amat.p, ldm, m, nn, kern.diag_value(), partials.p, status.p);
  sum_partials_kernel<<<1, 1024, 0, stream>>>(partials.p, blocks, e1 + mm2 + m, status.p);
  count_launch(2);
  {
    int S = (int)std::min<long long>(32, std::max<long long>(1, nn / 4096));
    if (splitbuf.ensure((size_t)S * ldm) != cudaSuccess) return set_error(GPRX_OUT_OF_MEMORY, "split buffer");
    GemmParams pp = gemm_params(m, 1, nn, Amat.p, ldm, y.p, nn, splitbuf.p, ldm, 1.0, 0.0, status.p);
    pp.mode = GEMM_SPLIT_K;
    pp.splits = S;
    pp.split_stride = ldm;
    GPRX_CUDA_TRY(dgemm(false, false, pp, stream));
    split_reduce_kernel<<<grid_for(m, 256), 256, 0, stream>>>(splitbuf.p, S, ldm, m, 0, 0.0, false, e1 + mm2,
                                                                status.p);
    count_launch();
  }
  res_h.p[20] = y2;
  res_h.p[21] = (double)n;
  GPRX_CUDA_TRY(cudaMemcpyAsync(e1 + mm2 + m + 1, res_h.p + 20, sizeof(double) * 2, cudaMemcpyHostToDevice, stream));
  GPRX_CUDA_TRY(cudaMemcpyAsync(res_h.p, res.p + 10, sizeof(double), cudaMemcpyDeviceToHost, stream));
  if (emu) GPRX_CUDA_TRY(cudaMemcpyAsync(emu_err_h.p, emu_err.p, sizeof(int), cudaMemcpyDeviceToHost, stream));
  if ((st = sync_check(GPRX_STAGE_FIT)) != GPRX_OK) return st;
  if (emu && *emu_err_h.p) return set_error(GPRX_TIMEOUT, "an emulated product's bounded wait ran out");
  pivot_ratio = res_h.p[0];
  assembled = false;  // the handle's B is not this shard's alone
  sharded = false;
  return GPRX_OK;
}

gprx_status SgprState::shard_nlml(const double* e1, double* nlml_out, double* e2) {
  if (!e1 || !nlml_out) return set_error(GPRX_INVALID_ARGUMENT, "null pointer");
  gprx_status st;
  if ((st = reset_status()) != GPRX_OK) return st;
  const long long mm2 = (long long)m * m;
  const double noise_v = noise();
  // B = Σ_s B_s + σ² I, L_B; Ay = Σ_s A_s y_s; the sums over n
  GPRX_CUDA_TRY(cudaMemcpy2DAsync(Bl.p, sizeof(double) * ldm, e1, sizeof(double) * m, sizeof(double) * m, m,
                                  cudaMemcpyDeviceToDevice, stream));
  add_diag_kernel<<<ceil_div(m, 256), 256, 0, stream>>>(Bl.p, ldm, m, noise_v);
  count_launch();
  GPRX_CUDA_TRY(potrf_blocked(Bl.p, ldm, m, linv_B.p, status.p, stream, &fctx));
  GPRX_CUDA_TRY(cudaMemcpyAsync(ay.p, e1 + mm2, sizeof(double) * m, cudaMemcpyDeviceToDevice, stream));
  GPRX_CUDA_TRY(cudaMemcpyAsync(res_h.p + 20, e1 + mm2 + m, sizeof(double) * 3, cudaMemcpyDeviceToHost, stream));
  if ((st = solve_w()) != GPRX_OK) return st;  // synchronises the stream
  trace_sum = res_h.p[20];
  const double y2_total = res_h.p[21];
  n_total = res_h.p[22];
  GPRX_CUDA_TRY(logdet_diag(Bl.p, ldm, m, false, res.p + 0, status.p, stream));
  GPRX_CUDA_TRY(dot_dev(ay.p, w.p, m, res.p + 1, status.p, stream));
  GPRX_CUDA_TRY(cudaMemcpyAsync(res_h.p, res.p, sizeof(double) * 2, cudaMemcpyDeviceToHost, stream));
  if ((st = sync_check(GPRX_STAGE_FIT)) != GPRX_OK) return st;
  shard_y2 = y2_total;
  const double logdet = (n_total - (double)m) * std::log(noise_v) + res_h.p[0];
  const double quad = (y2_total - res_h.p[1]) / noise_v;
  const double trace = trace_sum / (2.0 * noise_v);
  *nlml_out = 0.5 * (n_total * std::log(2.0 * M_PI) + logdet + quad) + trace;
  shard_ready = true;
  assembled = true;  // L, L_B and w are the global posterior's
  sharded = true;
  if (!e2) return GPRX_OK;
  // this shard's part of the gradient: G_s = B⁻¹A_s − (w r_sᵀ + A_s)/σ²,
  // H_s = G_s A_sᵀ, and the cross term with L⁻ᵀ G_s
  const int nn = (int)n;
  if (G.ensure((size_t)ldm * std::max(cap, 1LL)) != cudaSuccess)
    return set_error(GPRX_OUT_OF_MEMORY, "gradient buffers");
  const bool emu = use_emu();
  EmuWork ew;
  if (emu) {
    if ((st = ensure_emu(ew)) != GPRX_OK) return st;
    GPRX_CUDA_TRY(cudaMemsetAsync(emu_err.p, 0, sizeof(int), stream));
  }
  GPRX_CUDA_TRY(cudaMemcpyAsync(G.p, Amat.p, sizeof(double) * ldm * nn, cudaMemcpyDeviceToDevice, stream));
  GPRX_CUDA_TRY(trsm_lower_rec(Bl.p, ldm, m, linv_B.p, G.p, ldm, nn, TRSM_LEAF, status.p, stream));
  GPRX_CUDA_TRY(trsm_lower_t_rec(Bl.p, ldm, m, linv_B.p, G.p, ldm, nn, TRSM_LEAF, status.p, stream));
  adjoint_update_kernel<<<grid_for((long long)nn * 32, 256), 256, 0, stream>>>(Amat.p, G.p, ldm, m, nn, w.p, y.p,
                                                                                1.0 / noise_v, status.p);
  count_launch();
  if (emu) {
    GPRX_CUDA_TRY(emu_gram(G.p, Amat.p, ldm, m, nn, false, e2, m, ew, emu_part.p, ldm, EMU_GROUP, EMU_PART_K,
                           stream));
  } else {
    GPRX_CUDA_TRY(syrk_splitk(G.p, ldm, m, nn, Amat.p, ldm, false, 0.0, splitbuf, e2, m, status.p, stream));
  }
  GPRX_CUDA_TRY(trsm_lower_t_rec(Lmm.p, ldm, m, linv_mm.p, G.p, ldm, nn, TRSM_LEAF, status.p, stream));
  int b2 = 0;
  GPRX_CUDA_TRY(cross_contract(kern, z.p, m, m, x.p, cap, nn, G.p, ldm, partials.p, &b2, status.p, stream));
  GPRX_CUDA_TRY(grad_finalize(kern, partials.p, b2, slot_param.p, 1.0, 0.0, e2 + mm2, status.p, stream));
  if (emu) GPRX_CUDA_TRY(cudaMemcpyAsync(emu_err_h.p, emu_err.p, sizeof(int), cudaMemcpyDeviceToHost, stream));
  if ((st = sync_check(GPRX_STAGE_FIT)) != GPRX_OK) return st;
  if (emu && *emu_err_h.p) return set_error(GPRX_TIMEOUT, "an emulated product's bounded wait ran out");
  return GPRX_OK;
}

gprx_status SgprState::shard_gradient(const double* e2, double* grad) {
  if (!e2 || !grad) return set_error(GPRX_INVALID_ARGUMENT, "null pointer");
  if (!shard_ready) return set_error(GPRX_INVALID_CONFIG, "shard gradient before the shard NLML");
  gprx_status st;
  if (H.ensure((size_t)ldm * m) != cudaSuccess || Wm.ensure((size_t)ldm * m) != cudaSuccess ||
      Xb.ensure((size_t)ldm * m) != cudaSuccess || Xt.ensure((size_t)ldm * m) != cudaSuccess)
    return set_error(GPRX_OUT_OF_MEMORY, "gradient buffers");
  if ((st = reset_status()) != GPRX_OK) return st;
  const long long mm2 = (long long)m * m;
  const double noise_v = noise();
  const int nk = kern.n_params;
  // w_mm = −sym(L⁻ᵀ tril½(H) L⁻¹) from H = Σ_s H_s
  GPRX_CUDA_TRY(cudaMemcpy2DAsync(H.p, sizeof(double) * ldm, e2, sizeof(double) * m, sizeof(double) * m, m,
                                  cudaMemcpyDeviceToDevice, stream));
  tril_half_kernel<<<grid_for((long long)m * m, 256), 256, 0, stream>>>(H.p, ldm, m, Xb.p);
  count_launch();
  GPRX_CUDA_TRY(trsm_lower_t(Lmm.p, ldm, m, linv_mm.p, Xb.p, ldm, m, status.p, stream));
  {
    dim3 tb(32, 8), tg(ceil_div(m, 32), ceil_div(m, 32));
    transpose_kernel<<<tg, tb, 0, stream>>>(Xb.p, ldm, m, Xt.p);
    count_launch();
  }
  GPRX_CUDA_TRY(trsm_lower_t(Lmm.p, ldm, m, linv_mm.p, Xt.p, ldm, m, status.p, stream));
  neg_sym_half_kernel<<<grid_for((long long)m * m, 256), 256, 0, stream>>>(Xt.p, ldm, m, Wm.p);
  count_launch();
  int b1 = 0;
  GPRX_CUDA_TRY(grad_contract(kern, z.p, m, m, Wm.p, ldm, nullptr, partials.p, &b1, status.p, stream));
  GPRX_CUDA_TRY(grad_finalize(kern, partials.p, b1, slot_param.p, 1.0, 0.0, res.p + 20, status.p, stream));
  // the cross term after the K_mm term's nk + 1 values (nk ≤ 8 leaves ≤ 46 fits in 128)
  GPRX_CUDA_TRY(cudaMemcpyAsync(res.p + 21 + nk, e2 + mm2, sizeof(double) * nk, cudaMemcpyDeviceToDevice, stream));
  // tr(B⁻¹) = ‖L_B⁻¹‖²_F, ‖w‖², (Ay)ᵀw
  GPRX_CUDA_TRY(cudaMemsetAsync(Xt.p, 0, sizeof(double) * ldm * m, stream));
  if (H.ensure((size_t)((m + 1) / 2) * ((m + 1) / 2) + 1) != cudaSuccess) return set_error(GPRX_OUT_OF_MEMORY, "scratch");
  GPRX_CUDA_TRY(trtri_blocked(Bl.p, ldm, m, linv_B.p, Xt.p, ldm, H.p, status.p, stream));
  int blocks = grid_for((long long)m * m, 1024);
  sumsq_kernel<<<blocks, 256, 0, stream>>>(Xt.p, ldm, m, m, partials.p + 8192, status.p);
  sum_partials_kernel<<<1, 1024, 0, stream>>>(partials.p + 8192, blocks, res.p + 2, status.p);
  count_launch(2);
  GPRX_CUDA_TRY(dot_dev(w.p, w.p, m, res.p + 3, status.p, stream));
  GPRX_CUDA_TRY(dot_dev(ay.p, w.p, m, res.p + 4, status.p, stream));
  GPRX_CUDA_TRY(cudaMemcpyAsync(res_h.p, res.p, sizeof(double) * 128, cudaMemcpyDeviceToHost, stream));
  if ((st = sync_check(GPRX_STAGE_FIT)) != GPRX_OK) return st;
  std::vector<double> dg;
  diag_grad(kern, dg);
  const double wdiag = 0.5 / noise_v;
  for (int i = 0; i < nk; ++i) grad[i] = res_h.p[20 + i] + res_h.p[21 + nk + i] + wdiag * n_total * dg[i];
  const double trb = res_h.p[2], ww = res_h.p[3], ayw = res_h.p[4];
  const double quad = (shard_y2 - ayw) / noise_v;
  const double trace = trace_sum / (2.0 * noise_v);
  const double dn = noise_v;
  const double d_logdet_b = dn * trb;
  const double d_q = -dn * ww;
  const double d_quad = -d_q / noise_v - quad * dn / noise_v;
  const double d_trace = -trace * dn / noise_v;
  grad[nk] = 0.5 * ((n_total - (double)m) * dn / noise_v + d_logdet_b + d_quad) + d_trace;
  return GPRX_OK;
}

static gprx_status sgpr_eval_cb(void* ctx, const double* lt, double* f, double* g) {
  return ((SgprState*)ctx)->eval(lt, f, g);
}

}  // namespace gprx

struct gprx_sgpr {
  gprx::SgprState s;
};

using namespace gprx;

#define CHECK_SGPR(h) \
  if (!(h)) return set_error(GPRX_INVALID_ARGUMENT, "null handle")

extern "C" {

gprx_status gprx_sgpr_create(const double* x, uint64_t n, uint64_t d, const double* y, const double* z, uint64_t m,
                             const gprx_kernel_node* nodes, int32_t n_nodes, const double* theta, int32_t n_theta,
                             const gprx_options* options, gprx_sgpr** out) {
  if (!out) return set_error(GPRX_INVALID_ARGUMENT, "null output handle");
  *out = nullptr;
  gprx_sgpr* h = new (std::nothrow) gprx_sgpr;
  if (!h) return set_error(GPRX_OUT_OF_MEMORY, "host allocation");
  gprx_status st = h->s.create(x, n, d, y, z, m, nodes, n_nodes, theta, n_theta, options);
  if (st != GPRX_OK) {
    delete h;
    return st;
  }
  *out = h;
  return GPRX_OK;
}

gprx_status gprx_sgpr_destroy(gprx_sgpr* h) {
  delete h;
  return GPRX_OK;
}

uint64_t gprx_sgpr_num_params(const gprx_sgpr* h) { return h ? (uint64_t)h->s.num_params() : 0; }

gprx_status gprx_sgpr_get_params(gprx_sgpr* h, double* out, uint64_t p) {
  CHECK_SGPR(h);
  if (!out || p != (uint64_t)h->s.num_params()) return set_error(GPRX_SHAPE_MISMATCH, "parameter count");
  h->s.get_params(out);
  return GPRX_OK;
}

gprx_status gprx_sgpr_factor(gprx_sgpr* h) {
  CHECK_SGPR(h);
  return h->s.assemble();
}

gprx_status gprx_sgpr_set_params(gprx_sgpr* h, const double* params, uint64_t p) {
  CHECK_SGPR(h);
  SgprState& s = h->s;
  if (!params || p != (uint64_t)s.num_params()) return set_error(GPRX_SHAPE_MISMATCH, "parameter count");
  std::vector<double> prev(p);
  s.get_params(prev.data());
  gprx_status st = s.write_params(params);
  if (st == GPRX_OK) st = s.assemble();
  if (st != GPRX_OK) {
    gprx_error_info saved = last_error();
    s.write_params(prev.data());
    s.assemble();
    last_error() = saved;
  }
  return st;
}

gprx_status gprx_sgpr_eval(gprx_sgpr* h, const double* params, uint64_t p, double* nlml, double* grad) {
  CHECK_SGPR(h);
  if (!params || !nlml) return set_error(GPRX_INVALID_ARGUMENT, "null pointer");
  if (p != (uint64_t)h->s.num_params()) return set_error(GPRX_SHAPE_MISMATCH, "parameter count");
  return h->s.eval(params, nlml, grad);
}

gprx_status gprx_sgpr_nlml(gprx_sgpr* h, double* nlml) {
  CHECK_SGPR(h);
  if (!nlml) return set_error(GPRX_INVALID_ARGUMENT, "null pointer");
  return h->s.nlml(nlml);
}

gprx_status gprx_sgpr_shard_sizes(const gprx_sgpr* h, uint64_t* exchange1, uint64_t* exchange2) {
  CHECK_SGPR(h);
  if (!exchange1 || !exchange2) return set_error(GPRX_INVALID_ARGUMENT, "null pointer");
  *exchange1 = h->s.shard_e1();
  *exchange2 = h->s.shard_e2();
  return GPRX_OK;
}

gprx_status gprx_sgpr_shard_assemble(gprx_sgpr* h, const double* params, uint64_t p, double* exchange1) {
  CHECK_SGPR(h);
  if (p != (uint64_t)h->s.num_params()) return set_error(GPRX_SHAPE_MISMATCH, "parameter count");
  return h->s.shard_assemble(params, exchange1);
}

gprx_status gprx_sgpr_shard_nlml(gprx_sgpr* h, const double* exchange1, double* nlml, double* exchange2) {
  CHECK_SGPR(h);
  return h->s.shard_nlml(exchange1, nlml, exchange2);
}

gprx_status gprx_sgpr_shard_gradient(gprx_sgpr* h, const double* exchange2, double* grad) {
  CHECK_SGPR(h);
  return h->s.shard_gradient(exchange2, grad);
}

gprx_status gprx_sgpr_predict(gprx_sgpr* h, const double* xs, uint64_t q, int32_t kind, double* mean, double* var) {
  CHECK_SGPR(h);
  return h->s.predict(xs, q, kind, mean, var);
}

gprx_status gprx_sgpr_predict_covariance(gprx_sgpr* h, const double* xs, uint64_t q, int32_t kind, double* mean,
                                         double* cov) {
  CHECK_SGPR(h);
  return h->s.predict_covariance(xs, q, kind, mean, cov);
}

gprx_status gprx_sgpr_sample(gprx_sgpr* h, const double* xs, uint64_t q, int32_t kind, uint64_t n_draws,
                             uint64_t seed, double* out) {
  CHECK_SGPR(h);
  return h->s.sample(xs, q, kind, n_draws, seed, out);
}

gprx_status gprx_sgpr_fit(gprx_sgpr* h, const gprx_lbfgs_options* opt, gprx_fit_report* report) {
  CHECK_SGPR(h);
  SgprState& s = h->s;
  int p = s.num_params();
  std::vector<double> theta0(p), best;
  s.get_params(theta0.data());
  gprx_status st = fit_lbfgs(&s, sgpr_eval_cb, p, theta0.data(), opt, report, best);
  if (st != GPRX_OK) {
    gprx_error_info saved = last_error();
    s.write_params(theta0.data());
    s.assemble();
    last_error() = saved;
    return st;
  }
  st = s.write_params(best.data());
  if (st == GPRX_OK) st = s.assemble();
  if (st == GPRX_OK && report) st = s.nlml(&report->nlml);
  return st;
}

gprx_status gprx_sgpr_insert(gprx_sgpr* h, const double* x_new, double y_new, uint64_t* id) {
  CHECK_SGPR(h);
  return h->s.insert(x_new, y_new, id);
}

gprx_status gprx_sgpr_delete(gprx_sgpr* h, uint64_t id) {
  CHECK_SGPR(h);
  return h->s.remove(id);
}

gprx_status gprx_sgpr_set_inducing(gprx_sgpr* h, const double* z, uint64_t m) {
  CHECK_SGPR(h);
  SgprState& st = h->s;
  const gprx_status r = st.set_inducing(z, m);
  if (r == GPRX_OK) {  // a new set: new ids
    st.inducing_ids.clear();
    for (int i = 0; i < st.m; ++i) st.inducing_ids.push_back(st.next_inducing_id++);
  }
  return r;
}

gprx_status gprx_sgpr_insert_inducing(gprx_sgpr* h, const double* z_new, uint64_t* id) {
  CHECK_SGPR(h);
  return h->s.insert_inducing(z_new, id);
}

gprx_status gprx_sgpr_delete_inducing(gprx_sgpr* h, uint64_t id) {
  CHECK_SGPR(h);
  return h->s.delete_inducing(id);
}

uint64_t gprx_sgpr_m(const gprx_sgpr* h) { return h ? (uint64_t)h->s.m : 0; }

gprx_status gprx_sgpr_inducing_ids(const gprx_sgpr* h, uint64_t* out, uint64_t m) {
  CHECK_SGPR(h);
  if (!out || m != (uint64_t)h->s.m) return set_error(GPRX_SHAPE_MISMATCH, "inducing id count");
  std::copy(h->s.inducing_ids.begin(), h->s.inducing_ids.end(), out);
  return GPRX_OK;
}

uint64_t gprx_sgpr_n(const gprx_sgpr* h) { return h ? (uint64_t)h->s.n : 0; }

int32_t gprx_sgpr_last_step_in_place(const gprx_sgpr* h) { return h ? h->s.last_in_place : 0; }

gprx_status gprx_sgpr_point_ids(gprx_sgpr* h, uint64_t* out, uint64_t n) {
  CHECK_SGPR(h);
  if (!out || n != (uint64_t)h->s.n) return set_error(GPRX_SHAPE_MISMATCH, "id count");
  std::copy(h->s.ids.begin(), h->s.ids.end(), out);
  return GPRX_OK;
}

gprx_status gprx_sgpr_kmm_jitter(gprx_sgpr* h, double* jitter) {
  CHECK_SGPR(h);
  if (!jitter) return set_error(GPRX_INVALID_ARGUMENT, "null pointer");
  *jitter = h->s.kmm_jitter;
  return GPRX_OK;
}

gprx_status gprx_sgpr_stream(gprx_sgpr* h, void** stream) {
  CHECK_SGPR(h);
  if (!stream) return set_error(GPRX_INVALID_ARGUMENT, "null pointer");
  *stream = (void*)h->s.stream;
  return GPRX_OK;
}

gprx_status gprx_sgpr_stage_times(gprx_sgpr* h, double* out3) {
  CHECK_SGPR(h);
  if (!out3) return set_error(GPRX_INVALID_ARGUMENT, "null pointer");
  float ms;
  for (int i = 0; i < 3; ++i) {
    GPRX_CUDA_TRY(cudaEventElapsedTime(&ms, h->s.ev[i], h->s.ev[i + 1]));
    out3[i] = ms;
  }
  return GPRX_OK;
}

}  // extern "C"
