// batch.cu — thousands of independent exact GPs of uneven n: one persistent
// launch evaluates every pending point of a fitting round, and the per-problem
// L-BFGS state machines advance on the device between launches, so a whole
// fit runs as replays of one captured CUDA graph.
//
// Evaluation.  Each CTA pulls whole problems from an atomic queue (largest n
// first, so the long ones start early) and runs the complete NLML + gradient
// evaluation of ExactFit::value_and_gradient_into_fit (gprx
// src/gpr/exact_fit.rs:319-341) in its own workspace:
//   fill      lower K + (σn² + j) I                  (factor.rs:515-542)
//   LLT       128-wide block columns: diagonal block factor + inverse in
//             shared memory, panel P = A_below L_kk⁻ᵀ and trailing
//             A22 −= P Pᵀ as in-CTA DMMA tile GEMMs  (chol.rs:141-167)
//   log-det   2 Σ ln L_ii                             (factor.rs:555-568)
//   X = L⁻¹   block rows: X_i,<i = −L_ii⁻¹ (L_i,<i X_<i,<i)
//   α         Xᵀ (X y);  K⁻¹ = Xᵀ X (lower)          (workspace.rs:395-425)
//   gradient  −½⟨ααᵀ − K⁻¹, ∂K/∂θ⟩, noise −½σn² Σ_i W_ii (exact_fit.rs:665-729)
// A non-positive pivot retries with the next jitter offset (chol.rs:35-58);
// when every offset fails the problem reports CHOLESKY_FAILED and its
// optimizer sees the barrier (src/optimizer/adapter.rs:118-160).  The result
// of a problem does not depend on the batch it runs in: one CTA computes it
// in a fixed order.
//
// Fitting.  One LbfgsRC per problem (lbfgs.h) lives in device memory.  A round
// is {reset the queue, evaluate all active problems, advance every optimizer};
// several rounds are captured into one CUDA graph and replayed until no
// problem is active.

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <numeric>
#include <string>
#include <vector>

#include "cta_gemm.cuh"
#include "diag_block.cuh"
#include "kernels.cuh"
#include "lbfgs.h"
#include "runtime.cuh"

namespace gprx {

// ---------------------------------------------------------------------------
// device data
// ---------------------------------------------------------------------------
struct BatchProblem {
  const double* x;  // n × d, column-major (ld n)
  const double* y;
  int n;
  int pad;
};

constexpr int BATCH_MAX_JITTERS = 8;
struct JitterList {
  int count;  // offsets tried after the first attempt (which adds none)
  double j[BATCH_MAX_JITTERS];
};

// size classes of the autotuned schedule: n ≤ 64, ≤ 128, …, ≤ 4096, > 4096
constexpr int BATCH_SIZE_CLASSES = 8;
__host__ __device__ inline int batch_size_class(int n) {
  int c = 0;
  for (int lim = 64; c < BATCH_SIZE_CLASSES - 1 && n > lim; lim *= 2) ++c;
  return c;
}

struct BatchHeader {
  int queue;   // next position in the work order
  int active;  // problems the optimizer round left pending
  int pad[2];
};

struct BatchEvalArgs {
  const BatchProblem* probs;
  const int* order;  // problem indices, largest n first
  int nprob;
  int p;                    // kernel parameters + noise
  const double* log_theta;  // nprob × p
  const int* active;        // null: every problem
  double* nlml;             // nprob
  double* grad;             // nprob × p
  int* status;              // nprob
  BatchHeader* hdr;
  double* work;  // per-CTA workspaces
  long long work_stride;
  int8_t tile_of_class[BATCH_SIZE_CLASSES];  // in-CTA GEMM tile shape per size class (autotuned)
  int nmax;
  JitterList jit;
  KTree tmpl;  // tree structure (θ-dependent constants are set per problem)
  int slot_param[64];
};

constexpr int BT = 512;  // 16 warps: one CTA per SM holds a problem, so the warps hide the FP64 latencies
static_assert(BT == CG_THREADS, "the diagonal step and the CTA GEMM share the block");

__host__ __device__ inline long long batch_ld(int n) { return ((long long)n + 7) / 8 * 8; }

// Workspace of one CTA for problems of up to nmax points (doubles).
struct Work {
  double *A, *X, *T, *linv, *z, *alpha;
};
__host__ __device__ constexpr long long work_doubles(int nmax) {
  long long ld = ((long long)nmax + 7) / 8 * 8;
  long long nblk = (nmax + NB_DIAG - 1) / NB_DIAG;
  return 2 * ld * nmax + (long long)NB_DIAG * ld + nblk * NB_DIAG * NB_DIAG + 2 * ld;
}
__device__ inline Work work_of(double* base, int nmax) {
  long long ld = ((long long)nmax + 7) / 8 * 8;
  long long nblk = (nmax + NB_DIAG - 1) / NB_DIAG;
  Work w;
  w.A = base;
  w.X = w.A + ld * nmax;
  w.T = w.X + ld * nmax;
  w.linv = w.T + (long long)NB_DIAG * ld;
  w.z = w.linv + nblk * NB_DIAG * NB_DIAG;
  w.alpha = w.z + ld;
  return w;
}

// ---------------------------------------------------------------------------
// fill and gradient over 64×64 lower tiles
// ---------------------------------------------------------------------------
constexpr int FT_B = 64;
// pairs one thread evaluates together: more independent FP64 chains where
// the tree's leaves (NL at most) and ARD differences leave registers for them
template <int ARD_D, int NL>
constexpr int pairs_w() {
  return ARD_D == 0 ? (NL <= 2 ? 4 : 2) : 1;
}

template <int ARD_D>
__device__ double pair_dx(const double* xi, const double* xj, int d, double (&dx)[ARD_D > 0 ? ARD_D : 1]) {
  double r2 = 0.0;
  for (int f = 0; f < d; ++f) {
    double v = xi[f * FT_B] - xj[f * FT_B];
    r2 = fma(v, v, r2);
    if (ARD_D > 0) {
#pragma unroll
      for (int q = 0; q < (ARD_D > 0 ? ARD_D : 1); ++q)
        if (q == f) dx[q] = v;
    }
  }
  return r2;
}

__device__ inline void stage_points(const double* x, int n, int d, int i0, int j0, double* xi, double* xj) {
  for (int e = threadIdx.x; e < d * FT_B; e += BT) {
    const int r = e % FT_B, f = e / FT_B;
    xi[f * FT_B + r] = (i0 + r < n) ? x[(i0 + r) + (long long)f * n] : 0.0;
    xj[f * FT_B + r] = (j0 + r < n) ? x[(j0 + r) + (long long)f * n] : 0.0;
  }
}

// lower K + diag_add I into A (ld); returns true when every value is finite
// (trees of at most NL leaves)
template <int ARD_D, int NL>
__device__ bool cta_fill_lower(const KTree& t, const double* x, int n, double* A, long long ld, double diag_add,
                               double* smem, int* flag_sh) {
  double* xi = smem;
  double* xj = smem + GPRX_MAX_DIM * FT_B;
  const int d = t.d, tid = threadIdx.x;
  const int nt = (n + FT_B - 1) / FT_B;
  if (tid == 0) *flag_sh = 0;
  bool bad = false;
  for (int ti = 0; ti < nt; ++ti)
    for (int tj = 0; tj <= ti; ++tj) {
      const int i0 = ti * FT_B, j0 = tj * FT_B;
      __syncthreads();
      stage_points(x, n, d, i0, j0, xi, xj);
      __syncthreads();
      const int r = tid % FT_B, i = i0 + r;
      constexpr int CS = BT / FT_B;  // column stride of one thread
      constexpr int PW = pairs_w<ARD_D, NL>();
#pragma unroll 1
      for (int k0 = 0; k0 < FT_B / CS; k0 += PW) {
        const int cb = tid / FT_B + k0 * CS;
        if (i >= n || j0 + cb > i) continue;  // every pair of the group lies above the diagonal
        double dx[PW][ARD_D > 0 ? ARD_D : 1], r2[PW], kv[PW];
#pragma unroll
        for (int w = 0; w < PW; ++w) r2[w] = pair_dx<ARD_D>(xi + r, xj + cb + w * CS, d, dx[w]);
        kt_value_w<ARD_D, PW, NL>(t, dx, r2, kv);
#pragma unroll
        for (int w = 0; w < PW; ++w) {
          const int j = j0 + cb + w * CS;
          if (j >= n || i < j) continue;
          double v = kv[w];
          if (i == j) v += diag_add;
          if (!isfinite(v)) bad = true;
          A[i + (long long)j * ld] = v;
        }
      }
    }
  if (bad) *flag_sh = 1;
  __syncthreads();
  const bool ok = *flag_sh == 0;
  __syncthreads();
  return ok;
}

// Slot sums of Σ_{i≥j} c_ij W_ij ∂K_ij/∂θ (c = 1 on the diagonal, 2 off it),
// W = ααᵀ − K⁻¹ (K⁻¹ lower in kinv), and Σ W_ii in the last slot (trees of
// at most NL leaves; the slots of absent leaves are zero).
template <int ARD_D, int NL>
__device__ void cta_grad(const KTree& t, const double* x, int n, const double* kinv, long long ld,
                         const double* alpha, double* smem, double* slots) {
  constexpr int AD = ARD_D > 0 ? ARD_D : 1;
  constexpr int NS = GRAD_SLOTS_LEAF + AD + 1;
  double* xi = smem;
  double* xj = xi + GPRX_MAX_DIM * FT_B;
  double* ai = xj + GPRX_MAX_DIM * FT_B;
  double* aj = ai + FT_B;
  double* red = aj + FT_B;  // (BT / 32) × NS
  const int d = t.d, tid = threadIdx.x;
  double acc_leaf[NL][KT_ACC_PER_LEAF];
  double acc_ard[AD];
  double acc_noise = 0.0;
#pragma unroll
  for (int l = 0; l < NL; ++l) acc_leaf[l][0] = acc_leaf[l][1] = 0.0;
#pragma unroll
  for (int f = 0; f < AD; ++f) acc_ard[f] = 0.0;
  const int nt = (n + FT_B - 1) / FT_B;
  for (int ti = 0; ti < nt; ++ti)
    for (int tj = 0; tj <= ti; ++tj) {
      const int i0 = ti * FT_B, j0 = tj * FT_B;
      __syncthreads();
      stage_points(x, n, d, i0, j0, xi, xj);
      if (tid < FT_B) {
        ai[tid] = (i0 + tid < n) ? alpha[i0 + tid] : 0.0;
        aj[tid] = (j0 + tid < n) ? alpha[j0 + tid] : 0.0;
      }
      __syncthreads();
      const int r = tid % FT_B, i = i0 + r;
      constexpr int CS = BT / FT_B;
      constexpr int PW = pairs_w<ARD_D, NL>();
#pragma unroll 1
      for (int k0 = 0; k0 < FT_B / CS; k0 += PW) {
        const int cb = tid / FT_B + k0 * CS;
        if (i >= n || j0 + cb > i) continue;
        double dx[PW][AD], r2[PW], wt[PW];
#pragma unroll
        for (int w = 0; w < PW; ++w) {
          const int c = cb + w * CS, j = j0 + c;
          r2[w] = pair_dx<ARD_D>(xi + r, xj + c, d, dx[w]);
          double wv = 0.0;  // pairs outside the lower triangle weigh nothing
          if (j < n && i >= j) {
            wv = fma(ai[r], aj[c], -kinv[i + (long long)j * ld]);
            if (i == j) acc_noise += wv;
            else wv *= 2.0;
          }
          wt[w] = wv;
        }
        kt_accumulate_grad_w<ARD_D, PW, NL>(t, dx, r2, wt, acc_leaf, acc_ard);
      }
    }
  const int lane = tid & 31, warp = tid >> 5;
  __syncthreads();
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    double v;
    if (s < GRAD_SLOTS_LEAF) v = (s / KT_ACC_PER_LEAF < NL) ? acc_leaf[s / KT_ACC_PER_LEAF][s % KT_ACC_PER_LEAF] : 0.0;
    else if (s < GRAD_SLOTS_LEAF + AD) v = acc_ard[s - GRAD_SLOTS_LEAF];
    else v = acc_noise;
    v = warp_sum(v);
    if (lane == 0) red[warp * NS + s] = v;
  }
  __syncthreads();
  for (int s = tid; s < NS; s += BT) {
    double v = 0.0;
    for (int w = 0; w < BT / 32; ++w) v += red[w * NS + s];
    slots[s] = v;
  }
  __syncthreads();
}

// the two passes with the leaf bound of the problem's tree (isotropic trees
// of at most two leaves have their own, wider form)
template <int ARD_D>
__device__ bool cta_fill_any(const KTree& t, const double* x, int n, double* A, long long ld, double diag_add,
                             double* smem, int* flag_sh) {
  if (ARD_D == 0 && t.n_leaves <= 2) return cta_fill_lower<ARD_D, 2>(t, x, n, A, ld, diag_add, smem, flag_sh);
  return cta_fill_lower<ARD_D, KT_MAX_LEAVES>(t, x, n, A, ld, diag_add, smem, flag_sh);
}
template <int ARD_D>
__device__ void cta_grad_any(const KTree& t, const double* x, int n, const double* kinv, long long ld,
                             const double* alpha, double* smem, double* slots) {
  if (ARD_D == 0 && t.n_leaves <= 2) cta_grad<ARD_D, 2>(t, x, n, kinv, ld, alpha, smem, slots);
  else cta_grad<ARD_D, KT_MAX_LEAVES>(t, x, n, kinv, ld, alpha, smem, slots);
}

// ---------------------------------------------------------------------------
// one problem, one CTA
// ---------------------------------------------------------------------------
__device__ inline bool in_default_interval(double log_v) {
  // Interval::DEFAULT_POSITIVE = (1e-5, 1e5), open (src/param.rs:91)
  const double v = exp(log_v);
  return isfinite(v) && v > 1e-5 && v < 1e5;
}

// LLT of the lower n×n matrix in w.A with the diagonal-block inverses in
// w.linv.  Returns the failing column or −1.
__device__ int cta_potrf(const Work& w, int n, long long ld, double* smem, int* fail_sh, int cfg) {
  for (int k0 = 0; k0 < n; k0 += NB_DIAG) {
    const int nbk = min(NB_DIAG, n - k0);
    double* lk = w.linv + (long long)(k0 / NB_DIAG) * NB_DIAG * NB_DIAG;
    const int f = diag_block_factor_inv(w.A, ld, k0, nbk, lk, smem, fail_sh);
    if (f >= 0) return k0 + f;
    const int rest = n - k0 - nbk;
    if (rest <= 0) break;
    double* P = w.A + (k0 + nbk) + (long long)k0 * ld;
    // P := P L_kk⁻ᵀ (in place: one tile must span all nbk columns)
    cta_gemm<false, true>(nbk <= cg_tile_n(cfg) ? cfg : 0, rest, nbk, nbk, P, ld, lk, NB_DIAG, P, ld, 1.0, 0.0, false,
                          CG_FULL, smem);
    // A22 −= P Pᵀ (lower)
    double* A22 = w.A + (k0 + nbk) + (long long)(k0 + nbk) * ld;
    cta_gemm<false, true>(cfg, rest, rest, nbk, P, ld, P, ld, A22, ld, -1.0, 1.0, true, CG_FULL, smem);
  }
  return -1;
}

// X = L⁻¹ (lower, the upper part of every diagonal block zero), block rows
// top to bottom: X_ii = L_ii⁻¹, X_i,<i = −L_ii⁻¹ (L_i,<i X_<i,<i).
__device__ void cta_trtri(const Work& w, int n, long long ld, double* smem, int cfg) {
  for (int r0 = 0; r0 < n; r0 += NB_DIAG) {
    const int nbi = min(NB_DIAG, n - r0);
    const double* li = w.linv + (long long)(r0 / NB_DIAG) * NB_DIAG * NB_DIAG;
    for (int e = threadIdx.x; e < NB_DIAG * nbi; e += BT) {
      const int i = e % NB_DIAG, j = e / NB_DIAG;
      if (i < nbi) w.X[(r0 + i) + (long long)(r0 + j) * ld] = li[i + j * NB_DIAG];
    }
    if (r0 == 0) continue;
    // T = L_i,<i X_<i,<i  (X lower: k from the tile's first column)
    cta_gemm<false, false>(cfg, nbi, r0, r0, w.A + r0, ld, w.X, ld, w.T, NB_DIAG, 1.0, 0.0, false, CG_FROM_COL, smem);
    // X_i,<i = −L_ii⁻¹ T
    cta_gemm<false, false>(cfg, nbi, r0, nbi, li, NB_DIAG, w.T, NB_DIAG, w.X + r0, ld, -1.0, 0.0, false, CG_FULL,
                           smem);
  }
  __syncthreads();
}

template <int ARD_D>
__device__ void cta_eval(const BatchEvalArgs& a, int q, const Work& w, double* smem) {
  __shared__ KTree tree;
  __shared__ int flag_sh, code_sh;
  __shared__ double red[32];
  __shared__ double slots[64];
  __shared__ double noise_sh;
  const BatchProblem P = a.probs[q];
  const int n = P.n, tid = threadIdx.x, p = a.p;
  const long long ld = batch_ld(n);
  const int cfg = a.tile_of_class[batch_size_class(n)];
  const double* th = a.log_theta + (long long)q * p;
  if (tid == 0) {
    tree = a.tmpl;
    int code = kt_set_theta(tree, th);
    for (int i = 0; i < p; ++i)
      if (!in_default_interval(th[i])) code = GPRX_INVALID_HYPERPARAMETER;
    noise_sh = exp(th[p - 1]);
    code_sh = code;
  }
  __syncthreads();
  if (code_sh != GPRX_OK) {
    if (tid == 0) a.status[q] = code_sh;
    return;
  }
  const double noise = noise_sh;
  // fill + factor, retried with the jitter offsets
  int fail = 0;
  for (int attempt = 0; attempt <= a.jit.count; ++attempt) {
    const double j = attempt == 0 ? 0.0 : a.jit.j[attempt - 1];
    if (!cta_fill_any<ARD_D>(tree, P.x, n, w.A, ld, noise + j, smem, &flag_sh)) {
      if (tid == 0) a.status[q] = GPRX_NONFINITE_KERNEL;
      return;
    }
    fail = cta_potrf(w, n, ld, smem, &flag_sh, cfg);
    if (fail < 0) break;
  }
  if (fail >= 0) {
    if (tid == 0) a.status[q] = GPRX_CHOLESKY_FAILED;
    return;
  }
  double acc = 0.0;
  for (int i = tid; i < n; i += BT) acc += log(w.A[i + (long long)i * ld]);
  const double logdet = 2.0 * block_sum(acc, red);
  cta_trtri(w, n, ld, smem, cfg);
  // z = X y (rows), α = Xᵀ z (columns)
  for (int i = tid; i < n; i += BT) {
    double s = 0.0;
    for (int j = 0; j <= i; ++j) s = fma(w.X[i + (long long)j * ld], P.y[j], s);
    w.z[i] = s;
  }
  __syncthreads();
  {
    const int lane = tid & 31, warp = tid >> 5;
    for (int j = warp; j < n; j += BT / 32) {
      double s = 0.0;
      for (int i = j + lane; i < n; i += 32) s = fma(w.X[i + (long long)j * ld], w.z[i], s);
      s = warp_sum(s);
      if (lane == 0) w.alpha[j] = s;
    }
  }
  __syncthreads();
  acc = 0.0;
  for (int i = tid; i < n; i += BT) acc = fma(P.y[i], w.alpha[i], acc);
  const double quad = block_sum(acc, red);
  // K⁻¹ = Xᵀ X (lower) over L in A
  cta_gemm<true, false>(cfg, n, n, n, w.X, ld, w.X, ld, w.A, ld, 1.0, 0.0, true, CG_FROM_ROW, smem);
  cta_grad_any<ARD_D>(tree, P.x, n, w.A, ld, w.alpha, smem, slots);
  if (tid == 0) {
    constexpr int NS = GRAD_SLOTS_LEAF + (ARD_D > 0 ? ARD_D : 1) + 1;
    const double nl = 0.5 * (quad + logdet + (double)n * log(2.0 * M_PI));
    double* g = a.grad + (long long)q * p;
    for (int i = 0; i < p; ++i) g[i] = 0.0;
    for (int s = 0; s < NS - 1; ++s) {
      const int pi = a.slot_param[s];
      if (pi >= 0) g[pi] += slots[s];
    }
    for (int i = 0; i < p - 1; ++i) g[i] *= -0.5;
    g[p - 1] = -0.5 * noise * slots[NS - 1];
    a.nlml[q] = nl;
    a.status[q] = isfinite(nl) ? GPRX_OK : GPRX_NOT_CONVERGED;
  }
  __syncthreads();
}

template <int ARD_D>
__global__ void __launch_bounds__(BT, 1) batch_eval_kernel(BatchEvalArgs a) {
  extern __shared__ __align__(16) double smem[];
  __shared__ int pidx;
  const Work w = work_of(a.work + (long long)blockIdx.x * a.work_stride, a.nmax);
  for (;;) {
    if (threadIdx.x == 0) pidx = atomicAdd(&a.hdr->queue, 1);
    __syncthreads();
    const int at = pidx;
    __syncthreads();
    if (at >= a.nprob) break;
    const int q = a.order[at];
    if (a.active && !a.active[q]) continue;
    cta_eval<ARD_D>(a, q, w, smem);
  }
}

inline size_t batch_smem() {
  size_t gemm = cg_smem_bytes();
  size_t tiles = (size_t)(2 * GPRX_MAX_DIM * FT_B + 2 * FT_B + (BT / 32) * 64) * sizeof(double);
  return std::max(std::max(diag_block_smem(), gemm), tiles);
}

// ---------------------------------------------------------------------------
// per-problem optimizer on the device
// ---------------------------------------------------------------------------
constexpr int BATCH_MAX_VARS = 16;
constexpr int BATCH_MAX_HISTORY = 16;
using DevLbfgs = LbfgsRC<BATCH_MAX_VARS, BATCH_MAX_HISTORY>;

struct ProblemFit {
  DevLbfgs lb;
  int run;         // current run (0: from θ0, then restarts)
  int done;        // all runs finished
  int first_err;   // status of run 0 when it found no evaluable point
  int last_err;    // status of the last failed evaluation
  double best_f;
  double best_z[BATCH_MAX_VARS];
  uint64_t iters, total_evals;
  double gnorm;
  int converged;
};

struct FitArgs {
  ProblemFit* fits;
  int nprob, p, runs;
  LogitMap map;
  LbfgsConfig cfg;
  const double* z_start;  // nprob × runs × p
  double* log_theta;      // next point to evaluate (nprob × p)
  int* active;
  const double* nlml;
  const double* grad;
  const int* status;
  BatchHeader* hdr;
};

__device__ void fit_start_run(const FitArgs& a, ProblemFit& F, int q) {
  F.lb.start(a.cfg, a.z_start + ((long long)q * a.runs + F.run) * a.p, a.p);
}

// the run just ended: keep the best, start the next run or finish
__device__ void fit_end_run(const FitArgs& a, ProblemFit& F, int q) {
  DevLbfgs& lb = F.lb;
  F.total_evals += lb.evaluations();
  if (lb.best_value() < F.best_f) {
    F.best_f = lb.best_value();
    for (int i = 0; i < a.p; ++i) F.best_z[i] = lb.best()[i];
    F.iters = lb.iterations();
    F.gnorm = lb.grad_norm();
    F.converged = lb.converged() ? 1 : 0;
  }
  if (F.run == 0 && !(lb.best_value() < BARRIER_COST))
    F.first_err = F.last_err != GPRX_OK ? F.last_err : GPRX_NOT_CONVERGED;
  if (F.run + 1 < a.runs) {
    ++F.run;
    fit_start_run(a, F, q);
  } else {
    F.done = 1;
  }
}

__device__ void fit_emit(const FitArgs& a, ProblemFit& F, int q) {
  if (F.done) {
    a.active[q] = 0;
    return;
  }
  a.map.to_log(F.lb.point(), a.p, a.log_theta + (long long)q * a.p, nullptr);
  a.active[q] = 1;
  atomicAdd(&a.hdr->active, 1);
}

__global__ void fit_init_kernel(FitArgs a) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= a.nprob) return;
  ProblemFit& F = a.fits[q];
  F.run = 0;
  F.done = 0;
  F.first_err = GPRX_OK;
  F.last_err = GPRX_OK;
  F.best_f = BARRIER_COST;
  F.iters = F.total_evals = 0;
  F.gnorm = 0.0;
  F.converged = 0;
  for (int i = 0; i < a.p; ++i) F.best_z[i] = a.z_start[(long long)q * a.runs * a.p + i];
  fit_start_run(a, F, q);
  fit_emit(a, F, q);
}

// Consumes the evaluation of every active problem and emits its next point.
__global__ void fit_round_kernel(FitArgs a) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= a.nprob) return;
  ProblemFit& F = a.fits[q];
  if (F.done || !a.active[q]) {
    a.active[q] = 0;
    return;
  }
  double lt[BATCH_MAX_VARS], jac[BATCH_MAX_VARS], g[BATCH_MAX_VARS];
  a.map.to_log(F.lb.point(), a.p, lt, jac);
  double f = a.nlml[q];
  const int st = a.status[q];
  if (st != GPRX_OK || !isfinite(f)) {
    F.last_err = st != GPRX_OK ? st : GPRX_NOT_CONVERGED;
    f = BARRIER_COST;
    for (int i = 0; i < a.p; ++i) g[i] = 0.0;
  } else {
    for (int i = 0; i < a.p; ++i) g[i] = a.grad[(long long)q * a.p + i] * jac[i];
  }
  F.lb.resume(f, g);
  // a run that ends here is followed by the next run's first point
  while (!F.done && F.lb.task() == DevLbfgs::DONE) fit_end_run(a, F, q);
  fit_emit(a, F, q);
}

struct FitResult {
  double nlml;
  uint64_t iterations, evaluations;
  double grad_norm;
  int converged;
  int status;
};

__global__ void fit_finish_kernel(FitArgs a, double* log_theta_out, FitResult* out) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= a.nprob) return;
  const ProblemFit& F = a.fits[q];
  FitResult r;
  r.nlml = F.best_f;
  r.iterations = F.iters;
  r.evaluations = F.total_evals;
  r.grad_norm = F.gnorm;
  r.converged = F.converged;
  if (F.best_f < BARRIER_COST) {
    r.status = GPRX_OK;
  } else {
    r.status = F.first_err != GPRX_OK ? F.first_err : GPRX_NOT_CONVERGED;
  }
  a.map.to_log(F.best_z, a.p, log_theta_out + (long long)q * a.p, nullptr);
  out[q] = r;
}

// ---------------------------------------------------------------------------
// host state
// ---------------------------------------------------------------------------
struct BatchState {
  int device = 0;
  cudaStream_t stream = nullptr;
  int nprob = 0, d = 0, p = 0, nmax = 0;
  gprx_options opt{};
  HostKernel kern;
  std::vector<int> n_host;
  DevBuf<double> x, y, work, theta, nlml, grad, zstart, theta_out;
  DevBuf<BatchProblem> probs;
  DevBuf<int> order, status, active;
  DevBuf<BatchHeader> hdr;
  DevBuf<ProblemFit> fits;
  DevBuf<FitResult> results;
  HostPinned<BatchHeader> hdr_h;
  int ctas = 0;
  size_t smem = 0;
  cudaGraphExec_t graph = nullptr;
  int graph_rounds = 0;
  FitArgs graph_args{};
  bool graph_valid = false;
  // schedule: in-CTA GEMM tile shape per size class, autotuned at the first
  // evaluation unless set by the caller
  std::vector<int> ord_host;  // the work order (largest n first)
  std::string tree_sig;       // kernel tree, for the process-wide tuning cache
  int8_t tiles[BATCH_SIZE_CLASSES] = {};
  float tune_ms[BATCH_SIZE_CLASSES][CG_CONFIGS] = {};
  bool tuned = false, tiles_fixed = false;
  DevBuf<int> tune_order;

  ~BatchState() {
    if (stream) cudaStreamSynchronize(stream);
    if (graph) cudaGraphExecDestroy(graph);
    if (stream) cudaStreamDestroy(stream);
  }

  gprx_status create(const double* xh, const double* yh, const uint64_t* ns, uint64_t np, uint64_t dd,
                     const gprx_kernel_node* nodes, int n_nodes, int n_theta, const gprx_options* o);
  BatchEvalArgs eval_args(const int* active_dev, const double* log_theta);
  cudaError_t launch_eval(const BatchEvalArgs& a, bool count = true);
  cudaError_t set_eval_attributes();
  gprx_status eval(const double* log_theta, double* nl, double* g, int32_t* st);
  gprx_status fit(const double* theta0, const gprx_lbfgs_options* o, double* theta_out, gprx_fit_report* reports,
                  int32_t* st_out);
  gprx_status autotune(const double* log_theta_dev, bool force);
};

static JitterList jitter_list(const gprx_options& o) {
  JitterList jl{};
  if (o.jitter_kind == GPRX_JITTER_FIXED) {
    if (o.jitter_initial > 0.0) jl.j[jl.count++] = o.jitter_initial;
    return jl;
  }
  double j = o.jitter_initial;
  for (int r = 0; r < o.jitter_max_retries && jl.count < BATCH_MAX_JITTERS; ++r) {
    if (!(j <= o.jitter_max)) break;
    jl.j[jl.count++] = j;
    double g = j * o.jitter_multiplier;
    if (!std::isfinite(g)) break;
    j = g;
  }
  return jl;
}

gprx_status BatchState::create(const double* xh, const double* yh, const uint64_t* ns, uint64_t np, uint64_t dd,
                               const gprx_kernel_node* nodes, int n_nodes, int n_theta, const gprx_options* o) {
  if (!nodes || !ns || !xh || !yh) return set_error(GPRX_INVALID_ARGUMENT, "null pointer");
  if (np == 0) return set_error(GPRX_EMPTY_INPUT, "no problems");
  if (np > (uint64_t)INT32_MAX / 2) return set_error(GPRX_CAPACITY, "too many problems");
  if (dd == 0) return set_error(GPRX_EMPTY_INPUT, "no features (d = 0)");
  if (o) opt = *o;
  else gprx_options_default(&opt);
  if (opt.jitter_kind != GPRX_JITTER_FIXED && opt.jitter_max_retries > BATCH_MAX_JITTERS)
    return set_error(GPRX_INVALID_CONFIG, "at most 8 jitter retries in a batch");
  if (n_theta < 1) return set_error(GPRX_SHAPE_MISMATCH, "theta must hold the kernel parameters and log noise");
  if (n_theta > BATCH_MAX_VARS) return set_error(GPRX_INVALID_CONFIG, "a batched kernel has at most 15 parameters");
  nprob = (int)np;
  d = (int)dd;
  n_host.resize(nprob);
  long long total = 0;
  nmax = 0;
  for (int i = 0; i < nprob; ++i) {
    if (ns[i] == 0) return set_error(GPRX_EMPTY_INPUT, "a problem has no training points");
    if (ns[i] > GPRX_BATCH_MAX_N) return set_error(GPRX_CAPACITY, "a batched problem has more than 2048 points");
    n_host[i] = (int)ns[i];
    total += (long long)ns[i];
    nmax = std::max(nmax, n_host[i]);
  }
  if (!all_finite(xh, (size_t)total * d) || !all_finite(yh, (size_t)total))
    return set_error(GPRX_NONFINITE_INPUT, "non-finite input");
  // the template tree: every problem sets its own θ-dependent constants
  std::string why;
  std::vector<double> zeros(n_theta, 0.0);
  gprx_status s = kern.init(nodes, n_nodes, zeros.data(), n_theta - 1, d, &why);
  if (s != GPRX_OK) return set_error(s, why);
  p = n_theta;
  device = opt.device;
  GPRX_CUDA_TRY(cudaSetDevice(device));
  GPRX_CUDA_TRY(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
  int sms = 0;
  GPRX_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  smem = batch_smem();
  ctas = std::min(nprob, sms);
  GPRX_CUDA_TRY(set_eval_attributes());
  const long long wd = work_doubles(nmax);
  if (x.alloc((size_t)total * d) || y.alloc((size_t)total) || probs.alloc(nprob) || order.alloc(nprob) ||
      theta.alloc((size_t)nprob * p) || nlml.alloc(nprob) || grad.alloc((size_t)nprob * p) ||
      status.alloc(nprob) || active.alloc(nprob) || hdr.alloc(1) || work.alloc((size_t)wd * ctas))
    return set_error(GPRX_OUT_OF_MEMORY, "batch device allocation failed");
  GPRX_CUDA_TRY(hdr_h.ensure(1));
  GPRX_CUDA_TRY(cudaMemcpyAsync(x.p, xh, sizeof(double) * total * d, cudaMemcpyHostToDevice, stream));
  GPRX_CUDA_TRY(cudaMemcpyAsync(y.p, yh, sizeof(double) * total, cudaMemcpyHostToDevice, stream));
  // workspaces start at zero: no stale non-finite values anywhere
  GPRX_CUDA_TRY(cudaMemsetAsync(work.p, 0, sizeof(double) * wd * ctas, stream));
  std::vector<BatchProblem> ph(nprob);
  long long off = 0;
  for (int i = 0; i < nprob; ++i) {
    ph[i].x = x.p + off * d;
    ph[i].y = y.p + off;
    ph[i].n = n_host[i];
    ph[i].pad = 0;
    off += n_host[i];
  }
  // largest problems first (longest-processing-time order over the CTAs)
  std::vector<int> ord(nprob);
  std::iota(ord.begin(), ord.end(), 0);
  std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return n_host[a] > n_host[b]; });
  ord_host = ord;
  tree_sig = std::to_string(d) + ":";
  for (int i = 0; i < n_nodes; ++i) tree_sig += std::to_string(nodes[i].kind) + "," + std::to_string(nodes[i].arg) + ";";
  GPRX_CUDA_TRY(cudaMemcpyAsync(probs.p, ph.data(), sizeof(BatchProblem) * nprob, cudaMemcpyHostToDevice, stream));
  GPRX_CUDA_TRY(cudaMemcpyAsync(order.p, ord.data(), sizeof(int) * nprob, cudaMemcpyHostToDevice, stream));
  GPRX_CUDA_TRY(cudaStreamSynchronize(stream));
  return GPRX_OK;
}

BatchEvalArgs BatchState::eval_args(const int* active_dev, const double* log_theta) {
  BatchEvalArgs a{};
  a.probs = probs.p;
  a.order = order.p;
  a.nprob = nprob;
  a.p = p;
  a.log_theta = log_theta;
  a.active = active_dev;
  a.nlml = nlml.p;
  a.grad = grad.p;
  a.status = status.p;
  a.hdr = hdr.p;
  a.work = work.p;
  a.work_stride = work_doubles(nmax);
  a.nmax = nmax;
  a.jit = jitter_list(opt);
  a.tmpl = kern.tree;
  for (int i = 0; i < 64; ++i) a.slot_param[i] = i < (int)kern.slot_param.size() ? kern.slot_param[i] : -1;
  for (int c = 0; c < BATCH_SIZE_CLASSES; ++c) a.tile_of_class[c] = tiles[c];
  return a;
}

// ---------------------------------------------------------------------------
// autotuner: for every size class present, time one evaluation launch of a
// sample of that class's problems (up to two per CTA, at the given θ) with
// each tile shape, and keep the fastest.  Results are cached per device,
// kernel tree and class for the life of the process.  Every shape gives the
// same results bit for bit (cta_gemm.cuh), so tuning changes only the time.
// ---------------------------------------------------------------------------
static std::mutex g_tune_mu;
static std::map<std::string, int> g_tune_cache;

gprx_status BatchState::autotune(const double* log_theta_dev, bool force) {
  if (tiles_fixed || (tuned && !force)) return GPRX_OK;
  cudaDeviceProp prop;
  GPRX_CUDA_TRY(cudaGetDeviceProperties(&prop, device));
  const std::string key0 = std::string(prop.name) + "|" + std::to_string(device) + "|" + tree_sig + "|";
  std::vector<std::vector<int>> by_class(BATCH_SIZE_CLASSES);
  for (int q : ord_host) by_class[batch_size_class(n_host[q])].push_back(q);
  if (tune_order.ensure((size_t)std::max(nprob, 1)) != cudaSuccess)
    return set_error(GPRX_OUT_OF_MEMORY, "tuning buffers");
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  GPRX_CUDA_TRY(cudaEventCreate(&e0));
  GPRX_CUDA_TRY(cudaEventCreate(&e1));
  struct Ev {
    cudaEvent_t a, b;
    ~Ev() { cudaEventDestroy(a); cudaEventDestroy(b); }
  } guard{e0, e1};
  for (int c = 0; c < BATCH_SIZE_CLASSES; ++c) {
    if (by_class[c].empty()) continue;
    const std::string key = key0 + std::to_string(c);
    if (!force) {
      std::lock_guard<std::mutex> lk(g_tune_mu);
      auto it = g_tune_cache.find(key);
      if (it != g_tune_cache.end()) {
        tiles[c] = (int8_t)it->second;
        continue;
      }
    }
    const int ns = (int)std::min<size_t>(by_class[c].size(), (size_t)2 * ctas);
    GPRX_CUDA_TRY(cudaMemcpyAsync(tune_order.p, by_class[c].data(), sizeof(int) * ns, cudaMemcpyHostToDevice, stream));
    BatchEvalArgs a = eval_args(nullptr, log_theta_dev);
    a.order = tune_order.p;
    a.nprob = ns;
    int best = 0;
    for (int cfg = 0; cfg < CG_CONFIGS; ++cfg) {
      a.tile_of_class[c] = (int8_t)cfg;
      GPRX_CUDA_TRY(cudaMemsetAsync(hdr.p, 0, sizeof(BatchHeader), stream));
      GPRX_CUDA_TRY(launch_eval(a));  // warm-up
      float ms = 0.0f;
      GPRX_CUDA_TRY(cudaEventRecord(e0, stream));
      for (int r = 0; r < 2; ++r) {
        GPRX_CUDA_TRY(cudaMemsetAsync(hdr.p, 0, sizeof(BatchHeader), stream));
        GPRX_CUDA_TRY(launch_eval(a));
      }
      GPRX_CUDA_TRY(cudaEventRecord(e1, stream));
      GPRX_CUDA_TRY(cudaEventSynchronize(e1));
      GPRX_CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
      tune_ms[c][cfg] = ms / 2.0f;
      if (tune_ms[c][cfg] < tune_ms[c][best]) best = cfg;
    }
    tiles[c] = (int8_t)best;
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune_cache[key] = best;
  }
  tuned = true;
  return GPRX_OK;
}

template <int ARD_D>
static cudaError_t launch_eval_t(const BatchEvalArgs& a, int ctas, size_t smem, cudaStream_t s, bool count) {
  batch_eval_kernel<ARD_D><<<ctas, BT, smem, s>>>(a);
  if (count) count_launch();
  return cudaGetLastError();
}

cudaError_t BatchState::launch_eval(const BatchEvalArgs& a, bool count) {
  switch (kern.ard_d) {
    case 0: return launch_eval_t<0>(a, ctas, smem, stream, count);
    case 4: return launch_eval_t<4>(a, ctas, smem, stream, count);
    case 8: return launch_eval_t<8>(a, ctas, smem, stream, count);
    case 16: return launch_eval_t<16>(a, ctas, smem, stream, count);
    default: return launch_eval_t<32>(a, ctas, smem, stream, count);
  }
}

cudaError_t BatchState::set_eval_attributes() {
  const int b = (int)smem;
  switch (kern.ard_d) {
    case 0: return cudaFuncSetAttribute(batch_eval_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
    case 4: return cudaFuncSetAttribute(batch_eval_kernel<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
    case 8: return cudaFuncSetAttribute(batch_eval_kernel<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
    case 16: return cudaFuncSetAttribute(batch_eval_kernel<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
    default: return cudaFuncSetAttribute(batch_eval_kernel<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
  }
}

gprx_status BatchState::eval(const double* log_theta, double* nl, double* g, int32_t* st) {
  if (!log_theta || !nl || !st) return set_error(GPRX_INVALID_ARGUMENT, "null pointer");
  GPRX_CUDA_TRY(cudaSetDevice(device));
  GPRX_CUDA_TRY(
      cudaMemcpyAsync(theta.p, log_theta, sizeof(double) * nprob * p, cudaMemcpyHostToDevice, stream));
  gprx_status ts = autotune(theta.p, false);
  if (ts != GPRX_OK) return ts;
  GPRX_CUDA_TRY(cudaMemsetAsync(hdr.p, 0, sizeof(BatchHeader), stream));
  GPRX_CUDA_TRY(cudaMemsetAsync(nlml.p, 0, sizeof(double) * nprob, stream));
  GPRX_CUDA_TRY(launch_eval(eval_args(nullptr, theta.p)));
  GPRX_CUDA_TRY(cudaMemcpyAsync(nl, nlml.p, sizeof(double) * nprob, cudaMemcpyDeviceToHost, stream));
  if (g) GPRX_CUDA_TRY(cudaMemcpyAsync(g, grad.p, sizeof(double) * nprob * p, cudaMemcpyDeviceToHost, stream));
  GPRX_CUDA_TRY(cudaMemcpyAsync(st, status.p, sizeof(int32_t) * nprob, cudaMemcpyDeviceToHost, stream));
  GPRX_CUDA_TRY(cudaStreamSynchronize(stream));
  return GPRX_OK;
}

static constexpr int ROUNDS_PER_GRAPH = 8;

gprx_status BatchState::fit(const double* theta0, const gprx_lbfgs_options* o, double* theta_out,
                            gprx_fit_report* reports, int32_t* st_out) {
  if (!theta0 || !theta_out || !st_out) return set_error(GPRX_INVALID_ARGUMENT, "null pointer");
  gprx_lbfgs_options lo;
  if (o) lo = *o;
  else gprx_lbfgs_options_default(&lo);
  if (!(lo.interval_lo > 0.0) || !(lo.interval_hi > lo.interval_lo) || !std::isfinite(lo.interval_hi))
    return set_error(GPRX_INVALID_CONFIG, "parameter interval must be 0 < lo < hi");
  if (!(lo.tolerance >= 0.0) || !std::isfinite(lo.tolerance))
    return set_error(GPRX_INVALID_CONFIG, "L-BFGS gradient tolerance must be finite and >= 0");
  if (lo.history_size > BATCH_MAX_HISTORY) return set_error(GPRX_INVALID_CONFIG, "L-BFGS history must be at most 16");
  if (lo.restarts < 0) return set_error(GPRX_INVALID_CONFIG, "restarts must be >= 0");
  GPRX_CUDA_TRY(cudaSetDevice(device));
  const int runs = lo.restarts + 1;
  LogitMap map;
  map.init(lo.interval_lo, lo.interval_hi);
  LbfgsConfig cfg;
  cfg.history = lo.history_size > 0 ? lo.history_size : 10;
  cfg.max_iterations = lo.max_iterations;
  cfg.tol_grad = lo.tolerance;
  // starting points: θ0, then the restarts' log-uniform draws of the same
  // seeded stream the single-model fit uses (every problem draws the same)
  std::vector<double> zs((size_t)nprob * runs * p);
  std::vector<double> rz((size_t)std::max(runs - 1, 0) * p);
  {
    gprx_rng rng;
    gprx_rng_seed(&rng, lo.seed);
    for (int r = 1; r < runs; ++r)
      for (int i = 0; i < p; ++i) {
        double u = gprx_rng_unit(&rng);
        const double eps = 1.0 / 9007199254740992.0;
        u = std::min(std::max(u, eps), 1.0 - eps);
        double lt = map.ln_lo + u * (map.ln_hi - map.ln_lo);
        map.from_log(&lt, 1, &rz[(size_t)(r - 1) * p + i]);
      }
  }
  for (int q = 0; q < nprob; ++q) {
    double* z = &zs[(size_t)q * runs * p];
    if (!map.from_log(theta0 + (size_t)q * p, p, z))
      return set_error(GPRX_INVALID_HYPERPARAMETER, "initial θ of problem " + std::to_string(q) +
                                                         " outside the interval");
    for (int r = 1; r < runs; ++r)
      for (int i = 0; i < p; ++i) z[(size_t)r * p + i] = rz[(size_t)(r - 1) * p + i];
  }
  if (fits.ensure(nprob) || results.ensure(nprob) || zstart.ensure(zs.size()) ||
      this->theta_out.ensure((size_t)nprob * p))
    return set_error(GPRX_OUT_OF_MEMORY, "fit buffers");
  GPRX_CUDA_TRY(cudaMemcpyAsync(zstart.p, zs.data(), sizeof(double) * zs.size(), cudaMemcpyHostToDevice, stream));
  FitArgs fa{};
  fa.fits = fits.p;
  fa.nprob = nprob;
  fa.p = p;
  fa.runs = runs;
  fa.map = map;
  fa.cfg = cfg;
  fa.z_start = zstart.p;
  fa.log_theta = theta.p;
  fa.active = active.p;
  fa.nlml = nlml.p;
  fa.grad = grad.p;
  fa.status = status.p;
  fa.hdr = hdr.p;
  const int fb = 128, fg = (nprob + fb - 1) / fb;
  GPRX_CUDA_TRY(cudaMemsetAsync(hdr.p, 0, sizeof(BatchHeader), stream));
  GPRX_LAUNCH(fit_init_kernel, fg, fb, 0, stream, fa);
  GPRX_CUDA_TRY(cudaGetLastError());
  // the schedule at the starting points, then one graph: ROUNDS_PER_GRAPH ×
  // {reset header, evaluate, advance}, then the header back to the host
  gprx_status ts = autotune(theta.p, false);
  if (ts != GPRX_OK) return ts;
  GPRX_CUDA_TRY(cudaMemsetAsync(hdr.p, 0, sizeof(BatchHeader), stream));
  const BatchEvalArgs ea = eval_args(active.p, theta.p);
  if (graph) {
    cudaGraphExecDestroy(graph);
    graph = nullptr;
  }
  cudaGraph_t gr = nullptr;
  GPRX_CUDA_TRY(launch_eval(ea));  // evaluates the starting points
  GPRX_LAUNCH(fit_round_kernel, fg, fb, 0, stream, fa);
  GPRX_CUDA_TRY(cudaGetLastError());
  GPRX_CUDA_TRY(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
  for (int r = 0; r < ROUNDS_PER_GRAPH; ++r) {
    cudaMemsetAsync(hdr.p, 0, sizeof(BatchHeader), stream);
    launch_eval(ea, false);
    fit_round_kernel<<<fg, fb, 0, stream>>>(fa);
  }
  cudaMemcpyAsync(hdr_h.p, hdr.p, sizeof(BatchHeader), cudaMemcpyDeviceToHost, stream);
  cudaError_t ce = cudaStreamEndCapture(stream, &gr);
  if (ce != cudaSuccess) return set_cuda_error(ce, "capture of the fitting rounds");
  ce = cudaGraphInstantiate(&graph, gr, 0);
  cudaGraphDestroy(gr);
  if (ce != cudaSuccess) return set_cuda_error(ce, "graph instantiation");
  // the launch counter counts the graph's kernels per replay
  const uint64_t max_rounds = (uint64_t)runs * (lo.max_iterations + 1) * 21 + 4;
  uint64_t rounds = 1;
  for (;;) {
    GPRX_CUDA_TRY(cudaGraphLaunch(graph, stream));
    count_launch(2 * ROUNDS_PER_GRAPH);
    GPRX_CUDA_TRY(cudaStreamSynchronize(stream));
    rounds += ROUNDS_PER_GRAPH;
    if (hdr_h.p->active == 0) break;
    if (rounds > max_rounds) return set_error(GPRX_TIMEOUT, "batched fit did not finish in its round bound");
  }
  GPRX_LAUNCH(fit_finish_kernel, fg, fb, 0, stream, fa, this->theta_out.p, results.p);
  GPRX_CUDA_TRY(cudaGetLastError());
  std::vector<FitResult> rh(nprob);
  GPRX_CUDA_TRY(
      cudaMemcpyAsync(theta_out, this->theta_out.p, sizeof(double) * nprob * p, cudaMemcpyDeviceToHost, stream));
  GPRX_CUDA_TRY(cudaMemcpyAsync(rh.data(), results.p, sizeof(FitResult) * nprob, cudaMemcpyDeviceToHost, stream));
  GPRX_CUDA_TRY(cudaStreamSynchronize(stream));
  for (int q = 0; q < nprob; ++q) {
    st_out[q] = rh[q].status;
    if (reports) {
      reports[q].nlml = rh[q].nlml;
      reports[q].iterations = rh[q].iterations;
      reports[q].evaluations = rh[q].evaluations;
      reports[q].grad_norm = rh[q].grad_norm;
      reports[q].converged = rh[q].converged;
    }
  }
  return GPRX_OK;
}

// ---------------------------------------------------------------------------
// Allocation-free evaluation of one exact problem (gprx_exact_eval_noalloc).
//
// For callers that cannot allocate device memory at the moment they need an
// evaluation: code running while a CUDA graph is being captured on the
// stream, inside an allocator-owned memory pool (a framework that owns every
// byte of the device, a server under a fixed HBM budget), or in a real-time
// loop where the device-wide synchronisation of cudaMalloc/cudaFree is not
// acceptable.  The scratch the evaluation needs (the header of the persistent
// kernel and one CTA workspace) lives in the file-scope array below, sized for
// problems of up to NOALLOC_MAX_N points; every device that loads the library
// holds it until the process exits.  The caller passes device inputs and
// outputs; only the θ vector and the kernel tree come from host memory.
// ---------------------------------------------------------------------------
constexpr int NOALLOC_MAX_N = 512;
constexpr int NOALLOC_MAX_DEVICES = 64;

struct NoAllocHeader {
  BatchProblem prob;
  BatchHeader hdr;
  int order[1];
  int status[1];
  int input_bad[1];
  double log_theta[BATCH_MAX_VARS];
  double nlml[1];
  double grad[BATCH_MAX_VARS];
};
// the header is padded to 256 bytes so that the workspace keeps the alignment
// the CTA GEMM's 16-byte copies rely on
constexpr long long NOALLOC_HEADER_DOUBLES = ((long long)sizeof(NoAllocHeader) + 255) / 256 * 32;
constexpr long long NOALLOC_SCRATCH_DOUBLES = NOALLOC_HEADER_DOUBLES + work_doubles(NOALLOC_MAX_N);

// 5.3 MB per device.  Host code must not pass this name to a kernel: on the
// host it is a stand-in, not a device address (see noalloc_scratch_ptr).
static __device__ __align__(256) double g_noalloc_scratch[NOALLOC_SCRATCH_DOUBLES];

struct NoAllocTheta {
  double v[BATCH_MAX_VARS];
};

constexpr int NOALLOC_PREP_THREADS = 256;

// Writes the header of this call (everything the evaluation reads that must
// start fresh: the queue counter, the problem, θ, the status) and checks the
// caller's x and y for non-finite values, which the host cannot see here
// (TrainInput::validate, src/data.rs).
__global__ void __launch_bounds__(NOALLOC_PREP_THREADS) noalloc_prep_kernel(double* scratch, BatchProblem prob,
                                                                            NoAllocTheta th, int p, int d) {
  __shared__ int bad;
  NoAllocHeader* h = reinterpret_cast<NoAllocHeader*>(scratch);
  if (threadIdx.x == 0) bad = 0;
  __syncthreads();
  const long long nx = (long long)prob.n * d;
  int mine = 0;
  for (long long i = threadIdx.x; i < nx + prob.n; i += blockDim.x) {
    double v = i < nx ? prob.x[i] : prob.y[i - nx];
    if (!isfinite(v)) mine = 1;
  }
  if (mine) atomicOr(&bad, 1);
  __syncthreads();
  if (threadIdx.x != 0) return;
  h->prob = prob;
  h->hdr.queue = 0;
  h->hdr.active = 0;
  h->order[0] = 0;
  h->status[0] = GPRX_NOT_CONVERGED;  // overwritten by the evaluation
  h->input_bad[0] = bad;
  h->nlml[0] = 0.0;
  for (int i = 0; i < BATCH_MAX_VARS; ++i) {
    h->log_theta[i] = i < p ? th.v[i] : 0.0;
    h->grad[i] = 0.0;
  }
}

__global__ void noalloc_finish_kernel(const double* scratch, int p, double* nlml, double* grad, int32_t* status) {
  const NoAllocHeader* h = reinterpret_cast<const NoAllocHeader*>(scratch);
  const int i = threadIdx.x;
  const int st = h->input_bad[0] ? (int)GPRX_NONFINITE_INPUT : h->status[0];
  if (i == 0) {
    *status = st;
    *nlml = st == GPRX_OK ? h->nlml[0] : 0.0;
  }
  if (grad && i < p) grad[i] = st == GPRX_OK ? h->grad[i] : 0.0;
}

// Device address of g_noalloc_scratch on the current device, looked up once
// per device (with that device current) and kept.
static gprx_status noalloc_scratch_ptr(int dev, double** out) {
  static std::mutex mu;
  static double* ptrs[NOALLOC_MAX_DEVICES] = {};
  if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) return set_error(GPRX_INVALID_CONFIG, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(mu);
  if (!ptrs[dev]) {
    double* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress((void**)&p, g_noalloc_scratch);
    if (e != cudaSuccess) return set_cuda_error(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
    const int smem = (int)batch_smem();
    cudaFuncAttribute a = cudaFuncAttributeMaxDynamicSharedMemorySize;
    if ((e = cudaFuncSetAttribute(batch_eval_kernel<0>, a, smem)) != cudaSuccess ||
        (e = cudaFuncSetAttribute(batch_eval_kernel<4>, a, smem)) != cudaSuccess ||
        (e = cudaFuncSetAttribute(batch_eval_kernel<8>, a, smem)) != cudaSuccess ||
        (e = cudaFuncSetAttribute(batch_eval_kernel<16>, a, smem)) != cudaSuccess ||
        (e = cudaFuncSetAttribute(batch_eval_kernel<32>, a, smem)) != cudaSuccess)
      return set_cuda_error(e, "shared-memory attribute of the evaluation kernel");
    ptrs[dev] = p;
  }
  *out = ptrs[dev];
  return GPRX_OK;
}

// Makes `dev` the current device for the life of the guard.
struct NoAllocDeviceGuard {
  int prev = -1;
  cudaError_t set(int dev) {
    cudaError_t e = cudaGetDevice(&prev);
    if (e != cudaSuccess) return e;
    return prev == dev ? cudaSuccess : cudaSetDevice(dev);
  }
  ~NoAllocDeviceGuard() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

static gprx_status exact_eval_noalloc(const double* x, const double* y, uint64_t n, uint64_t d,
                                      const gprx_kernel_node* nodes, int32_t n_nodes, const double* params,
                                      uint64_t p, const gprx_options* opts, double* nlml, double* grad,
                                      int32_t* status, void* stream) {
  // The scratch and the launch belong to the device that owns the stream
  // (the current device for the NULL stream); options.device must name it.
  cudaStream_t s = (cudaStream_t)stream;
  int dev = 0;
  if (s) {
    GPRX_CUDA_TRY(cudaStreamGetDevice(s, &dev));
  } else {
    GPRX_CUDA_TRY(cudaGetDevice(&dev));
  }
  if (opts && opts->device != dev)
    return set_error(GPRX_INVALID_CONFIG, "options.device must be the device that owns the stream");
  NoAllocDeviceGuard guard;
  GPRX_CUDA_TRY(guard.set(dev));
  double* scratch = nullptr;
  gprx_status st = noalloc_scratch_ptr(dev, &scratch);
  if (st != GPRX_OK) return st;
  if (n == 0) return GPRX_OK;  // set-up only: nothing is enqueued
  if (!x || !y || !nodes || !params || !nlml || !status) return set_error(GPRX_INVALID_ARGUMENT, "null pointer");
  if (d == 0) return set_error(GPRX_EMPTY_INPUT, "no features (d = 0)");
  if (n > (uint64_t)NOALLOC_MAX_N)
    return set_error(GPRX_CAPACITY, "gprx_exact_eval_noalloc takes at most 512 points (its fixed scratch size); "
                                    "use gprx_exact_eval or gprx_batch_eval for larger problems");
  if (p < 1 || p > (uint64_t)BATCH_MAX_VARS)
    return set_error(GPRX_INVALID_CONFIG, "gprx_exact_eval_noalloc takes 1..16 parameters");
  gprx_options o;
  if (opts) o = *opts;
  else gprx_options_default(&o);
  if (o.jitter_kind != GPRX_JITTER_FIXED && o.jitter_max_retries > BATCH_MAX_JITTERS)
    return set_error(GPRX_INVALID_CONFIG, "at most 8 jitter retries");
  HostKernel kern;
  std::string why;
  st = kern.init(nodes, n_nodes, params, (int)p - 1, (int)d, &why);
  if (st != GPRX_OK) return set_error(st, why);
  NoAllocHeader* h = reinterpret_cast<NoAllocHeader*>(scratch);  // a device address
  BatchProblem prob{x, y, (int)n, 0};
  NoAllocTheta th{};
  for (uint64_t i = 0; i < p; ++i) th.v[i] = params[i];
  BatchEvalArgs a{};
  a.probs = &h->prob;
  a.order = h->order;
  a.nprob = 1;
  a.p = (int)p;
  a.log_theta = h->log_theta;
  a.active = nullptr;
  a.nlml = h->nlml;
  a.grad = h->grad;
  a.status = h->status;
  a.hdr = &h->hdr;
  a.work = scratch + NOALLOC_HEADER_DOUBLES;
  a.work_stride = 0;
  a.nmax = (int)n;
  a.jit = jitter_list(o);
  a.tmpl = kern.tree;
  for (int i = 0; i < 64; ++i) a.slot_param[i] = i < (int)kern.slot_param.size() ? kern.slot_param[i] : -1;
  const size_t smem = batch_smem();
  noalloc_prep_kernel<<<1, NOALLOC_PREP_THREADS, 0, s>>>(scratch, prob, th, (int)p, (int)d);
  switch (kern.ard_d) {
    case 0: batch_eval_kernel<0><<<1, BT, smem, s>>>(a); break;
    case 4: batch_eval_kernel<4><<<1, BT, smem, s>>>(a); break;
    case 8: batch_eval_kernel<8><<<1, BT, smem, s>>>(a); break;
    case 16: batch_eval_kernel<16><<<1, BT, smem, s>>>(a); break;
    default: batch_eval_kernel<32><<<1, BT, smem, s>>>(a); break;
  }
  noalloc_finish_kernel<<<1, 32, 0, s>>>(scratch, (int)p, nlml, grad, status);
  count_launch(3);
  GPRX_CUDA_TRY(cudaGetLastError());
  return GPRX_OK;
}

}  // namespace gprx

using namespace gprx;

struct gprx_batch {
  BatchState s;
};

extern "C" {

gprx_status gprx_batch_create(const double* x, const double* y, const uint64_t* n, uint64_t n_problems,
                              uint64_t d, const gprx_kernel_node* nodes, int32_t n_nodes, int32_t n_theta,
                              const gprx_options* options, gprx_batch** out) {
  if (!out) return set_error(GPRX_INVALID_ARGUMENT, "null out");
  *out = nullptr;
  std::unique_ptr<gprx_batch> h(new (std::nothrow) gprx_batch());
  if (!h) return set_error(GPRX_OUT_OF_MEMORY, "handle");
  gprx_status st = h->s.create(x, y, n, n_problems, d, nodes, n_nodes, n_theta, options);
  if (st != GPRX_OK) return st;
  *out = h.release();
  return GPRX_OK;
}

gprx_status gprx_batch_destroy(gprx_batch* h) {
  delete h;
  return GPRX_OK;
}

uint64_t gprx_batch_num_params(const gprx_batch* h) { return h ? (uint64_t)h->s.p : 0; }

gprx_status gprx_batch_eval(gprx_batch* h, const double* params, uint64_t p, double* nlml, double* grad,
                            int32_t* status) {
  if (!h) return set_error(GPRX_INVALID_ARGUMENT, "null handle");
  if (p != (uint64_t)h->s.p) return set_error(GPRX_SHAPE_MISMATCH, "params must hold p values per problem");
  return h->s.eval(params, nlml, grad, status);
}

gprx_status gprx_batch_fit(gprx_batch* h, const double* params0, uint64_t p, const gprx_lbfgs_options* opt,
                           double* params_out, gprx_fit_report* reports, int32_t* status) {
  if (!h) return set_error(GPRX_INVALID_ARGUMENT, "null handle");
  if (p != (uint64_t)h->s.p) return set_error(GPRX_SHAPE_MISMATCH, "params must hold p values per problem");
  return h->s.fit(params0, opt, params_out, reports, status);
}

gprx_status gprx_batch_autotune(gprx_batch* h, const double* params, uint64_t p) {
  if (!h || !params) return set_error(GPRX_INVALID_ARGUMENT, "null pointer");
  if (p != (uint64_t)h->s.p) return set_error(GPRX_SHAPE_MISMATCH, "params must hold p values per problem");
  BatchState& s = h->s;
  GPRX_CUDA_TRY(cudaSetDevice(s.device));
  GPRX_CUDA_TRY(cudaMemcpyAsync(s.theta.p, params, sizeof(double) * s.nprob * s.p, cudaMemcpyHostToDevice, s.stream));
  s.tiles_fixed = false;
  return s.autotune(s.theta.p, true);
}

gprx_status gprx_batch_set_schedule(gprx_batch* h, const int32_t* tile_of_class) {
  if (!h || !tile_of_class) return set_error(GPRX_INVALID_ARGUMENT, "null pointer");
  for (int c = 0; c < BATCH_SIZE_CLASSES; ++c)
    if (tile_of_class[c] < 0 || tile_of_class[c] >= CG_CONFIGS)
      return set_error(GPRX_INVALID_CONFIG, "tile shape index out of range");
  for (int c = 0; c < BATCH_SIZE_CLASSES; ++c) h->s.tiles[c] = (int8_t)tile_of_class[c];
  h->s.tiles_fixed = true;
  return GPRX_OK;
}

gprx_status gprx_batch_schedule(const gprx_batch* h, int32_t* tile_of_class, float* tune_ms, int32_t* tuned) {
  if (!h) return set_error(GPRX_INVALID_ARGUMENT, "null handle");
  for (int c = 0; c < BATCH_SIZE_CLASSES; ++c) {
    if (tile_of_class) tile_of_class[c] = h->s.tiles[c];
    for (int k = 0; k < CG_CONFIGS && tune_ms; ++k) tune_ms[c * CG_CONFIGS + k] = h->s.tune_ms[c][k];
  }
  if (tuned) *tuned = h->s.tuned ? 1 : 0;
  return GPRX_OK;
}

gprx_status gprx_batch_stream(gprx_batch* h, void** stream) {
  if (!h || !stream) return set_error(GPRX_INVALID_ARGUMENT, "null pointer");
  *stream = (void*)h->s.stream;
  return GPRX_OK;
}

gprx_status gprx_exact_eval_noalloc(const double* x, const double* y, uint64_t n, uint64_t d,
                                    const gprx_kernel_node* nodes, int32_t n_nodes, const double* params, uint64_t p,
                                    const gprx_options* options, double* nlml, double* grad, int32_t* status,
                                    void* stream) {
  return exact_eval_noalloc(x, y, n, d, nodes, n_nodes, params, p, options, nlml, grad, status, stream);
}

}  // extern "C"
