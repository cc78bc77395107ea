// common.cuh — shared device infrastructure of the gprx B200 backend.
//
//  * DevStatus: the device-side status word every kernel of a pipeline reads
//    first and writes on failure (non-positive pivot, non-finite kernel value,
//    bounded wait that ran out).  Kernels never trap; the host reads the word
//    after the stream drains and maps it onto a gprx_status.
//  * KTree: a KernelSpec tree (src/kernel/spec.rs:106) in sum-of-products
//    form, evaluated per matrix entry with static register indexing.
//  * launch bookkeeping (gprx_launch_count).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/gprx_cuda.h"

namespace gprx {

// ---------------------------------------------------------------------------
// status word
// ---------------------------------------------------------------------------
struct DevStatus {
  int code;       // GPRX_OK or a gprx_status
  int stage;      // GPRX_STAGE_* for CHOLESKY_FAILED
  long long info; // failing row / index
};

__device__ __forceinline__ bool dev_failed(const DevStatus* st) {
  return st != nullptr && *(volatile const int*)&st->code != GPRX_OK;
}

__device__ __forceinline__ void dev_fail(DevStatus* st, int code, long long info) {
  if (st == nullptr) return;
  if (atomicCAS(&st->code, GPRX_OK, code) == GPRX_OK) {
    st->info = info;
  }
}

// ---------------------------------------------------------------------------
// launch accounting
// ---------------------------------------------------------------------------
void count_launch(int k = 1);
uint64_t launches();

#define GPRX_LAUNCH(kernel, grid, block, smem, stream, ...)            \
  do {                                                                 \
    kernel<<<(grid), (block), (smem), (stream)>>>(__VA_ARGS__);        \
    ::gprx::count_launch();                                            \
  } while (0)

// ---------------------------------------------------------------------------
// kernel tree in sum-of-products form
// ---------------------------------------------------------------------------
constexpr int KT_MAX_LEAVES = 8;
constexpr int KT_MAX_TERMS = 8;
constexpr int KT_ACC_PER_LEAF = 2;  // ∂/∂ of a non-ARD leaf: ≤ 2 parameters

struct KLeaf {
  int kind;      // GPRX_LEAF_*
  int param;     // first θ index
  double c0;     // RBF: 1/(2ℓ²); CONSTANT: c; PERIODIC: π/p
  double c1;     // PERIODIC: 1/ℓ²
};

struct KTree {
  int n_leaves;
  int n_terms;
  int n_params;               // kernel parameters
  int d;
  int ard_leaf;               // index of the single RBF_ARD leaf, or -1
  int ard_param;              // its first θ index
  unsigned term_mask[KT_MAX_TERMS];
  KLeaf leaf[KT_MAX_LEAVES];
  double inv_ell2[GPRX_MAX_DIM];  // ARD 1/ℓ_f²
  double diag_value;          // k(x, x) (stationary: the same for every x)
};

#ifndef GPRX_HD
#define GPRX_HD __host__ __device__
#endif

// Derived constants of every leaf from θ (log space, depth-first order) and
// k(x, x).  Returns GPRX_OK or GPRX_INVALID_HYPERPARAMETER.  Host and device
// use the same formulas (rbf.rs:18, constant.rs:12, periodic.rs:598-638,
// rbf_ard.rs:16).
GPRX_HD inline int kt_set_theta(KTree& t, const double* th) {
  for (int i = 0; i < t.n_params; ++i)
    if (!isfinite(th[i])) return GPRX_INVALID_HYPERPARAMETER;
  double v0[KT_MAX_LEAVES];
  for (int l = 0; l < t.n_leaves; ++l) {
    KLeaf& lf = t.leaf[l];
    const double* p = th + lf.param;
    switch (lf.kind) {
      case GPRX_LEAF_RBF: {
        double ell = exp(p[0]);
        lf.c0 = 0.5 / (ell * ell);
        v0[l] = 1.0;
        break;
      }
      case GPRX_LEAF_CONSTANT:
        lf.c0 = exp(p[0]);
        v0[l] = lf.c0;
        break;
      case GPRX_LEAF_PERIODIC: {
        double ell = exp(p[0]), per = exp(p[1]);
        lf.c0 = M_PI / per;
        lf.c1 = 1.0 / (ell * ell);
        v0[l] = 1.0;
        break;
      }
      case GPRX_LEAF_RBF_ARD:
        for (int f = 0; f < t.d; ++f) {
          double ell = exp(p[f]);
          t.inv_ell2[f] = 1.0 / (ell * ell);
        }
        v0[l] = 1.0;
        break;
      default:
        v0[l] = 0.0;
    }
    if (!isfinite(lf.c0) || !isfinite(lf.c1)) return GPRX_INVALID_HYPERPARAMETER;
  }
  double k0 = 0.0;
  for (int tt = 0; tt < t.n_terms; ++tt) {
    double pr = 1.0;
    for (int l = 0; l < t.n_leaves; ++l)
      if ((t.term_mask[tt] >> l) & 1u) pr *= v0[l];
    k0 += pr;
  }
  t.diag_value = k0;
  return GPRX_OK;
}

// The pair evaluators take W pairs at once: the W evaluations are
// independent chains of FP64 math that the scheduler interleaves, which keeps
// the FP64 pipe busy when few warps are resident (one 256-thread CTA per SM in
// the batched path).  W = 1 is the single-pair form of the large kernels.

// Leaf values at W pairs.  dx[w][f] = x1_f − x2_f of pair w, r2[w] = |dx|².
// NL bounds the leaves a caller's trees have (registers scale with it).
template <int ARD_D, int W, int NL = KT_MAX_LEAVES>
__device__ __forceinline__ void kt_leaf_values_w(const KTree& t, const double (&dx)[W][ARD_D > 0 ? ARD_D : 1],
                                                 const double (&r2)[W], double (&v)[NL][W]) {
  double ard_q[W];
#pragma unroll
  for (int w = 0; w < W; ++w) {
    ard_q[w] = 0.0;
    if (ARD_D > 0) {
#pragma unroll
      for (int f = 0; f < (ARD_D > 0 ? ARD_D : 1); ++f)
        if (f < t.d) ard_q[w] = fma(dx[w][f] * dx[w][f], t.inv_ell2[f], ard_q[w]);
    }
  }
#pragma unroll
  for (int l = 0; l < NL; ++l) {
    if (l >= t.n_leaves) {
#pragma unroll
      for (int w = 0; w < W; ++w) v[l][w] = 0.0;
      continue;
    }
    const KLeaf& lf = t.leaf[l];
    switch (lf.kind) {
      case GPRX_LEAF_CONSTANT:
#pragma unroll
        for (int w = 0; w < W; ++w) v[l][w] = lf.c0;
        break;
      case GPRX_LEAF_RBF:
#pragma unroll
        for (int w = 0; w < W; ++w) v[l][w] = exp(-r2[w] * lf.c0);
        break;
      case GPRX_LEAF_RBF_ARD:
#pragma unroll
        for (int w = 0; w < W; ++w) v[l][w] = exp(-0.5 * ard_q[w]);
        break;
      case GPRX_LEAF_PERIODIC: {
        double s[W];
#pragma unroll
        for (int w = 0; w < W; ++w) s[w] = sin(lf.c0 * sqrt(fmax(r2[w], 0.0)));
#pragma unroll
        for (int w = 0; w < W; ++w) v[l][w] = exp(-2.0 * s[w] * s[w] * lf.c1);
        break;
      }
      default:
#pragma unroll
        for (int w = 0; w < W; ++w) v[l][w] = 0.0;
    }
  }
}

template <int W, int NL = KT_MAX_LEAVES>
__device__ __forceinline__ void kt_combine_w(const KTree& t, const double (&v)[NL][W], double (&k)[W]) {
#pragma unroll
  for (int w = 0; w < W; ++w) k[w] = 0.0;
#pragma unroll
  for (int tt = 0; tt < KT_MAX_TERMS; ++tt) {
    if (tt >= t.n_terms) break;
    const unsigned mask = t.term_mask[tt];
    double p[W];
#pragma unroll
    for (int w = 0; w < W; ++w) p[w] = 1.0;
#pragma unroll
    for (int l = 0; l < NL; ++l)
      if ((mask >> l) & 1u) {
#pragma unroll
        for (int w = 0; w < W; ++w) p[w] *= v[l][w];
      }
#pragma unroll
    for (int w = 0; w < W; ++w) k[w] += p[w];
  }
}

// k(x1, x2) at W pairs.
template <int ARD_D, int W, int NL = KT_MAX_LEAVES>
__device__ __forceinline__ void kt_value_w(const KTree& t, const double (&dx)[W][ARD_D > 0 ? ARD_D : 1],
                                           const double (&r2)[W], double (&k)[W]) {
  double v[NL][W];
  kt_leaf_values_w<ARD_D, W, NL>(t, dx, r2, v);
  kt_combine_w<W, NL>(t, v, k);
}

// k(x1, x2) at one pair.
template <int ARD_D>
__device__ __forceinline__ double kt_value(const KTree& t, const double* dx, double r2) {
  constexpr int AD = ARD_D > 0 ? ARD_D : 1;
  double d1[1][AD];
#pragma unroll
  for (int f = 0; f < AD; ++f) d1[0][f] = dx[f];
  const double r[1] = {r2};
  double k[1];
  kt_value_w<ARD_D, 1>(t, d1, r, k);
  return k[0];
}

// Accumulates wt[w] · ∂k/∂θ of W pairs into per-leaf slots (acc_leaf[l][0..1])
// and per-dim ARD slots (acc_ard[f]); the host maps slots to θ indices.  A Sum
// gives each term the same weight; a Product gives a factor the weight times
// the other factors (src/kernel/compiled/weighted.rs:274-345).
template <int ARD_D, int W, int NL = KT_MAX_LEAVES>
__device__ __forceinline__ void kt_accumulate_grad_w(const KTree& t, const double (&dx)[W][ARD_D > 0 ? ARD_D : 1],
                                                     const double (&r2)[W], const double (&wt)[W],
                                                     double (&acc_leaf)[NL][KT_ACC_PER_LEAF],
                                                     double (&acc_ard)[ARD_D > 0 ? ARD_D : 1]) {
  double v[NL][W];
  kt_leaf_values_w<ARD_D, W, NL>(t, dx, r2, v);
  double adj[NL][W];
#pragma unroll
  for (int l = 0; l < NL; ++l)
#pragma unroll
    for (int w = 0; w < W; ++w) adj[l][w] = 0.0;
#pragma unroll
  for (int tt = 0; tt < KT_MAX_TERMS; ++tt) {
    if (tt >= t.n_terms) break;
    const unsigned mask = t.term_mask[tt];
#pragma unroll
    for (int l = 0; l < NL; ++l) {
      if (!((mask >> l) & 1u)) continue;
      double others[W];
#pragma unroll
      for (int w = 0; w < W; ++w) others[w] = 1.0;
#pragma unroll
      for (int o = 0; o < NL; ++o)
        if (o != l && ((mask >> o) & 1u)) {
#pragma unroll
          for (int w = 0; w < W; ++w) others[w] *= v[o][w];
        }
#pragma unroll
      for (int w = 0; w < W; ++w) adj[l][w] += others[w];
    }
  }
#pragma unroll
  for (int l = 0; l < NL; ++l) {
    if (l >= t.n_leaves) break;
    const KLeaf& lf = t.leaf[l];
    switch (lf.kind) {
      case GPRX_LEAF_CONSTANT:
#pragma unroll
        for (int w = 0; w < W; ++w) acc_leaf[l][0] = fma(wt[w] * adj[l][w], lf.c0, acc_leaf[l][0]);
        break;
      case GPRX_LEAF_RBF:
#pragma unroll
        for (int w = 0; w < W; ++w)
          acc_leaf[l][0] = fma(wt[w] * adj[l][w] * v[l][w], 2.0 * lf.c0 * r2[w], acc_leaf[l][0]);
        break;
      case GPRX_LEAF_RBF_ARD:
        if (ARD_D > 0) {
#pragma unroll
          for (int w = 0; w < W; ++w) {
            const double wv = wt[w] * adj[l][w] * v[l][w];
#pragma unroll
            for (int f = 0; f < (ARD_D > 0 ? ARD_D : 1); ++f)
              if (f < t.d) acc_ard[f] = fma(wv, dx[w][f] * dx[w][f] * t.inv_ell2[f], acc_ard[f]);
          }
        }
        break;
      case GPRX_LEAF_PERIODIC: {
        double a[W], s[W], c[W];
#pragma unroll
        for (int w = 0; w < W; ++w) {
          a[w] = lf.c0 * sqrt(fmax(r2[w], 0.0));
          sincos(a[w], &s[w], &c[w]);
        }
#pragma unroll
        for (int w = 0; w < W; ++w) {
          const double wv = wt[w] * adj[l][w] * v[l][w] * 4.0 * lf.c1 * s[w];
          acc_leaf[l][0] = fma(wv, s[w], acc_leaf[l][0]);
          acc_leaf[l][1] = fma(wv, c[w] * a[w], acc_leaf[l][1]);
        }
        break;
      }
      default:
        break;
    }
  }
}

template <int ARD_D>
__device__ __forceinline__ void kt_accumulate_grad(const KTree& t, const double* dx, double r2, double w,
                                                   double (&acc_leaf)[KT_MAX_LEAVES][KT_ACC_PER_LEAF],
                                                   double (&acc_ard)[ARD_D > 0 ? ARD_D : 1]) {
  constexpr int AD = ARD_D > 0 ? ARD_D : 1;
  double d1[1][AD];
#pragma unroll
  for (int f = 0; f < AD; ++f) d1[0][f] = dx[f];
  const double r[1] = {r2};
  const double wt[1] = {w};
  kt_accumulate_grad_w<ARD_D, 1>(t, d1, r, wt, acc_leaf, acc_ard);
}

// Number of accumulator slots and the θ index of each (host side).
int kt_num_slots(int ard_d);

// ---------------------------------------------------------------------------
// small device helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Block-wide sum; `red` holds ≥ 32 doubles of shared memory.  All threads get
// the result.  Fixed order: deterministic for a fixed block size.
__device__ __forceinline__ double block_sum(double v, double* red) {
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int nw = (blockDim.x + 31) >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  double s = 0.0;
  if (warp == 0) {
    s = lane < nw ? red[lane] : 0.0;
    s = warp_sum(s);
    if (lane == 0) red[0] = s;
  }
  __syncthreads();
  s = red[0];
  __syncthreads();
  return s;
}

inline int ceil_div(long long a, long long b) { return (int)((a + b - 1) / b); }

}  // namespace gprx
