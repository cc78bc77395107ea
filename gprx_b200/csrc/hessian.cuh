// hessian.cuh — device pieces of the exact NLML's Hessian (hessian.cu).
#pragma once

#include <algorithm>
#include <string>

#include "kernels.cuh"

namespace gprx {

constexpr int HESS_MAX_PARAMS = 40;   // GPRX_MAX_PARAMS
constexpr int HESS_MAX_BLOCKS = 148 * 4;

// θ index → (leaf, index among that leaf's parameters), for the kernel's
// parameters (the noise is handled on the host).
struct HessMap {
  int n_par;
  int leaf_of[HESS_MAX_PARAMS];
  int local_of[HESS_MAX_PARAMS];
  unsigned terms_of[HESS_MAX_PARAMS];  // bit t: term t holds the parameter's leaf
};

// All rows of the second-order part in one launch when the kernel has at
// most HESS_FUSE_K parameters; the Frobenius products of at most HESS_FUSE_P
// matrices in one pass.
constexpr int HESS_FUSE_K = 10;
constexpr int HESS_FUSE_P = 11;
struct HessMats {
  const double* m[HESS_FUSE_P];
};

// Partial sums (HESS_MAX_PARAMS per block, blocks in *blocks_out) of
// Σ_{a ≥ b} c_ab W_ab ∂²K_ab/∂θ_i∂θ_j for j = i..n_par−1 at slot j − i,
// W = ααᵀ − M, M the lower triangle of A⁻¹ (ld).
cudaError_t hess_second(const HostKernel& k, const HessMap& hm, int i, const double* x, long long ldx, int n,
                        const double* kinv, long long ld, const double* alpha, double* partials, int* blocks_out,
                        cudaStream_t s);
// Partial sums (HESS_FUSE_K·(HESS_FUSE_K+1)/2 per block, packed upper
// triangle row by row) of the same contraction for every i ≤ j < n_par in one
// launch; n_par ≤ HESS_FUSE_K.
constexpr int HESS_FUSE_SLOTS = HESS_FUSE_K * (HESS_FUSE_K + 1) / 2;
cudaError_t hess_second_all(const HostKernel& k, const HessMap& hm, const double* x, long long ldx, int n,
                            const double* kinv, long long ld, const double* alpha, double* partials, int* blocks_out,
                            cudaStream_t s);
constexpr int HESS_TRACE_SLOTS = HESS_FUSE_P * (HESS_FUSE_P + 1) / 2;
// Partial sums (HESS_TRACE_SLOTS per block, packed lower triangle row by
// row) of ⟨M_i, M_j⟩_F = Σ_{a≥b} c_ab M_i(a,b) M_j(a,b) for symmetric M_i
// stored in their lower triangles (c = 1 on the diagonal, 2 off it), every
// j ≤ i < np, np ≤ HESS_FUSE_P.
cudaError_t sym_products(const HessMats& mats, int np, long long ld, int n, double* partials, int* blocks_out,
                         cudaStream_t s);
// out (n×n, both triangles, ld) = ∂K/∂θ_i.
cudaError_t fill_deriv(const HostKernel& k, const HessMap& hm, int i, const double* x, long long ldx, int n,
                       double* out, long long ld, cudaStream_t s);
// out[q] = Σ_b partials[b·stride + q], q < nq.
cudaError_t reduce_slots(const double* partials, int blocks, int stride, int nq, double* out, cudaStream_t s);
// out = trace of M (n×n, ld).
cudaError_t trace_dev(const double* M, long long ld, int n, double* out, cudaStream_t s);

}  // namespace gprx
