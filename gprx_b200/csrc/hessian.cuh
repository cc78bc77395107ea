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
};

// Partial sums (HESS_MAX_PARAMS per block, blocks in *blocks_out) of
// Σ_{a ≥ b} c_ab W_ab ∂²K_ab/∂θ_i∂θ_j for j = i..n_par−1 at slot j − i,
// W = ααᵀ − M, M the lower triangle of A⁻¹ (ld).
cudaError_t hess_second(const HostKernel& k, const HessMap& hm, int i, const double* x, long long ldx, int n,
                        const double* kinv, long long ld, const double* alpha, double* partials, int* blocks_out,
                        cudaStream_t s);
// out (n×n, both triangles, ld) = ∂K/∂θ_i.
cudaError_t fill_deriv(const HostKernel& k, const HessMap& hm, int i, const double* x, long long ldx, int n,
                       double* out, long long ld, cudaStream_t s);
// Partial sums of Σ X ∘ Y over the n×n blocks (ld).
cudaError_t dot_nn(const double* X, const double* Y, long long ld, int n, double* partials, int* blocks_out,
                   cudaStream_t s);

// Partial sums of Σ_{a,b} X(a,b) Y(b,a) = tr(X Y) over the n×n blocks (ld).
cudaError_t dot_nt(const double* X, const double* Y, long long ld, int n, double* partials, int* blocks_out,
                   cudaStream_t s);
// M (n×n, ldm, both triangles) from the lower triangle of Lw (ldl).
cudaError_t symmetrize(const double* Lw, long long ldl, int n, double* M, long long ldm, cudaStream_t s);
// out[q] = Σ_b partials[b·stride + q], q < nq.
cudaError_t reduce_slots(const double* partials, int blocks, int stride, int nq, double* out, cudaStream_t s);
// out = trace of M (n×n, ld).
cudaError_t trace_dev(const double* M, long long ld, int n, double* out, cudaStream_t s);

}  // namespace gprx
