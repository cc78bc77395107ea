// dense_f64.cuh — blocked FP64 dense kernels and drivers (host API).
#pragma once

#include "common.cuh"
#include <vector>

#include "gemm_f64.cuh"

namespace gprx {

// Panel width of the blocked factor / inverse / solves.  The in-place GEMM
// steps need it ≤ the 128-wide GEMM tile.
constexpr int NB = 128;

// C = alpha·opA·opB + beta·C with the 128×128 DMMA tile (see gemm_f64.cuh).
cudaError_t dgemm(bool ta, bool tb, const GemmParams& p, cudaStream_t s, int batch = 1);
// A·B (NN) with 64×64 tiles when 128×128 tiles would leave most SMs idle
// (fewer than two waves); C must not alias A or B.
cudaError_t dgemm_nn_fill(const GemmParams& p, cudaStream_t s, int batch);

// Small helper building GemmParams.
GemmParams gemm_params(int M, int N, int K, const double* A, long long lda, const double* B, long long ldb,
                       double* C, long long ldc, double alpha, double beta, const DevStatus* st);

// Side streams and events of the look-ahead factorization (one per handle):
// aux carries the chain, aux2 the column update's rows below the diagonal
// block (concurrent with the diagonal block).
struct FactorCtx {
  int device = -1;
  cudaStream_t aux = nullptr;
  cudaStream_t aux2 = nullptr;
  std::vector<cudaEvent_t> ev;
  ~FactorCtx();
  cudaError_t ensure(int nblk);
};

// In-place lower Cholesky of A (n×n, ld) by right-looking blocks of NB.
// linv receives the inverse of every diagonal block (ceil(n/NB) blocks of
// NB×NB, column-major, ld NB).  A non-positive pivot sets st (CHOLESKY_FAILED,
// info = global row) and every later kernel of the stream returns at once.
// With ctx, the chain column update → diagonal block → panel solve of step
// k+1 runs on ctx->aux (high priority) while the trailing update of step k
// runs on s; on return all work is ordered before later work on s.
cudaError_t potrf_blocked(double* A, long long ld, int n, double* linv, DevStatus* st, cudaStream_t s,
                          FactorCtx* ctx = nullptr);

// Inverses of the diagonal NB-blocks of a lower triangle (unit: unit diagonal).
cudaError_t tri_inv_blocks(const double* L, long long ld, int n, bool unit, double* linv, DevStatus* st,
                           cudaStream_t s);

// X = L⁻¹ into X (n×n, ldx), from L and its diagonal block inverses.  X's
// strict upper triangle must be zero on entry; scratch holds ceil(n/2)²
// doubles.
cudaError_t trtri_blocked(const double* L, long long ld, int n, const double* linv, double* X, long long ldx,
                          double* scratch, DevStatus* st, cudaStream_t s);

// C (lower) = Xᵀ X for lower-triangular X: K⁻¹ from X = L⁻¹.
cudaError_t lauum_lower(const double* X, long long ldx, int n, double* C, long long ldc, DevStatus* st,
                        cudaStream_t s);

struct EmuWork;

// B (n×q, ldb) := L⁻¹ B   /   := L⁻ᵀ B, with L's diagonal block inverses.
cudaError_t trsm_lower(const double* L, long long ld, int n, const double* linv, double* B, long long ldb, int q,
                       DevStatus* st, cudaStream_t s);
cudaError_t trsm_lower_t(const double* L, long long ld, int n, const double* linv, double* B, long long ldb, int q,
                         DevStatus* st, cudaStream_t s);

// The same two solves for wide B (q ≫ n) by recursive halving: X1 from the
// top half, one rank-n1 update B2 −= L21 X1 (L21ᵀ X2 for the transpose), then
// the bottom half; blocks of at most `leaf` rows use trsm_lower /
// trsm_lower_t.  The updates have K = n/2, n/4, … instead of NB, so the
// DGEMMs run near their large-K rate.
cudaError_t trsm_lower_rec(const double* L, long long ld, int n, const double* linv, double* B, long long ldb, int q,
                           int leaf, DevStatus* st, cudaStream_t s);
cudaError_t trsm_lower_t_rec(const double* L, long long ld, int n, const double* linv, double* B, long long ldb,
                             int q, int leaf, DevStatus* st, cudaStream_t s);

// out = log|det L|² contribution: 2 Σ ln L_ii (lower LLT) or Σ ln D_i (ldlt=true).
cudaError_t logdet_diag(const double* L, long long ld, int n, bool ldlt, double* out, DevStatus* st,
                        cudaStream_t s);

// z = X y for lower-triangular X (n×n, ld).
cudaError_t trmv_lower(const double* X, long long ld, int n, const double* y, double* z, DevStatus* st,
                       cudaStream_t s);
// out_j = Σ_{i ≥ (lower ? j : 0)} M(i,j) v_i  for j < ncols (one warp per column).
cudaError_t gemv_t(const double* M, long long ld, int nrows, int ncols, bool lower, const double* v, double* out,
                   DevStatus* st, cudaStream_t s);
// out_j = Σ_i M(i,j)² (/ w_i when w != nullptr) for j < ncols.
cudaError_t col_sumsq(const double* M, long long ld, int nrows, int ncols, const double* w, double* out,
                      DevStatus* st, cudaStream_t s);

// out = Σ_i a_i b_i (single block, deterministic).
cudaError_t dot_dev(const double* a, const double* b, int n, double* out, DevStatus* st, cudaStream_t s);

// The same two products with the FP64 GEMMs emulated on the int8 tensor
// cores (emu_gemm.cuh) wherever the blocks are at least emu_min wide; the
// narrower levels stay on DMMA.  X's strict upper triangle must be zero.
cudaError_t trtri_blocked_emu(const double* L, long long ld, int n, const double* linv, double* X, long long ldx,
                              double* scratch, const EmuWork& w, int emu_min, DevStatus* st, cudaStream_t s);
cudaError_t lauum_lower_emu(const double* X, long long ldx, int n, double* C, long long ldc, const EmuWork& w,
                            DevStatus* st, cudaStream_t s);

// Lower LLT of A (n×n) and X = L⁻¹ together by recursive halving: A11 → (L11,
// X11) recursively, L21 = A21 X11ᵀ, A22 −= L21 L21ᵀ, A22 → (L22, X22),
// X21 = −X22 (L21 X11), the coupling products as emulated FP64 GEMMs; blocks
// of at most `leaf` rows use potrf_blocked and trtri_blocked_emu.  linv gets
// the diagonal-block inverses (block index = row / NB); scratch holds
// ceil(n/2)² doubles.  X's strict upper triangle must be zero.
cudaError_t potrf_trtri_rec(double* A, long long ld, int n, double* X, long long ldx, double* linv,
                            double* scratch, const EmuWork& w, int leaf, int emu_min, DevStatus* st,
                            cudaStream_t s, FactorCtx* ctx);

// Sets X (n×n, ld) to the identity (full columns, zero off the diagonal).
cudaError_t set_identity(double* X, long long ld, int n, cudaStream_t s);

}  // namespace gprx
