// dense_f64.cu — blocked FP64 Cholesky, triangular inverse, Xᵀ X and
// triangular solves on the DMMA GEMM (gemm_f64.cuh).
//
// Replaces faer's llt::factor::cholesky_in_place (gprx src/linalg/chol.rs:141-167),
// llt::solve (chol.rs:334-339, src/workspace.rs:395-425) and
// solve_lower_triangular_in_place (src/gpr/shared.rs:831-842).
//
// Layout: column-major, element (i, j) at i + j·ld, lower triangle.  A panel
// width NB = 128 matches the GEMM tile so the panel solve and the diagonal
// block applications can run in place (one CTA covers a whole panel row /
// column strip and reads it fully before writing).

#include <algorithm>

#include "dense_f64.cuh"

namespace gprx {

cudaError_t dgemm(bool ta, bool tb, const GemmParams& p, cudaStream_t s, int batch) {
  if (!ta && !tb) return launch_dgemm<128, 128, 16, 64, 32, 3, false, false>(p, batch, s);
  if (!ta && tb) return launch_dgemm<128, 128, 16, 64, 32, 3, false, true>(p, batch, s);
  if (ta && !tb) return launch_dgemm<128, 128, 16, 64, 32, 3, true, false>(p, batch, s);
  return launch_dgemm<128, 128, 16, 64, 32, 3, true, true>(p, batch, s);
}

GemmParams gemm_params(int M, int N, int K, const double* A, long long lda, const double* B, long long ldb,
                       double* C, long long ldc, double alpha, double beta, const DevStatus* st) {
  GemmParams p{};
  p.M = M;
  p.N = N;
  p.K = K;
  p.A = A;
  p.lda = lda;
  p.B = B;
  p.ldb = ldb;
  p.C = C;
  p.ldc = ldc;
  p.alpha = alpha;
  p.beta = beta;
  p.mode = 0;
  p.row0 = p.col0 = p.krow0 = 0;
  p.splits = 1;
  p.split_stride = 0;
  p.status = st;
  p.strideA = p.strideB = p.strideC = 0;
  return p;
}

// ---------------------------------------------------------------------------
// diagonal block: factor and invert in shared memory
// ---------------------------------------------------------------------------
constexpr int DIAG_THREADS = 256;

__device__ void blk_load_lower(double* s, int ls, const double* A, long long lda, long long k0, int nb) {
  for (int e = threadIdx.x; e < nb * nb; e += blockDim.x) {
    int i = e % nb, j = e / nb;
    s[i + j * ls] = (i >= j) ? A[(k0 + i) + (k0 + j) * lda] : 0.0;
  }
  __syncthreads();
}

// Unblocked right-looking LLT of the nb×nb lower block in shared memory.
// Returns the first failing column, or -1.
__device__ int blk_potf2(double* s, int ls, int nb) {
  __shared__ int fail;
  if (threadIdx.x == 0) fail = -1;
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int j = 0; j < nb; ++j) {
    if (threadIdx.x == 0) {
      double dj = s[j + j * ls];
      if (!(dj > 0.0)) fail = j;
      else s[j + j * ls] = sqrt(dj);
    }
    __syncthreads();
    if (fail >= 0) return fail;
    double ljj = s[j + j * ls];
    for (int i = j + 1 + threadIdx.x; i < nb; i += blockDim.x) s[i + j * ls] = s[i + j * ls] / ljj;
    __syncthreads();
    for (int c = j + 1 + warp; c < nb; c += nw) {
      double lc = s[c + j * ls];
      for (int i = c + lane; i < nb; i += 32) s[i + c * ls] = fma(-s[i + j * ls], lc, s[i + c * ls]);
    }
    __syncthreads();
  }
  return -1;
}

// In-place inverse of the lower nb×nb triangle (LAPACK trti2 order: columns
// from the right, each a product with the already inverted trailing block).
__device__ void blk_trti2(double* s, int ls, int nb, bool unit, double* tmp) {
  for (int j = nb - 1; j >= 0; --j) {
    double inv = unit ? 1.0 : 1.0 / s[j + j * ls];
    for (int i = j + 1 + threadIdx.x; i < nb; i += blockDim.x) tmp[i] = s[i + j * ls];
    __syncthreads();
    for (int i = j + 1 + threadIdx.x; i < nb; i += blockDim.x) {
      double v = 0.0;
      for (int c = j + 1; c <= i; ++c) v = fma(s[i + c * ls], tmp[c], v);
      s[i + j * ls] = -v * inv;
    }
    __syncthreads();
    if (threadIdx.x == 0) s[j + j * ls] = inv;
    __syncthreads();
  }
}

__device__ void blk_store_full(double* dst, int ldd, const double* s, int ls, int nb) {
  for (int e = threadIdx.x; e < nb * nb; e += blockDim.x) {
    int i = e % nb, j = e / nb;
    dst[i + j * ldd] = (i >= j) ? s[i + j * ls] : 0.0;
  }
}

// ---------------------------------------------------------------------------
// Fast diagonal block (nb ≤ 128): LLT by 32-column sub-panels and the block's
// inverse, all in shared memory.
//   per sub-panel p:  one warp factors the 32×32 diagonal sub-block in
//                     registers (lane = row, pivots broadcast by shuffles) and
//                     inverts it (lane = column);
//                     all warps: P = A_below · L_pp⁻ᵀ, then A22 −= P Pᵀ.
//   inverse:          column blocks right to left from X L = I:
//                     X_ij = −(Σ_{k=j+1..i} X_ik L_kj) X_jj, in place.
// ---------------------------------------------------------------------------
constexpr int FD_THREADS = 512;
constexpr int SB = 32;         // sub-panel width
constexpr int SBL = SB + 1;    // ld of a 32×32 scratch block

__device__ __forceinline__ void warp_factor_inv(double* s, int ls, int c0, int w, double* xd, int* fail) {
  // lane r holds row r of the diagonal sub-block (columns ≤ r)
  const int lane = threadIdx.x & 31;
  double d[SB];
#pragma unroll
  for (int c = 0; c < SB; ++c) d[c] = (lane < w && c <= lane) ? s[(c0 + lane) + (c0 + c) * ls] : 0.0;
  int bad = -1;
#pragma unroll
  for (int j = 0; j < SB; ++j) {
    if (j < w && bad < 0) {
      double piv = __shfl_sync(0xffffffffu, d[j], j);
      if (!(piv > 0.0)) {
        bad = j;
      } else {
        double ljj = sqrt(piv);
        if (lane == j) d[j] = ljj;
        else if (lane > j) d[j] = d[j] / ljj;
#pragma unroll
        for (int c = j + 1; c < SB; ++c) {
          double lcj = __shfl_sync(0xffffffffu, d[j], c);
          if (lane >= c) d[c] = fma(-d[j], lcj, d[c]);
        }
      }
    }
  }
  if (bad >= 0) {
    if (lane == 0) *fail = c0 + bad;
    return;
  }
  if (lane < w) {
#pragma unroll
    for (int c = 0; c < SB; ++c)
      if (c <= lane) s[(c0 + lane) + (c0 + c) * ls] = d[c];
  }
  __syncwarp();
  // inverse of the sub-block: lane c computes column c
  if (lane < w) {
    const int c = lane;
    for (int r = 0; r < c; ++r) xd[r + c * SBL] = 0.0;
    xd[c + c * SBL] = 1.0 / s[(c0 + c) + (c0 + c) * ls];
    for (int r = c + 1; r < w; ++r) {
      double acc = 0.0;
      for (int t = c; t < r; ++t) acc = fma(s[(c0 + r) + (c0 + t) * ls], xd[t + c * SBL], acc);
      xd[r + c * SBL] = -acc / s[(c0 + r) + (c0 + r) * ls];
    }
  }
}

__global__ void __launch_bounds__(FD_THREADS) potrf_diag_kernel(double* A, long long lda, long long k0, int nb,
                                                                 double* linv, DevStatus* st) {
  extern __shared__ double smem[];
  __shared__ int fail;
  if (dev_failed(st)) return;
  const int ls = nb + 1;
  double* s = smem;                       // nb × ls
  double* xd = s + nb * ls;               // 4 × (32 × 33) diagonal sub-block inverses
  double* tmp = xd + 4 * SB * SBL;        // 3 × (32 × 33)
  const int tid = threadIdx.x, nt = blockDim.x;
  if (tid == 0) fail = -1;
  for (int e = tid; e < nb * nb; e += nt) {
    int i = e % nb, j = e / nb;
    s[i + j * ls] = (i >= j) ? A[(k0 + i) + (k0 + j) * lda] : 0.0;
  }
  __syncthreads();
  const int np = (nb + SB - 1) / SB;
  for (int p = 0; p < np; ++p) {
    const int c0 = p * SB, w = min(SB, nb - c0);
    if (tid < 32) warp_factor_inv(s, ls, c0, w, xd + p * SB * SBL, &fail);
    __syncthreads();
    if (fail >= 0) {
      if (tid == 0) dev_fail(st, GPRX_CHOLESKY_FAILED, k0 + fail);
      return;
    }
    const int r0 = c0 + w, cnt = nb - r0;
    if (cnt <= 0) break;
    // P = A_below · X_ppᵀ  (P(r, c) = Σ_{t ≤ c} A(r, t) X(c, t))
    const double* X = xd + p * SB * SBL;
    const int items = cnt * (SB / 4);  // ≤ 96 · 8 = 768 ≤ 2 · FD_THREADS
    // each thread: up to two items, results held until all reads finish
    double res0[4] = {0, 0, 0, 0}, res1[4] = {0, 0, 0, 0};
    auto item = [&](int it, double (&acc)[4]) {
      int r = r0 + it % cnt, cg = (it / cnt) * 4;
      for (int t = 0; t < w; ++t) {
        double a = s[r + (c0 + t) * ls];
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[q] = fma(a, X[(cg + q) + t * SBL], acc[q]);
      }
    };
    auto put = [&](int it, const double (&acc)[4]) {
      int r = r0 + it % cnt, cg = (it / cnt) * 4;
#pragma unroll
      for (int q = 0; q < 4; ++q)
        if (cg + q < w) s[r + (c0 + cg + q) * ls] = acc[q];
    };
    if (tid < items) item(tid, res0);
    if (tid + nt < items) item(tid + nt, res1);
    __syncthreads();
    if (tid < items) put(tid, res0);
    if (tid + nt < items) put(tid + nt, res1);
    __syncthreads();
    // A22 −= P Pᵀ over 4×4 blocks of the lower triangle
    const int nb4 = (cnt + 3) / 4;
    const int nblk = nb4 * (nb4 + 1) / 2;
    for (int b = tid; b < nblk; b += nt) {
      int bi = (int)((sqrt(8.0 * b + 1.0) - 1.0) * 0.5);
      while ((bi + 1) * (bi + 2) / 2 <= b) ++bi;
      while (bi * (bi + 1) / 2 > b) --bi;
      int bj = b - bi * (bi + 1) / 2;
      int i0 = r0 + bi * 4, j0 = r0 + bj * 4;
      double a4[4][4];
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) a4[u][v] = 0.0;
      for (int t = 0; t < w; ++t) {
        double pi[4], pj[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          pi[u] = (i0 + u < nb) ? s[(i0 + u) + (c0 + t) * ls] : 0.0;
          pj[u] = (j0 + u < nb) ? s[(j0 + u) + (c0 + t) * ls] : 0.0;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
          for (int v = 0; v < 4; ++v) a4[u][v] = fma(pi[u], pj[v], a4[u][v]);
      }
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) {
          int i = i0 + u, j = j0 + v;
          if (i < nb && j < nb && i >= j) s[i + j * ls] -= a4[u][v];
        }
    }
    __syncthreads();
  }
  // L back to global
  for (int e = tid; e < nb * nb; e += nt) {
    int i = e % nb, j = e / nb;
    if (i >= j) A[(k0 + i) + (k0 + j) * lda] = s[i + j * ls];
  }
  __syncthreads();
  // block inverse in place, column blocks right to left
  for (int jb = np - 1; jb >= 0; --jb) {
    const int j0 = jb * SB, wj = min(SB, nb - j0);
    const double* Xjj = xd + jb * SB * SBL;
    // T_ib = Σ_{k=jb+1..ib} X_ik L_kj  for ib > jb (X_ik already in s for k > jb)
    const int nout = np - 1 - jb;
    for (int e = tid; e < nout * SB * SB; e += nt) {
      int ib = jb + 1 + e / (SB * SB);
      int rr = (e % (SB * SB)) % SB, cc = (e % (SB * SB)) / SB;
      int i = ib * SB + rr, j = j0 + cc;
      double acc = 0.0;
      if (i < nb && cc < wj) {
        // X (columns > jb, including the inverted diagonal blocks, zero above
        // their diagonals) is already in s; column block jb still holds L.
        const int kend = min(nb, (ib + 1) * SB);
        for (int k = (jb + 1) * SB; k < kend; ++k) acc = fma(s[i + k * ls], s[k + j * ls], acc);
      }
      tmp[(ib - jb - 1) * SB * SBL + rr + cc * SBL] = acc;
    }
    __syncthreads();
    // X_ib,jb = −T X_jj ; then X_jj onto the diagonal block
    for (int e = tid; e < nout * SB * SB; e += nt) {
      int ib = jb + 1 + e / (SB * SB);
      int rr = (e % (SB * SB)) % SB, cc = (e % (SB * SB)) / SB;
      int i = ib * SB + rr, j = j0 + cc;
      if (i < nb && cc < wj) {
        const double* T = tmp + (ib - jb - 1) * SB * SBL;
        double acc = 0.0;
        for (int k = cc; k < wj; ++k) acc = fma(T[rr + k * SBL], Xjj[k + cc * SBL], acc);
        s[i + j * ls] = -acc;
      }
    }
    for (int e = tid; e < SB * SB; e += nt) {
      int rr = e % SB, cc = e / SB;
      if (rr < wj && cc < wj) s[(j0 + rr) + (j0 + cc) * ls] = (rr >= cc) ? Xjj[rr + cc * SBL] : 0.0;
    }
    __syncthreads();
  }
  blk_store_full(linv, NB, s, ls, nb);
}

__global__ void __launch_bounds__(DIAG_THREADS) tri_inv_blocks_kernel(const double* L, long long ld, int n,
                                                                       bool unit, double* linv, DevStatus* st) {
  extern __shared__ double s[];
  if (dev_failed(st)) return;
  long long k0 = (long long)blockIdx.x * NB;
  int nb = (int)min((long long)NB, n - k0);
  const int ls = nb + 1;
  double* tmp = s + nb * ls;
  blk_load_lower(s, ls, L, ld, k0, nb);
  blk_trti2(s, ls, nb, unit, tmp);
  blk_store_full(linv + (long long)blockIdx.x * NB * NB, NB, s, ls, nb);
}

static size_t diag_smem(int nb) { return (size_t)(nb * (nb + 1) + nb) * sizeof(double); }
static size_t fast_diag_smem(int nb) { return (size_t)(nb * (nb + 1) + 7 * SB * SBL) * sizeof(double); }

static cudaError_t diag_attrs() {
  static bool done = false;
  if (done) return cudaSuccess;
  cudaError_t e = cudaFuncSetAttribute(potrf_diag_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)fast_diag_smem(NB));
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(tri_inv_blocks_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)diag_smem(NB));
  if (e != cudaSuccess) return e;
  done = true;
  return cudaSuccess;
}

#define CK(x)                                \
  do {                                       \
    cudaError_t e_ = (x);                    \
    if (e_ != cudaSuccess) return e_;        \
  } while (0)

cudaError_t potrf_blocked(double* A, long long ld, int n, double* linv, DevStatus* st, cudaStream_t s) {
  CK(diag_attrs());
  for (int k0 = 0; k0 < n; k0 += NB) {
    int nbk = min(NB, n - k0);
    double* lk = linv + (long long)(k0 / NB) * NB * NB;
    GPRX_LAUNCH(potrf_diag_kernel, 1, FD_THREADS, fast_diag_smem(nbk), s, A, ld, (long long)k0, nbk, lk, st);
    int rest = n - k0 - nbk;
    if (rest <= 0) break;
    double* P = A + (k0 + nbk) + (long long)k0 * ld;
    // panel: P := P · L_kk⁻ᵀ (in place; the 128-wide tile covers all nbk columns)
    GemmParams pp = gemm_params(rest, nbk, nbk, P, ld, lk, NB, P, ld, 1.0, 0.0, st);
    CK(dgemm(false, true, pp, s));
    // trailing: A22 −= P Pᵀ (lower tiles)
    double* A22 = A + (k0 + nbk) + (long long)(k0 + nbk) * ld;
    GemmParams ps = gemm_params(rest, rest, nbk, P, ld, P, ld, A22, ld, -1.0, 1.0, st);
    ps.mode = GEMM_LOWER_TILES;
    CK(dgemm(false, true, ps, s));
  }
  return cudaGetLastError();
}

cudaError_t tri_inv_blocks(const double* L, long long ld, int n, bool unit, double* linv, DevStatus* st,
                           cudaStream_t s) {
  CK(diag_attrs());
  int nblk = ceil_div(n, NB);
  if (nblk == 0) return cudaSuccess;
  GPRX_LAUNCH(tri_inv_blocks_kernel, nblk, DIAG_THREADS, diag_smem(min(n, NB)), s, L, ld, n, unit, linv, st);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// identity / triangular inverse / Xᵀ X
// ---------------------------------------------------------------------------
__global__ void set_identity_kernel(double* X, long long ld, int n) {
  long long total = (long long)n * n;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    int i = (int)(e % n), j = (int)(e / n);
    X[i + j * ld] = (i == j) ? 1.0 : 0.0;
  }
}

cudaError_t set_identity(double* X, long long ld, int n, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  long long total = (long long)n * n;
  int blocks = (int)std::min<long long>((total + 255) / 256, 148LL * 16);
  GPRX_LAUNCH(set_identity_kernel, blocks, 256, 0, s, X, ld, n);
  return cudaGetLastError();
}

// Solves L X = I right-looking over block rows: X_k = L_kk⁻¹ B_k, then
// B_{>k} −= L_{>k,k} X_k (columns ≤ the block only; the rest stays zero).
cudaError_t trtri_blocked(const double* L, long long ld, int n, const double* linv, double* X, long long ldx,
                          DevStatus* st, cudaStream_t s) {
  CK(set_identity(X, ldx, n, s));
  for (int k0 = 0; k0 < n; k0 += NB) {
    int nbk = min(NB, n - k0);
    int cols = k0 + nbk;
    const double* lk = linv + (long long)(k0 / NB) * NB * NB;
    double* Xk = X + k0;
    GemmParams p1 = gemm_params(nbk, cols, nbk, lk, NB, Xk, ldx, Xk, ldx, 1.0, 0.0, st);
    CK(dgemm(false, false, p1, s));
    int rest = n - cols;
    if (rest <= 0) break;
    GemmParams p2 = gemm_params(rest, cols, nbk, L + cols + (long long)k0 * ld, ld, Xk, ldx, X + cols, ldx, -1.0,
                                1.0, st);
    CK(dgemm(false, false, p2, s));
  }
  return cudaGetLastError();
}

cudaError_t lauum_lower(const double* X, long long ldx, int n, double* C, long long ldc, DevStatus* st,
                        cudaStream_t s) {
  GemmParams p = gemm_params(n, n, n, X, ldx, X, ldx, C, ldc, 1.0, 0.0, st);
  p.mode = GEMM_LOWER_TILES | GEMM_K_FROM_ROW;
  return dgemm(true, false, p, s);
}

cudaError_t trsm_lower(const double* L, long long ld, int n, const double* linv, double* B, long long ldb, int q,
                       DevStatus* st, cudaStream_t s) {
  for (int k0 = 0; k0 < n; k0 += NB) {
    int nbk = min(NB, n - k0);
    const double* lk = linv + (long long)(k0 / NB) * NB * NB;
    double* Bk = B + k0;
    GemmParams p1 = gemm_params(nbk, q, nbk, lk, NB, Bk, ldb, Bk, ldb, 1.0, 0.0, st);
    CK(dgemm(false, false, p1, s));
    int rest = n - k0 - nbk;
    if (rest <= 0) break;
    GemmParams p2 = gemm_params(rest, q, nbk, L + (k0 + nbk) + (long long)k0 * ld, ld, Bk, ldb, B + k0 + nbk, ldb,
                                -1.0, 1.0, st);
    CK(dgemm(false, false, p2, s));
  }
  return cudaGetLastError();
}

cudaError_t trsm_lower_t(const double* L, long long ld, int n, const double* linv, double* B, long long ldb, int q,
                         DevStatus* st, cudaStream_t s) {
  int nblk = ceil_div(n, NB);
  for (int kb = nblk - 1; kb >= 0; --kb) {
    int k0 = kb * NB;
    int nbk = min(NB, n - k0);
    const double* lk = linv + (long long)kb * NB * NB;
    double* Bk = B + k0;
    // B_k := L_kk⁻ᵀ B_k
    GemmParams p1 = gemm_params(nbk, q, nbk, lk, NB, Bk, ldb, Bk, ldb, 1.0, 0.0, st);
    CK(dgemm(true, false, p1, s));
    if (k0 == 0) break;
    // B_{<k} −= L_{k,<k}ᵀ B_k
    GemmParams p2 = gemm_params(k0, q, nbk, L + k0, ld, Bk, ldb, B, ldb, -1.0, 1.0, st);
    CK(dgemm(true, false, p2, s));
  }
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// reductions and matrix-vector products (HBM-bound)
// ---------------------------------------------------------------------------
__global__ void logdet_kernel(const double* L, long long ld, int n, bool ldlt, double* out, const DevStatus* st) {
  __shared__ double red[32];
  if (dev_failed(st)) return;
  double acc = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) acc += log(L[i + (long long)i * ld]);
  double s = block_sum(acc, red);
  if (threadIdx.x == 0) *out = ldlt ? s : 2.0 * s;
}

cudaError_t logdet_diag(const double* L, long long ld, int n, bool ldlt, double* out, DevStatus* st,
                        cudaStream_t s) {
  GPRX_LAUNCH(logdet_kernel, 1, 1024, 0, s, L, ld, n, ldlt, out, st);
  return cudaGetLastError();
}

// z_i = Σ_{j ≤ i} X_ij y_j: a block owns 32 rows and walks the columns.
constexpr int TRMV_ROWS = 32;
__global__ void trmv_lower_kernel(const double* X, long long ld, int n, const double* y, double* z,
                                  const DevStatus* st) {
  __shared__ double part[8][TRMV_ROWS];
  if (dev_failed(st)) return;
  int r = threadIdx.x % TRMV_ROWS, cg = threadIdx.x / TRMV_ROWS;  // 8 column groups
  int i = blockIdx.x * TRMV_ROWS + r;
  int jmax = min(n, (blockIdx.x + 1) * TRMV_ROWS);
  double acc = 0.0;
  if (i < n) {
    for (int j = cg; j < jmax; j += 8) {
      if (j <= i) acc = fma(X[i + (long long)j * ld], y[j], acc);
    }
  }
  part[cg][r] = acc;
  __syncthreads();
  if (cg == 0 && i < n) {
    double s = 0.0;
#pragma unroll
    for (int c = 0; c < 8; ++c) s += part[c][r];
    z[i] = s;
  }
}

cudaError_t trmv_lower(const double* X, long long ld, int n, const double* y, double* z, DevStatus* st,
                       cudaStream_t s) {
  GPRX_LAUNCH(trmv_lower_kernel, ceil_div(n, TRMV_ROWS), TRMV_ROWS * 8, 0, s, X, ld, n, y, z, st);
  return cudaGetLastError();
}

__global__ void gemv_t_kernel(const double* M, long long ld, int nrows, int ncols, bool lower, const double* v,
                              double* out, const DevStatus* st) {
  if (dev_failed(st)) return;
  int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (warp >= ncols) return;
  const double* col = M + (long long)warp * ld;
  int i0 = lower ? warp : 0;
  double acc = 0.0;
  for (int i = i0 + lane; i < nrows; i += 32) acc = fma(col[i], v[i], acc);
  acc = warp_sum(acc);
  if (lane == 0) out[warp] = acc;
}

cudaError_t gemv_t(const double* M, long long ld, int nrows, int ncols, bool lower, const double* v, double* out,
                   DevStatus* st, cudaStream_t s) {
  if (ncols <= 0) return cudaSuccess;
  GPRX_LAUNCH(gemv_t_kernel, ceil_div((long long)ncols * 32, 256), 256, 0, s, M, ld, nrows, ncols, lower, v, out, st);
  return cudaGetLastError();
}

__global__ void col_sumsq_kernel(const double* M, long long ld, int nrows, int ncols, const double* w, double* out,
                                 const DevStatus* st) {
  if (dev_failed(st)) return;
  int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (warp >= ncols) return;
  const double* col = M + (long long)warp * ld;
  double acc = 0.0;
  for (int i = lane; i < nrows; i += 32) {
    double v = col[i];
    acc = w ? fma(v, v / w[i], acc) : fma(v, v, acc);
  }
  acc = warp_sum(acc);
  if (lane == 0) out[warp] = acc;
}

cudaError_t col_sumsq(const double* M, long long ld, int nrows, int ncols, const double* w, double* out,
                      DevStatus* st, cudaStream_t s) {
  if (ncols <= 0) return cudaSuccess;
  GPRX_LAUNCH(col_sumsq_kernel, ceil_div((long long)ncols * 32, 256), 256, 0, s, M, ld, nrows, ncols, w, out, st);
  return cudaGetLastError();
}

__global__ void dot_kernel(const double* a, const double* b, int n, double* out, const DevStatus* st) {
  __shared__ double red[32];
  if (dev_failed(st)) return;
  double acc = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) acc = fma(a[i], b[i], acc);
  double s = block_sum(acc, red);
  if (threadIdx.x == 0) *out = s;
}

cudaError_t dot_dev(const double* a, const double* b, int n, double* out, DevStatus* st, cudaStream_t s) {
  GPRX_LAUNCH(dot_kernel, 1, 1024, 0, s, a, b, n, out, st);
  return cudaGetLastError();
}

}  // namespace gprx
