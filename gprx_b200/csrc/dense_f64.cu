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
  p.max_ctas = 0;
  p.splits_tiles = 0;
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
// Diagonal block (nb ≤ 128): LLT and the block's inverse in shared memory.
// The block is padded to a multiple of 32 with an identity tail.
//   per 32-column sub-panel p:
//     warp 0 factors the 32×32 diagonal sub-block in registers (lane = row,
//     pivots broadcast by shuffles) and inverts it (lane = column);
//     all warps (DMMA m16n8k4): P = A_below · L_pp⁻ᵀ, then A22 −= P Pᵀ.
//   inverse, column blocks right to left from X L = I (DMMA):
//     X_ij = −(Σ_{k=j+1..i} X_ik L_kj) X_jj, in place.
// ---------------------------------------------------------------------------
constexpr int FD_THREADS = 256;
constexpr int SB = 32;          // sub-panel width
constexpr int FLS = NB + 4;     // ld of the block (≡ 4 mod 16: conflict-free fragments)
constexpr int XLD = SB + 4;     // ld of a 32×32 scratch block

// C(16×8) += A(16×K) · B(K×8) with A(i,k) = a[i·ai + k·ak], B(k,j) = b[k·bk + j·bj].
__device__ __forceinline__ void mma_tile_smem(double (&c)[4], const double* a, int ai, int ak, const double* b, int bk,
                                              int bj, int K) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll 4
  for (int kk = 0; kk < K; kk += 4) {
    double a0 = a[g * ai + (kk + t) * ak];
    double a1 = a[(g + 8) * ai + (kk + t) * ak];
    double b0 = b[(kk + t) * bk + g * bj];
    dmma_16x8x4(c, a0, a1, b0);
  }
}

// 16×16 leaf, one warp: lanes r and r+16 both hold row r of the block at
// (off, off) of s in registers; pivots are broadcast by shuffles.  Writes L
// back to s and L⁻¹ (column-major, ld XLD) to xo.  Returns the failing column
// or −1.  Kept out of line so one compact copy serves every call (the fully
// unrolled 32-wide form overflowed the instruction cache).
__device__ __noinline__ int leaf16_factor_inv(double* s, int off, double* xo) {
  const int lane = threadIdx.x & 31, r = lane & 15;
  double d[16];
#pragma unroll
  for (int c = 0; c < 16; ++c) d[c] = (c <= r) ? s[(off + r) + (off + c) * FLS] : 0.0;
  int bad = -1;
  double my_inv = 1.0;
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    double piv = __shfl_sync(0xffffffffu, d[j], j);
    if (!(piv > 0.0) && bad < 0) bad = j;
    double rs = rsqrt(fmax(piv, 1e-300));
    if (r == j) {
      d[j] = piv * rs;
      my_inv = rs;
    } else if (r > j) {
      d[j] = d[j] * rs;
    }
#pragma unroll
    for (int c = 0; c < 16; ++c) {
      if (c > j) {
        double lcj = __shfl_sync(0xffffffffu, d[j], c);
        if (r >= c) d[c] = fma(-d[j], lcj, d[c]);
      }
    }
  }
  if (bad >= 0) return bad;
  if (lane < 16) {
#pragma unroll
    for (int c = 0; c < 16; ++c)
      if (c <= r) s[(off + r) + (off + c) * FLS] = d[c];
  }
  double x[16];
#pragma unroll
  for (int q = 0; q < 16; ++q) {
    double acc = (q == r) ? 1.0 : 0.0;
#pragma unroll
    for (int t = 0; t < 16; ++t)
      if (t < q) acc = fma(-__shfl_sync(0xffffffffu, d[t], q), x[t], acc);
    x[q] = acc * __shfl_sync(0xffffffffu, my_inv, q);
  }
  if (lane < 16) {
#pragma unroll
    for (int q = 0; q < 16; ++q) xo[q + r * XLD] = x[q];
  }
  __syncwarp();
  return -1;
}

// Factor + invert the 32×32 sub-block at (c0, c0) of s with one warp, as two
// 16×16 leaves: L21 = A21 X11ᵀ, A22 −= L21 L21ᵀ, then X21 = −X22 (L21 X11),
// the products on DMMA.  L goes back to s, L⁻¹ to xd (ld XLD, zero above the
// diagonal).  Returns the failing column or −1 (uniform over the warp).
__device__ __forceinline__ int warp_factor_inv32(double* s, int c0, double* xd) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t4 = lane & 3;
  int f = leaf16_factor_inv(s, c0, xd);
  if (f >= 0) return f;
  // L21 = A21 · X11ᵀ  (B(k, j) = X11(j, k))
  double c[2][4] = {{0, 0, 0, 0}, {0, 0, 0, 0}};
#pragma unroll
  for (int tn = 0; tn < 2; ++tn) mma_tile_smem(c[tn], s + (c0 + 16) + c0 * FLS, 1, FLS, xd + 8 * tn, XLD, 1, 16);
  __syncwarp();
#pragma unroll
  for (int tn = 0; tn < 2; ++tn) {
    int row = c0 + 16 + g, col = c0 + 8 * tn + 2 * t4;
    s[row + col * FLS] = c[tn][0];
    s[row + (col + 1) * FLS] = c[tn][1];
    s[(row + 8) + col * FLS] = c[tn][2];
    s[(row + 8) + (col + 1) * FLS] = c[tn][3];
  }
  __syncwarp();
  // A22 −= L21 L21ᵀ (lower part)
#pragma unroll
  for (int tn = 0; tn < 2; ++tn) {
    double u[4] = {0, 0, 0, 0};
    mma_tile_smem(u, s + (c0 + 16) + c0 * FLS, 1, FLS, s + (c0 + 16 + 8 * tn) + c0 * FLS, FLS, 1, 16);
    int i = g, j = 8 * tn + 2 * t4;  // within the 16×16 block
    double* b = s + (c0 + 16) + (c0 + 16) * FLS;
    if (i >= j) b[i + j * FLS] -= u[0];
    if (i >= j + 1) b[i + (j + 1) * FLS] -= u[1];
    if (i + 8 >= j) b[(i + 8) + j * FLS] -= u[2];
    if (i + 8 >= j + 1) b[(i + 8) + (j + 1) * FLS] -= u[3];
  }
  __syncwarp();
  f = leaf16_factor_inv(s, c0 + 16, xd + 16 + 16 * XLD);
  if (f >= 0) return 16 + f;
  // T = L21 · X11 into the (zero) upper-right quarter of xd, then
  // X21 = −X22 · T, and the quarter back to zero
  double* T = xd + 16 * XLD;  // rows 0..15, columns 16..31
#pragma unroll
  for (int tn = 0; tn < 2; ++tn) {
    double u[4] = {0, 0, 0, 0};
    mma_tile_smem(u, s + (c0 + 16) + c0 * FLS, 1, FLS, xd + 8 * tn * XLD, 1, XLD, 16);
    int i = g, j = 8 * tn + 2 * t4;
    T[i + j * XLD] = u[0];
    T[i + (j + 1) * XLD] = u[1];
    T[(i + 8) + j * XLD] = u[2];
    T[(i + 8) + (j + 1) * XLD] = u[3];
  }
  __syncwarp();
#pragma unroll
  for (int tn = 0; tn < 2; ++tn) {
    double u[4] = {0, 0, 0, 0};
    mma_tile_smem(u, xd + 16 + 16 * XLD, 1, XLD, T + 8 * tn * XLD, 1, XLD, 16);
    int i = g, j = 8 * tn + 2 * t4;
    double* X21 = xd + 16;
    X21[i + j * XLD] = -u[0];
    X21[i + (j + 1) * XLD] = -u[1];
    X21[(i + 8) + j * XLD] = -u[2];
    X21[(i + 8) + (j + 1) * XLD] = -u[3];
  }
  __syncwarp();
  for (int e = lane; e < 256; e += 32) T[(e % 16) + (e / 16) * XLD] = 0.0;
  __syncwarp();
  return -1;
}

// A22 −= P Pᵀ on the 16×8 tiles of rows [rlo, npad) × columns [clo, chi) that
// are not strictly above the diagonal; tiles dealt to warps w0.. in steps of nws.
__device__ __forceinline__ void diag_syrk_tiles(double* s, int c0, int rlo, int clo, int chi, int npad, int w0,
                                                int nws) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t4 = lane & 3;
  const int tm_n = (npad - rlo) / 16, tn_n = (chi - clo) / 8;
  for (int tile = warp - w0; tile < tm_n * tn_n; tile += nws) {
    int tm = tile % tm_n, tn = tile / tm_n;
    int rbeg = rlo + 16 * tm, cbeg = clo + 8 * tn;
    if (rbeg + 15 < cbeg) continue;
    double c[4] = {0, 0, 0, 0};
    mma_tile_smem(c, s + rbeg + c0 * FLS, 1, FLS, s + cbeg + c0 * FLS, FLS, 1, SB);
    int row = rbeg + g, col = cbeg + 2 * t4;
    if (row >= col) s[row + col * FLS] -= c[0];
    if (row >= col + 1) s[row + (col + 1) * FLS] -= c[1];
    if (row + 8 >= col) s[(row + 8) + col * FLS] -= c[2];
    if (row + 8 >= col + 1) s[(row + 8) + (col + 1) * FLS] -= c[3];
  }
}

__global__ void __launch_bounds__(FD_THREADS) potrf_diag_kernel(double* A, long long lda, long long k0, int nb,
                                                                 double* linv, DevStatus* st) {
  extern __shared__ __align__(16) double smem[];
  __shared__ int fail;
  if (dev_failed(st)) return;
  double* s = smem;                       // NB × FLS
  double* xd = s + NB * FLS;              // 4 × (32 × XLD) sub-block inverses
  double* tmp = xd + 4 * SB * XLD;        // 3 × (32 × XLD)
  const int tid = threadIdx.x, nt = blockDim.x, warp = tid >> 5, nw = nt >> 5;
  const int lane = tid & 31, g = lane >> 2, t4 = lane & 3;
  const int npad = (nb + SB - 1) / SB * SB;
  if (tid == 0) fail = -1;
  // block load: every lower entry in flight at once (16-byte cp.async pairs
  // from the even row at or above the diagonal), then zero / pad
  const bool vec = ((lda & 1) == 0) && ((((unsigned long long)(A + k0 + k0 * lda)) & 15) == 0);
  for (int j = warp; j < nb; j += nw) {
    if (vec) {
      for (int i = (j & ~1) + 2 * lane; i < nb; i += 64) {
        if (i + 1 < nb) {
          unsigned sa = (unsigned)__cvta_generic_to_shared(s + i + j * FLS);
          asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(A + (k0 + i) + (k0 + j) * lda));
        } else {
          cp_async8(s + i + j * FLS, A + (k0 + i) + (k0 + j) * lda, true);
        }
      }
    } else {
      for (int i = j + lane; i < nb; i += 32) cp_async8(s + i + j * FLS, A + (k0 + i) + (k0 + j) * lda, true);
    }
  }
  cp_async_commit();
  cp_async_wait<0>();
  __syncthreads();
  for (int e = tid; e < npad * npad; e += nt) {
    int i = e % npad, j = e / npad;
    if (i < j) s[i + j * FLS] = 0.0;
    else if (i >= nb || j >= nb) s[i + j * FLS] = (i == j) ? 1.0 : 0.0;
  }
  __syncthreads();
  const int np = npad / SB;
  // one call site of the warp factor (a second inlined copy ran several times
  // slower)
  for (int p = 0; p < np; ++p) {
    const int c0 = p * SB;
    if (warp == 0) {
      int f = warp_factor_inv32(s, c0, xd + p * SB * XLD);
      if (f >= 0 && lane == 0) fail = c0 + f;
    }
    __syncthreads();
    if (fail >= 0) break;
    const int r0 = c0 + SB, cnt = npad - r0;
    if (cnt <= 0) break;
    // P = A_below · X_ppᵀ: tiles (cnt/16) × 4, held in registers until all read
    const double* X = xd + p * SB * XLD;
    const int tiles = (cnt / 16) * 4;
    double pc[3][4];  // ≤ 24 tiles over 8 warps
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      int tile = warp + q * nw;
#pragma unroll
      for (int r = 0; r < 4; ++r) pc[q][r] = 0.0;
      if (tile < tiles) {
        int tm = tile % (cnt / 16), tn = tile / (cnt / 16);
        mma_tile_smem(pc[q], s + (r0 + 16 * tm) + c0 * FLS, 1, FLS, X + 8 * tn, XLD, 1, SB);
      }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      int tile = warp + q * nw;
      if (tile < tiles) {
        int tm = tile % (cnt / 16), tn = tile / (cnt / 16);
        int row = r0 + 16 * tm + g, col = c0 + 8 * tn + 2 * t4;
        s[row + col * FLS] = pc[q][0];
        s[row + (col + 1) * FLS] = pc[q][1];
        s[(row + 8) + col * FLS] = pc[q][2];
        s[(row + 8) + (col + 1) * FLS] = pc[q][3];
      }
    }
    __syncthreads();
    // trailing update of the rest of the block (all warps)
    diag_syrk_tiles(s, c0, r0, r0, npad, npad, 0, nw);
    __syncthreads();
  }
  if (fail >= 0) {
    if (tid == 0) dev_fail(st, GPRX_CHOLESKY_FAILED, k0 + fail);
    return;
  }
  // L back to global
  for (int j = warp; j < nb; j += nw)
    for (int i = j + lane; i < nb; i += 32) A[(k0 + i) + (k0 + j) * lda] = s[i + j * FLS];
  // block inverse in place, column blocks right to left
  for (int jb = np - 1; jb >= 0; --jb) {
    const int j0 = jb * SB;
    const int nout = np - 1 - jb;
    // T_ib = Σ_{k=(jb+1)·32}^{(ib+1)·32−1} X(i, k) L(k, j): tiles (ib, 2 m-tiles, 4 n-tiles)
    for (int tile = warp; tile < nout * 8; tile += nw) {
      int ib = jb + 1 + tile / 8, tm = (tile % 8) / 4, tn = tile % 4;
      double c[4] = {0, 0, 0, 0};
      int kbeg = (jb + 1) * SB, kcnt = (ib - jb) * SB;
      mma_tile_smem(c, s + (ib * SB + 16 * tm) + kbeg * FLS, 1, FLS, s + kbeg + (j0 + 8 * tn) * FLS, 1, FLS, kcnt);
      double* T = tmp + (ib - jb - 1) * SB * XLD;
      int row = 16 * tm + g, col = 8 * tn + 2 * t4;
      T[row + col * XLD] = c[0];
      T[row + (col + 1) * XLD] = c[1];
      T[(row + 8) + col * XLD] = c[2];
      T[(row + 8) + (col + 1) * XLD] = c[3];
    }
    __syncthreads();
    const double* Xjj = xd + jb * SB * XLD;
    for (int tile = warp; tile < nout * 8; tile += nw) {
      int ib = jb + 1 + tile / 8, tm = (tile % 8) / 4, tn = tile % 4;
      const double* T = tmp + (ib - jb - 1) * SB * XLD;
      double c[4] = {0, 0, 0, 0};
      mma_tile_smem(c, T + 16 * tm, 1, XLD, Xjj + 8 * tn * XLD, 1, XLD, SB);
      int row = ib * SB + 16 * tm + g, col = j0 + 8 * tn + 2 * t4;
      s[row + col * FLS] = -c[0];
      s[row + (col + 1) * FLS] = -c[1];
      s[(row + 8) + col * FLS] = -c[2];
      s[(row + 8) + (col + 1) * FLS] = -c[3];
    }
    for (int e = tid; e < SB * SB; e += nt) {
      int rr = e % SB, cc = e / SB;
      s[(j0 + rr) + (j0 + cc) * FLS] = (rr >= cc) ? Xjj[rr + cc * XLD] : 0.0;
    }
    __syncthreads();
  }
  for (int j = warp; j < NB; j += nw)
    for (int i = lane; i < NB; i += 32) linv[i + j * NB] = (i < nb && j < nb && i >= j) ? s[i + j * FLS] : 0.0;
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
static size_t fast_diag_smem(int nb) { (void)nb; return (size_t)(NB * FLS + 7 * SB * XLD) * sizeof(double); }

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

FactorCtx::~FactorCtx() {
  for (auto e : ev) cudaEventDestroy(e);
  if (aux) cudaStreamDestroy(aux);
}

cudaError_t FactorCtx::ensure(int nblk) {
  if (!aux) {
    int lo, hi;
    CK(cudaDeviceGetStreamPriorityRange(&lo, &hi));
    CK(cudaStreamCreateWithPriority(&aux, cudaStreamNonBlocking, hi));
  }
  while ((int)ev.size() < 2 * nblk + 2) {
    cudaEvent_t e;
    CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    ev.push_back(e);
  }
  return cudaSuccess;
}

static cudaError_t diag_and_panel(double* A, long long ld, int n, int k0, double* linv, DevStatus* st,
                                  cudaStream_t s) {
  int nbk = min(NB, n - k0);
  double* lk = linv + (long long)(k0 / NB) * NB * NB;
  GPRX_LAUNCH(potrf_diag_kernel, 1, FD_THREADS, fast_diag_smem(nbk), s, A, ld, (long long)k0, nbk, lk, st);
  int rest = n - k0 - nbk;
  if (rest > 0) {
    double* P = A + (k0 + nbk) + (long long)k0 * ld;
    // panel: P := P · L_kk⁻ᵀ (in place; the 128-wide tile covers all nbk columns)
    GemmParams pp = gemm_params(rest, nbk, nbk, P, ld, lk, NB, P, ld, 1.0, 0.0, st);
    CK(dgemm(false, true, pp, s));
  }
  return cudaGetLastError();
}

// CTAs of the bulk trailing update in the look-ahead factor (of 148 SMs).
constexpr int BULK_CTAS = 132;

cudaError_t potrf_blocked(double* A, long long ld, int n, double* linv, DevStatus* st, cudaStream_t s,
                          FactorCtx* ctx) {
  CK(diag_attrs());
  const int nblk = ceil_div(n, NB);
  if (!ctx) {
    for (int k0 = 0; k0 < n; k0 += NB) {
      CK(diag_and_panel(A, ld, n, k0, linv, st, s));
      int nbk = min(NB, n - k0), rest = n - k0 - nbk;
      if (rest <= 0) break;
      double* P = A + (k0 + nbk) + (long long)k0 * ld;
      double* A22 = A + (k0 + nbk) + (long long)(k0 + nbk) * ld;
      GemmParams ps = gemm_params(rest, rest, nbk, P, ld, P, ld, A22, ld, -1.0, 1.0, st);
      ps.mode = GEMM_LOWER_TILES;
      CK(dgemm(false, true, ps, s));
    }
    return cudaGetLastError();
  }
  CK(ctx->ensure(nblk));
  cudaStream_t X = ctx->aux;
  cudaEvent_t* Ep = ctx->ev.data();          // panel k done (on X)
  cudaEvent_t* Es = ctx->ev.data() + nblk;   // trailing update of step k done (on s)
  cudaEvent_t Ein = ctx->ev[2 * nblk];
  CK(cudaEventRecord(Ein, s));
  CK(cudaStreamWaitEvent(X, Ein, 0));
  CK(diag_and_panel(A, ld, n, 0, linv, st, X));
  CK(cudaEventRecord(Ep[0], X));
  int last = 0;
  for (int k = 0; k < nblk; ++k) {
    const int c1 = (k + 1) * NB;  // first column of block k+1
    if (c1 >= n) break;
    const int k0 = k * NB;
    const double* Pk = A + c1 + (long long)k0 * ld;  // panel k, rows from c1
    // critical chain of block k+1 (side stream)
    if (k >= 1) CK(cudaStreamWaitEvent(X, Es[k - 1], 0));
    {
      int m = n - c1, w = min(NB, n - c1);
      GemmParams pc = gemm_params(m, w, NB, Pk, ld, Pk, ld, A + c1 + (long long)c1 * ld, ld, -1.0, 1.0, st);
      pc.mode = GEMM_LOWER_TILES;
      CK(dgemm(false, true, pc, X));
    }
    CK(diag_and_panel(A, ld, n, c1, linv, st, X));
    CK(cudaEventRecord(Ep[k + 1], X));
    last = k + 1;
    // bulk trailing update of step k (main stream): columns from c2
    CK(cudaStreamWaitEvent(s, Ep[k], 0));
    const int c2 = c1 + NB;
    if (c2 < n) {
      int m = n - c2;
      const double* Pk2 = A + c2 + (long long)k0 * ld;
      GemmParams ps = gemm_params(m, m, NB, Pk2, ld, Pk2, ld, A + c2 + (long long)c2 * ld, ld, -1.0, 1.0, st);
      ps.mode = GEMM_LOWER_TILES;
      ps.max_ctas = BULK_CTAS;  // leave SMs free for the side stream's chain
      CK(dgemm(false, true, ps, s));
    }
    CK(cudaEventRecord(Es[k], s));
  }
  CK(cudaStreamWaitEvent(s, Ep[last], 0));
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

// X = L⁻¹ by recursive doubling over the NB-blocks: the diagonal blocks are
// the inverses the factor left in linv; at each level every pair of sibling
// blocks gets X21 = −X22 (L21 X11), two batched triangular products with the
// k-ranges cut to the nonzero triangles.  X's strict upper triangle must be
// zero on entry (it is never written).  scratch holds ceil(n/2)² doubles.
__global__ void copy_diag_blocks_kernel(const double* linv, int n, double* X, long long ldx) {
  long long k0 = (long long)blockIdx.x * NB;
  int nb = (int)min((long long)NB, n - k0);
  const double* src = linv + (long long)blockIdx.x * NB * NB;
  for (int e = threadIdx.x; e < nb * nb; e += blockDim.x) {
    int i = e % nb, j = e / nb;
    X[(k0 + i) + (k0 + j) * ldx] = src[i + j * NB];
  }
}

cudaError_t trtri_blocked(const double* L, long long ld, int n, const double* linv, double* X, long long ldx,
                          double* scratch, DevStatus* st, cudaStream_t s) {
  int nblk = ceil_div(n, NB);
  GPRX_LAUNCH(copy_diag_blocks_kernel, nblk, 256, 0, s, linv, n, X, ldx);
  for (long long b = 2LL * NB; b < 2LL * n; b *= 2) {
    long long h = b / 2;
    if (h >= n) break;
    long long full = n / b;            // pairs with both halves of size h
    long long r = n - full * b;        // tail: a pair when it reaches past h
    for (int part = 0; part < 2; ++part) {
      long long s0, cnt, h2;
      if (part == 0) {
        if (full == 0) continue;
        s0 = 0;
        cnt = full;
        h2 = h;
      } else {
        if (r <= h) continue;
        s0 = full * b;
        cnt = 1;
        h2 = r - h;
      }
      // T = L21 · X11   (h2 × h, K = h; X11 lower → k from the column)
      GemmParams p1 = gemm_params((int)h2, (int)h, (int)h, L + (s0 + h) + s0 * ld, ld, X + s0 + s0 * ldx, ldx,
                                  scratch, h2, 1.0, 0.0, st);
      p1.mode = GEMM_K_FROM_COL;
      p1.strideA = b + b * ld;
      p1.strideB = b + b * ldx;
      p1.strideC = h2 * h;
      CK(dgemm(false, false, p1, s, (int)cnt));
      // X21 = −X22 · T   (h2 × h, K = h2; X22 lower → k up to the row)
      GemmParams p2 = gemm_params((int)h2, (int)h, (int)h2, X + (s0 + h) + (s0 + h) * ldx, ldx, scratch, h2,
                                  X + (s0 + h) + s0 * ldx, ldx, -1.0, 0.0, st);
      p2.mode = GEMM_K_TO_ROW;
      p2.strideA = b + b * ldx;
      p2.strideB = h2 * h;
      p2.strideC = b + b * ldx;
      CK(dgemm(false, false, p2, s, (int)cnt));
    }
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
