// diag_block.cuh — the diagonal-block step of the blocked Cholesky (LLT of an
// nb×nb block and its inverse, one CTA), shared by the blocked factor and the
// batched per-problem evaluation.
#pragma once

#include "gemm_f64.cuh"

namespace gprx {

constexpr int NB_DIAG = 128;

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
constexpr int FLS = NB_DIAG + 4;     // ld of the block (≡ 4 mod 16: conflict-free fragments)
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
static __device__ __noinline__ int leaf16_factor_inv(double* s, int off, double* xo) {
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

// The whole diagonal-block step for one CTA of FD_THREADS threads: load the
// nb×nb lower block at (k0, k0) of A, factor it (L back into A), invert it
// (L⁻¹ into linv, ld NB_DIAG, zero above the diagonal; it also stays in smem[0 ..
// NB_DIAG·FLS) with ld FLS).  fail_sh is a shared int.  Returns the failing column
// (uniform over the CTA) or −1.
static __device__ int diag_block_factor_inv(double* A, long long lda, long long k0, int nb, double* linv, double* smem,
                                     int* fail_sh) {
  int& fail = *fail_sh;
  double* s = smem;                       // NB_DIAG × FLS
  double* xd = s + NB_DIAG * FLS;              // 4 × (32 × XLD) sub-block inverses
  double* tmp = xd + 4 * SB * XLD;        // 3 × (32 × XLD)
  const int tid = threadIdx.x, nt = blockDim.x, warp = tid >> 5, nw = nt >> 5;
  const int lane = tid & 31, g = lane >> 2, t4 = lane & 3;
  const int npad = (nb + SB - 1) / SB * SB;
  if (tid == 0) fail = -1;
  __syncthreads();
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
  for (int j = warp; j < npad; j += nw)
    for (int i = lane; i < npad; i += 32) {
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
  if (fail >= 0) return fail;
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
  for (int j = warp; j < NB_DIAG; j += nw)
    for (int i = 2 * lane; i < NB_DIAG; i += 64) {
      const double a = (i < nb && j < nb && i >= j) ? s[i + j * FLS] : 0.0;
      const double b = (i + 1 < nb && j < nb && i + 1 >= j) ? s[i + 1 + j * FLS] : 0.0;
      *reinterpret_cast<double2*>(linv + i + j * NB_DIAG) = make_double2(a, b);
    }
  __syncthreads();
  return -1;
}


inline size_t diag_block_smem() { return (size_t)(NB_DIAG * FLS + 7 * SB * XLD) * sizeof(double); }

}  // namespace gprx
