// diag_block.cuh — the diagonal-block step of the blocked Cholesky (LLT of an
// nb×nb block and its inverse, one CTA), shared by the blocked factor and the
// batched per-problem evaluation.
#pragma once

#include "gemm_f64.cuh"

namespace gprx {

constexpr int NB_DIAG = 128;

// ---------------------------------------------------------------------------
// Diagonal block (nb ≤ 128): LLT and the block's inverse in shared memory,
// one CTA of FD_THREADS threads.  The block is padded to a multiple of 16
// with an identity tail.
//   factor, per 16-column panel p (right-looking, with look-ahead inside the
//   CTA):
//     warp 0 factors the 16×16 leaf in registers (lane = row, pivots by
//     shuffles) and keeps the reciprocal pivots; meanwhile warps 1..7 apply
//     the previous panel's trailing update (DMMA m16n8k4, K = 16) to the rest
//     of the block;
//     all warps: the panel below the leaf by column-oriented substitution
//     (lane = row, L entries broadcast from shared memory);
//     warp 0: the next leaf's own update, then its factor.
//   inverse (off the chain): every warp inverts one 16×16 leaf, then
//   recursive doubling 16 → 32 → 64 → 128 on DMMA:
//     X21 = −X22 (L21 X11), in place.
// ---------------------------------------------------------------------------
constexpr int FD_THREADS = 256;
constexpr int LF = 16;               // leaf / panel width
constexpr int FLS = NB_DIAG + 4;     // ld of the block (≡ 4 mod 16: conflict-free fragments)
constexpr int TMP_DOUBLES = 64 * 68; // the doubling step's T (ld h + 4 ≡ 4 mod 16)

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

// 16×16 leaf LLT, one warp: lanes r and r+16 both hold row r of the block at
// (off, off) of s in registers; pivots are broadcast by shuffles.  Writes L
// back to s and 1/L_jj to rinv[off + j].  Returns the failing column or −1
// (uniform over the warp).  Out of line: one compact copy for every panel.
static __device__ __noinline__ int leaf16_factor(double* s, int off, double* rinv) {
  const int lane = threadIdx.x & 31, r = lane & 15;
  double d[16];
#pragma unroll
  for (int c = 0; c < 16; ++c) d[c] = (c <= r) ? s[(off + r) + (off + c) * FLS] : 0.0;
  int bad = -1;
  double my_inv = 1.0;
  // the next pivot is formed first, by its own row from its own entry, so
  // that the chain from one pivot to the next is a shuffle, the reciprocal
  // square root, a product and an FMA; the other updates of the step overlap
  // it (the values are those of the plain order, bit for bit)
  double piv = __shfl_sync(0xffffffffu, d[0], 0);
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    if (!(piv > 0.0) && bad < 0) bad = j;
    const double rs = rsqrt(fmax(piv, 1e-300));
    if (r == j) {
      d[j] = piv * rs;
      my_inv = rs;
    } else if (r > j) {
      d[j] = d[j] * rs;
    }
    if (j + 1 < 16) {
      const double cand = (r == j + 1) ? fma(-d[j], d[j], d[j + 1]) : 0.0;
      const double nxt = __shfl_sync(0xffffffffu, cand, j + 1);
#pragma unroll
      for (int c = 0; c < 16; ++c) {
        if (c > j) {
          const double lcj = __shfl_sync(0xffffffffu, d[j], c);
          if (r >= c) d[c] = fma(-d[j], lcj, d[c]);
        }
      }
      piv = nxt;
    }
  }
  if (bad >= 0) return bad;
  if (lane < 16) {
#pragma unroll
    for (int c = 0; c < 16; ++c)
      if (c <= r) s[(off + r) + (off + c) * FLS] = d[c];
    rinv[off + r] = my_inv;
  }
  __syncwarp();
  return -1;
}

// Lower 16×8 tiles of A[i][j] −= Σ_{t<16} A[i][k0+t] A[j][k0+t] over rows and
// columns [r0, npad); `which` = 0: every tile but those of the 16×16 block at
// (r0, r0), dealt to warps w0.. in steps of nws; 1: only that block's tiles
// (the calling warp does both).
__device__ __forceinline__ void syrk16_tiles(double* s, int k0, int r0, int npad, int which, int w0, int nws) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t4 = lane & 3;
  const int tm_n = (npad - r0) / 16, tn_n = (npad - r0) / 8;
  const int first = which ? 0 : warp - w0, count = which ? 2 : tm_n * tn_n, step = which ? 1 : nws;
  for (int tile = first; tile < count; tile += step) {
    const int tm = which ? 0 : tile % tm_n, tn = which ? tile : tile / tm_n;
    if (!which && tm == 0 && tn < 2) continue;
    const int rbeg = r0 + 16 * tm, cbeg = r0 + 8 * tn;
    if (rbeg + 15 < cbeg) continue;
    double c[4] = {0, 0, 0, 0};
    mma_tile_smem(c, s + rbeg + k0 * FLS, 1, FLS, s + cbeg + k0 * FLS, FLS, 1, LF);
    const int row = rbeg + g, col = cbeg + 2 * t4;
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
  double* s = smem;                     // NB_DIAG × FLS
  double* tmp = s + NB_DIAG * FLS;      // TMP_DOUBLES
  double* rinv = tmp + TMP_DOUBLES;     // NB_DIAG reciprocal pivots
  const int tid = threadIdx.x, nt = blockDim.x, warp = tid >> 5, nw = nt >> 5;
  const int lane = tid & 31, g = lane >> 2, t4 = lane & 3;
  const int npad = (nb + LF - 1) / LF * LF;
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
  const int np = npad / LF;
  for (int p = 0; p < np; ++p) {
    const int c0 = p * LF;
    if (warp == 0) {
      // leaf p (its own update by the previous panel was done by this warp)
      const int f = leaf16_factor(s, c0, rinv);
      if (f >= 0 && lane == 0) fail = c0 + f;
    } else if (p > 0) {
      // the previous panel's update of the rest of the trailing block
      syrk16_tiles(s, c0 - LF, c0, npad, 0, 1, nw - 1);
    }
    __syncthreads();
    if (fail >= 0) break;
    const int r0 = c0 + LF;
    if (r0 >= npad) break;
    // panel: rows below the leaf solve X L_ppᵀ = A (32 rows per warp)
    for (int grp = warp; grp * 32 < npad - r0; grp += nw) {
      const int row = r0 + grp * 32 + lane;
      const bool act = row < npad;
      double a[LF];
#pragma unroll
      for (int c = 0; c < LF; ++c) a[c] = act ? s[row + (c0 + c) * FLS] : 0.0;
#pragma unroll
      for (int t = 0; t < LF; ++t) {
        const double x = a[t] * rinv[c0 + t];
        a[t] = x;
#pragma unroll
        for (int j = t + 1; j < LF; ++j) a[j] = fma(-x, s[(c0 + j) + (c0 + t) * FLS], a[j]);
      }
      if (act) {
#pragma unroll
        for (int c = 0; c < LF; ++c) s[row + (c0 + c) * FLS] = a[c];
      }
    }
    __syncthreads();
    // the next leaf's own update (warp 0, which factors it next)
    if (warp == 0) {
      syrk16_tiles(s, c0, r0, npad, 1, 0, 1);
      __syncwarp();
    }
  }
  if (fail >= 0) return fail;
  // L back to global (16-byte stores from the first even row below the diagonal)
  for (int j = warp; j < nb; j += nw) {
    double* col = A + k0 + (k0 + j) * lda;
    const double* sc = s + j * FLS;
    if (vec) {
      const int i0 = (j + 1) & ~1;
      if ((j & 1) && lane == 0) col[j] = sc[j];
      for (int i = i0 + 2 * lane; i + 1 < nb; i += 64)
        *reinterpret_cast<double2*>(col + i) = *reinterpret_cast<const double2*>(sc + i);
      if (((nb - i0) & 1) && lane == 0) col[nb - 1] = sc[nb - 1];
    } else {
      for (int i = j + lane; i < nb; i += 32) col[i] = sc[i];
    }
  }
  __syncthreads();
  // leaf inverses: lane q computes column q of L_pp⁻¹ by column-oriented
  // substitution, written over L_pp (its off-diagonal blocks stay L)
  for (int p = warp; p < np; p += nw) {
    const int off = p * LF, q = lane & 15;
    double acc[LF];
#pragma unroll
    for (int i = 0; i < LF; ++i) acc[i] = (i == q) ? 1.0 : 0.0;
#pragma unroll
    for (int t = 0; t < LF; ++t) {
      const double x = acc[t] * rinv[off + t];
      acc[t] = x;
#pragma unroll
      for (int j = t + 1; j < LF; ++j) acc[j] = fma(-s[(off + j) + (off + t) * FLS], x, acc[j]);
    }
    __syncwarp();
    if (lane < 16) {
#pragma unroll
      for (int i = 0; i < LF; ++i)
        if (i >= q) s[(off + i) + (off + q) * FLS] = acc[i];
    }
  }
  __syncthreads();
  // recursive doubling: for sibling blocks (a, b) of h columns,
  // T = L21 X11 (X11 lower: k from the column), X21 = −X22 T (k up to the row)
  for (int h = LF; h < npad; h *= 2) {
    const int TL = h + 4;
    const int pairs = (npad + 2 * h - 1) / (2 * h);
    int ntile = 0;
    for (int k = 0; k < pairs; ++k) {
      const int b = 2 * k * h + h;
      if (b < npad) ntile += (min(h, npad - b) / 16) * (h / 8);
    }
    for (int tile = warp; tile < ntile; tile += nw) {
      int rest = tile, k = 0, h2 = 0;
      for (;; ++k) {
        const int b = 2 * k * h + h;
        h2 = min(h, npad - b);
        const int cnt = (h2 / 16) * (h / 8);
        if (rest < cnt) break;
        rest -= cnt;
      }
      const int a0 = 2 * k * h, b0 = a0 + h;
      const int tm = rest % (h2 / 16), tn = rest / (h2 / 16);
      const int i0 = 16 * tm, j0 = 8 * tn, kb = j0 & ~3;
      double c[4] = {0, 0, 0, 0};
      mma_tile_smem(c, s + (b0 + i0) + (a0 + kb) * FLS, 1, FLS, s + (a0 + kb) + (a0 + j0) * FLS, 1, FLS, h - kb);
      double* T = tmp + k * h * TL;
      const int row = i0 + g, col = j0 + 2 * t4;
      T[row + col * TL] = c[0];
      T[row + (col + 1) * TL] = c[1];
      T[(row + 8) + col * TL] = c[2];
      T[(row + 8) + (col + 1) * TL] = c[3];
    }
    __syncthreads();
    for (int tile = warp; tile < ntile; tile += nw) {
      int rest = tile, k = 0, h2 = 0;
      for (;; ++k) {
        const int b = 2 * k * h + h;
        h2 = min(h, npad - b);
        const int cnt = (h2 / 16) * (h / 8);
        if (rest < cnt) break;
        rest -= cnt;
      }
      const int a0 = 2 * k * h, b0 = a0 + h;
      const int tm = rest % (h2 / 16), tn = rest / (h2 / 16);
      const int i0 = 16 * tm, j0 = 8 * tn;
      const double* T = tmp + k * h * TL;
      double c[4] = {0, 0, 0, 0};
      mma_tile_smem(c, s + (b0 + i0) + b0 * FLS, 1, FLS, T + j0 * TL, 1, TL, i0 + 16);
      const int row = b0 + i0 + g, col = a0 + j0 + 2 * t4;
      s[row + col * FLS] = -c[0];
      s[row + (col + 1) * FLS] = -c[1];
      s[(row + 8) + col * FLS] = -c[2];
      s[(row + 8) + (col + 1) * FLS] = -c[3];
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


inline size_t diag_block_smem() { return (size_t)(NB_DIAG * FLS + TMP_DOUBLES + NB_DIAG) * sizeof(double); }

}  // namespace gprx
