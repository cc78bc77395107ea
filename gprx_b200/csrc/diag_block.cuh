// diag_block.cuh — the diagonal-block step of the blocked Cholesky (LLT of an
// nb×nb block and its inverse, one CTA), shared by the blocked factor and the
// batched per-problem evaluation.
#pragma once

#include "gemm_f64.cuh"

namespace gprx {

constexpr int NB_DIAG = 128;

// ---------------------------------------------------------------------------
// Diagonal block (nb ≤ 128): LLT and the block's inverse X = L⁻¹ in shared
// memory, one CTA of FD_THREADS threads (warp 0 and seven helper warps).  The
// block is padded to a multiple of 16 with an identity tail.
//
// Left-looking by 16-column blocks p, two barriers per step:
//   warp 0   : the leaf (p, p) takes panel p−1 (its earlier panels are in),
//              then its 16×16 LLT in registers (lane = row, pivots by shuffles);
//   helpers  : column block p below the leaf takes panel p−1; column block
//              p+1 takes panels 0..p−1 in one product; block row p−1 of X:
//              X_{p−1,p−1} = L_{p−1,p−1}⁻¹ (one warp), T = L_{p−1,<p−1} X_{<p−1,<p−1},
//              then X_{p−1,<p−1} = −X_{p−1,p−1} T; and the stores of L column
//              block p−1 and of X block row p−2 to global memory;
//   all      : the panel below leaf p by column-oriented substitution.
// Column block q arrives by its own cp.async group, waited for one step
// before its first use, so the factor starts while the block still loads.
//
// Storage: L lower in s (ld FLS); X(i, j) for j < i in the transposed slot
// s[j + i·FLS] (the upper triangle), X(i, i) = 1/L_ii on the diagonal once
// block row i of X is formed (L's diagonal is kept in ldiag for the store).
// ---------------------------------------------------------------------------
constexpr int FD_THREADS = 256;
constexpr int LF = 16;                      // leaf / panel width
constexpr int FLS = NB_DIAG + 4;            // ld of the block (≡ 4 mod 16: conflict-free fragments)
constexpr int TLD = 20;                     // ld of T (16 rows; ≡ 4 mod 16)
constexpr int TMP_DOUBLES = TLD * NB_DIAG;  // T: 16 rows × up to 112 columns

// C(16×8) += A(16×K) · B(K×8) with A(i,k) = a[i·ai + k·ak], B(k,j) = b[k·bk + j·bj].
// AMASK: A(i,k) = 0 for k > i + moff;  BMASK: B(k,j) = 0 for k < j + moff.
template <bool AMASK = false, bool BMASK = false>
__device__ __forceinline__ void mma_tile_smem(double (&c)[4], const double* a, int ai, int ak, const double* b, int bk,
                                              int bj, int K, int moff = 0) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll 4
  for (int kk = 0; kk < K; kk += 4) {
    const int k = kk + t;
    double a0 = a[g * ai + k * ak];
    double a1 = a[(g + 8) * ai + k * ak];
    double b0 = b[k * bk + g * bj];
    if (AMASK) {
      if (k > g + moff) a0 = 0.0;
      if (k > g + 8 + moff) a1 = 0.0;
    }
    if (BMASK && k < g + moff) b0 = 0.0;
    dmma_16x8x4(c, a0, a1, b0);
  }
}

// 16×16 leaf LLT, one warp: lanes r and r+16 both hold row r of the block at
// (off, off) of s in registers; pivots are broadcast by shuffles.  Writes L
// back to s, 1/L_jj to rinv[off + j] and L_jj to ldiag[off + j].  Returns the
// failing column or −1 (uniform over the warp).  Out of line: one compact
// copy for every panel.
static __device__ __noinline__ int leaf16_factor(double* s, int off, double* rinv, double* ldiag) {
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
    ldiag[off + r] = d[r];
  }
  __syncwarp();
  return -1;
}

// One lower 16×8 tile of A[rbeg.., cbeg..] −= Σ_{k<K} L[rbeg+i, k0+k] L[cbeg+j, k0+k]
// (entries above the diagonal are left alone).
__device__ __forceinline__ void syrk_tile(double* s, int rbeg, int cbeg, int k0, int K) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t4 = lane & 3;
  double c[4] = {0, 0, 0, 0};
  mma_tile_smem(c, s + rbeg + k0 * FLS, 1, FLS, s + cbeg + k0 * FLS, FLS, 1, K);
  const int row = rbeg + g, col = cbeg + 2 * t4;
  if (row >= col) s[row + col * FLS] -= c[0];
  if (row >= col + 1) s[row + (col + 1) * FLS] -= c[1];
  if (row + 8 >= col) s[(row + 8) + col * FLS] -= c[2];
  if (row + 8 >= col + 1) s[(row + 8) + (col + 1) * FLS] -= c[3];
}

// 16×8 tiles of a 16-column block from row r0 to npad (tile u: rows
// r0 + 16·(u/2), columns + 8·(u%2)).
__device__ __forceinline__ int colblock_tiles(int r0, int npad) { return ((npad - r0) / 16) * 2; }

// The 16×16 leaf inverse of block q (one warp): lane c computes column c of
// L_qq⁻¹ by substitution; X(i, c) goes to s[c + i·FLS] (i ≥ c: the diagonal
// and the transposed slot above it).
__device__ __forceinline__ void leaf16_inverse(double* s, int q, const double* rinv) {
  const int lane = threadIdx.x & 31, c = lane & 15, off = q * LF;
  double acc[LF];
#pragma unroll
  for (int i = 0; i < LF; ++i) acc[i] = (i == c) ? 1.0 : 0.0;
#pragma unroll
  for (int t = 0; t < LF; ++t) {
    const double x = acc[t] * rinv[off + t];
    acc[t] = x;
#pragma unroll
    for (int j = t + 1; j < LF; ++j) acc[j] = fma(-s[(off + j) + (off + t) * FLS], x, acc[j]);
  }
  if (lane < 16) {
#pragma unroll
    for (int i = 0; i < LF; ++i)
      if (i >= c) s[(off + c) + (off + i) * FLS] = acc[i];
  }
}

// T tile tn of block row q (a0 = 16q): T(:, j0..j0+7) = L_{q,<q}(:, kb..) X_{<q,<q}(kb.., j0..),
// k from kb = j0 rounded down to 4 (X(k, j) = 0 for k < j), T in tmp (ld TLD).
__device__ __forceinline__ void inv_t_tile(const double* s, double* tmp, int q, int tn) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t4 = lane & 3;
  const int a0 = q * LF, j0 = 8 * tn, kb = j0 & ~3;
  double c[4] = {0, 0, 0, 0};
  // A(i, k) = L(a0 + i, kb + k);  B(k, j) = X(kb + k, j0 + j) = s[(j0 + j) + (kb + k)·FLS], 0 for kb + k < j0 + j
  mma_tile_smem<false, true>(c, s + a0 + kb * FLS, 1, FLS, s + j0 + kb * FLS, FLS, 1, a0 - kb, j0 - kb);
  const int row = g, col = j0 + 2 * t4;
  tmp[row + col * TLD] = c[0];
  tmp[row + (col + 1) * TLD] = c[1];
  tmp[(row + 8) + col * TLD] = c[2];
  tmp[(row + 8) + (col + 1) * TLD] = c[3];
}

// X tile tn of block row q: X(a0+i, j0+j) = −Σ_{k ≤ i} X_qq(i, k) T(k, j0+j), into the transposed slot.
__device__ __forceinline__ void inv_x_tile(double* s, const double* tmp, int q, int tn) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t4 = lane & 3;
  const int a0 = q * LF, j0 = 8 * tn;
  double c[4] = {0, 0, 0, 0};
  // A(i, k) = X_qq(i, k) = s[(a0 + k) + (a0 + i)·FLS] for k ≤ i;  B(k, j) = T(k, j0 + j)
  mma_tile_smem<true, false>(c, s + a0 + a0 * FLS, FLS, 1, tmp + j0 * TLD, 1, TLD, LF, 0);
  const int row = a0 + g, col = j0 + 2 * t4;
  s[col + row * FLS] = -c[0];
  s[(col + 1) + row * FLS] = -c[1];
  s[col + (row + 8) * FLS] = -c[2];
  s[(col + 1) + (row + 8) * FLS] = -c[3];
}

// Stores of finished parts, one warp each.
// L column block q, columns q·16 + 8·half .. +8, rows from the diagonal (L_jj
// from ldiag; 16-byte stores from the first even row when vec).
__device__ __forceinline__ void store_l_part(const double* s, const double* ldiag, double* A, long long lda,
                                             long long k0, int nb, bool vec, int q, int half) {
  const int lane = threadIdx.x & 31;
  for (int j = q * LF + 8 * half; j < q * LF + 8 * half + 8 && j < nb; ++j) {
    double* col = A + k0 + (k0 + j) * lda;
    const double* sc = s + j * FLS;
    if (vec) {
      const int i0 = (j + 1) & ~1;
      if ((j & 1) && lane == 0) col[j] = ldiag[j];
      for (int i = i0 + 2 * lane; i + 1 < nb; i += 64)
        *reinterpret_cast<double2*>(col + i) = make_double2(i == j ? ldiag[j] : sc[i], sc[i + 1]);
      if (((nb - i0) & 1) && lane == 0) col[nb - 1] = (nb - 1 == j) ? ldiag[j] : sc[nb - 1];
    } else {
      for (int i = j + lane; i < nb; i += 32) col[i] = (i == j) ? ldiag[j] : sc[i];
    }
  }
}

// Block row q of X into linv (ld NB_DIAG, zero above the diagonal and in the
// padding), columns [part·cw, (part+1)·cw), cw = NB_DIAG / nparts.
__device__ __forceinline__ void store_x_part(const double* s, double* linv, int nb, int q, int part, int nparts) {
  const int lane = threadIdx.x & 31, cw = NB_DIAG / nparts;
  const int i = q * LF + 2 * (lane & 7);
  for (int jb = part * cw; jb < (part + 1) * cw; jb += 4) {
    const int j = jb + (lane >> 3);
    const double a = (i < nb && j < nb && j <= i) ? s[j + i * FLS] : 0.0;
    const double b = (i + 1 < nb && j < nb && j <= i + 1) ? s[j + (i + 1) * FLS] : 0.0;
    *reinterpret_cast<double2*>(linv + i + j * NB_DIAG) = make_double2(a, b);
  }
}

// cp.async.wait_group with a run-time count (0 ≤ n ≤ 7 groups left in flight)
__device__ __forceinline__ void cp_async_wait_n(int n) {
  switch (n < 0 ? 0 : n) {
    case 0: cp_async_wait<0>(); break;
    case 1: cp_async_wait<1>(); break;
    case 2: cp_async_wait<2>(); break;
    case 3: cp_async_wait<3>(); break;
    case 4: cp_async_wait<4>(); break;
    case 5: cp_async_wait<5>(); break;
    case 6: cp_async_wait<6>(); break;
    default: cp_async_wait<7>(); break;
  }
}

// The work of step p that is off warp 0's chain, dealt over nh warps (h =
// this warp's index among them): inverse block row q = p − 1 (leaf inverse
// and T, then — after the barrier of the nh warps — X_{q,<q}), the updates
// of column blocks p (panel p−1, below the leaf) and p+1 (panels 0..p−1),
// the store of L column block p−1 and of X block row p−2.  With tail, p = np
// and the whole CTA takes part (barriers are __syncthreads).
static __device__ void diag_helpers(double* s, double* tmp, const double* rinv, const double* ldiag, double* A, long long lda,
                             long long k0, int nb, double* linv, bool vec, int p, int np, int h, int nh, bool tail) {
  const int npad = np * LF, c0 = p * LF, r1 = c0 + LF, q = p - 1;
  const int n_inv = p >= 1 ? 1 : 0;
  const int n_t = p >= 2 ? 2 * q : 0;
  const int n_next = (!tail && p >= 1 && p + 1 < np) ? colblock_tiles(r1, npad) : 0;
  const int n_cur = (!tail && p >= 1 && r1 < npad) ? colblock_tiles(r1, npad) : 0;
  const int n_ls = p >= 1 ? 2 : 0;
  const int xs_parts = tail ? 4 : 2;
  const int n_xs = p >= 2 ? xs_parts : 0;
  const int total = n_inv + n_t + n_next + n_cur + n_ls + n_xs;
  for (int t = h; t < total; t += nh) {
    int u = t;
    if (u < n_inv) { leaf16_inverse(s, q, rinv); continue; }
    u -= n_inv;
    if (u < n_t) { inv_t_tile(s, tmp, q, u); continue; }
    u -= n_t;
    if (u < n_next) {  // column block p+1, rows from r1, panels 0..p−1
      const int rbeg = r1 + 16 * (u >> 1), cbeg = r1 + 8 * (u & 1);
      if (rbeg + 15 >= cbeg) syrk_tile(s, rbeg, cbeg, 0, c0);
      continue;
    }
    u -= n_next;
    if (u < n_cur) {  // column block p below the leaf, panel p−1
      syrk_tile(s, r1 + 16 * (u >> 1), c0 + 8 * (u & 1), c0 - LF, LF);
      continue;
    }
    u -= n_cur;
    if (u < n_ls) { store_l_part(s, ldiag, A, lda, k0, nb, vec, q, u); continue; }
    u -= n_ls;
    store_x_part(s, linv, nb, p - 2, u, xs_parts);
  }
  if (p < 2) return;
  if (tail) __syncthreads();
  else asm volatile("bar.sync 1, %0;" ::"r"(32 * nh) : "memory");
  for (int t = h; t < 2 * q; t += nh) inv_x_tile(s, tmp, q, t);
}

// The whole diagonal-block step for one CTA of FD_THREADS threads: load the
// nb×nb lower block at (k0, k0) of A, factor it (L back into A), invert it
// (L⁻¹ into linv, ld NB_DIAG, zero above the diagonal).  fail_sh is a shared
// int.  Returns the failing column (uniform over the CTA) or −1; either way
// no copy into shared memory is in flight on return.
static __device__ int diag_block_factor_inv(double* A, long long lda, long long k0, int nb, double* linv, double* smem,
                                            int* fail_sh) {
  int& fail = *fail_sh;
  double* s = smem;                  // NB_DIAG × FLS
  double* tmp = s + NB_DIAG * FLS;   // TMP_DOUBLES
  double* rinv = tmp + TMP_DOUBLES;  // NB_DIAG reciprocal pivots
  double* ldiag = rinv + NB_DIAG;    // NB_DIAG diagonal entries of L
  const int tid = threadIdx.x, nt = blockDim.x, warp = tid >> 5, nw = nt >> 5, lane = tid & 31;
  const int npad = (nb + LF - 1) / LF * LF, np = npad / LF;
  if (tid == 0) fail = -1;
  // column block q is cp.async group q of every thread (16-byte copies from
  // the even row at or above the diagonal); blocks 0 and 1 go first alone and
  // are waited for, the rest then loads during the first steps
  const bool vec = ((lda & 1) == 0) && ((((unsigned long long)(A + k0 + k0 * lda)) & 15) == 0);
  for (int q = 0; q < np; ++q) {
    if (q == 2) cp_async_wait<0>();
    for (int j = q * LF + warp; j < q * LF + LF && j < nb; j += nw) {
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
  }
  // identity padding (lower part; the copies never reach these entries)
  for (int j = warp; j < npad; j += nw)
    for (int i = j + lane; i < npad; i += 32)
      if (i >= nb || j >= nb) s[i + j * FLS] = (i == j) ? 1.0 : 0.0;
  cp_async_wait_n(np - 2);  // column blocks 0 and 1
  __syncthreads();
  for (int p = 0; p < np; ++p) {
    const int c0 = p * LF, r1 = c0 + LF;
    if (warp == 0) {
      if (p > 0) {  // the leaf's last update: panel p−1
        syrk_tile(s, c0, c0, c0 - LF, LF);
        syrk_tile(s, c0, c0 + 8, c0 - LF, LF);
        __syncwarp();
      }
      const int f = leaf16_factor(s, c0, rinv, ldiag);
      if (f >= 0 && lane == 0) fail = c0 + f;
    } else {
      diag_helpers(s, tmp, rinv, ldiag, A, lda, k0, nb, linv, vec, p, np, warp - 1, nw - 1, false);
    }
    __syncthreads();
    if (fail >= 0) break;
    // panel: rows below the leaf solve X L_ppᵀ = A (32 rows per warp)
    for (int grp = warp; grp * 32 < npad - r1; grp += nw) {
      const int row = r1 + grp * 32 + lane;
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
    cp_async_wait_n(np - 3 - p);  // column block p+2, used by the next step's helpers
    __syncthreads();
  }
  if (fail >= 0) {
    cp_async_wait<0>();
    __syncthreads();
    return fail;
  }
  // the last block row of X, the last column block of L, the last two block
  // rows of X into linv (all warps)
  diag_helpers(s, tmp, rinv, ldiag, A, lda, k0, nb, linv, vec, np, np, warp, nw, true);
  __syncthreads();
  // block rows np−1 .. NB_DIAG/16 − 1 (those past the block are zeros)
  for (int t = warp; t < (NB_DIAG / LF - np + 1) * 4; t += nw) store_x_part(s, linv, nb, np - 1 + t / 4, t % 4, 4);
  __syncthreads();
  return -1;
}

inline size_t diag_block_smem() { return (size_t)(NB_DIAG * FLS + TMP_DOUBLES + 2 * NB_DIAG) * sizeof(double); }

}  // namespace gprx
