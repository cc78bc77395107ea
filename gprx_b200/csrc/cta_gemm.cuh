// cta_gemm.cuh — FP64 GEMM run by ONE CTA of 512 threads over all output
// tiles of a small matrix product: the building block of the batched
// per-problem evaluation, where each CTA owns a whole problem.
//
//   C = alpha · Σ_{k∈[kb,K)} opA(i,k) opB(k,j) + beta · C
//   opA(i,k) = TA ? A[k + i·lda] : A[i + k·lda]
//   opB(k,j) = TB ? B[j + k·ldb] : B[k + j·ldb]
//
// Output tiles are TM×TN, 16 warps in a WGM×WGN grid of (TM/WGM)×(TN/WGN)
// DMMA m16n8k4 blocks (32×32 tiles keep eight warps busy and let the other
// eight load); the shapes the autotuner picks from are listed in CgTile
// below.  The k chunks (TK deep) of ALL tiles form one stream through
// a 2- or 3-stage cp.async ring, so the next tile's first chunks load while the
// current tile computes, and the C values a tile needs (beta ≠ 0) are fetched
// into registers when the tile starts.  Shared-memory layouts follow each
// operand's contiguous direction (16-byte copies) with leading dimensions
// ≡ 4 mod 16 doubles, which keeps every fragment load free of bank conflicts.
//
// Every tile shape sums each output's k terms in the same order (k ascending
// from a multiple of 4, four per DMMA), so the results do not depend on the
// shape.
//
// lower: only entries i ≥ j are written; tiles wholly above the diagonal are
// skipped and warps whose block is wholly above it only help load.
// kmode: CG_FULL kb = 0; CG_FROM_ROW kb = the tile's first row (opA(i,k) = 0
// for k < i); CG_FROM_COL kb = the tile's first column (opB(k,j) = 0 for
// k < j).  A tile reads all its inputs before it writes C, so C may alias A's
// rows when one tile spans all of N.
#pragma once

#include "gemm_f64.cuh"

namespace gprx {

constexpr int CG_THREADS = 512;
constexpr int CG_FULL = 0, CG_FROM_ROW = 1, CG_FROM_COL = 2;

// tile shapes (TM × TN, k chunk TK, warp grid WGM × WGN, copy-ring stages ST)
// by configuration index; the 64×128 tile takes 64-deep chunks in two stages
// (half the barriers of 32-deep chunks in three; a chunk's DMMA work covers
// the next chunk's copy)
constexpr int CG_CONFIGS = 4;
template <int CFG>
struct CgTile;
template <> struct CgTile<0> { static constexpr int M = 64, N = 128, K = 64, WGM = 4, WGN = 4, ST = 2; };
template <> struct CgTile<1> { static constexpr int M = 64, N = 64, K = 32, WGM = 4, WGN = 4, ST = 3; };
template <> struct CgTile<2> { static constexpr int M = 32, N = 64, K = 32, WGM = 2, WGN = 8, ST = 3; };
template <> struct CgTile<3> { static constexpr int M = 32, N = 32, K = 16, WGM = 2, WGN = 4, ST = 3; };
__host__ __device__ constexpr int cg_tile_n(int cfg) { return cfg == 0 ? 128 : cfg == 3 ? 32 : 64; }
__host__ __device__ constexpr int cg_tile_m(int cfg) { return cfg <= 1 ? 64 : 32; }

template <bool TA, int TM, int TK>
struct CgA {  // A chunk: TM (i) × TK (k)
  static constexpr int LD = TA ? TK + 4 : TM + 4;
  static constexpr int ELEMS = TA ? TM * LD : TK * LD;
  __device__ static int at(int i, int k) { return TA ? i * LD + k : k * LD + i; }
};
template <bool TB, int TN, int TK>
struct CgB {  // B chunk: TK (k) × TN (j)
  static constexpr int LD = TB ? TN + 4 : TK + 4;
  static constexpr int ELEMS = TB ? TK * LD : TN * LD;
  __device__ static int at(int k, int j) { return TB ? k * LD + j : j * LD + k; }
};

template <int CFG>
constexpr size_t cg_smem_bytes_cfg() {
  using T = CgTile<CFG>;
  constexpr int a = CgA<true, T::M, T::K>::ELEMS > CgA<false, T::M, T::K>::ELEMS ? CgA<true, T::M, T::K>::ELEMS
                                                                                 : CgA<false, T::M, T::K>::ELEMS;
  constexpr int b = CgB<true, T::N, T::K>::ELEMS > CgB<false, T::N, T::K>::ELEMS ? CgB<true, T::N, T::K>::ELEMS
                                                                                 : CgB<false, T::N, T::K>::ELEMS;
  return (size_t)T::ST * (a + b) * sizeof(double);
}
constexpr size_t cg_max2(size_t a, size_t b) { return a > b ? a : b; }
// the largest stage ring over the shapes and the four orientations
constexpr size_t cg_smem_bytes() {
  return cg_max2(cg_max2(cg_smem_bytes_cfg<0>(), cg_smem_bytes_cfg<1>()),
                 cg_max2(cg_smem_bytes_cfg<2>(), cg_smem_bytes_cfg<3>()));
}

// 16-byte copy of src_bytes ∈ {0, 8, 16} (the rest zero-filled)
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, int src_bytes) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(src_bytes));
}

template <bool TA, bool TB, int CFG>
__device__ void cta_gemm_tile(int M, int N, int K, const double* A, long long lda, const double* B, long long ldb,
                         double* C, long long ldc, double alpha, double beta, bool lower, int kmode, double* smem) {
  constexpr int CG_M = CgTile<CFG>::M, CG_N = CgTile<CFG>::N, CG_K = CgTile<CFG>::K;
  constexpr int WGM = CgTile<CFG>::WGM, WGN = CgTile<CFG>::WGN, ST = CgTile<CFG>::ST;
  constexpr int WM = CG_M / WGM, WN = CG_N / WGN, MI = WM / 16, NJ = WN / 8;
  static_assert(WGM * WGN <= CG_THREADS / 32 && MI >= 1 && NJ >= 1, "warp grid");
  using SA = CgA<TA, CG_M, CG_K>;
  using SB = CgB<TB, CG_N, CG_K>;
  constexpr int STAGE = SA::ELEMS + SB::ELEMS;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, g = lane >> 2, t4 = lane & 3;
  const int wm = warp % WGM, wn = warp / WGM;
  const bool wact = warp < WGM * WGN;  // warps past the grid only load
  const int tm_n = (M + CG_M - 1) / CG_M, tn_n = (N + CG_N - 1) / CG_N;
  const int ntiles = tm_n * tn_n;
  // 16-byte copies need even leading dimensions and 16-byte aligned bases
  const bool a16 = ((lda & 1) == 0) && ((reinterpret_cast<unsigned long long>(A) & 15) == 0);
  const bool b16 = ((ldb & 1) == 0) && ((reinterpret_cast<unsigned long long>(B) & 15) == 0);

  auto tile_used = [&](int t) {
    const int m0 = (t % tm_n) * CG_M, n0 = (t / tm_n) * CG_N;
    return !(lower && m0 + CG_M - 1 < n0);
  };
  auto tile_kb = [&](int t) {
    const int m0 = (t % tm_n) * CG_M, n0 = (t / tm_n) * CG_N;
    int kb = kmode == CG_FROM_ROW ? m0 : kmode == CG_FROM_COL ? n0 : 0;
    return kb < K ? kb : K;
  };
  auto tile_nch = [&](int t) {
    const int n = (K - tile_kb(t) + CG_K - 1) / CG_K;
    return n > 0 ? n : 1;  // an empty k range still runs one zero chunk
  };
  auto next_used = [&](int t) {
    while (t < ntiles && !tile_used(t)) ++t;
    return t;
  };

  // loader cursor
  int lt = next_used(0), lc = 0;
  auto load_next = [&](int st) {
    if (lt < ntiles) {
      const int m0 = (lt % tm_n) * CG_M, n0 = (lt / tm_n) * CG_N;
      const int k0 = tile_kb(lt) + lc * CG_K;
      double* sA = smem + st * STAGE;
      double* sB = sA + SA::ELEMS;
      // A chunk
      if (a16) {
        for (int e = tid; e < CG_M * CG_K / 2; e += CG_THREADS) {
          int i, k, bytes;
          const double* src;
          if (TA) {  // pairs along k
            k = 2 * (e % (CG_K / 2));
            i = e / (CG_K / 2);
            const int gi = m0 + i, gk = k0 + k;
            bytes = (gi < M && gk < K) ? (gk + 1 < K ? 16 : 8) : 0;
            src = bytes ? A + gk + (long long)gi * lda : A;
          } else {  // pairs along i
            i = 2 * (e % (CG_M / 2));
            k = e / (CG_M / 2);
            const int gi = m0 + i, gk = k0 + k;
            bytes = (gi < M && gk < K) ? (gi + 1 < M ? 16 : 8) : 0;
            src = bytes ? A + gi + (long long)gk * lda : A;
          }
          cp_async16(sA + SA::at(i, k), src, bytes);
        }
      } else {
        for (int e = tid; e < CG_M * CG_K; e += CG_THREADS) {
          int i, k;
          if (TA) { k = e % CG_K; i = e / CG_K; } else { i = e % CG_M; k = e / CG_M; }
          const int gi = m0 + i, gk = k0 + k;
          const bool ok = gi < M && gk < K;
          cp_async8(sA + SA::at(i, k), ok ? (TA ? A + gk + (long long)gi * lda : A + gi + (long long)gk * lda) : A,
                    ok);
        }
      }
      // B chunk
      if (b16) {
        for (int e = tid; e < CG_K * CG_N / 2; e += CG_THREADS) {
          int j, k, bytes;
          const double* src;
          if (TB) {  // pairs along j
            j = 2 * (e % (CG_N / 2));
            k = e / (CG_N / 2);
            const int gj = n0 + j, gk = k0 + k;
            bytes = (gj < N && gk < K) ? (gj + 1 < N ? 16 : 8) : 0;
            src = bytes ? B + gj + (long long)gk * ldb : B;
          } else {  // pairs along k
            k = 2 * (e % (CG_K / 2));
            j = e / (CG_K / 2);
            const int gj = n0 + j, gk = k0 + k;
            bytes = (gj < N && gk < K) ? (gk + 1 < K ? 16 : 8) : 0;
            src = bytes ? B + gk + (long long)gj * ldb : B;
          }
          cp_async16(sB + SB::at(k, j), src, bytes);
        }
      } else {
        for (int e = tid; e < CG_K * CG_N; e += CG_THREADS) {
          int k, j;
          if (TB) { j = e % CG_N; k = e / CG_N; } else { k = e % CG_K; j = e / CG_K; }
          const int gj = n0 + j, gk = k0 + k;
          const bool ok = gj < N && gk < K;
          cp_async8(sB + SB::at(k, j), ok ? (TB ? B + gj + (long long)gk * ldb : B + gk + (long long)gj * ldb) : B,
                    ok);
        }
      }
      if (++lc == tile_nch(lt)) {
        lc = 0;
        lt = next_used(lt + 1);
      }
    }
    cp_async_commit();  // an empty group past the end keeps the counting uniform
  };

  __syncthreads();  // the previous user of the stages is done
#pragma unroll
  for (int s = 0; s < ST - 1; ++s) load_next(s);
  int gch = 0;  // chunks consumed so far
  for (int ct = next_used(0); ct < ntiles; ct = next_used(ct + 1)) {
    const int m0 = (ct % tm_n) * CG_M, n0 = (ct / tm_n) * CG_N;
    const int nch = tile_nch(ct);
    const bool wskip = !wact || (lower && (m0 + wm * WM + WM - 1 < n0 + wn * WN));
    // C of this tile into registers now; consumed after the k loop
    double cv[MI][NJ][4];
#pragma unroll
    for (int mi = 0; mi < MI; ++mi)
#pragma unroll
      for (int nj = 0; nj < NJ; ++nj)
#pragma unroll
        for (int r = 0; r < 4; ++r) {
          const int row = m0 + wm * WM + mi * 16 + g + ((r & 2) ? 8 : 0);
          const int col = n0 + wn * WN + nj * 8 + 2 * t4 + (r & 1);
          const bool ok = wact && beta != 0.0 && row < M && col < N && !(lower && row < col);
          cv[mi][nj][r] = ok ? C[row + (long long)col * ldc] : 0.0;
        }
    double acc[MI][NJ][4];
#pragma unroll
    for (int mi = 0; mi < MI; ++mi)
#pragma unroll
      for (int nj = 0; nj < NJ; ++nj)
#pragma unroll
        for (int r = 0; r < 4; ++r) acc[mi][nj][r] = 0.0;
    for (int c = 0; c < nch; ++c, ++gch) {
      cp_async_wait<ST - 2>();
      __syncthreads();
      load_next((gch + ST - 1) % ST);
      if (!wskip) {
        const double* sA = smem + (gch % ST) * STAGE;
        const double* sB = sA + SA::ELEMS;
#pragma unroll
        for (int kk = 0; kk < CG_K; kk += 4) {
          double a[MI][2], b[NJ];
#pragma unroll
          for (int mi = 0; mi < MI; ++mi) {
            a[mi][0] = sA[SA::at(wm * WM + mi * 16 + g, kk + t4)];
            a[mi][1] = sA[SA::at(wm * WM + mi * 16 + g + 8, kk + t4)];
          }
#pragma unroll
          for (int nj = 0; nj < NJ; ++nj) b[nj] = sB[SB::at(kk + t4, wn * WN + nj * 8 + g)];
#pragma unroll
          for (int mi = 0; mi < MI; ++mi)
#pragma unroll
            for (int nj = 0; nj < NJ; ++nj) dmma_16x8x4(acc[mi][nj], a[mi][0], a[mi][1], b[nj]);
        }
      }
    }
#pragma unroll
    for (int mi = 0; mi < MI; ++mi)
#pragma unroll
      for (int nj = 0; nj < NJ; ++nj)
#pragma unroll
        for (int r = 0; r < 4; ++r) {
          const int row = m0 + wm * WM + mi * 16 + g + ((r & 2) ? 8 : 0);
          const int col = n0 + wn * WN + nj * 8 + 2 * t4 + (r & 1);
          if (wact && row < M && col < N && !(lower && row < col)) {
            double v = alpha * acc[mi][nj][r];
            if (beta != 0.0) v = fma(beta, cv[mi][nj][r], v);
            C[row + (long long)col * ldc] = v;
          }
        }
  }
  cp_async_wait<0>();
  __syncthreads();
}

// cta_gemm_tile with the tile shape chosen at run time (cfg < CG_CONFIGS)
template <bool TA, bool TB>
__device__ __forceinline__ void cta_gemm(int cfg, int M, int N, int K, const double* A, long long lda, const double* B,
                                         long long ldb, double* C, long long ldc, double alpha, double beta, bool lower,
                                         int kmode, double* smem) {
  switch (cfg) {
    case 1: cta_gemm_tile<TA, TB, 1>(M, N, K, A, lda, B, ldb, C, ldc, alpha, beta, lower, kmode, smem); break;
    case 2: cta_gemm_tile<TA, TB, 2>(M, N, K, A, lda, B, ldb, C, ldc, alpha, beta, lower, kmode, smem); break;
    case 3: cta_gemm_tile<TA, TB, 3>(M, N, K, A, lda, B, ldb, C, ldc, alpha, beta, lower, kmode, smem); break;
    default: cta_gemm_tile<TA, TB, 0>(M, N, K, A, lda, B, ldb, C, ldc, alpha, beta, lower, kmode, smem); break;
  }
}

}  // namespace gprx
