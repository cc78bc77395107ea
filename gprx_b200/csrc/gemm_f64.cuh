// gemm_f64.cuh — FP64 tensor-core GEMM for sm_100a (DMMA, mma.sync f64).
//
// tcgen05 has no f64 kind, so the FP64 contractions of the blocked Cholesky,
// the triangular inverse / solves and the Sgpr products run on the FP64 MMA
// pipe through `mma.sync.aligned.m16n8k4.row.col.f64`.  Tiles are staged in
// shared memory by `cp.async` in a multi-stage ring; the padding of every
// shared tile (row stride ≡ 4 doubles mod 16) makes the fragment loads
// conflict-free.
//
//   C(i,j) = alpha · Σ_k opA(i,k) · opB(k,j) + beta · C(i,j)
//   opA(i,k) = TA ? A[k + i·lda] : A[i + k·lda]
//   opB(k,j) = TB ? B[j + k·ldb] : B[k + j·ldb]
//
// Modes: LOWER_TILES skips output tiles strictly above the diagonal and stores
// only i ≥ j (global row/col offsets row0/col0 decide "diagonal");
// K_FROM_ROW starts the k-loop at the tile's first global row (the lower-
// triangular X in Xᵀ X); SPLIT_K writes partial sums into C + z·split_stride.
#pragma once

#include "common.cuh"

namespace gprx {

enum GemmMode : int {
  GEMM_LOWER_TILES = 1,
  GEMM_K_FROM_ROW = 2,
  GEMM_SPLIT_K = 4,
  GEMM_K_TO_ROW = 8,   // k-loop stops at the tile's last global row + 1 (lower-triangular A)
  GEMM_K_FROM_COL = 16, // k-loop starts at the tile's first global column (lower-triangular B)
  GEMM_K_TO_COL = 32,   // k-loop stops at the tile's last global column + 1 (op(B)(k, j) = 0 for k > j)
};

struct GemmParams {
  int M, N, K;
  const double* A;
  long long lda;
  const double* B;
  long long ldb;
  double* C;
  long long ldc;
  double alpha, beta;
  int mode;
  long long row0, col0;     // global offsets of C(0,0) for the triangle tests
  long long krow0;          // global row of k = 0 (K_FROM_ROW / K_TO_ROW)
  int splits;               // SPLIT_K: number of k slices (grid.z)
  long long split_stride;   // SPLIT_K: distance between partial outputs
  const DevStatus* status;
  // batched: pointer strides per blockIdx.z when splits == 1 and batch > 1
  long long strideA, strideB, strideC;
  int max_ctas;             // > 0: at most this many CTAs, each looping over tiles
  int splits_tiles;         // set by the launcher: tile count when max_ctas > 0
};

__device__ __forceinline__ void cp_async8(void* smem, const void* gmem, bool pred) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  int n = pred ? 8 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(n));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

__device__ __forceinline__ void dmma_16x8x4(double (&c)[4], double a0, double a1, double b0) {
  asm volatile(
      "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};\n"
      : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
      : "d"(a0), "d"(a1), "d"(b0));
}

template <int BM, int BN, int BK, int WM, int WN, int STAGES, bool TA, bool TB>
struct GemmCfg {
  static constexpr int WARPS_M = BM / WM;
  static constexpr int WARPS_N = BN / WN;
  static constexpr int THREADS = WARPS_M * WARPS_N * 32;
  static constexpr int MT = WM / 16;  // m16 tiles per warp
  static constexpr int NT = WN / 8;   // n8 tiles per warp
  // shared layout of one stage
  static constexpr int SA_LD = TA ? (BK + 4) : (BM + 4);
  static constexpr int SA_ROWS = TA ? BM : BK;
  static constexpr int SB_LD = TB ? (BN + 4) : (BK + 4);
  static constexpr int SB_ROWS = TB ? BK : BN;
  static constexpr int SA_SIZE = SA_LD * SA_ROWS;
  static constexpr int SB_SIZE = SB_LD * SB_ROWS;
  static constexpr int STAGE = SA_SIZE + SB_SIZE;
  static constexpr size_t SMEM = (size_t)STAGE * STAGES * sizeof(double);
};

template <int BM, int BN, int BK, int WM, int WN, int STAGES, bool TA, bool TB>
__global__ void __launch_bounds__(GemmCfg<BM, BN, BK, WM, WN, STAGES, TA, TB>::THREADS)
    dgemm_kernel(GemmParams p) {
  using Cfg = GemmCfg<BM, BN, BK, WM, WN, STAGES, TA, TB>;
  extern __shared__ __align__(16) double smem[];
  if (dev_failed(p.status)) return;
  const int ntiles_total = p.max_ctas > 0 ? p.max_ctas : 0;  // set by the launcher when capped
  for (int tile_idx = blockIdx.x;; tile_idx += gridDim.x) {
  if (p.max_ctas > 0) {
    if (tile_idx >= p.splits_tiles) break;
    __syncthreads();  // the previous tile's shared-memory reads are done
  } else if (tile_idx != (int)blockIdx.x) {
    break;
  }
  (void)ntiles_total;

  // ---- which output tile ----
  int tile_m, tile_n;
  const int tiles_m = (p.M + BM - 1) / BM;
  if (p.mode & GEMM_LOWER_TILES) {
    // tile_idx enumerates (tm, tn) with the tile not strictly above the
    // diagonal; when row0 == col0 and BM == BN that is tn ≤ tm.
    int idx = tile_idx;
    // general enumeration: walk columns; tile (tm, tn) is kept when its last
    // global row ≥ its first global column.
    const int tiles_n = (p.N + BN - 1) / BN;
    tile_m = -1;
    tile_n = -1;
    for (int tn = 0; tn < tiles_n; ++tn) {
      long long c_first = p.col0 + (long long)tn * BN;
      // first tm with row_last >= c_first
      long long need = c_first - p.row0 - (BM - 1);
      int tm0 = need <= 0 ? 0 : (int)((need + BM - 1) / BM);
      int cnt = tiles_m - tm0;
      if (cnt < 0) cnt = 0;
      if (idx < cnt) { tile_m = tm0 + idx; tile_n = tn; break; }
      idx -= cnt;
    }
    if (tile_m < 0) return;
  } else {
    tile_m = tile_idx % tiles_m;
    tile_n = tile_idx / tiles_m;
  }
  const int m0 = tile_m * BM;
  const int n0 = tile_n * BN;

  const double* A = p.A;
  const double* B = p.B;
  double* C = p.C;
  int kbeg = 0, kend = p.K;
  if (p.mode & GEMM_SPLIT_K) {
    int z = blockIdx.z;
    int per = (p.K + p.splits - 1) / p.splits;
    per = (per + BK - 1) / BK * BK;
    kbeg = z * per;
    kend = min(p.K, kbeg + per);
    C = C + (long long)z * p.split_stride;
  } else if (gridDim.z > 1) {
    A += (long long)blockIdx.z * p.strideA;
    B += (long long)blockIdx.z * p.strideB;
    C += (long long)blockIdx.z * p.strideC;
  }
  if (p.mode & GEMM_K_FROM_ROW) {
    long long first_row = p.row0 + m0;  // global row of this tile
    long long kb = first_row - p.krow0;
    if (kb > kbeg) kbeg = (int)(kb / BK * BK);
  }
  if (p.mode & GEMM_K_FROM_COL) {
    long long first_col = p.col0 + n0;
    long long kb = first_col - p.krow0;
    if (kb > kbeg) kbeg = (int)(kb / BK * BK);
  }
  if (p.mode & GEMM_K_TO_ROW) {
    long long last_row = p.row0 + min(m0 + BM, p.M);  // exclusive
    long long ke = last_row - p.krow0;
    if (ke < kend) kend = (int)max(ke, 0LL);
  }
  if (p.mode & GEMM_K_TO_COL) {
    long long last_col = p.col0 + min(n0 + BN, p.N);  // exclusive
    long long ke = last_col - p.krow0;
    if (ke < kend) kend = (int)max(ke, 0LL);
  }

  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  const int wm = warp % Cfg::WARPS_M, wn = warp / Cfg::WARPS_M;
  const int g = lane >> 2, t4 = lane & 3;

  double acc[Cfg::MT][Cfg::NT][4];
#pragma unroll
  for (int i = 0; i < Cfg::MT; ++i)
#pragma unroll
    for (int j = 0; j < Cfg::NT; ++j)
#pragma unroll
      for (int r = 0; r < 4; ++r) acc[i][j][r] = 0.0;

  const int nk = kend > kbeg ? (kend - kbeg + BK - 1) / BK : 0;

  auto load_stage = [&](int stage, int kt) {
    double* sA = smem + stage * Cfg::STAGE;
    double* sB = sA + Cfg::SA_SIZE;
    const int k0 = kbeg + kt * BK;
    // A tile: BM x BK
    for (int e = tid; e < BM * BK; e += Cfg::THREADS) {
      int i, k;
      if (TA) { k = e % BK; i = e / BK; } else { i = e % BM; k = e / BM; }
      int gi = m0 + i, gk = k0 + k;
      bool ok = gi < p.M && gk < kend;
      const double* src = TA ? (A + (long long)(ok ? gi : 0) * p.lda + (ok ? gk : 0))
                             : (A + (ok ? gi : 0) + (long long)(ok ? gk : 0) * p.lda);
      double* dst = TA ? (sA + i * Cfg::SA_LD + k) : (sA + k * Cfg::SA_LD + i);
      cp_async8(dst, src, ok);
    }
    // B tile: BK x BN
    for (int e = tid; e < BK * BN; e += Cfg::THREADS) {
      int k, j;
      if (TB) { j = e % BN; k = e / BN; } else { k = e % BK; j = e / BK; }
      int gj = n0 + j, gk = k0 + k;
      bool ok = gj < p.N && gk < kend;
      const double* src = TB ? (B + (ok ? gj : 0) + (long long)(ok ? gk : 0) * p.ldb)
                             : (B + (ok ? gk : 0) + (long long)(ok ? gj : 0) * p.ldb);
      double* dst = TB ? (sB + k * Cfg::SB_LD + j) : (sB + j * Cfg::SB_LD + k);
      cp_async8(dst, src, ok);
    }
  };

  // prologue
#pragma unroll
  for (int s = 0; s < STAGES - 1; ++s) {
    if (s < nk) load_stage(s, s);
    cp_async_commit();
  }

  for (int kt = 0; kt < nk; ++kt) {
    cp_async_wait<STAGES - 2>();
    __syncthreads();
    {
      int nxt = kt + STAGES - 1;
      if (nxt < nk) load_stage(nxt % STAGES, nxt);
      cp_async_commit();
    }
    const double* sA = smem + (kt % STAGES) * Cfg::STAGE;
    const double* sB = sA + Cfg::SA_SIZE;
#pragma unroll
    for (int kk = 0; kk < BK; kk += 4) {
      double af[Cfg::MT][2];
      double bf[Cfg::NT];
#pragma unroll
      for (int i = 0; i < Cfg::MT; ++i) {
        int r0 = wm * WM + i * 16 + g;
        int kc = kk + t4;
        if (TA) {
          af[i][0] = sA[r0 * Cfg::SA_LD + kc];
          af[i][1] = sA[(r0 + 8) * Cfg::SA_LD + kc];
        } else {
          af[i][0] = sA[kc * Cfg::SA_LD + r0];
          af[i][1] = sA[kc * Cfg::SA_LD + r0 + 8];
        }
      }
#pragma unroll
      for (int j = 0; j < Cfg::NT; ++j) {
        int c0 = wn * WN + j * 8 + g;
        int kc = kk + t4;
        bf[j] = TB ? sB[kc * Cfg::SB_LD + c0] : sB[c0 * Cfg::SB_LD + kc];
      }
#pragma unroll
      for (int i = 0; i < Cfg::MT; ++i)
#pragma unroll
        for (int j = 0; j < Cfg::NT; ++j) dmma_16x8x4(acc[i][j], af[i][0], af[i][1], bf[j]);
    }
  }
  cp_async_wait<0>();

  // ---- epilogue ----
  // Per m16 row group, every C value is loaded before any store of the group
  // (a load after a store to a possibly aliasing address cannot be hoisted,
  // and each would pay the full memory latency).
  const bool lower = (p.mode & GEMM_LOWER_TILES) != 0;
  const bool split = (p.mode & GEMM_SPLIT_K) != 0;
  const bool use_beta = !split && p.beta != 0.0;
#pragma unroll
  for (int i = 0; i < Cfg::MT; ++i) {
    double cv[Cfg::NT][4];
    bool ok[Cfg::NT][4];
#pragma unroll
    for (int j = 0; j < Cfg::NT; ++j)
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        int row = m0 + wm * WM + i * 16 + g + ((r & 2) ? 8 : 0);
        int col = n0 + wn * WN + j * 8 + t4 * 2 + (r & 1);
        ok[j][r] = row < p.M && col < p.N && !(lower && p.row0 + row < p.col0 + col);
        cv[j][r] = (use_beta && ok[j][r]) ? C[row + (long long)col * p.ldc] : 0.0;
      }
#pragma unroll
    for (int j = 0; j < Cfg::NT; ++j)
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        if (!ok[j][r]) continue;
        int row = m0 + wm * WM + i * 16 + g + ((r & 2) ? 8 : 0);
        int col = n0 + wn * WN + j * 8 + t4 * 2 + (r & 1);
        double v = p.alpha * acc[i][j][r];
        if (use_beta) v = fma(p.beta, cv[j][r], v);
        C[row + (long long)col * p.ldc] = v;
      }
  }
  }  // tile loop
}

// Host-side launcher for one configuration.
template <int BM, int BN, int BK, int WM, int WN, int STAGES, bool TA, bool TB>
cudaError_t launch_dgemm(const GemmParams& p, int batch, cudaStream_t stream) {
  using Cfg = GemmCfg<BM, BN, BK, WM, WN, STAGES, TA, TB>;
  auto kern = dgemm_kernel<BM, BN, BK, WM, WN, STAGES, TA, TB>;
  static bool attr_set = false;
  if (!attr_set) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Cfg::SMEM);
    if (e != cudaSuccess) return e;
    attr_set = true;
  }
  if (p.M <= 0 || p.N <= 0) return cudaSuccess;
  int tiles_m = (p.M + BM - 1) / BM, tiles_n = (p.N + BN - 1) / BN;
  int nblocks;
  if (p.mode & GEMM_LOWER_TILES) {
    nblocks = 0;
    for (int tn = 0; tn < tiles_n; ++tn) {
      long long c_first = p.col0 + (long long)tn * BN;
      long long need = c_first - p.row0 - (BM - 1);
      int tm0 = need <= 0 ? 0 : (int)((need + BM - 1) / BM);
      if (tm0 < tiles_m) nblocks += tiles_m - tm0;
    }
    if (nblocks == 0) return cudaSuccess;
  } else {
    nblocks = tiles_m * tiles_n;
  }
  GemmParams q = p;
  q.splits_tiles = nblocks;
  if (p.max_ctas > 0 && nblocks > p.max_ctas) nblocks = p.max_ctas;
  dim3 grid(nblocks, 1, (p.mode & GEMM_SPLIT_K) ? p.splits : batch);
  kern<<<grid, Cfg::THREADS, Cfg::SMEM, stream>>>(q);
  count_launch();
  return cudaGetLastError();
}

}  // namespace gprx
