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
#include "emu_gemm.cuh"
#include "diag_block.cuh"

namespace gprx {

cudaError_t dgemm(bool ta, bool tb, const GemmParams& p, cudaStream_t s, int batch) {
  if (!ta && !tb) return launch_dgemm<128, 128, 16, 64, 32, 3, false, false>(p, batch, s);
  if (!ta && tb) return launch_dgemm<128, 128, 16, 64, 32, 3, false, true>(p, batch, s);
  if (ta && !tb) return launch_dgemm<128, 128, 16, 64, 32, 3, true, false>(p, batch, s);
  return launch_dgemm<128, 128, 16, 64, 32, 3, true, true>(p, batch, s);
}

cudaError_t dgemm_nn_fill(const GemmParams& p, cudaStream_t s, int batch) {
  const long long tiles128 = (long long)ceil_div(p.M, 128) * ceil_div(p.N, 128) * batch;
  if (tiles128 >= 2 * 148) return launch_dgemm<128, 128, 16, 64, 32, 3, false, false>(p, batch, s);
  return launch_dgemm<64, 64, 16, 32, 16, 3, false, false>(p, batch, s);
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

// Programmatic dependent launch on the factor's chain: a chain kernel first
// waits for its predecessor in the stream to complete (its writes visible),
// then lets its own dependent start launching, so the launch of the next
// chain kernel overlaps this one instead of following its completion.  Both
// instructions are no-ops for a kernel launched without the attribute.
__device__ __forceinline__ void chain_dependency_wait_and_release() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

__global__ void __launch_bounds__(FD_THREADS) potrf_diag_kernel(double* A, long long lda, long long k0, int nb,
                                                                 double* linv, DevStatus* st) {
  extern __shared__ __align__(16) double smem[];
  __shared__ int fail;
  chain_dependency_wait_and_release();
  if (dev_failed(st)) return;
  int f = diag_block_factor_inv(A, lda, k0, nb, linv, smem, &fail);
  if (f >= 0 && threadIdx.x == 0) dev_fail(st, GPRX_CHOLESKY_FAILED, k0 + f);
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
static size_t fast_diag_smem(int nb) { (void)nb; return diag_block_smem(); }

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
  if (aux2) cudaStreamDestroy(aux2);
}

cudaError_t FactorCtx::ensure(int nblk) {
  if (!aux) {
    int lo, hi;
    CK(cudaDeviceGetStreamPriorityRange(&lo, &hi));
    CK(cudaStreamCreateWithPriority(&aux, cudaStreamNonBlocking, hi));
  }
  if (!aux2) {
    int lo, hi;
    CK(cudaDeviceGetStreamPriorityRange(&lo, &hi));
    CK(cudaStreamCreateWithPriority(&aux2, cudaStreamNonBlocking, hi));
  }
  while ((int)ev.size() < 3 * nblk + 2) {
    cudaEvent_t e;
    CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    ev.push_back(e);
  }
  return cudaSuccess;
}

// ---------------------------------------------------------------------------
// the chain's panel products: K ≤ NB, N ≤ NB
// ---------------------------------------------------------------------------
// C(M×N) = alpha · A(M×K) · B(N×K)ᵀ + beta · C with A(i,k) = A[i + k·lda],
// B(j,k) = B[j + k·ldb], C column-major; lower: only i ≥ j is written.  One
// CTA of 256 threads per PG_TM-row strip stages the strip of A and all of B
// in shared memory in one go (K is one panel: no k pipeline, one memory
// latency instead of one per k chunk), prefetches its C values meanwhile,
// then runs the DMMA k steps.  A strip is read whole before it is written,
// so C may be A's rows when beta = 0 (the in-place panel solve).
constexpr int PG_TM = 32;
constexpr int PG_LDA = PG_TM + 4;  // ≡ 4 mod 16 doubles: conflict-free fragments
constexpr int PG_LDB = NB + 4;
inline size_t panel_gemm_smem() { return (size_t)(NB * PG_LDA + NB * PG_LDB) * sizeof(double); }

struct PanelGemmArgs {
  int M, N, K;
  const double* A;
  long long lda;
  const double* B;
  long long ldb;
  double* C;
  long long ldc;
  double alpha, beta;
  int lower;
  const DevStatus* st;
};

__global__ void __launch_bounds__(256) panel_gemm_kernel(PanelGemmArgs g) {
  extern __shared__ __align__(16) double smem[];
  chain_dependency_wait_and_release();
  if (dev_failed(g.st)) return;
  double* sA = smem;                 // [k][i], ld PG_LDA
  double* sB = smem + NB * PG_LDA;   // [k][j], ld PG_LDB
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, gq = lane >> 2, t4 = lane & 3;
  const int m0 = blockIdx.x * PG_TM;
  const int KP = (g.K + 3) & ~3;
  const bool a16 = ((g.lda & 1) == 0) && ((reinterpret_cast<unsigned long long>(g.A) & 15) == 0);
  const bool b16 = ((g.ldb & 1) == 0) && ((reinterpret_cast<unsigned long long>(g.B) & 15) == 0);
  // A strip: PG_TM × KP (zero past M and K)
  if (a16) {
    for (int e = tid; e < (PG_TM / 2) * KP; e += 256) {
      const int i = 2 * (e % (PG_TM / 2)), k = e / (PG_TM / 2), gi = m0 + i;
      const int bytes = (gi < g.M && k < g.K) ? (gi + 1 < g.M ? 16 : 8) : 0;
      const unsigned d = (unsigned)__cvta_generic_to_shared(sA + k * PG_LDA + i);
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d),
                   "l"(bytes ? g.A + gi + (long long)k * g.lda : g.A), "r"(bytes));
    }
  } else {
    for (int e = tid; e < PG_TM * KP; e += 256) {
      const int i = e % PG_TM, k = e / PG_TM, gi = m0 + i;
      const bool ok = gi < g.M && k < g.K;
      cp_async8(sA + k * PG_LDA + i, ok ? g.A + gi + (long long)k * g.lda : g.A, ok);
    }
  }
  // B: NB × KP (zero past N and K)
  if (b16) {
    for (int e = tid; e < (NB / 2) * KP; e += 256) {
      const int j = 2 * (e % (NB / 2)), k = e / (NB / 2);
      const int bytes = (j < g.N && k < g.K) ? (j + 1 < g.N ? 16 : 8) : 0;
      const unsigned d = (unsigned)__cvta_generic_to_shared(sB + k * PG_LDB + j);
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d),
                   "l"(bytes ? g.B + j + (long long)k * g.ldb : g.B), "r"(bytes));
    }
  } else {
    for (int e = tid; e < NB * KP; e += 256) {
      const int j = e % NB, k = e / NB;
      const bool ok = j < g.N && k < g.K;
      cp_async8(sB + k * PG_LDB + j, ok ? g.B + j + (long long)k * g.ldb : g.B, ok);
    }
  }
  cp_async_commit();
  // warps in a 2 × 4 grid of 16 × 32 blocks (MI = 1, NJ = 4)
  const int wm = warp & 1, wn = warp >> 1;
  const int rb = wm * 16, cb = wn * 32;
  const bool wskip = (cb >= g.N) || (g.lower && m0 + rb + 15 < cb);
  double cv[4][4];
#pragma unroll
  for (int nj = 0; nj < 4; ++nj)
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const int row = m0 + rb + gq + ((r & 2) ? 8 : 0), col = cb + nj * 8 + 2 * t4 + (r & 1);
      const bool ok = !wskip && g.beta != 0.0 && row < g.M && col < g.N && !(g.lower && row < col);
      cv[nj][r] = ok ? g.C[row + (long long)col * g.ldc] : 0.0;
    }
  cp_async_wait<0>();
  __syncthreads();
  if (wskip) return;
  double acc[4][4];
#pragma unroll
  for (int nj = 0; nj < 4; ++nj)
#pragma unroll
    for (int r = 0; r < 4; ++r) acc[nj][r] = 0.0;
#pragma unroll 4
  for (int kk = 0; kk < KP; kk += 4) {
    const double a0 = sA[(kk + t4) * PG_LDA + rb + gq];
    const double a1 = sA[(kk + t4) * PG_LDA + rb + gq + 8];
    double b[4];
#pragma unroll
    for (int nj = 0; nj < 4; ++nj) b[nj] = sB[(kk + t4) * PG_LDB + cb + nj * 8 + gq];
#pragma unroll
    for (int nj = 0; nj < 4; ++nj) dmma_16x8x4(acc[nj], a0, a1, b[nj]);
  }
#pragma unroll
  for (int nj = 0; nj < 4; ++nj)
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const int row = m0 + rb + gq + ((r & 2) ? 8 : 0), col = cb + nj * 8 + 2 * t4 + (r & 1);
      if (row < g.M && col < g.N && !(g.lower && row < col)) {
        double v = g.alpha * acc[nj][r];
        if (g.beta != 0.0) v = fma(g.beta, cv[nj][r], v);
        g.C[row + (long long)col * g.ldc] = v;
      }
    }
}

// launch with programmatic stream serialization (the kernel waits for its
// predecessor itself: chain_dependency_wait_and_release)
template <typename... Params, typename... Args>
static cudaError_t launch_chain(void (*kernel)(Params...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                                Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  count_launch();
  return cudaLaunchKernelEx(&cfg, kernel, args...);
}

static cudaError_t panel_gemm(int M, int N, int K, const double* A, long long lda, const double* B, long long ldb,
                              double* C, long long ldc, double alpha, double beta, bool lower, const DevStatus* st,
                              cudaStream_t s, bool chained = false) {
  static bool attr = false;
  if (!attr) {
    CK(cudaFuncSetAttribute(panel_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)panel_gemm_smem()));
    attr = true;
  }
  if (M <= 0 || N <= 0) return cudaSuccess;
  if (N > NB || K > NB || K < 0) return cudaErrorInvalidValue;
  PanelGemmArgs g{M, N, K, A, lda, B, ldb, C, ldc, alpha, beta, lower ? 1 : 0, st};
  if (chained) return launch_chain(panel_gemm_kernel, dim3(ceil_div(M, PG_TM)), dim3(256), panel_gemm_smem(), s, g);
  GPRX_LAUNCH(panel_gemm_kernel, ceil_div(M, PG_TM), 256, panel_gemm_smem(), s, g);
  return cudaGetLastError();
}

// rows below the diagonal block up to which the chain uses dependent launch
// (at larger trailing blocks the bulk update fills the GPU, and panel CTAs
// launched early would sit waiting on SMs it could use)
constexpr int CHAIN_PDL_ROWS = 4096;

// The diagonal block at k0 and the panel below it.  before_panel: an event
// the panel waits for (the rest of the column update on another stream).
static cudaError_t diag_and_panel(double* A, long long ld, int n, int k0, double* linv, DevStatus* st,
                                  cudaStream_t s, cudaEvent_t before_panel = nullptr) {
  int nbk = min(NB, n - k0);
  double* lk = linv + (long long)(k0 / NB) * NB * NB;
  int rest = n - k0 - nbk;
  const bool chained = rest <= CHAIN_PDL_ROWS;
  if (chained) {
    CK(launch_chain(potrf_diag_kernel, dim3(1), dim3(FD_THREADS), fast_diag_smem(nbk), s, A, ld, (long long)k0, nbk,
                    lk, st));
  } else {
    GPRX_LAUNCH(potrf_diag_kernel, 1, FD_THREADS, fast_diag_smem(nbk), s, A, ld, (long long)k0, nbk, lk, st);
  }
  if (rest > 0) {
    double* P = A + (k0 + nbk) + (long long)k0 * ld;
    // panel: P := P · L_kk⁻ᵀ, i.e. P(i,j) = Σ_k P(i,k) L_kk⁻¹(j,k) (in place:
    // a strip is staged whole before it is written); after an event wait the
    // launch is a plain one
    if (before_panel) CK(cudaStreamWaitEvent(s, before_panel, 0));
    CK(panel_gemm(rest, nbk, nbk, P, ld, lk, NB, P, ld, 1.0, 0.0, false, st, s, chained && !before_panel));
  }
  return cudaGetLastError();
}

// The bulk trailing update of the look-ahead factor (K = NB) runs on 64×128
// tiles: half the registers of the 128×128 tile, so two CTAs share an SM and
// one's copies and epilogue overlap the other's DMMA work, and CTAs short
// enough that the chain's high-priority kernels get SMs as they retire (no
// SM is held back).  Measured (FP64 factor probe, n = 4096 / 8192): 2.42 /
// 10.35 ms, against 2.55 / 11.67 ms with 128×128 tiles capped at 132 CTAs
// while the trailing block has at most 4096 rows, 3.14 / 11.34 ms with the
// 64×128 tiles capped at 132 CTAs and 2.53 / 10.40 ms capped at 264.

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
  cudaEvent_t* Ec = ctx->ev.data() + 2 * nblk + 2;  // column update's lower rows of step k done (on aux2)
  cudaEvent_t Ein = ctx->ev[2 * nblk];
  cudaStream_t X2 = ctx->aux2;
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
    // critical chain of block k+1 (side stream): column block k+1 −= panel
    // k · (its top rows)ᵀ — the diagonal block's rows on the chain, the rows
    // below on aux2 while the diagonal block is factored; the panel solve
    // waits for both
    if (k >= 1) CK(cudaStreamWaitEvent(X, Es[k - 1], 0));
    const int m = n - c1, w = min(NB, n - c1);
    cudaEvent_t lower_done = nullptr;
    if (m > NB) {
      if (k >= 1) CK(cudaStreamWaitEvent(X2, Es[k - 1], 0));
      CK(cudaStreamWaitEvent(X2, Ep[k], 0));
      CK(panel_gemm(m - NB, w, NB, Pk + NB, ld, Pk, ld, A + (c1 + NB) + (long long)c1 * ld, ld, -1.0, 1.0, false, st,
                    X2));
      CK(cudaEventRecord(Ec[k], X2));
      lower_done = Ec[k];
    }
    CK(panel_gemm(min(m, NB), w, NB, Pk, ld, Pk, ld, A + c1 + (long long)c1 * ld, ld, -1.0, 1.0, true, st, X));
    CK(diag_and_panel(A, ld, n, c1, linv, st, X, lower_done));
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
      CK((launch_dgemm<64, 128, 16, 32, 32, 3, false, true>(ps, 1, s)));
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
      CK(dgemm_nn_fill(p1, s, (int)cnt));
      // X21 = −X22 · T   (h2 × h, K = h2; X22 lower → k up to the row)
      GemmParams p2 = gemm_params((int)h2, (int)h, (int)h2, X + (s0 + h) + (s0 + h) * ldx, ldx, scratch, h2,
                                  X + (s0 + h) + s0 * ldx, ldx, -1.0, 0.0, st);
      p2.mode = GEMM_K_TO_ROW;
      p2.strideA = b + b * ldx;
      p2.strideB = h2 * h;
      p2.strideC = b + b * ldx;
      CK(dgemm_nn_fill(p2, s, (int)cnt));
    }
  }
  return cudaGetLastError();
}

cudaError_t trtri_blocked_emu(const double* L, long long ld, int n, const double* linv, double* X, long long ldx,
                              double* scratch, const EmuWork& w, int emu_min, DevStatus* st, cudaStream_t s) {
  int nblk = ceil_div(n, NB);
  GPRX_LAUNCH(copy_diag_blocks_kernel, nblk, 256, 0, s, linv, n, X, ldx);
  for (long long b = 2LL * NB; b < 2LL * n; b *= 2) {
    long long h = b / 2;
    if (h >= n) break;
    long long full = n / b;
    long long r = n - full * b;
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
      if (h < emu_min) {
        GemmParams p1 = gemm_params((int)h2, (int)h, (int)h, L + (s0 + h) + s0 * ld, ld, X + s0 + s0 * ldx, ldx,
                                    scratch, h2, 1.0, 0.0, st);
        p1.mode = GEMM_K_FROM_COL;
        p1.strideA = b + b * ld;
        p1.strideB = b + b * ldx;
        p1.strideC = h2 * h;
        CK(dgemm_nn_fill(p1, s, (int)cnt));
        GemmParams p2 = gemm_params((int)h2, (int)h, (int)h2, X + (s0 + h) + (s0 + h) * ldx, ldx, scratch, h2,
                                    X + (s0 + h) + s0 * ldx, ldx, -1.0, 0.0, st);
        p2.mode = GEMM_K_TO_ROW;
        p2.strideA = b + b * ldx;
        p2.strideB = h2 * h;
        p2.strideC = b + b * ldx;
        CK(dgemm_nn_fill(p2, s, (int)cnt));
        continue;
      }
      for (long long c = 0; c < cnt; ++c) {
        const long long o = s0 + c * b;
        // T = L21 · X11 (rows of L21 against the columns of X11; X11 lower:
        // k from the tile's first column)
        EmuOperand a = w.op_a((int)h2, (int)h), bo = w.op_b((int)h, (int)h);
        CK(emu_slice(L + (o + h) + o * ld, ld, false, a, s));
        CK(emu_slice(X + o + o * ldx, ldx, true, bo, s));
        CK(emu_gemm(a, bo, scratch, h2, 1.0, 0.0, false, 0, 0, 2, w.err, s));
        // X21 = −X22 · T (X22 lower: k up to the tile's last row)
        EmuOperand a2 = w.op_a((int)h2, (int)h2), b2 = w.op_b((int)h, (int)h2);
        CK(emu_slice(X + (o + h) + (o + h) * ldx, ldx, false, a2, s));
        CK(emu_slice(scratch, h2, true, b2, s));
        CK(emu_gemm(a2, b2, X + (o + h) + o * ldx, ldx, -1.0, 0.0, false, 0, 0, 3, w.err, s));
      }
    }
  }
  return cudaGetLastError();
}

cudaError_t potrf_trtri_rec(double* A, long long ld, int n, double* X, long long ldx, double* linv,
                            double* scratch, const EmuWork& w, int leaf, int emu_min, DevStatus* st,
                            cudaStream_t s, FactorCtx* ctx) {
  if (n <= leaf) {
    CK(potrf_blocked(A, ld, n, linv, st, s, ctx));
    return trtri_blocked_emu(A, ld, n, linv, X, ldx, scratch, w, emu_min, st, s);
  }
  const int n1 = (n / 2 + NB - 1) / NB * NB, n2 = n - n1;
  CK(potrf_trtri_rec(A, ld, n1, X, ldx, linv, scratch, w, leaf, emu_min, st, s, ctx));
  double* A21 = A + n1;
  double* A22 = A + n1 + (long long)n1 * ld;
  // L21 = A21 X11ᵀ (rows of A21 against the rows of X11, k ≤ j), written over A21
  {
    EmuOperand a = w.op_a(n2, n1), b = w.op_b(n1, n1);
    CK(emu_slice(A21, ld, false, a, s));
    CK(emu_slice(X, ldx, false, b, s));
    CK(emu_gemm(a, b, A21, ld, 1.0, 0.0, false, 0, 0, 4, w.err, s));
  }
  // A22 −= L21 L21ᵀ (lower)
  {
    EmuOperand l = w.op_a(n2, n1);
    CK(emu_slice(A21, ld, false, l, s));
    CK(emu_gemm(l, l, A22, ld, -1.0, 1.0, true, 0, 0, 0, w.err, s));
  }
  CK(potrf_trtri_rec(A22, ld, n2, X + n1 + (long long)n1 * ldx, ldx, linv + (long long)(n1 / NB) * NB * NB, scratch,
                     w, leaf, emu_min, st, s, ctx));
  // T = L21 X11 (X11 lower: k from the tile's first column), X21 = −X22 T
  // (X22 lower: k up to the tile's last row)
  {
    EmuOperand a = w.op_a(n2, n1), b = w.op_b(n1, n1);
    CK(emu_slice(A21, ld, false, a, s));
    CK(emu_slice(X, ldx, true, b, s));
    CK(emu_gemm(a, b, scratch, n2, 1.0, 0.0, false, 0, 0, 2, w.err, s));
    EmuOperand a2 = w.op_a(n2, n2), b2 = w.op_b(n1, n2);
    CK(emu_slice(X + n1 + (long long)n1 * ldx, ldx, false, a2, s));
    CK(emu_slice(scratch, n2, true, b2, s));
    CK(emu_gemm(a2, b2, X + n1, ldx, -1.0, 0.0, false, 0, 0, 3, w.err, s));
  }
  return cudaGetLastError();
}

cudaError_t lauum_lower_emu(const double* X, long long ldx, int n, double* C, long long ldc, const EmuWork& w,
                            DevStatus* st, cudaStream_t s) {
  (void)st;
  // C(i, j) = Σ_k X(k,i) X(k,j): both operands are the rows of Xᵀ; lower,
  // k from the tile's first row
  EmuOperand a = w.op_a(n, n);
  CK(emu_slice(X, ldx, true, a, s));
  return emu_gemm(a, a, C, ldc, 1.0, 0.0, true, 0, 0, 1, w.err, s);
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

// split point of a recursive solve: half of n rounded up to whole NB blocks
// (the diagonal-block inverses are indexed by row / NB)
static int rec_split(int n) { return ceil_div(ceil_div(n, 2), NB) * NB; }

cudaError_t trsm_lower_rec(const double* L, long long ld, int n, const double* linv, double* B, long long ldb, int q,
                           int leaf, DevStatus* st, cudaStream_t s) {
  const int n1 = rec_split(n);
  if (n <= leaf || n1 >= n) return trsm_lower(L, ld, n, linv, B, ldb, q, st, s);
  const int n2 = n - n1;
  CK(trsm_lower_rec(L, ld, n1, linv, B, ldb, q, leaf, st, s));
  GemmParams p = gemm_params(n2, q, n1, L + n1, ld, B, ldb, B + n1, ldb, -1.0, 1.0, st);
  CK(dgemm(false, false, p, s));
  return trsm_lower_rec(L + n1 + (long long)n1 * ld, ld, n2, linv + (long long)(n1 / NB) * NB * NB, B + n1, ldb, q,
                        leaf, st, s);
}

cudaError_t trsm_lower_t_rec(const double* L, long long ld, int n, const double* linv, double* B, long long ldb,
                             int q, int leaf, DevStatus* st, cudaStream_t s) {
  const int n1 = rec_split(n);
  if (n <= leaf || n1 >= n) return trsm_lower_t(L, ld, n, linv, B, ldb, q, st, s);
  const int n2 = n - n1;
  CK(trsm_lower_t_rec(L + n1 + (long long)n1 * ld, ld, n2, linv + (long long)(n1 / NB) * NB * NB, B + n1, ldb, q,
                      leaf, st, s));
  GemmParams p = gemm_params(n1, q, n2, L + n1, ld, B + n1, ldb, B, ldb, -1.0, 1.0, st);
  CK(dgemm(true, false, p, s));
  return trsm_lower_t_rec(L, ld, n1, linv, B, ldb, q, leaf, st, s);
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
__global__ void __launch_bounds__(1024) trmv_lower_kernel(const double* X, long long ld, int n, const double* y,
                                                            double* z, const DevStatus* st) {
  constexpr int CG = 32;  // column groups: 32 rows × 32 groups, four loads in flight per thread
  __shared__ double part[CG][TRMV_ROWS + 1];
  if (dev_failed(st)) return;
  const int r = threadIdx.x % TRMV_ROWS, cg = threadIdx.x / TRMV_ROWS;
  const int i = blockIdx.x * TRMV_ROWS + r;
  const int jmax = min(n, (blockIdx.x + 1) * TRMV_ROWS);
  double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
  if (i < n) {
    int j = cg;
    for (; j + 3 * CG < jmax; j += 4 * CG) {
      const double x0 = j <= i ? X[i + (long long)j * ld] : 0.0;
      const double x1 = j + CG <= i ? X[i + (long long)(j + CG) * ld] : 0.0;
      const double x2 = j + 2 * CG <= i ? X[i + (long long)(j + 2 * CG) * ld] : 0.0;
      const double x3 = j + 3 * CG <= i ? X[i + (long long)(j + 3 * CG) * ld] : 0.0;
      a0 = fma(x0, y[j], a0);
      a1 = fma(x1, y[j + CG], a1);
      a2 = fma(x2, y[j + 2 * CG], a2);
      a3 = fma(x3, y[j + 3 * CG], a3);
    }
    for (; j < jmax; j += CG)
      if (j <= i) a0 = fma(X[i + (long long)j * ld], y[j], a0);
  }
  part[cg][r] = (a0 + a1) + (a2 + a3);
  __syncthreads();
  if (cg == 0 && i < n) {
    double s = 0.0;
#pragma unroll
    for (int c = 0; c < CG; ++c) s += part[c][r];
    z[i] = s;
  }
}

cudaError_t trmv_lower(const double* X, long long ld, int n, const double* y, double* z, DevStatus* st,
                       cudaStream_t s) {
  GPRX_LAUNCH(trmv_lower_kernel, ceil_div(n, TRMV_ROWS), TRMV_ROWS * 32, 0, s, X, ld, n, y, z, st);
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
