// emu_gemm.cu — see emu_gemm.cuh.
//
// Slice planes are stored pre-tiled: for plane p, 128-row tile rt and
// 64-byte K chunk kc, one 8 KB block at ((p·ntr + rt)·nkc + kc)·8 KB holds the
// chunk in the K-major, no-swizzle UMMA layout (8-row × 16-byte core
// matrices; the four K-adjacent core matrices of a row group 128 B apart, row
// groups 512 B apart), so a pipeline stage is filled by 2S bulk copies
// (cp.async.bulk, completion counted on the stage's "full" mbarrier).
//
// Kernel shape: one CTA of 128 threads per 128×64 output tile.  One thread
// issues the bulk copies and another the MMAs (tcgen05.mma.cta_group::1.kind::i8,
// M = 128, K = 32): slice p of A against the stacked B slices q = 0..S-1-p,
// so term p+q lands in TMEM columns 64(p+q) and one MMA of N = 64(S − p)
// (split at 256) covers every term of slice p; tcgen05.commit to the stage's
// "empty" mbarrier frees it for the next copy.
// The epilogue (all four warps, TMEM lane = output row) loads the S terms,
// combines them in FP64 and writes beta·C + alpha·2^-(e_i+e_j)·Σ_t 2^-7t C_t.
// Every wait on an mbarrier is bounded by a clock limit; a wait that runs
// out sets the error flag and the kernel still frees its TMEM and returns.

#include <cmath>

#include "emu_gemm.cuh"
#include "gemm_f64.cuh"

namespace gprx {

// ---------------------------------------------------------------------------
// slicing
// ---------------------------------------------------------------------------
// Row maxima of |op(r,k)| over 32 × 64 tiles (atomicMax on the bit pattern:
// non-negative doubles order like their bits).
__global__ void __launch_bounds__(256) emu_rowmax_kernel(const double* M, long long ld, bool trans, int R, int K,
                                                         unsigned long long* rmax) {
  __shared__ double t[32][65];
  const int r0 = blockIdx.x * 32, k0 = blockIdx.y * 64, tid = threadIdx.x;
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    int r, k;
    if (!trans) {
      r = tid & 31;
      k = (tid >> 5) + 8 * i;
    } else {
      k = tid & 63;
      r = (tid >> 6) + 4 * i;
    }
    const int gr = r0 + r, gk = k0 + k;
    double a = 0.0;
    if (gr < R && gk < K) a = fabs(trans ? M[gk + (long long)gr * ld] : M[gr + (long long)gk * ld]);
    t[r][k] = a;
  }
  __syncthreads();
  if (tid < 32) {
    double m = 0.0;
    for (int k = 0; k < 64; ++k) m = fmax(m, t[tid][k]);
    if (r0 + tid < R && m > 0.0) atomicMax(rmax + r0 + tid, (unsigned long long)__double_as_longlong(m));
  }
}

// One block per 32 rows × 64 columns of K: the tile is staged in shared
// memory (coalesced reads in either storage order), then each thread writes
// 8 digits of one row for every slice plane into the pre-tiled layout.
template <int S>
__global__ void __launch_bounds__(256) emu_slice_kernel(const double* M, long long ld, bool trans, int R, int K,
                                                        int Rpad, int Kpad, const unsigned long long* rmax,
                                                        int* exps, int8_t* out) {
  __shared__ double t[32][65];
  const int r0 = blockIdx.x * 32, kc = blockIdx.y, k0 = kc * 64, tid = threadIdx.x;
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    int r, k;
    if (!trans) {
      r = tid & 31;
      k = (tid >> 5) + 8 * i;
    } else {
      k = tid & 63;
      r = (tid >> 6) + 4 * i;
    }
    const int gr = r0 + r, gk = k0 + k;
    double a = 0.0;
    if (gr < R && gk < K) a = trans ? M[gk + (long long)gr * ld] : M[gr + (long long)gk * ld];
    t[r][k] = a;
  }
  __syncthreads();
  const int r = tid >> 3, c8 = tid & 7, gr = r0 + r;
  if (gr >= Rpad) return;
  // exponent e = 6 − E with max_k |op(r,k)| = m·2^E, m ∈ [0.5, 1): the scaled
  // row maximum lies in [32, 64)
  const double mx = __longlong_as_double((long long)rmax[gr]);
  int E = 0;
  frexp(mx, &E);
  const int e = mx > 0.0 ? 6 - E : 0;
  if (blockIdx.y == 0 && c8 == 0) exps[gr] = e;
  uint32_t w[S][2];
#pragma unroll
  for (int p = 0; p < S; ++p) w[p][0] = w[p][1] = 0u;
#pragma unroll
  for (int u = 0; u < 8; ++u) {
    double a = ldexp(t[r][c8 * 8 + u], e);
#pragma unroll
    for (int p = 0; p < S; ++p) {
      const double d = rint(a);
      w[p][u >> 2] |= ((uint32_t)(uint8_t)(int8_t)(int)d) << (8 * (u & 3));
      a = (a - d) * 128.0;
    }
  }
  const int ntr = Rpad / EMU_M, nkc = Kpad / EMU_KC, rt = gr / EMU_M, rr = gr % EMU_M;
  const size_t within = (size_t)(rr >> 3) * 512 + (c8 >> 1) * 128 + (rr & 7) * 16 + (c8 & 1) * 8;
#pragma unroll
  for (int p = 0; p < S; ++p) {
    const size_t blk = ((size_t)p * ntr + rt) * nkc + kc;
    *reinterpret_cast<uint2*>(out + blk * 8192 + within) = make_uint2(w[p][0], w[p][1]);
  }
}

cudaError_t emu_slice(const double* M, long long ld, bool trans, const EmuOperand& op, cudaStream_t s) {
  if (op.S < 4 || op.S > EMU_MAX_S || op.Rpad % EMU_M || op.Kpad % EMU_KC || !op.rmax) return cudaErrorInvalidValue;
  cudaError_t e = cudaMemsetAsync(op.rmax, 0, sizeof(unsigned long long) * op.Rpad, s);
  if (e != cudaSuccess) return e;
  const dim3 grid(op.Rpad / 32, op.Kpad / 64);
  GPRX_LAUNCH(emu_rowmax_kernel, grid, 256, 0, s, M, ld, trans, op.R, op.K, op.rmax);
  switch (op.S) {
    case 4: GPRX_LAUNCH(emu_slice_kernel<4>, grid, 256, 0, s, M, ld, trans, op.R, op.K, op.Rpad, op.Kpad, op.rmax, op.exps, op.slices); break;
    case 5: GPRX_LAUNCH(emu_slice_kernel<5>, grid, 256, 0, s, M, ld, trans, op.R, op.K, op.Rpad, op.Kpad, op.rmax, op.exps, op.slices); break;
    case 6: GPRX_LAUNCH(emu_slice_kernel<6>, grid, 256, 0, s, M, ld, trans, op.R, op.K, op.Rpad, op.Kpad, op.rmax, op.exps, op.slices); break;
    case 7: GPRX_LAUNCH(emu_slice_kernel<7>, grid, 256, 0, s, M, ld, trans, op.R, op.K, op.Rpad, op.Kpad, op.rmax, op.exps, op.slices); break;
    default: GPRX_LAUNCH(emu_slice_kernel<8>, grid, 256, 0, s, M, ld, trans, op.R, op.K, op.Rpad, op.Kpad, op.rmax, op.exps, op.slices); break;
  }
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// tcgen05 helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

// K-major, no swizzle: LBO = 128 B between K-adjacent core matrices, SBO =
// 512 B between 8-row groups, version 1 (sm100).
__device__ __forceinline__ uint64_t emu_desc(uint32_t addr) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)(128u >> 4) << 16) | ((uint64_t)(512u >> 4) << 32) |
         (1ull << 46);
}

__device__ __forceinline__ void umma_i8(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

// Waits for the phase of `parity` with a clock limit (about two seconds).
__device__ bool emu_wait(uint64_t* bar, uint32_t parity, int* err) {
  const uint32_t a = smem_u32(bar);
  const long long t0 = clock64();
  for (;;) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, P1;\n\t}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
    if (clock64() - t0 > 4000000000LL) {
      if (err) atomicExch(err, 1);
      return false;
    }
  }
}

__device__ __forceinline__ void tmem_ld16(uint32_t addr, uint32_t (&v)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];\n"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]),
        "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
      : "r"(addr));
}

// ---------------------------------------------------------------------------
// GEMM
// ---------------------------------------------------------------------------
struct EmuGemmArgs {
  const int8_t* A;
  const int8_t* B;
  const int* expA;
  const int* expB;
  int ntrA, ntrB;  // 128-row tiles per plane
  int M, N, Kpad;
  double* C;
  long long ldc;
  double alpha, beta;
  int lower;
  long long row0, col0;
  int kmode;
  int* err;
  int kz;              // > 0: blockIdx.z takes K chunks [z·kz, (z+1)·kz) into C + z·zstride
  long long zstride;
  int nsm;             // SMs of the device (one resident CTA each): the size of a wave
};

template <int S>
constexpr int emu_stages() {
  return S <= 6 ? 3 : 2;
}
template <int S>
constexpr int emu_stage_bytes() {
  return S * (EMU_M + EMU_N) * EMU_KC;
}

template <int S>
__global__ void __launch_bounds__(EMU_THREADS, 1) emu_gemm_kernel(EmuGemmArgs g) {
  constexpr int STAGES = emu_stages<S>();
  constexpr int A_SL = EMU_M * EMU_KC, B_SL = EMU_N * EMU_KC;
  constexpr int STAGE = emu_stage_bytes<S>();
  extern __shared__ __align__(1024) uint8_t emu_smem[];
  uint8_t* smem = emu_smem;
  __shared__ __align__(8) uint64_t full[STAGES], empty[STAGES];
  __shared__ uint32_t tmem_sh;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  // bands of 8 row tiles: the CTAs launched together share their A rows and
  // sweep the column tiles, so a band's A slices stay in L2 while B streams
  // (a bijection of the grid onto the tiles)
  constexpr int BAND = 8;
  const long long lid = blockIdx.x + (long long)blockIdx.y * gridDim.x;
  const long long band = lid / ((long long)BAND * gridDim.y), within = lid % ((long long)BAND * gridDim.y);
  const int rows_in_band = (int)min((long long)BAND, (long long)gridDim.x - band * BAND);
  const int bx = (int)(band * BAND + within % rows_in_band), by = (int)(within / rows_in_band);
  const long long i0 = (long long)bx * EMU_M, j0 = (long long)by * EMU_N;
  if (g.lower && i0 + g.row0 + EMU_M - 1 < j0 + g.col0) return;  // wholly above the diagonal
  const int nkc = g.Kpad / EMU_KC;
  int kc0 = 0, kc1 = nkc;
  if (g.kmode == 1) kc0 = (int)(i0 / EMU_KC);
  else if (g.kmode == 2) kc0 = (int)(j0 / EMU_KC);
  else if (g.kmode == 3) kc1 = (int)min((long long)nkc, (i0 + EMU_M + EMU_KC - 1) / EMU_KC);
  else if (g.kmode == 4) kc1 = (int)min((long long)nkc, (j0 + EMU_N + EMU_KC - 1) / EMU_KC);
  if (g.kz > 0) {
    kc0 = (int)blockIdx.z * g.kz;
    kc1 = min(nkc, kc0 + g.kz);
  }
  const int nch = kc0 < kc1 ? kc1 - kc0 : 0;
  // odd waves of CTAs walk K backwards: a wave then starts on the chunks the
  // wave before it read last, which are still in L2 (the int32 sums are
  // exact, so the order of the chunks does not change the result)
  const bool rev = g.nsm > 0 && ((lid / g.nsm) & 1);
  double* const Cz = g.C + (long long)blockIdx.z * g.zstride;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_sh)),
                 "r"(512));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    for (int s2 = 0; s2 < STAGES; ++s2) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&full[s2])), "r"(1));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&empty[s2])), "r"(1));
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_sh;

  // warp-specialised issue: lane 0 of warp 1 fills the stages, lane 0 of
  // warp 0 issues the MMAs as soon as a stage is full, so the tensor pipe
  // holds the next chunk's MMAs while the current chunk's run
  if (warp == 1 && lane == 0) {
    const int8_t* Ab = g.A + ((size_t)bx * nkc) * 8192;
    const int8_t* Bb = g.B + ((size_t)(by >> 1) * nkc) * 8192 + (by & 1) * 4096;
    const size_t planeA = (size_t)g.ntrA * nkc * 8192, planeB = (size_t)g.ntrB * nkc * 8192;
    int issued = 0;
    for (int c = 0; c < nch; ++c) {
      const int st = c % STAGES;
      if (c >= STAGES && !emu_wait(&empty[st], (uint32_t)(((c / STAGES) - 1) & 1), g.err)) break;
      uint8_t* base = smem + st * STAGE;
      expect_tx(&full[st], (uint32_t)STAGE);
      const size_t off = (size_t)(rev ? kc1 - 1 - c : kc0 + c) * 8192;
#pragma unroll
      for (int p = 0; p < S; ++p) bulk_load(base + p * A_SL, Ab + p * planeA + off, A_SL, &full[st]);
#pragma unroll
      for (int q = 0; q < S; ++q) bulk_load(base + S * A_SL + q * B_SL, Bb + q * planeB + off, B_SL, &full[st]);
      issued = c + 1;
    }
    // no copy still in flight when the CTA leaves (the last phase of each
    // stage; already complete unless a wait above gave up)
    for (int j = issued > STAGES ? issued - STAGES : 0; j < issued; ++j)
      emu_wait(&full[j % STAGES], (uint32_t)((j / STAGES) & 1), g.err);
  } else if (warp == 0 && lane == 0) {
    // s32 accumulate, signed A and B, K-major both, M = 128 (N set per MMA)
    const uint32_t idesc = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(EMU_M >> 4) << 24);
    bool ok = true;
    for (int m = 0; m < nch && ok; ++m) {
      const int st = m % STAGES;
      ok = emu_wait(&full[st], (uint32_t)((m / STAGES) & 1), g.err);
      if (!ok) break;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint8_t* base = smem + st * STAGE;
      const uint32_t a0 = smem_u32(base), b0 = smem_u32(base + S * A_SL);
#pragma unroll
      for (int p = 0; p < S; ++p)
#pragma unroll
        for (int q0 = 0; q0 < S - p; q0 += 4) {
          const int nq = (S - p - q0) < 4 ? (S - p - q0) : 4;
          const uint32_t id = idesc | ((uint32_t)(nq * EMU_N >> 3) << 17);
#pragma unroll
          for (int kk = 0; kk < 2; ++kk)
            umma_i8(tmem + (p + q0) * EMU_N, emu_desc(a0 + p * A_SL + kk * 256),
                    emu_desc(b0 + q0 * B_SL + kk * 256), id, (m > 0 || p > 0 || kk > 0) ? 1u : 0u);
        }
      umma_commit(&empty[st]);
    }
    // every MMA done before the epilogue reads TMEM
    if (nch > 0 && ok) emu_wait(&empty[(nch - 1) % STAGES], (uint32_t)(((nch - 1) / STAGES) & 1), g.err);
  }
  // epilogue: thread = output row.  With beta ≠ 0 the C values of a 16-column
  // group are read all at once, one group ahead (the first group before the
  // MMAs are waited for), so the memory latency is not paid per element.
  const long long i = i0 + warp * 32 + lane;
  const bool has_beta = g.beta != 0.0;
  auto live = [&](long long j) { return i < g.M && j < g.N && !(g.lower && i + g.row0 < j + g.col0); };
  double cv[16];
#pragma unroll
  for (int u = 0; u < 16; ++u) cv[u] = (has_beta && live(j0 + u)) ? Cz[i + (j0 + u) * g.ldc] : 0.0;
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");

  const int ea = i < g.M ? g.expA[i] : 0;
  const uint32_t trow = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll 1
  for (int cb = 0; cb < EMU_N; cb += 16) {
    uint32_t v[S][16];
#pragma unroll
    for (int t = 0; t < S; ++t) tmem_ld16(trow + t * EMU_N + cb, v[t]);
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
    double nx[16];
#pragma unroll
    for (int u = 0; u < 16; ++u) {
      const long long j = j0 + cb + 16 + u;
      nx[u] = (has_beta && cb + 16 < EMU_N && live(j)) ? Cz[i + j * g.ldc] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < 16; ++u) {
      const long long j = j0 + cb + u;
      if (!live(j)) continue;
      double acc = (double)(int)v[S - 1][u];
#pragma unroll
      for (int t = S - 2; t >= 0; --t) acc = fma(acc, 0.0078125, (double)(int)v[t][u]);
      if (nch == 0) acc = 0.0;
      const double val = ldexp(acc, -(ea + g.expB[j]));
      Cz[i + j * g.ldc] = has_beta ? fma(g.alpha, val, g.beta * cv[u]) : g.alpha * val;
    }
#pragma unroll
    for (int u = 0; u < 16; ++u) cv[u] = nx[u];
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512));
}

size_t emu_gemm_smem(int S) {
  return (size_t)(S <= 6 ? 3 : 2) * S * (EMU_M + EMU_N) * EMU_KC;
}

// SM count of the current device (cached per device)
static int emu_sm_count() {
  static int cached[64] = {0};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 0;
  if (cached[dev] == 0) {
    int v = 0;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
    cached[dev] = v;
  }
  return cached[dev];
}

template <int S>
static cudaError_t launch_emu(const EmuGemmArgs& g, dim3 grid, cudaStream_t s) {
  const int smem = (int)emu_gemm_smem(S);
  cudaError_t e = cudaFuncSetAttribute(emu_gemm_kernel<S>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e != cudaSuccess) return e;
  GPRX_LAUNCH(emu_gemm_kernel<S>, grid, EMU_THREADS, smem, s, g);
  return cudaGetLastError();
}

static cudaError_t launch_emu_any(const EmuGemmArgs& g, int S, dim3 grid, cudaStream_t s) {
  switch (S) {
    case 4: return launch_emu<4>(g, grid, s);
    case 5: return launch_emu<5>(g, grid, s);
    case 6: return launch_emu<6>(g, grid, s);
    case 7: return launch_emu<7>(g, grid, s);
    default: return launch_emu<8>(g, grid, s);
  }
}

static EmuGemmArgs emu_args(const EmuOperand& A, const EmuOperand& B, double* C, long long ldc, double alpha,
                            double beta, bool lower, long long row0, long long col0, int kmode, int* err) {
  EmuGemmArgs g;
  g.A = A.slices;
  g.B = B.slices;
  g.expA = A.exps;
  g.expB = B.exps;
  g.ntrA = A.Rpad / EMU_M;
  g.ntrB = B.Rpad / EMU_M;
  g.M = A.R;
  g.N = B.R;
  g.Kpad = A.Kpad;
  g.C = C;
  g.ldc = ldc;
  g.alpha = alpha;
  g.beta = beta;
  g.lower = lower ? 1 : 0;
  g.row0 = row0;
  g.col0 = col0;
  g.kmode = kmode;
  g.err = err;
  g.kz = 0;
  g.zstride = 0;
  g.nsm = emu_sm_count();
  return g;
}

cudaError_t emu_gemm(const EmuOperand& A, const EmuOperand& B, double* C, long long ldc, double alpha, double beta,
                     bool lower, long long row0, long long col0, int kmode, int* err, cudaStream_t s) {
  if (A.S != B.S || A.Kpad != B.Kpad || A.S < 4 || A.S > EMU_MAX_S) return cudaErrorInvalidValue;
  if (A.R <= 0 || B.R <= 0) return cudaSuccess;
  const EmuGemmArgs g = emu_args(A, B, C, ldc, alpha, beta, lower, row0, col0, kmode, err);
  // B's padded rows (multiple of 128) cover every 64-row tile the grid touches
  return launch_emu_any(g, A.S, dim3(A.Rpad / EMU_M, ceil_div(B.R, EMU_N)), s);
}

cudaError_t emu_gemm_splitk(const EmuOperand& A, const EmuOperand& B, double* C, long long ldc, long long zstride,
                            int kz, bool lower, int* err, cudaStream_t s) {
  if (A.S != B.S || A.Kpad != B.Kpad || A.S < 4 || A.S > EMU_MAX_S || kz <= 0) return cudaErrorInvalidValue;
  if (A.R <= 0 || B.R <= 0) return cudaSuccess;
  EmuGemmArgs g = emu_args(A, B, C, ldc, 1.0, 0.0, lower, 0, 0, 0, err);
  g.kz = kz;
  g.zstride = zstride;
  return launch_emu_any(g, A.S, dim3(A.Rpad / EMU_M, ceil_div(B.R, EMU_N), emu_splitk_parts(A.Kpad, kz)), s);
}

}  // namespace gprx
