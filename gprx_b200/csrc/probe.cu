// probe.cu — device microbenchmarks of the FP64 building blocks (timed with
// CUDA events on a private stream).  They measure the roofline denominators
// that MEASURED_PEAKS.json does not carry (FP64 GEMM on this part) and
// the blocked factor in isolation.

#include <cmath>
#include <cstring>
#include <vector>

#include "dense_f64.cuh"
#include "emu_gemm.cuh"
#include "runtime.cuh"

namespace gprx {

__global__ void fill_pattern_kernel(double* a, long long n, unsigned seed) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    unsigned h = (unsigned)(i * 2654435761u) ^ seed;
    h ^= h >> 13;
    h *= 0x5bd1e995u;
    h ^= h >> 15;
    a[i] = ((double)(h & 0xffffff) / 16777216.0) - 0.5;
  }
}

// SPD test matrix: A = B Bᵀ/n + n·I is replaced by a cheap diagonally dominant
// fill: a_ij = 0.5^|i−j| mixed with the pattern, plus n on the diagonal.
__global__ void fill_spd_kernel(double* a, long long ld, int n) {
  long long total = (long long)n * n;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    int i = (int)(e % n), j = (int)(e / n);
    if (i < j) continue;
    double v = exp(-0.01 * (double)(i - j) * (double)(i - j));
    if (i == j) v += 1.0;
    a[i + (long long)j * ld] = v;
  }
}

__global__ void abs_copy_kernel(const double* a, double* b, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    b[i] = fabs(a[i]);
}

// rows of a scaled by 2^((r % 9) − 4): the per-row exponents differ
__global__ void scale_rows_kernel(double* a, long long ld, int rows, int cols) {
  const long long total = (long long)rows * cols;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(e % rows);
    a[r + (e / rows) * ld] = ldexp(a[r + (e / rows) * ld], (r % 9) - 4);
  }
}

// max over entries of |c − ref| / max(cabs, tiny)
__global__ void rel_err_kernel(const double* c, const double* ref, const double* cabs, long long n,
                               unsigned long long* out_bits) {
  double m = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    m = fmax(m, fabs(c[i] - ref[i]) / fmax(cabs[i], 1e-300));
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out_bits, (unsigned long long)__double_as_longlong(m));
}

}  // namespace gprx

using namespace gprx;

extern "C" {

gprx_status gprx_probe_dgemm(int32_t m, int32_t n, int32_t k, int32_t trans_a, int32_t trans_b, int32_t reps,
                             double* ms_per_launch) {
  if (m <= 0 || n <= 0 || k <= 0 || reps <= 0 || !ms_per_launch) return set_error(GPRX_INVALID_ARGUMENT, "sizes");
  long long lda = trans_a ? k : m, ldb = trans_b ? n : k;
  size_t sa = (size_t)lda * (trans_a ? m : k), sb = (size_t)ldb * (trans_b ? k : n), sc = (size_t)m * n;
  DevBuf<double> A, B, Cm;
  if (A.alloc(sa) || B.alloc(sb) || Cm.alloc(sc)) return set_error(GPRX_OUT_OF_MEMORY, "probe buffers");
  cudaStream_t s;
  GPRX_CUDA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  fill_pattern_kernel<<<1184, 256, 0, s>>>(A.p, (long long)sa, 1u);
  fill_pattern_kernel<<<1184, 256, 0, s>>>(B.p, (long long)sb, 2u);
  GemmParams p = gemm_params(m, n, k, A.p, lda, B.p, ldb, Cm.p, m, 1.0, 0.0, nullptr);
  cudaError_t e = dgemm(trans_a != 0, trans_b != 0, p, s);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, s);
  for (int r = 0; r < reps && e == cudaSuccess; ++r) e = dgemm(trans_a != 0, trans_b != 0, p, s);
  cudaEventRecord(e1, s);
  cudaError_t e2 = cudaStreamSynchronize(s);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaStreamDestroy(s);
  if (e != cudaSuccess) return set_cuda_error(e, "probe dgemm");
  if (e2 != cudaSuccess) return set_cuda_error(e2, "probe dgemm sync");
  *ms_per_launch = ms / reps;
  return GPRX_OK;
}

// Times the blocked Cholesky (potrf) alone on an SPD n×n matrix; out[0] ms
// per factor, out[1] ms of the diagonal-block kernel chain alone is not
// separated (use ncu for that).
gprx_status gprx_probe_potrf(int32_t n, int32_t reps, double* ms_per_factor) {
  if (n <= 0 || reps <= 0 || !ms_per_factor) return set_error(GPRX_INVALID_ARGUMENT, "sizes");
  long long ld = round_ld(n);
  DevBuf<double> A, linv;
  DevBuf<DevStatus> st;
  if (A.alloc((size_t)ld * n) || linv.alloc((size_t)ceil_div(n, NB) * NB * NB) || st.alloc(1))
    return set_error(GPRX_OUT_OF_MEMORY, "probe buffers");
  cudaStream_t s;
  GPRX_CUDA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float total = 0.f;
  cudaError_t e = cudaSuccess;
  FactorCtx ctx;
  for (int r = 0; r < reps + 1 && e == cudaSuccess; ++r) {
    cudaMemsetAsync(st.p, 0, sizeof(DevStatus), s);
    fill_spd_kernel<<<1184, 256, 0, s>>>(A.p, ld, n);
    cudaEventRecord(e0, s);
    e = potrf_blocked(A.p, ld, n, linv.p, st.p, s, &ctx);
    cudaEventRecord(e1, s);
    cudaStreamSynchronize(s);
    float ms;
    cudaEventElapsedTime(&ms, e0, e1);
    if (r > 0) total += ms;
  }
  DevStatus hs;
  cudaMemcpy(&hs, st.p, sizeof(hs), cudaMemcpyDeviceToHost);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaStreamDestroy(s);
  if (e != cudaSuccess) return set_cuda_error(e, "probe potrf");
  if (hs.code != GPRX_OK) return set_error(hs.code, "probe potrf status");
  *ms_per_factor = total / reps;
  return GPRX_OK;
}

// The int8-sliced FP64 product C = A·Bᵀ (A m×k, B n×k, S slices) against the
// FP64 DMMA product: out[0] ms per emulated GEMM, out[1] ms to slice both
// operands, out[2] ms per DMMA GEMM, out[3] max |C − C_ref| / (|A|·|B|ᵀ).
gprx_status gprx_probe_emu_gemm(int32_t m, int32_t n, int32_t k, int32_t S, int32_t reps, double* out) {
  if (m <= 0 || n <= 0 || k <= 0 || reps <= 0 || !out || S < 4 || S > EMU_MAX_S)
    return set_error(GPRX_INVALID_ARGUMENT, "sizes");
  DevBuf<double> A, B, Aa, Ba, C, R, Cabs;
  DevBuf<int8_t> sa, sb;
  DevBuf<int> ea, eb, err;
  DevBuf<unsigned long long> mx, rma, rmb;
  EmuOperand a, b;
  a.R = m; a.K = k; a.S = S; a.Rpad = emu_pad_rows(m); a.Kpad = emu_pad_k(k);
  b.R = n; b.K = k; b.S = S; b.Rpad = emu_pad_rows(n); b.Kpad = emu_pad_k(k);
  const size_t sza = (size_t)m * k, szb = (size_t)n * k, szc = (size_t)m * n;
  if (A.alloc(sza) || B.alloc(szb) || Aa.alloc(sza) || Ba.alloc(szb) || C.alloc(szc) || R.alloc(szc) ||
      Cabs.alloc(szc) || sa.alloc(emu_slice_bytes(m, k, S)) || sb.alloc(emu_slice_bytes(n, k, S)) ||
      ea.alloc(a.Rpad) || eb.alloc(b.Rpad) || err.alloc(1) || mx.alloc(1) || rma.alloc(a.Rpad) ||
      rmb.alloc(b.Rpad))
    return set_error(GPRX_OUT_OF_MEMORY, "probe buffers");
  a.slices = sa.p; a.exps = ea.p; a.rmax = rma.p; b.slices = sb.p; b.exps = eb.p; b.rmax = rmb.p;
  cudaStream_t s;
  GPRX_CUDA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  fill_pattern_kernel<<<1184, 256, 0, s>>>(A.p, (long long)sza, 3u);
  fill_pattern_kernel<<<1184, 256, 0, s>>>(B.p, (long long)szb, 4u);
  scale_rows_kernel<<<1184, 256, 0, s>>>(A.p, m, m, k);
  abs_copy_kernel<<<1184, 256, 0, s>>>(A.p, Aa.p, (long long)sza);
  abs_copy_kernel<<<1184, 256, 0, s>>>(B.p, Ba.p, (long long)szb);
  cudaMemsetAsync(err.p, 0, sizeof(int), s);
  cudaMemsetAsync(mx.p, 0, sizeof(unsigned long long), s);
  GemmParams pr = gemm_params(m, n, k, A.p, m, B.p, n, R.p, m, 1.0, 0.0, nullptr);
  GemmParams pa = gemm_params(m, n, k, Aa.p, m, Ba.p, n, Cabs.p, m, 1.0, 0.0, nullptr);
  cudaError_t e = dgemm(false, true, pr, s);
  if (e == cudaSuccess) e = dgemm(false, true, pa, s);
  if (e == cudaSuccess) e = emu_slice(A.p, m, false, a, s);
  if (e == cudaSuccess) e = emu_slice(B.p, n, false, b, s);
  if (e == cudaSuccess) e = emu_gemm(a, b, C.p, m, 1.0, 0.0, false, 0, 0, 0, err.p, s);
  if (e == cudaSuccess) {
    rel_err_kernel<<<592, 256, 0, s>>>(C.p, R.p, Cabs.p, (long long)szc, mx.p);
    e = cudaGetLastError();
  }
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float t_emu = 0.f, t_slice = 0.f, t_d = 0.f, t_beta = 0.f;
  if (e == cudaSuccess) {
    cudaEventRecord(e0, s);
    for (int r = 0; r < reps && e == cudaSuccess; ++r) e = emu_gemm(a, b, C.p, m, 1.0, 0.0, false, 0, 0, 0, err.p, s);
    cudaEventRecord(e1, s);
    cudaEventSynchronize(e1);
    cudaEventElapsedTime(&t_emu, e0, e1);
    // the update form C = C − A·Bᵀ (every C value read and written)
    cudaEventRecord(e0, s);
    for (int r = 0; r < reps && e == cudaSuccess; ++r) e = emu_gemm(a, b, C.p, m, -1.0, 1.0, false, 0, 0, 0, err.p, s);
    cudaEventRecord(e1, s);
    cudaEventSynchronize(e1);
    cudaEventElapsedTime(&t_beta, e0, e1);
    cudaEventRecord(e0, s);
    for (int r = 0; r < reps && e == cudaSuccess; ++r) {
      e = emu_slice(A.p, m, false, a, s);
      if (e == cudaSuccess) e = emu_slice(B.p, n, false, b, s);
    }
    cudaEventRecord(e1, s);
    cudaEventSynchronize(e1);
    cudaEventElapsedTime(&t_slice, e0, e1);
    cudaEventRecord(e0, s);
    for (int r = 0; r < reps && e == cudaSuccess; ++r) e = dgemm(false, true, pr, s);
    cudaEventRecord(e1, s);
    cudaEventSynchronize(e1);
    cudaEventElapsedTime(&t_d, e0, e1);
  }
  cudaError_t e2 = cudaStreamSynchronize(s);
  int herr = 0;
  unsigned long long hm = 0;
  cudaMemcpy(&herr, err.p, sizeof(int), cudaMemcpyDeviceToHost);
  cudaMemcpy(&hm, mx.p, sizeof(hm), cudaMemcpyDeviceToHost);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaStreamDestroy(s);
  if (e != cudaSuccess) return set_cuda_error(e, "probe emu gemm");
  if (e2 != cudaSuccess) return set_cuda_error(e2, "probe emu gemm sync");
  if (herr) return set_error(GPRX_TIMEOUT, "emulated GEMM: a bounded wait ran out");
  out[0] = t_emu / reps;
  out[1] = t_slice / reps;
  out[2] = t_d / reps;
  double hd;
  std::memcpy(&hd, &hm, sizeof(hd));
  out[3] = hd;
  out[4] = t_beta / reps;
  return GPRX_OK;
}

}  // extern "C"
