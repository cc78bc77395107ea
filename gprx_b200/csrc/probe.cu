// probe.cu — device microbenchmarks of the FP64 building blocks (timed with
// CUDA events on a private stream).  They measure the roofline denominators
// that the driver's peak file does not carry (FP64 GEMM on this part) and
// the blocked factor in isolation.

#include <cmath>
#include <vector>

#include "dense_f64.cuh"
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

}  // extern "C"
