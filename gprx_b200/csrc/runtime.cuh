// runtime.cuh — host runtime shared by the handles: device buffers, the
// per-thread error record, status mapping.
#pragma once

#include <cstring>
#include <string>
#include <vector>

#include "common.cuh"

namespace gprx {

// Thread-local record behind gprx_last_error().
gprx_error_info& last_error();
gprx_status set_error(gprx_status st, const std::string& msg);
gprx_status set_cuda_error(cudaError_t e, const char* where);
gprx_status set_cholesky_error(double jitter, uint64_t size, int stage);

#define GPRX_CUDA_TRY(expr)                                   \
  do {                                                        \
    cudaError_t e_ = (expr);                                  \
    if (e_ != cudaSuccess) return ::gprx::set_cuda_error(e_, #expr); \
  } while (0)

// Owning device buffer.
template <typename T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { reset(); }
  cudaError_t alloc(size_t count) {
    reset();
    if (count == 0) return cudaSuccess;
    cudaError_t e = cudaMalloc((void**)&p, count * sizeof(T));
    if (e != cudaSuccess) {
      p = nullptr;
      return e;
    }
    n = count;
    return cudaSuccess;
  }
  // grows (never shrinks); contents are not kept
  cudaError_t ensure(size_t count) { return count <= n ? cudaSuccess : alloc(count); }
  void reset() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
};

// Pinned host scratch.
template <typename T>
struct HostPinned {
  T* p = nullptr;
  size_t n = 0;
  ~HostPinned() {
    if (p) cudaFreeHost(p);
  }
  cudaError_t ensure(size_t count) {
    if (count <= n) return cudaSuccess;
    if (p) cudaFreeHost(p);
    p = nullptr;
    n = 0;
    cudaError_t e = cudaMallocHost((void**)&p, count * sizeof(T));
    if (e == cudaSuccess) n = count;
    return e;
  }
};

inline long long round_ld(long long n) { return (n + 31) / 32 * 32; }

bool all_finite(const double* v, size_t n);

// Reads the device status word (after the stream drained) and maps it.
gprx_status status_to_error(const DevStatus& st, double jitter, uint64_t size, int stage);

}  // namespace gprx
