// Shared host-side helpers for the C ABI: error reporting and CUDA checks.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstring>

#include "../../include/stwo_b200.h"

namespace stwo_b200 {

inline int set_err(char* err, size_t err_len, int code, const char* fmt, ...) {
  if (err && err_len) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(err, err_len, fmt, ap);
    va_end(ap);
  }
  return code;
}

inline int ok(char* err, size_t err_len) {
  if (err && err_len) err[0] = 0;
  return STWO_B200_OK;
}

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// Raises a kernel's dynamic shared-memory limit on the current device the
// first time it is launched there.  The attribute is per device, so `done`
// keeps one bit per device; threads that race to set it both set the same
// value, which is harmless.
template <typename Kernel>
inline cudaError_t ensure_smem_limit(Kernel* kernel, int bytes, std::atomic<uint32_t>& done) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const uint32_t bit = dev >= 0 && dev < 32 ? 1u << dev : 0u;
  if (bit && (done.load(std::memory_order_acquire) & bit)) return cudaSuccess;
  e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess && bit) done.fetch_or(bit, std::memory_order_release);
  return e;
}

// Number of kernels this library has launched (read by stwo_b200_launch_count).
extern std::atomic<uint64_t> g_kernel_launches;

// Host/device index helpers.
__host__ __device__ __forceinline__ uint32_t bitrev32(uint32_t x, uint32_t bits) {
#ifdef __CUDA_ARCH__
  return bits ? (__brev(x) >> (32 - bits)) : 0;
#else
  uint32_t r = 0;
  for (uint32_t b = 0; b < bits; b++) r |= ((x >> b) & 1u) << (bits - 1 - b);
  return r;
#endif
}

}  // namespace stwo_b200

#define STWO_CUDA_TRY(expr)                                                                              \
  do {                                                                                                   \
    cudaError_t e_ = (expr);                                                                             \
    if (e_ != cudaSuccess)                                                                               \
      return ::stwo_b200::set_err(err, err_len, e_ == cudaErrorMemoryAllocation ? STWO_B200_ENOMEM       \
                                                                                : STWO_B200_ECUDA,       \
                                  "%s: %s (%s:%d)", #expr, cudaGetErrorString(e_), __FILE__, __LINE__); \
  } while (0)

#define STWO_CHECK_LAUNCH()                                                                                 \
  do {                                                                                                      \
    ::stwo_b200::g_kernel_launches.fetch_add(1, std::memory_order_relaxed);                                 \
    cudaError_t e_ = cudaGetLastError();                                                                    \
    if (e_ != cudaSuccess)                                                                                  \
      return ::stwo_b200::set_err(err, err_len, STWO_B200_ECUDA, "kernel launch: %s (%s:%d)",               \
                                  cudaGetErrorString(e_), __FILE__, __LINE__);                              \
  } while (0)

#define STWO_ARG_CHECK(cond, ...)                                                  \
  do {                                                                             \
    if (!(cond)) return ::stwo_b200::set_err(err, err_len, STWO_B200_EARG, __VA_ARGS__); \
  } while (0)
