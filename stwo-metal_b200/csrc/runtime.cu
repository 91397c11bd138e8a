// Runtime entry points: device selection, stream-ordered pool memory, copies,
// streams.  The B200 counterpart of the reference's Objective-C runtime
// (crates/stwo-metal-sys/metal/runtime.m: device/queue/buffer management).
#include <cuda_runtime.h>

#include <cstdint>

#include "common.cuh"

namespace stwo_b200 {
std::atomic<uint64_t> g_kernel_launches{0};
}

using namespace stwo_b200;

extern "C" {

const char* stwo_b200_version(void) { return "stwo_b200 0.1 (sm_100a)"; }

uint64_t stwo_b200_launch_count(void) { return g_kernel_launches.load(std::memory_order_relaxed); }

int stwo_b200_init(int device, char* err, size_t err_len) {
  int n = 0;
  STWO_CUDA_TRY(cudaGetDeviceCount(&n));
  STWO_ARG_CHECK(device >= 0 && device < n, "device %d out of range (%d devices)", device, n);
  STWO_CUDA_TRY(cudaSetDevice(device));
  cudaDeviceProp prop;
  STWO_CUDA_TRY(cudaGetDeviceProperties(&prop, device));
  if (prop.major != 10)
    return set_err(err, err_len, STWO_B200_ESTATE, "device %d is sm_%d%d; this library is built for sm_100a", device,
                   prop.major, prop.minor);
  // Keep freed pool memory cached for reuse instead of returning it to the OS
  // at every synchronisation: the prover allocates the same shapes repeatedly.
  cudaMemPool_t pool;
  STWO_CUDA_TRY(cudaDeviceGetDefaultMemPool(&pool, device));
  uint64_t threshold = UINT64_MAX;
  STWO_CUDA_TRY(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold));
  return ok(err, err_len);
}

int stwo_b200_alloc(size_t bytes, void** d_out, void* stream, char* err, size_t err_len) {
  STWO_ARG_CHECK(d_out != nullptr, "d_out is null");
  *d_out = nullptr;
  if (bytes == 0) return ok(err, err_len);
  STWO_CUDA_TRY(cudaMallocAsync(d_out, bytes, as_stream(stream)));
  return ok(err, err_len);
}

int stwo_b200_free(void* d_ptr, void* stream, char* err, size_t err_len) {
  if (d_ptr) STWO_CUDA_TRY(cudaFreeAsync(d_ptr, as_stream(stream)));
  return ok(err, err_len);
}

int stwo_b200_memcpy_h2d(void* d_dst, const void* h_src, size_t bytes, void* stream, char* err, size_t err_len) {
  if (bytes) STWO_CUDA_TRY(cudaMemcpyAsync(d_dst, h_src, bytes, cudaMemcpyHostToDevice, as_stream(stream)));
  return ok(err, err_len);
}

int stwo_b200_memcpy_d2h(void* h_dst, const void* d_src, size_t bytes, void* stream, char* err, size_t err_len) {
  if (bytes) STWO_CUDA_TRY(cudaMemcpyAsync(h_dst, d_src, bytes, cudaMemcpyDeviceToHost, as_stream(stream)));
  return ok(err, err_len);
}

int stwo_b200_memcpy_d2d(void* d_dst, const void* d_src, size_t bytes, void* stream, char* err, size_t err_len) {
  if (bytes) STWO_CUDA_TRY(cudaMemcpyAsync(d_dst, d_src, bytes, cudaMemcpyDeviceToDevice, as_stream(stream)));
  return ok(err, err_len);
}

int stwo_b200_memset(void* d_dst, int value, size_t bytes, void* stream, char* err, size_t err_len) {
  if (bytes) STWO_CUDA_TRY(cudaMemsetAsync(d_dst, value, bytes, as_stream(stream)));
  return ok(err, err_len);
}

int stwo_b200_stream_create(void** stream_out, char* err, size_t err_len) {
  STWO_ARG_CHECK(stream_out != nullptr, "stream_out is null");
  cudaStream_t s;
  STWO_CUDA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  *stream_out = s;
  return ok(err, err_len);
}

int stwo_b200_stream_destroy(void* stream, char* err, size_t err_len) {
  if (stream) STWO_CUDA_TRY(cudaStreamDestroy(as_stream(stream)));
  return ok(err, err_len);
}

int stwo_b200_stream_sync(void* stream, char* err, size_t err_len) {
  STWO_CUDA_TRY(cudaStreamSynchronize(as_stream(stream)));
  return ok(err, err_len);
}

int stwo_b200_host_alloc(size_t bytes, void** h_out, char* err, size_t err_len) {
  STWO_ARG_CHECK(h_out != nullptr, "h_out is null");
  STWO_CUDA_TRY(cudaMallocHost(h_out, bytes ? bytes : 1));
  return ok(err, err_len);
}

int stwo_b200_host_free(void* h_ptr, char* err, size_t err_len) {
  if (h_ptr) STWO_CUDA_TRY(cudaFreeHost(h_ptr));
  return ok(err, err_len);
}

}  // extern "C"
