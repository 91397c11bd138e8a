// FRI folds for sm_100a: fold_line, fold_circle_into_line, decompose.
//
// QM31 columns are four M31 coordinate columns; each kernel streams them with
// one thread per output (fold) or per element (decompose).
//  fold_line (crates/stwo/src/prover/backend/cpu/fri.rs:67-92, simd/fri.rs:32-122):
//    f' = (f(x) + f(-x)) + alpha * (f(x) - f(-x)) * x^-1, fold_step layers fused
//    with alpha <- alpha^2 per layer; x^-1 from the inverse twiddle tree.
//  fold_circle_into_line (cpu/fri.rs:95-123, simd/fri.rs:124-172):
//    dst <- dst * alpha^2 + (f(p) + f(-p)) + alpha * (f(p) - f(-p)) * p.y^-1.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>

#include "common.cuh"
#include "field.cuh"

namespace stwo_b200 {

struct Cols4 {
  const uint32_t* c[4];
};
struct Cols4W {
  uint32_t* c[4];
};

__device__ __forceinline__ qm31 load_q(const Cols4& s, uint64_t i) {
  return {__ldg(s.c[0] + i), __ldg(s.c[1] + i), __ldg(s.c[2] + i), __ldg(s.c[3] + i)};
}
__device__ __forceinline__ void store_q(const Cols4W& d, uint64_t i, qm31 v) {
  d.c[0][i] = v.a;
  d.c[1][i] = v.b;
  d.c[2][i] = v.c;
  d.c[3][i] = v.d;
}

constexpr int kMaxFoldStep = 6;
struct FoldAlphas {
  qm31 a[kMaxFoldStep];
};

// One thread per output; reads 2^fold_step consecutive inputs.
__global__ void fold_line_kernel(Cols4 in, uint32_t log_m, uint32_t fold_step, FoldAlphas alphas,
                                 const uint32_t* itw, uint64_t tw_len, Cols4W out) {
  uint64_t n_out = 1ull << (log_m - fold_step);
  for (uint64_t o = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; o < n_out; o += (uint64_t)gridDim.x * blockDim.x) {
    if (fold_step == 1) {
      const uint32_t* lt = itw + (tw_len - (1ull << log_m));
      qm31 fx = load_q(in, 2 * o), fnx = load_q(in, 2 * o + 1);
      qm31 f0 = qm31_add(fx, fnx);
      qm31 f1 = qm31_mul_m31(qm31_sub(fx, fnx), __ldg(lt + o));
      store_q(out, o, qm31_add(f0, qm31_mul(alphas.a[0], f1)));
      continue;
    }
    qm31 v[1 << kMaxFoldStep];
    const uint32_t w = 1u << fold_step;
    for (uint32_t j = 0; j < w; j++) v[j] = load_q(in, o * w + j);
    for (uint32_t s = 0; s < fold_step; s++) {
      const uint32_t* lt = itw + (tw_len - (1ull << (log_m - s)));
      uint32_t pairs = w >> (s + 1);
      for (uint32_t j = 0; j < pairs; j++) {
        qm31 fx = v[2 * j], fnx = v[2 * j + 1];
        qm31 f0 = qm31_add(fx, fnx);
        qm31 f1 = qm31_mul_m31(qm31_sub(fx, fnx), __ldg(lt + o * pairs + j));
        v[j] = qm31_add(f0, qm31_mul(alphas.a[s], f1));
      }
    }
    store_q(out, o, v[0]);
  }
}

// fold_line with fold_step 1, two outputs per thread: the four inputs of
// outputs 2k, 2k + 1 are one 16-byte load per coordinate, their twiddles one
// 8-byte load, the outputs one 8-byte store per coordinate.  Same arithmetic
// per output as fold_line_kernel.  Inputs 16-byte and outputs 8-byte aligned,
// at least 2 outputs.
__global__ void __launch_bounds__(256) fold_line2_kernel(Cols4 in, uint32_t log_m, qm31 alpha, const uint32_t* itw,
                                                         uint64_t tw_len, Cols4W out) {
  const uint64_t n_pairs = 1ull << (log_m - 2);
  const uint32_t* lt = itw + (tw_len - (1ull << log_m));
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < n_pairs;
       k += (uint64_t)gridDim.x * blockDim.x) {
    uint4 w[4];
#pragma unroll
    for (int c = 0; c < 4; c++) w[c] = __ldg(reinterpret_cast<const uint4*>(in.c[c]) + k);
    const uint2 t = __ldg(reinterpret_cast<const uint2*>(lt) + k);
    const qm31 f0x{w[0].x, w[1].x, w[2].x, w[3].x}, f0n{w[0].y, w[1].y, w[2].y, w[3].y};
    const qm31 f1x{w[0].z, w[1].z, w[2].z, w[3].z}, f1n{w[0].w, w[1].w, w[2].w, w[3].w};
    const qm31 v0 = qm31_add(qm31_add(f0x, f0n), qm31_mul(alpha, qm31_mul_m31(qm31_sub(f0x, f0n), t.x)));
    const qm31 v1 = qm31_add(qm31_add(f1x, f1n), qm31_mul(alpha, qm31_mul_m31(qm31_sub(f1x, f1n), t.y)));
    reinterpret_cast<uint2*>(out.c[0])[k] = make_uint2(v0.a, v1.a);
    reinterpret_cast<uint2*>(out.c[1])[k] = make_uint2(v0.b, v1.b);
    reinterpret_cast<uint2*>(out.c[2])[k] = make_uint2(v0.c, v1.c);
    reinterpret_cast<uint2*>(out.c[3])[k] = make_uint2(v0.d, v1.d);
  }
}

// Circle-layer inverse twiddle of pair i, derived from line layer 1 of the
// source domain: [y, -y, -x, x] (simd/fft/mod.rs:61-97).
__device__ __forceinline__ uint32_t circle_itw(const uint32_t* lt0, uint64_t i) {
  uint32_t b = __ldg(lt0 + ((i >> 1) ^ 1));
  return ((i ^ (i >> 1)) & 1) ? m31_neg(b) : b;
}

struct SmallYinv {
  uint32_t v[8];
};

__global__ void fold_circle_kernel(Cols4W dst, Cols4 src, uint32_t log_n, qm31 alpha, qm31 alpha_sq,
                                   const uint32_t* itw, uint64_t tw_len, SmallYinv small) {
  uint64_t n_out = 1ull << (log_n - 1);
  const uint32_t* lt0 = log_n > 4 ? itw + (tw_len - (1ull << (log_n - 1))) : nullptr;
  const Cols4 dr{{dst.c[0], dst.c[1], dst.c[2], dst.c[3]}};
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n_out; i += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t yinv = log_n > 4 ? circle_itw(lt0, i) : small.v[i];
    qm31 fp = load_q(src, 2 * i), fnp = load_q(src, 2 * i + 1);
    qm31 f0 = qm31_add(fp, fnp);
    qm31 f1 = qm31_mul_m31(qm31_sub(fp, fnp), yinv);
    qm31 fprime = qm31_add(f0, qm31_mul(alpha, f1));
    qm31 d = load_q(dr, i);
    store_q(dst, i, qm31_add(qm31_mul(d, alpha_sq), fprime));
  }
}

// fold_circle_kernel, two outputs per thread (log_n > 4): the four source
// values of outputs 2k, 2k + 1 are one 16-byte load per coordinate, dst one
// 8-byte load and store.  The circle twiddles of outputs 2k, 2k + 1 are
// [y, -y] or [-x, x] of one line-layer-1 entry (circle_itw).  Same arithmetic
// per output as fold_circle_kernel.
__global__ void __launch_bounds__(256) fold_circle2_kernel(Cols4W dst, Cols4 src, uint32_t log_n, qm31 alpha,
                                                           qm31 alpha_sq, const uint32_t* itw, uint64_t tw_len) {
  const uint64_t n_pairs = 1ull << (log_n - 2);
  const uint32_t* lt0 = itw + (tw_len - (1ull << (log_n - 1)));
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < n_pairs;
       k += (uint64_t)gridDim.x * blockDim.x) {
    uint4 w[4];
    uint2 d[4];
#pragma unroll
    for (int c = 0; c < 4; c++) {
      w[c] = __ldg(reinterpret_cast<const uint4*>(src.c[c]) + k);
      d[c] = reinterpret_cast<const uint2*>(dst.c[c])[k];
    }
    const uint32_t y0 = circle_itw(lt0, 2 * k), y1 = circle_itw(lt0, 2 * k + 1);
    const qm31 p0{w[0].x, w[1].x, w[2].x, w[3].x}, n0{w[0].y, w[1].y, w[2].y, w[3].y};
    const qm31 p1{w[0].z, w[1].z, w[2].z, w[3].z}, n1{w[0].w, w[1].w, w[2].w, w[3].w};
    const qm31 f0 = qm31_add(qm31_add(p0, n0), qm31_mul(alpha, qm31_mul_m31(qm31_sub(p0, n0), y0)));
    const qm31 f1 = qm31_add(qm31_add(p1, n1), qm31_mul(alpha, qm31_mul_m31(qm31_sub(p1, n1), y1)));
    const qm31 v0 = qm31_add(qm31_mul(qm31{d[0].x, d[1].x, d[2].x, d[3].x}, alpha_sq), f0);
    const qm31 v1 = qm31_add(qm31_mul(qm31{d[0].y, d[1].y, d[2].y, d[3].y}, alpha_sq), f1);
    reinterpret_cast<uint2*>(dst.c[0])[k] = make_uint2(v0.a, v1.a);
    reinterpret_cast<uint2*>(dst.c[1])[k] = make_uint2(v0.b, v1.b);
    reinterpret_cast<uint2*>(dst.c[2])[k] = make_uint2(v0.c, v1.c);
    reinterpret_cast<uint2*>(dst.c[3])[k] = make_uint2(v0.d, v1.d);
  }
}

static bool aligned4(const void* const* p, uintptr_t a) {
  for (int c = 0; c < 4; c++)
    if (reinterpret_cast<uintptr_t>(p[c]) % a) return false;
  return true;
}

// decompose: per-block signed sums (+ on [0, 16*half_a), - on [16*half_a,
// 16*range)), then lambda = sum / n, then g = f -/+ lambda.
__global__ void decompose_sums_kernel(Cols4 in, uint64_t split, uint64_t end, uint32_t* partial) {
  __shared__ uint32_t red[4][256];
  uint32_t acc[4] = {0, 0, 0, 0};
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < end; i += (uint64_t)gridDim.x * blockDim.x) {
    qm31 v = load_q(in, i);
    uint32_t w[4] = {v.a, v.b, v.c, v.d};
#pragma unroll
    for (int k = 0; k < 4; k++) acc[k] = i < split ? m31_add(acc[k], w[k]) : m31_sub(acc[k], w[k]);
  }
#pragma unroll
  for (int k = 0; k < 4; k++) red[k][threadIdx.x] = acc[k];
  __syncthreads();
  for (uint32_t s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
#pragma unroll
      for (int k = 0; k < 4; k++) red[k][threadIdx.x] = m31_add(red[k][threadIdx.x], red[k][threadIdx.x + s]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < 4; k++) partial[blockIdx.x * 4 + k] = red[k][0];
  }
}

__global__ void decompose_finish_kernel(const uint32_t* partial, uint32_t n_blocks, uint32_t inv_n, uint32_t* lambda) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  uint32_t s[4] = {0, 0, 0, 0};
  for (uint32_t b = 0; b < n_blocks; b++)
    for (int k = 0; k < 4; k++) s[k] = m31_add(s[k], partial[b * 4 + k]);
  for (int k = 0; k < 4; k++) lambda[k] = m31_mul(s[k], inv_n);
}

__global__ void decompose_apply_kernel(Cols4 in, uint64_t n, uint64_t split, const uint32_t* lambda, Cols4W out) {
  qm31 l{lambda[0], lambda[1], lambda[2], lambda[3]};
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    qm31 v = load_q(in, i);
    store_q(out, i, i < split ? qm31_sub(v, l) : qm31_add(v, l));
  }
}

static unsigned grid_for(uint64_t n, unsigned threads) {
  uint64_t b = (n + threads - 1) / threads;
  return (unsigned)std::min<uint64_t>(std::max<uint64_t>(b, 1), 148ull * 64);
}

static void host_point(uint64_t idx, uint32_t& x, uint32_t& y) {
  uint32_t gx = 2, gy = 1268011823u;
  x = 1;
  y = 0;
  idx &= (1ull << 31) - 1;
  for (int b = 0; b < 31; b++) {
    if ((idx >> b) & 1) {
      uint32_t nx = m31_sub(m31_mul(x, gx), m31_mul(y, gy));
      uint32_t ny = m31_add(m31_mul(x, gy), m31_mul(y, gx));
      x = nx;
      y = ny;
    }
    uint32_t dx = m31_sub(m31_mul(gx, gx), m31_mul(gy, gy));
    uint32_t dy = m31_add(m31_mul(gx, gy), m31_mul(gy, gx));
    gx = dx;
    gy = dy;
  }
}

}  // namespace stwo_b200

using namespace stwo_b200;

extern "C" int stwo_b200_fold_line(const uint32_t* const* d_in4, uint32_t log_size, const uint32_t* alpha,
                                   uint32_t fold_step, const uint32_t* d_itwiddles, uint32_t tree_log_size,
                                   uint32_t* const* d_out4, void* stream, char* err, size_t err_len) {
  STWO_ARG_CHECK(d_in4 && d_out4 && alpha, "null argument");
  STWO_ARG_CHECK(fold_step >= 1 && fold_step <= (uint32_t)kMaxFoldStep && fold_step <= log_size,
                 "fold_step %u invalid for log size %u", fold_step, log_size);
  STWO_ARG_CHECK(d_itwiddles && log_size <= tree_log_size, "twiddle tree (log %u) too small for line log size %u",
                 tree_log_size, log_size);
  Cols4 in{{d_in4[0], d_in4[1], d_in4[2], d_in4[3]}};
  Cols4W out{{d_out4[0], d_out4[1], d_out4[2], d_out4[3]}};
  FoldAlphas al;
  qm31 a{alpha[0], alpha[1], alpha[2], alpha[3]};
  for (uint32_t s = 0; s < fold_step; s++) {
    al.a[s] = a;
    a = qm31_mul(a, a);
  }
  uint64_t n_out = 1ull << (log_size - fold_step);
  if (fold_step == 1 && log_size >= 2 && aligned4(reinterpret_cast<const void* const*>(in.c), 16) &&
      aligned4(reinterpret_cast<const void* const*>(out.c), 8))
    fold_line2_kernel<<<grid_for(n_out / 2, 256), 256, 0, as_stream(stream)>>>(in, log_size, al.a[0], d_itwiddles,
                                                                              1ull << tree_log_size, out);
  else
    fold_line_kernel<<<grid_for(n_out, 256), 256, 0, as_stream(stream)>>>(in, log_size, fold_step, al, d_itwiddles,
                                                                          1ull << tree_log_size, out);
  STWO_CHECK_LAUNCH();
  return ok(err, err_len);
}

extern "C" int stwo_b200_fold_circle_into_line(uint32_t* const* d_dst4, const uint32_t* const* d_src4,
                                               uint32_t log_size, uint64_t half_initial_index, const uint32_t* alpha,
                                               const uint32_t* d_itwiddles, uint32_t tree_log_size, void* stream,
                                               char* err, size_t err_len) {
  STWO_ARG_CHECK(d_dst4 && d_src4 && alpha, "null argument");
  STWO_ARG_CHECK(log_size >= 1 && log_size <= 30, "bad log size %u", log_size);
  SmallYinv small{};
  if (log_size <= 4) {
    // simd/fri.rs:130-140: CPU path, y^-1 of circle domain point bitrev(2i).
    uint64_t half_size = 1ull << (log_size - 1);
    uint64_t step = 1ull << (31 - (log_size - 1));
    for (uint64_t i = 0; i < half_size; i++) {
      uint64_t pos = bitrev32((uint32_t)(i << 1), log_size);
      uint64_t idx = pos < half_size ? (half_initial_index + step * pos)
                                     : ((1ull << 31) - ((half_initial_index + step * (pos - half_size)) & ((1ull << 31) - 1)));
      uint32_t x, y;
      host_point(idx, x, y);
      small.v[i] = m31_inv(y);
    }
  } else {
    STWO_ARG_CHECK(d_itwiddles && log_size - 1 <= tree_log_size, "twiddle tree (log %u) too small for log size %u",
                   tree_log_size, log_size);
  }
  Cols4W dst{{d_dst4[0], d_dst4[1], d_dst4[2], d_dst4[3]}};
  Cols4 src{{d_src4[0], d_src4[1], d_src4[2], d_src4[3]}};
  qm31 a{alpha[0], alpha[1], alpha[2], alpha[3]};
  uint64_t n_out = 1ull << (log_size - 1);
  if (log_size > 4 && aligned4(reinterpret_cast<const void* const*>(src.c), 16) &&
      aligned4(reinterpret_cast<const void* const*>(dst.c), 8))
    fold_circle2_kernel<<<grid_for(n_out / 2, 256), 256, 0, as_stream(stream)>>>(dst, src, log_size, a, qm31_mul(a, a),
                                                                                d_itwiddles, 1ull << tree_log_size);
  else
    fold_circle_kernel<<<grid_for(n_out, 256), 256, 0, as_stream(stream)>>>(
        dst, src, log_size, a, qm31_mul(a, a), d_itwiddles, d_itwiddles ? (1ull << tree_log_size) : 0, small);
  STWO_CHECK_LAUNCH();
  return ok(err, err_len);
}

extern "C" int stwo_b200_decompose(const uint32_t* const* d_in4, uint32_t log_size, uint32_t* const* d_out4,
                                   uint32_t* lambda_out, void* stream, char* err, size_t err_len) {
  STWO_ARG_CHECK(d_in4 && d_out4 && lambda_out, "null argument");
  STWO_ARG_CHECK(log_size <= 30, "bad log size %u", log_size);
  cudaStream_t s = as_stream(stream);
  uint64_t n = 1ull << log_size;
  uint64_t range = n / 16, half_a = range / 2;
  uint64_t split_sum = 16 * half_a, end_sum = 16 * range;
  uint64_t split_apply = 16 * (((n + 15) / 16) / 2);
  Cols4 in{{d_in4[0], d_in4[1], d_in4[2], d_in4[3]}};
  Cols4W out{{d_out4[0], d_out4[1], d_out4[2], d_out4[3]}};
  unsigned blocks = grid_for(std::max<uint64_t>(end_sum, 1), 256);
  uint32_t* scratch = nullptr;
  STWO_CUDA_TRY(cudaMallocAsync(&scratch, (blocks * 4 + 4) * sizeof(uint32_t), s));
  uint32_t* lam = scratch + blocks * 4;
  decompose_sums_kernel<<<blocks, 256, 0, s>>>(in, split_sum, end_sum, scratch);
  STWO_CHECK_LAUNCH();
  decompose_finish_kernel<<<1, 32, 0, s>>>(scratch, blocks, m31_inv(m31_reduce_u32((uint32_t)n)), lam);
  STWO_CHECK_LAUNCH();
  decompose_apply_kernel<<<grid_for(n, 256), 256, 0, s>>>(in, n, split_apply, lam, out);
  STWO_CHECK_LAUNCH();
  STWO_CUDA_TRY(cudaMemcpyAsync(lambda_out, lam, 16, cudaMemcpyDeviceToHost, s));
  STWO_CUDA_TRY(cudaFreeAsync(scratch, s));
  STWO_CUDA_TRY(cudaStreamSynchronize(s));
  return ok(err, err_len);
}

// ---------------------------------------------------------------------------
// decompose without allocation.
//
// Some callers cannot let a library allocate device memory while they run: a
// prover service whose admission controller has already divided the GPU's
// memory between requests (a cudaMalloc from inside a request could fail
// under that pressure or bypass the accounting), or a host runtime that owns
// every device allocation itself.  stwo_b200_decompose_noalloc gives them
// FriOps::decompose with its reduction scratch in the fixed array below
// instead of cudaMallocAsync.
//
// The array is a file-scope __device__ symbol: every GPU that loads this
// library holds its kNoAllocScratchWords words until the process exits.  In
// host code the symbol's name is a host-side stand-in, not a device address,
// so the address is fetched once per device with cudaGetSymbolAddress (with
// that device current) and cached; the first call on a device does that
// set-up.  The cache is keyed by device ordinal: a cudaDeviceReset between
// calls (which recreates the device's context and may move the array) is not
// supported.  All calls on a device share
// the array and it keeps the last call's contents: each call overwrites every
// word it reads, and calls that overlap on the GPU (different streams, or
// host threads without ordering) race on it.
namespace stwo_b200 {

constexpr uint32_t kNoAllocBlocks = 148 * 8;                  // reduction blocks (one wave)
constexpr uint32_t kNoAllocScratchWords = kNoAllocBlocks * 4 + 4;  // partials + lambda: 18,960 bytes
// A launch of at most kNoAllocBlocks blocks writes 4 partial words per block,
// and lambda sits after the last block's partials.
static_assert(kNoAllocScratchWords >= kNoAllocBlocks * 4 + 4, "partials and lambda must fit the fixed array");
static __device__ __align__(256) uint32_t g_decompose_scratch[kNoAllocScratchWords];

static uint32_t* noalloc_scratch(int device, char* err, size_t err_len, int* rc) {
  static std::atomic<uint32_t*> cache[64];
  *rc = STWO_B200_OK;
  if (device < 0 || device >= 64) {
    *rc = set_err(err, err_len, STWO_B200_ESTATE, "device ordinal %d out of range", device);
    return nullptr;
  }
  uint32_t* p = cache[device].load(std::memory_order_acquire);
  if (p) return p;
  void* addr = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&addr, g_decompose_scratch);
  if (e != cudaSuccess) {
    *rc = set_err(err, err_len, STWO_B200_ECUDA, "cudaGetSymbolAddress(decompose scratch): %s",
                  cudaGetErrorString(e));
    return nullptr;
  }
  p = static_cast<uint32_t*>(addr);
  cache[device].store(p, std::memory_order_release);
  return p;
}

}  // namespace stwo_b200

extern "C" int stwo_b200_decompose_noalloc(const uint32_t* const* d_in4, uint32_t log_size, uint32_t* const* d_out4,
                                           uint32_t* lambda_out, void* stream, char* err, size_t err_len) {
  STWO_ARG_CHECK(d_in4 && d_out4 && lambda_out, "null argument");
  STWO_ARG_CHECK(log_size <= 30, "log size %u exceeds the maximum of 30 (2^30 elements per coordinate)", log_size);
  cudaStream_t s = as_stream(stream);
  int device = 0;
  STWO_CUDA_TRY(cudaGetDevice(&device));
  int rc;
  uint32_t* scratch = noalloc_scratch(device, err, err_len, &rc);
  if (!scratch) return rc;
  uint64_t n = 1ull << log_size;
  uint64_t range = n / 16, half_a = range / 2;
  uint64_t split_sum = 16 * half_a, end_sum = 16 * range;
  uint64_t split_apply = 16 * (((n + 15) / 16) / 2);
  // At most kNoAllocBlocks blocks, so the partials and lambda fit the array
  // (static_assert above).
  unsigned blocks = (unsigned)std::min<uint64_t>(std::max<uint64_t>((end_sum + 255) / 256, 1), kNoAllocBlocks);
  uint32_t* lam = scratch + blocks * 4;
  Cols4 in{{d_in4[0], d_in4[1], d_in4[2], d_in4[3]}};
  Cols4W out{{d_out4[0], d_out4[1], d_out4[2], d_out4[3]}};
  // Every partial word read below is written first by decompose_sums_kernel
  // (one word per block and coordinate, zero sums included), so no clearing
  // is needed between calls.
  decompose_sums_kernel<<<blocks, 256, 0, s>>>(in, split_sum, end_sum, scratch);
  STWO_CHECK_LAUNCH();
  decompose_finish_kernel<<<1, 32, 0, s>>>(scratch, blocks, m31_inv(m31_reduce_u32((uint32_t)n)), lam);
  STWO_CHECK_LAUNCH();
  decompose_apply_kernel<<<grid_for(n, 256), 256, 0, s>>>(in, n, split_apply, lam, out);
  STWO_CHECK_LAUNCH();
  STWO_CUDA_TRY(cudaMemcpyAsync(lambda_out, lam, 16, cudaMemcpyDeviceToHost, s));
  STWO_CUDA_TRY(cudaStreamSynchronize(s));
  return ok(err, err_len);
}
