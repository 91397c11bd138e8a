// PolyOps::precompute_twiddles on the device.
//
// Layout (crates/stwo/src/prover/backend/cpu/circle.rs:294-311): for a root
// coset of log size R the tree holds, for k = 0..R-1, the x coordinates of the
// first half of coset_k = root.repeated_double(k) in bit-reversed order, at
// [2^R - 2^(R-k), 2^R - 2^(R-k-1)), then a trailing 1.  itwiddles are the
// inverses.  One thread per entry: the coset point is a product of
// precomputed generator powers GEN^(2^b) selected by the bits of its index.
#include <cuda_runtime.h>

#include "common.cuh"
#include "field.cuh"

namespace stwo_b200 {

struct GenPowers {
  uint32_t x[31], y[31];  // GEN^(2^b), b = 0..30
};

__host__ __device__ __forceinline__ void point_add(uint32_t& x, uint32_t& y, uint32_t x2, uint32_t y2) {
  uint32_t nx = m31_sub(m31_mul(x, x2), m31_mul(y, y2));
  uint32_t ny = m31_add(m31_mul(x, y2), m31_mul(y, x2));
  x = nx;
  y = ny;
}

__global__ void twiddle_tree_kernel(GenPowers g, uint64_t initial_index, uint32_t R, uint32_t* tw, uint32_t* itw) {
  uint64_t total = 1ull << R;
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < total; e += (uint64_t)gridDim.x * blockDim.x) {
    if (e == total - 1) {
      tw[e] = 1;
      itw[e] = 1;
      continue;
    }
    uint64_t r = total - e;  // in [2, 2^R]
    uint32_t lg = 64 - __clzll(r - 1);  // ceil(log2(r))
    uint32_t k = R - lg;                // level
    uint64_t j = e - (total - (1ull << lg));
    uint32_t half_log = lg - 1;  // log2 of entries in this level
    uint64_t m = half_log ? (__brevll(j) >> (64 - half_log)) : 0;
    uint64_t idx = ((initial_index << k) + (m << (31 - lg))) & ((1ull << 31) - 1);
    uint32_t x = 1, y = 0;
#pragma unroll 1
    for (int b = 0; b < 31; b++)
      if ((idx >> b) & 1) point_add(x, y, g.x[b], g.y[b]);
    tw[e] = x;
    itw[e] = m31_inv(x);
  }
}

static GenPowers gen_powers() {
  GenPowers g;
  uint32_t x = 2, y = 1268011823u;  // M31_CIRCLE_GEN, crates/stwo/src/core/circle.rs:202-205
  for (int b = 0; b < 31; b++) {
    g.x[b] = x;
    g.y[b] = y;
    point_add(x, y, x, y);
  }
  return g;
}

}  // namespace stwo_b200

using namespace stwo_b200;

extern "C" int stwo_b200_precompute_twiddles(uint64_t initial_index, uint32_t log_size, uint32_t* d_twiddles,
                                             uint32_t* d_itwiddles, void* stream, char* err, size_t err_len) {
  STWO_ARG_CHECK(log_size <= 30, "coset log size %u > 30", log_size);
  STWO_ARG_CHECK(d_twiddles && d_itwiddles, "null output");
  static const GenPowers g = gen_powers();
  uint64_t total = 1ull << log_size;
  uint32_t threads = 256;
  uint64_t blocks = (total + threads - 1) / threads;
  if (blocks > 148 * 64) blocks = 148 * 64;
  twiddle_tree_kernel<<<(unsigned)blocks, threads, 0, as_stream(stream)>>>(g, initial_index & ((1ull << 31) - 1),
                                                                           log_size, d_twiddles, d_itwiddles);
  STWO_CHECK_LAUNCH();
  return ok(err, err_len);
}
