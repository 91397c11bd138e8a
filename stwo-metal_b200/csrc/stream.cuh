// Column streaming through shared memory with TMA bulk copies (sm_100a).
//
// Row-wise kernels of the prover (composition, quotients) combine ~100
// column-major columns at every row.  A block owns a tile of ROWS consecutive
// rows and walks the columns in groups of G; one elected thread issues one
// `cp.async.bulk` global->shared copy per column segment (ROWS * 4 bytes,
// 16-byte aligned) into an S-stage ring, each stage completing on its own
// mbarrier.  All threads consume the stages in order, so DRAM traffic for the
// next S-1 groups is in flight while the current group is combined.  No
// multicast: every copy lands in the issuing CTA's own shared memory.
//
// Every wait is bounded: a stage that does not complete within kStreamSpin
// polls sets *err = 1 and the whole block leaves (uniformly, decided with a
// barrier reduction) after a second bounded wait for its copies in flight.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace stwo_b200 {

constexpr uint32_t kStreamSpin = 1u << 22;  // try_wait polls before giving up

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_addr(dst)),
               "l"(src), "r"(bytes), "r"(smem_addr(bar))
               : "memory");
}
// Waits for phase `parity` of `bar`; false when kStreamSpin polls ran out.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  const uint32_t a = smem_addr(bar);
  for (uint32_t it = 0; it < kStreamSpin; it++) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// S-stage ring of column groups for a persistent block that walks tiles
// blockIdx.x, blockIdx.x + gridDim.x, ... (ROWS rows each).  Groups are
// numbered across tiles (gg = local tile * n_groups + g), so the copies of the
// next tile's first groups are in flight while the current tile finishes.
// Usage, by every thread of the block:
//   ColumnRing<G, S, ROWS> ring(buf, bars, n_cols, n_tiles);  // then a barrier
//   ring.start(col);                                           // thread 0 issues
//   for (t = 0; t < ring.my_tiles; t++)
//     for (g = 0; g < ring.n_groups; g++) {
//       gg = t * ring.n_groups + g;
//       if (!ring.wait(gg, err)) return;                       // uniform
//       ... read ring.seg(gg, k) for k < ring.cols_in(g) ...
//       ring.release(gg, col);                                  // barrier + refill
//     }
template <int G, int S, int ROWS>
struct ColumnRing {
  uint32_t* buf;  // S * G * ROWS words, 16-byte aligned
  uint64_t* bars;
  uint32_t n_cols, n_groups, my_tiles, total;
  __device__ ColumnRing(uint32_t* b, uint64_t* m, uint32_t n, uint32_t n_tiles)
      : buf(b), bars(m), n_cols(n), n_groups((n + G - 1) / G) {
    my_tiles = blockIdx.x < n_tiles ? (n_tiles - blockIdx.x + gridDim.x - 1) / gridDim.x : 0;
    total = my_tiles * n_groups;
    if (threadIdx.x == 0) {
      for (int st = 0; st < S; st++) mbar_init(bars + st, 1);
      mbar_fence_init();
    }
  }
  __device__ __forceinline__ uint64_t tile_row0(uint32_t t) const {
    return (uint64_t)(blockIdx.x + t * gridDim.x) * ROWS;
  }
  __device__ __forceinline__ uint32_t cols_in(uint32_t g) const {
    const uint32_t c0 = g * G;
    return n_cols - c0 < (uint32_t)G ? n_cols - c0 : (uint32_t)G;
  }
  __device__ __forceinline__ const uint32_t* seg(uint32_t gg, uint32_t k) const {
    return buf + ((size_t)(gg % S) * G + k) * ROWS;
  }
  template <typename ColFn>
  __device__ __forceinline__ void issue(uint32_t gg, ColFn col) {
    const int st = gg % S;
    const uint32_t g = gg % n_groups;
    const uint64_t r0 = tile_row0(gg / n_groups);
    const uint32_t nc = cols_in(g);
    mbar_expect_tx(bars + st, nc * ROWS * 4u);
    for (uint32_t k = 0; k < nc; k++)
      bulk_load(buf + ((size_t)st * G + k) * ROWS, col(g * G + k) + r0, ROWS * 4u, bars + st);
  }
  template <typename ColFn>
  __device__ __forceinline__ void start(ColFn col) {
    if (threadIdx.x == 0)
      for (uint32_t gg = 0; gg < total && gg < (uint32_t)S; gg++) issue(gg, col);
  }
  // Bounded wait for group gg; false (uniformly, with *err set and the copies
  // in flight drained) when it timed out.  Thread 0 alone polls the mbarrier
  // (its acquire makes the bulk-copied bytes visible to it) and the block
  // barrier that follows orders them before every other thread's reads, so
  // the other warps sleep at the barrier instead of spending issue slots.
  __device__ __forceinline__ bool wait(uint32_t gg, uint32_t* err) {
    bool ok = true;
    if (threadIdx.x == 0) ok = mbar_wait(bars + gg % S, (gg / S) & 1);
    if (__syncthreads_or(!ok)) {
      if (threadIdx.x == 0) {
        atomicExch(err, 1u);
        for (uint32_t h = gg; h < total && h < gg + S; h++) (void)mbar_wait(bars + h % S, (h / S) & 1);
      }
      __syncthreads();
      return false;
    }
    return true;
  }
  template <typename ColFn>
  __device__ __forceinline__ void release(uint32_t gg, ColFn col) {
    __syncthreads();  // stage of gg fully read before it is refilled
    if (threadIdx.x == 0 && gg + S < total) issue(gg + S, col);
  }
};

}  // namespace stwo_b200
