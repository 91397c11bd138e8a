// Column streaming through shared memory with TMA bulk copies (sm_100a).
//
// Row-wise kernels of the prover (composition, quotients) combine ~100
// column-major columns at every row.  A block owns a tile of ROWS consecutive
// rows and walks the columns in groups of G; a producer thread issues one
// `cp.async.bulk` global->shared copy per column segment (ROWS * 4 bytes,
// 16-byte aligned) into an S-stage ring, each stage completing on its own
// mbarrier, while the consumer warps combine the stages in order.  DRAM
// traffic for the next groups is in flight while the current group is
// combined.  No multicast: every copy lands in the issuing CTA's own shared
// memory.
//
// Every wait is bounded: a consumer's wait for a stage by the pipe's `spin`
// polls (a kernel argument, kStreamSpin by default), every producer wait by
// kStreamSpin.  A wait that runs out sets an error word and the block leaves
// after its copies in flight have landed.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/stwo_b200.h"

namespace stwo_b200 {

constexpr uint32_t kStreamSpin = STWO_B200_STREAM_SPIN_DEFAULT;  // try_wait polls before giving up

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

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// Warp-specialised column ring: threads [0, CONSUMERS) consume, lane 0 of the
// warp after them produces, and no block barrier is taken per group.
// Stage st has a "full" mbarrier (the producer's expect_tx arrival plus the
// copied bytes) and an "empty" one (one arrival per consumer thread after it
// has read the stage); the producer refills a stage once its empty phase
// completes.  Each stage also carries a small header the producer writes
// before arming the first group of a tile (per-tile constants such as a
// domain point), read by consumers while they hold that stage.
//
// Failure: a wait that runs out of polls, or sees another thread's abort,
// sets *err = 1 and the shared abort word; consumers then return, the
// producer stops issuing and waits (bounded) for its copies in flight before
// it exits, so no copy lands after the block's shared memory is released.
// Usage (block = CONSUMERS + 32 threads, CONSUMERS % 32 == 0):
//   ColumnPipe<G, S, ROWS, C> pipe(buf, bars, n_cols, n_tiles, spin);   // then one barrier
//   if (threadIdx.x >= C) { if (threadIdx.x == C) pipe.produce(col, head, err); return; }
//   for (t ...) for (g ...) { gg = t * n_groups + g;
//     if (!pipe.wait(gg, err)) return;  ... read pipe.seg(gg, k) ...;  pipe.release(gg); }
constexpr uint32_t kPipeHeaderWords = 4;
template <int G, int S, int ROWS, int CONSUMERS>
struct ColumnPipe {
  static_assert(CONSUMERS % 32 == 0, "the producer warp follows whole consumer warps");
  uint32_t* buf;     // S * G * ROWS words, 16-byte aligned
  uint64_t* full;    // S mbarriers
  uint64_t* empty;   // S mbarriers
  uint32_t* header;  // S * kPipeHeaderWords words
  volatile uint32_t* abort_word;
  uint32_t n_cols, n_groups, my_tiles, total;
  uint32_t spin;  // polls of a consumer's stage wait before it gives up (0: at once)
  // `bars` holds 2 * S mbarriers followed by S * kPipeHeaderWords + 1 words
  // (8-byte aligned shared memory).
  __device__ ColumnPipe(uint32_t* b, uint64_t* bars, uint32_t n, uint32_t n_tiles, uint32_t consumer_spin)
      : buf(b), full(bars), empty(bars + S), n_cols(n), n_groups((n + G - 1) / G), spin(consumer_spin) {
    header = reinterpret_cast<uint32_t*>(bars + 2 * S);
    abort_word = header + S * kPipeHeaderWords;
    my_tiles = blockIdx.x < n_tiles ? (n_tiles - blockIdx.x + gridDim.x - 1) / gridDim.x : 0;
    total = my_tiles * n_groups;
    if (threadIdx.x == 0) {
      for (int st = 0; st < S; st++) {
        mbar_init(full + st, 1);
        mbar_init(empty + st, CONSUMERS);
      }
      *abort_word = 0;
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
  __device__ __forceinline__ const uint32_t* head(uint32_t gg) const {
    return header + (gg % S) * kPipeHeaderWords;
  }
  // Poll of phase `parity`, at most `limit` times, that also gives up when
  // another thread has aborted.
  __device__ __forceinline__ bool poll(uint64_t* bar, uint32_t parity, uint32_t limit) const {
    const uint32_t a = smem_addr(bar);
    for (uint32_t it = 0; it < limit; it++) {
      uint32_t done;
      asm volatile(
          "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
          : "=r"(done)
          : "r"(a), "r"(parity)
          : "memory");
      if (done) return true;
      if ((it & 255) == 255 && *abort_word) return false;
    }
    return false;
  }
  __device__ __forceinline__ void fail(uint32_t* err) const {
    atomicExch(err, 1u);
    *abort_word = 1;
  }
  // Consumer side.
  __device__ __forceinline__ bool wait(uint32_t gg, uint32_t* err) const {
    if (poll(full + gg % S, (gg / S) & 1, spin)) return true;
    fail(err);
    return false;
  }
  __device__ __forceinline__ void release(uint32_t gg) const { mbar_arrive(empty + gg % S); }
  // Producer side (one thread).  head_fn(t, words) fills the header of the
  // stage that carries tile t's first group.
  template <typename ColFn, typename HeadFn>
  __device__ void produce(ColFn col, HeadFn head_fn, uint32_t* err) {
    uint32_t gg = 0;
    for (; gg < total; gg++) {
      const uint32_t st = gg % S;
      if (gg >= (uint32_t)S && !poll(empty + st, (gg / S - 1) & 1, kStreamSpin)) {
        fail(err);
        break;
      }
      if (*abort_word) break;
      const uint32_t g = gg % n_groups;
      const uint32_t t = gg / n_groups;
      if (g == 0) head_fn(t, header + st * kPipeHeaderWords);
      const uint64_t r0 = tile_row0(t);
      const uint32_t nc = cols_in(g);
      mbar_expect_tx(full + st, nc * ROWS * 4u);  // release: orders the header before the phase completes
      for (uint32_t k = 0; k < nc; k++)
        bulk_load(buf + ((size_t)st * G + k) * ROWS, col(g * G + k) + r0, ROWS * 4u, full + st);
    }
    // Copies of the last min(gg, S) groups may still be in flight; older ones
    // were read by every consumer before their stage was re-armed.
    for (uint32_t h = gg > (uint32_t)S ? gg - S : 0; h < gg; h++) (void)mbar_wait(full + h % S, (h / S) & 1);
  }
};

}  // namespace stwo_b200
