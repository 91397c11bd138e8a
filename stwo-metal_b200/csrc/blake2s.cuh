// Blake2s-256 compression for sm_100a (RFC 7693), one compression per thread.
//
// The message block lives in 16 registers; the round loop is fully unrolled so
// every SIGMA index is a compile-time constant.  Rotations by 16 and 8 are byte
// permutes, by 12 and 7 funnel shifts.  Two forms of the same function:
//  - blake2s_compress (throughput): XORs and rotations keep the integer ALU
//    pipe busy, so the additions go to the multiply-add pipe: x + y is written
//    x * kB2sOne + y with kB2sOne a constant-bank 1 that the compiler cannot
//    fold.  About 20% more compressions per second on a full GPU.
//  - blake2s_compress_lat (latency): a + b + m as one three-input add, the
//    shortest dependency chain, for the one-CTA tree tops and channel steps.
// This is the hash of crate blake2 0.10.6 as called by stwo
// (crates/stwo/src/core/vcs/blake2_hash.rs:84-94).
#pragma once
#include <cstdint>

namespace stwo_b200 {

__device__ __constant__ static const uint32_t kBlake2sIV[8] = {0x6A09E667u, 0xBB67AE85u, 0x3C6EF372u,
                                                                0xA54FF53Au, 0x510E527Fu, 0x9B05688Cu,
                                                                0x1F83D9ABu, 0x5BE0CD19u};

__device__ __forceinline__ uint32_t rotr16(uint32_t x) { return __byte_perm(x, x, 0x1032); }
__device__ __forceinline__ uint32_t rotr8(uint32_t x) { return __byte_perm(x, x, 0x0321); }
__device__ __forceinline__ uint32_t rotr12(uint32_t x) { return __funnelshift_r(x, x, 12); }
__device__ __forceinline__ uint32_t rotr7(uint32_t x) { return __funnelshift_r(x, x, 7); }

// 1, but not a compile-time constant (see the header comment).
__device__ __constant__ uint32_t kB2sOne = 1;
__device__ __forceinline__ uint32_t madd(uint32_t x, uint32_t y) { return x * kB2sOne + y; }

#define STWO_B2S_G(a, b, c, d, x, y)      \
  do {                                    \
    v[a] = madd(v[b], madd((x), v[a]));   \
    v[d] = rotr16(v[d] ^ v[a]);           \
    v[c] = madd(v[d], v[c]);              \
    v[b] = rotr12(v[b] ^ v[c]);           \
    v[a] = madd(v[b], madd((y), v[a]));   \
    v[d] = rotr8(v[d] ^ v[a]);            \
    v[c] = madd(v[d], v[c]);              \
    v[b] = rotr7(v[b] ^ v[c]);            \
  } while (0)

#define STWO_B2S_G_LAT(a, b, c, d, x, y) \
  do {                                   \
    v[a] = v[a] + v[b] + (x);            \
    v[d] = rotr16(v[d] ^ v[a]);          \
    v[c] = v[c] + v[d];                  \
    v[b] = rotr12(v[b] ^ v[c]);          \
    v[a] = v[a] + v[b] + (y);            \
    v[d] = rotr8(v[d] ^ v[a]);           \
    v[c] = v[c] + v[d];                  \
    v[b] = rotr7(v[b] ^ v[c]);           \
  } while (0)

#define STWO_B2S_ROUND(G, s0, s1, s2, s3, s4, s5, s6, s7, s8, s9, s10, s11, s12, s13, s14, s15) \
  do {                                                                                          \
    G(0, 4, 8, 12, m[s0], m[s1]);                                                               \
    G(1, 5, 9, 13, m[s2], m[s3]);                                                               \
    G(2, 6, 10, 14, m[s4], m[s5]);                                                              \
    G(3, 7, 11, 15, m[s6], m[s7]);                                                              \
    G(0, 5, 10, 15, m[s8], m[s9]);                                                              \
    G(1, 6, 11, 12, m[s10], m[s11]);                                                            \
    G(2, 7, 8, 13, m[s12], m[s13]);                                                             \
    G(3, 4, 9, 14, m[s14], m[s15]);                                                             \
  } while (0)

#define STWO_B2S_COMPRESS(G)                                                     \
  uint32_t v[16];                                                                \
  _Pragma("unroll") for (int i = 0; i < 8; i++) v[i] = h[i];                     \
  v[8] = 0x6A09E667u;                                                            \
  v[9] = 0xBB67AE85u;                                                            \
  v[10] = 0x3C6EF372u;                                                           \
  v[11] = 0xA54FF53Au;                                                           \
  v[12] = 0x510E527Fu ^ t;                                                       \
  v[13] = 0x9B05688Cu; /* high word of t is zero for every input here */         \
  v[14] = last ? ~0x1F83D9ABu : 0x1F83D9ABu;                                     \
  v[15] = 0x5BE0CD19u;                                                           \
  STWO_B2S_ROUND(G, 0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15);       \
  STWO_B2S_ROUND(G, 14, 10, 4, 8, 9, 15, 13, 6, 1, 12, 0, 2, 11, 7, 5, 3);       \
  STWO_B2S_ROUND(G, 11, 8, 12, 0, 5, 2, 15, 13, 10, 14, 3, 6, 7, 1, 9, 4);       \
  STWO_B2S_ROUND(G, 7, 9, 3, 1, 13, 12, 11, 14, 2, 6, 5, 10, 4, 0, 15, 8);       \
  STWO_B2S_ROUND(G, 9, 0, 5, 7, 2, 4, 10, 15, 14, 1, 11, 12, 6, 8, 3, 13);       \
  STWO_B2S_ROUND(G, 2, 12, 6, 10, 0, 11, 8, 3, 4, 13, 7, 5, 15, 14, 1, 9);       \
  STWO_B2S_ROUND(G, 12, 5, 1, 15, 14, 13, 4, 10, 0, 7, 6, 3, 9, 2, 8, 11);       \
  STWO_B2S_ROUND(G, 13, 11, 7, 14, 12, 1, 3, 9, 5, 0, 15, 4, 8, 6, 2, 10);       \
  STWO_B2S_ROUND(G, 6, 15, 14, 9, 11, 3, 0, 8, 12, 2, 13, 7, 1, 4, 10, 5);       \
  STWO_B2S_ROUND(G, 10, 2, 8, 4, 7, 6, 1, 5, 15, 11, 9, 14, 3, 12, 13, 0);       \
  _Pragma("unroll") for (int i = 0; i < 8; i++) h[i] ^= v[i] ^ v[i + 8];

// h <- compress(h, m, t, last).  t = total bytes hashed including this block.
__device__ __forceinline__ void blake2s_compress(uint32_t h[8], const uint32_t m[16], uint32_t t, bool last) {
  STWO_B2S_COMPRESS(STWO_B2S_G)
}
__device__ __forceinline__ void blake2s_compress_lat(uint32_t h[8], const uint32_t m[16], uint32_t t, bool last) {
  STWO_B2S_COMPRESS(STWO_B2S_G_LAT)
}

// Initial chaining value for a 32-byte unkeyed digest.
__device__ __forceinline__ void blake2s_init(uint32_t h[8]) {
  h[0] = 0x6A09E667u ^ 0x01010020u;
  h[1] = 0xBB67AE85u;
  h[2] = 0x3C6EF372u;
  h[3] = 0xA54FF53Au;
  h[4] = 0x510E527Fu;
  h[5] = 0x9B05688Cu;
  h[6] = 0x1F83D9ABu;
  h[7] = 0x5BE0CD19u;
}

}  // namespace stwo_b200
