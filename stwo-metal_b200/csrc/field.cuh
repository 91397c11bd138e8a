// M31 / CM31 / QM31 device arithmetic for sm_100a.
//
// Values are u32 words in [0, P].  add / sub use the same min-based reduction
// as stwo's packed SimdBackend (crates/stwo/src/prover/backend/simd/m31.rs:
// 150-162, 253-265), so a word equal to P propagates exactly as it does there;
// mul is a full 31-bit Mersenne reduction of the 62-bit product and always
// returns a canonical value (like simd/m31.rs:579-626 mul_doubled).
#pragma once
#include <cstdint>

namespace stwo_b200 {

constexpr uint32_t M31_P = 0x7fffffffu;

__host__ __device__ __forceinline__ uint32_t m31_add(uint32_t a, uint32_t b) {
  uint32_t c = a + b;
  uint32_t d = c - M31_P;
  return c < d ? c : d;
}
__host__ __device__ __forceinline__ uint32_t m31_sub(uint32_t a, uint32_t b) {
  uint32_t c = a - b;
  uint32_t d = c + M31_P;
  return d < c ? d : c;
}
// Scalar negation (core/fields/m31.rs Neg): 0 -> 0.
__host__ __device__ __forceinline__ uint32_t m31_neg(uint32_t a) {
  uint32_t c = M31_P - a;
  return c >= M31_P ? c - M31_P : c;
}
__host__ __device__ __forceinline__ uint32_t m31_mul(uint32_t a, uint32_t b) {
  uint64_t x = (uint64_t)a * b;
  uint32_t lo = (uint32_t)x & M31_P;
  uint32_t hi = (uint32_t)(x >> 31);
  return m31_add(lo, hi);
}
__host__ __device__ __forceinline__ uint32_t m31_sqr(uint32_t a) { return m31_mul(a, a); }
__host__ __device__ inline uint32_t m31_pow(uint32_t a, uint64_t e) {
  uint32_t r = 1;
  while (e) {
    if (e & 1) r = m31_mul(r, a);
    a = m31_mul(a, a);
    e >>= 1;
  }
  return r;
}
__host__ __device__ inline uint32_t m31_inv(uint32_t a) { return m31_pow(a, (uint64_t)M31_P - 2); }
// M31::reduce of a u32 (core/fields/m31.rs:58-60 restricted to 32-bit input).
__host__ __device__ __forceinline__ uint32_t m31_reduce_u32(uint32_t v) {
  uint32_t r = (v & M31_P) + (v >> 31);
  return r >= M31_P ? r - M31_P : r;
}

struct cm31 {
  uint32_t a, b;
};
__host__ __device__ __forceinline__ cm31 cm31_add(cm31 x, cm31 y) { return {m31_add(x.a, y.a), m31_add(x.b, y.b)}; }
__host__ __device__ __forceinline__ cm31 cm31_sub(cm31 x, cm31 y) { return {m31_sub(x.a, y.a), m31_sub(x.b, y.b)}; }
__host__ __device__ __forceinline__ cm31 cm31_mul(cm31 x, cm31 y) {
  return {m31_sub(m31_mul(x.a, y.a), m31_mul(x.b, y.b)), m31_add(m31_mul(x.a, y.b), m31_mul(x.b, y.a))};
}

// QM31 = (a + b i) + (c + d i) u, u^2 = 2 + i (core/fields/qm31.rs:14-88).
struct qm31 {
  uint32_t a, b, c, d;
};
__host__ __device__ __forceinline__ qm31 qm31_add(qm31 x, qm31 y) {
  return {m31_add(x.a, y.a), m31_add(x.b, y.b), m31_add(x.c, y.c), m31_add(x.d, y.d)};
}
__host__ __device__ __forceinline__ qm31 qm31_sub(qm31 x, qm31 y) {
  return {m31_sub(x.a, y.a), m31_sub(x.b, y.b), m31_sub(x.c, y.c), m31_sub(x.d, y.d)};
}
__host__ __device__ __forceinline__ qm31 qm31_mul_m31(qm31 x, uint32_t m) {
  return {m31_mul(x.a, m), m31_mul(x.b, m), m31_mul(x.c, m), m31_mul(x.d, m)};
}
__host__ __device__ __forceinline__ qm31 qm31_mul(qm31 x, qm31 y) {
  cm31 x0{x.a, x.b}, x1{x.c, x.d}, y0{y.a, y.b}, y1{y.c, y.d};
  cm31 ac = cm31_mul(x0, y0);
  cm31 bd = cm31_mul(x1, y1);
  // R * bd with R = 2 + i: (2bd.a - bd.b) + (2bd.b + bd.a) i
  cm31 rbd{m31_sub(m31_add(bd.a, bd.a), bd.b), m31_add(m31_add(bd.b, bd.b), bd.a)};
  cm31 l = cm31_add(ac, rbd);
  cm31 r = cm31_add(cm31_mul(x0, y1), cm31_mul(x1, y0));
  return {l.a, l.b, r.a, r.b};
}

}  // namespace stwo_b200

namespace stwo_b200 {

// ---- host/device helpers beyond the kernels' hot arithmetic ----
__host__ __device__ __forceinline__ bool qm31_eq(qm31 x, qm31 y) {
  return x.a == y.a && x.b == y.b && x.c == y.c && x.d == y.d;
}
__host__ __device__ __forceinline__ qm31 qm31_from_m31(uint32_t v) { return {v, 0, 0, 0}; }
__host__ __device__ __forceinline__ qm31 qm31_one() { return {1, 0, 0, 0}; }
__host__ __device__ __forceinline__ qm31 qm31_zero() { return {0, 0, 0, 0}; }
__host__ __device__ __forceinline__ qm31 qm31_neg(qm31 x) { return {m31_neg(x.a), m31_neg(x.b), m31_neg(x.c), m31_neg(x.d)}; }
// Complex conjugate over CM31: (x0 + x1 u) -> (x0 - x1 u) (core/fields/mod.rs:413-415).
__host__ __device__ __forceinline__ qm31 qm31_conj(qm31 x) { return {x.a, x.b, m31_neg(x.c), m31_neg(x.d)}; }
__host__ __device__ __forceinline__ cm31 cm31_neg(cm31 x) { return {m31_neg(x.a), m31_neg(x.b)}; }
__host__ __device__ inline cm31 cm31_inv(cm31 x) {  // (a - bi) / (a^2 + b^2)
  uint32_t d = m31_inv(m31_add(m31_sqr(x.a), m31_sqr(x.b)));
  return cm31_mul({x.a, m31_neg(x.b)}, {d, 0});
}
__host__ __device__ inline qm31 qm31_inv(qm31 x) {  // core/fields/qm31.rs:125-133
  cm31 x0{x.a, x.b}, x1{x.c, x.d};
  cm31 b2 = cm31_mul(x1, x1);
  cm31 ib2{m31_neg(b2.b), b2.a};
  cm31 denom = cm31_sub(cm31_mul(x0, x0), cm31_add(cm31_add(b2, b2), ib2));
  cm31 di = cm31_inv(denom);
  cm31 r0 = cm31_mul(x0, di), r1 = cm31_mul(cm31_neg(x1), di);
  return {r0.a, r0.b, r1.a, r1.b};
}
__host__ __device__ __forceinline__ qm31 qm31_mul_cm31(qm31 x, cm31 c) {
  cm31 a = cm31_mul({x.a, x.b}, c), b = cm31_mul({x.c, x.d}, c);
  return {a.a, a.b, b.a, b.b};
}

// Circle points over M31 and QM31.
struct cpoint {
  uint32_t x, y;
};
__host__ __device__ __forceinline__ cpoint cpoint_add(cpoint p, cpoint q) {
  return {m31_sub(m31_mul(p.x, q.x), m31_mul(p.y, q.y)), m31_add(m31_mul(p.x, q.y), m31_mul(p.y, q.x))};
}
struct spoint {
  qm31 x, y;
};
__host__ __device__ inline spoint spoint_add(spoint p, spoint q) {
  return {qm31_sub(qm31_mul(p.x, q.x), qm31_mul(p.y, q.y)), qm31_add(qm31_mul(p.x, q.y), qm31_mul(p.y, q.x))};
}
__host__ __device__ inline qm31 qm31_double_x(qm31 x) {
  qm31 s = qm31_mul(x, x);
  return qm31_sub(qm31_add(s, s), qm31_one());
}
__host__ __device__ inline spoint spoint_repeated_double(spoint p, uint32_t n) {
  for (uint32_t i = 0; i < n; i++) p = spoint_add(p, p);
  return p;
}

// Circle point of index i (GEN^i, GEN = M31_CIRCLE_GEN of crates/stwo/src/core/circle.rs:202-205).
__host__ __device__ inline cpoint index_to_cpoint(uint64_t idx) {
  cpoint g{2u, 1268011823u}, r{1u, 0u};
  idx &= (1ull << 31) - 1;
  for (int b = 0; b < 31; b++) {
    if ((idx >> b) & 1) r = cpoint_add(r, g);
    g = cpoint_add(g, g);
  }
  return r;
}

}  // namespace stwo_b200
