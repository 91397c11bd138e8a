// Row-wise exact M31/QM31 accumulation helpers shared by the prover's row
// kernels (composition, quotients, OODS sampling) and the stand-alone
// QuotientOps / AccumulationOps / PolyOps::eval_at_point entry points.
#pragma once
#include <cstdint>

#include "field.cuh"

namespace stwo_b200 {

// Exact M31 dot products: products of words <= P with canonical weights
// (<= P (P - 1)) are summed in 64 bits and folded with 2^31 = 1 (mod P) every
// four terms (a folded value is < 2^33 + 2^31, and that plus four products
// stays below 2^64), then reduced once to the canonical value.  The residue is exact, so the result equals the
// canonical value SimdBackend's reduced-per-operation arithmetic produces.
__device__ __forceinline__ uint64_t fold64(uint64_t x) { return (x & M31_P) + (x >> 31); }  // < 2^34
__device__ __forceinline__ uint32_t reduce_acc(uint64_t x) {
  x = fold64(fold64(x));  // < P + 8
  uint32_t y = (uint32_t)x;
  return y >= M31_P ? y - M31_P : y;
}
struct acc4 {
  uint64_t a, b, c, d;
};
__device__ __forceinline__ void acc4_mad(acc4& s, const qm31& w, uint32_t v) {
  s.a += (uint64_t)w.a * v;
  s.b += (uint64_t)w.b * v;
  s.c += (uint64_t)w.c * v;
  s.d += (uint64_t)w.d * v;
}
__device__ __forceinline__ void acc4_fold(acc4& s) {
  s.a = fold64(s.a);
  s.b = fold64(s.b);
  s.c = fold64(s.c);
  s.d = fold64(s.d);
}
__device__ __forceinline__ qm31 acc4_reduce(const acc4& s) {
  return {reduce_acc(s.a), reduce_acc(s.b), reduce_acc(s.c), reduce_acc(s.d)};
}

__device__ __forceinline__ uint4 ldg4(const uint32_t* p) { return __ldg(reinterpret_cast<const uint4*>(p)); }
__device__ __forceinline__ uint32_t u4get(const uint4& v, int r) {
  return r == 0 ? v.x : r == 1 ? v.y : r == 2 ? v.z : v.w;
}

// Polynomial values at one secure point: sum_j coeff_j * w_j where
// w_j = prod over set bits b of j of f_b, f = [y, x, pi(x), pi^2(x), ...]
// (the coefficient fold of prover/backend/cpu/circle.rs:82-99), w_j =
// w_hi[j >> h] * w_lo[j & (2^h - 1)]; see oods_eval_kernel.
constexpr int kMaxPolys = 1024;
struct PolyTable {
  const uint32_t* p[kMaxPolys];
};

}  // namespace stwo_b200
