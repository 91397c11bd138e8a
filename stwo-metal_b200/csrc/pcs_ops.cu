// The trait methods stwo's generic prover calls beyond the commit and FRI
// operations, as stand-alone entry points (sm_100a):
//
//   QuotientOps::accumulate_numerators / compute_quotients_and_combine
//     (crates/stwo/src/prover/pcs/quotient_ops.rs:22-45; SimdBackend
//     prover/backend/simd/quotients.rs:34-164),
//   AccumulationOps::accumulate / generate_secure_powers / lift_and_accumulate
//     (prover/air/accumulation.rs:127-145; simd/accumulation.rs:13-80),
//   PolyOps::eval_at_point / batch_eval_at_point (prover/poly/circle/ops.rs:44-63;
//     simd/circle.rs:168-230),
//   GrindOps::grind (prover/backend/simd/grind.rs:25-96),
//   ColumnOps<SecureField>::bit_reverse_column (prover/backend/mod.rs:37-39).
//
// Every result is an exact M31/QM31 value.  All inputs that these operations
// combine are canonical or reduce to canonical values through a multiply (the
// only place a word equal to P could survive is the first column of
// lift_and_accumulate and the add of accumulate, which use SimdBackend's own
// min-form add), so the order of the exact sums does not change a bit.  The
// OODS sampling and the grind of the Wide-Fibonacci prover run the same
// kernels (pcs.hpp).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "channel.hpp"
#include "common.cuh"
#include "field.cuh"
#include "pcs.hpp"
#include "rowops.cuh"

namespace stwo_b200 {

namespace {

struct Col4 {
  uint32_t* c[4];
};
struct Col4R {
  const uint32_t* c[4];
};

// ------------------------------------------------ accumulate_numerators ----
// out[p] (+)= sum_i c_i * col_i[p] - negb: up to kNumTerms terms per launch.
constexpr int kNumTerms = 256;
struct NumeratorTerms {
  const uint32_t* col[kNumTerms];
  qm31 c[kNumTerms];
};

template <bool VEC>
__global__ void __launch_bounds__(256) numerators_kernel(NumeratorTerms t, uint32_t n_terms, qm31 b_sum, uint64_t n,
                                                         int accumulate, Col4 out) {
  constexpr int R = VEC ? 4 : 1;
  const uint64_t n_units = n / R;
  for (uint64_t u = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; u < n_units;
       u += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t i = u * R;
    acc4 s[R];
#pragma unroll
    for (int r = 0; r < R; r++) s[r] = {0, 0, 0, 0};
    for (uint32_t k = 0; k < n_terms; k++) {
      const qm31 c = t.c[k];
      if (VEC) {
        const uint4 v = ldg4(t.col[k] + i);
#pragma unroll
        for (int r = 0; r < R; r++) acc4_mad(s[r], c, u4get(v, r));
      } else {
        acc4_mad(s[0], c, __ldg(t.col[k] + i));
      }
      if ((k & 3) == 3) {
#pragma unroll
        for (int r = 0; r < R; r++) acc4_fold(s[r]);
      }
    }
#pragma unroll
    for (int r = 0; r < R; r++) {
      qm31 v = acc4_reduce(s[r]);
      if (accumulate)
        v = qm31_add(qm31{out.c[0][i + r], out.c[1][i + r], out.c[2][i + r], out.c[3][i + r]}, v);
      else
        v = qm31_sub(v, b_sum);
      out.c[0][i + r] = v.a;
      out.c[1][i + r] = v.b;
      out.c[2][i + r] = v.c;
      out.c[3][i + r] = v.d;
    }
  }
}

// ------------------------------------------------- lift_and_accumulate -----
// Columns of strictly increasing log size (at most 31); row i of the largest
// reads column k at the lifted index l(i, L - l_k) = ((i >> (r + 1)) << 1) +
// (i & 1) (r > 0), the composition of the per-step lifts of
// simd/accumulation.rs:45-80.  r = c_0, then r = c_k + r, as SimdBackend adds.
constexpr int kMaxLift = 31;
struct LiftCols {
  const uint32_t* c[kMaxLift][4];
  uint32_t shift[kMaxLift];
};

__device__ __forceinline__ uint64_t lift_index(uint64_t i, uint32_t r) {
  return r == 0 ? i : (((i >> (r + 1)) << 1) | (i & 1));
}

__global__ void __launch_bounds__(256) lift_accumulate_kernel(LiftCols t, uint32_t n_cols, uint64_t n, Col4 out) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t j0 = lift_index(i, t.shift[0]);
    qm31 r{__ldg(t.c[0][0] + j0), __ldg(t.c[0][1] + j0), __ldg(t.c[0][2] + j0), __ldg(t.c[0][3] + j0)};
    for (uint32_t k = 1; k < n_cols; k++) {
      const uint64_t j = lift_index(i, t.shift[k]);
      r = qm31_add(qm31{__ldg(t.c[k][0] + j), __ldg(t.c[k][1] + j), __ldg(t.c[k][2] + j), __ldg(t.c[k][3] + j)}, r);
    }
    out.c[0][i] = r.a;
    out.c[1][i] = r.b;
    out.c[2][i] = r.c;
    out.c[3][i] = r.d;
  }
}

// ------------------------------------------ compute_quotients_and_combine --
// q(p_i) = sum_z (lift(num_z)[i] - A_z * p_i.y) * den_z(p_i)^-1 on the
// bit-reversed CanonicCoset(L) circle domain, den_z(p) = (Re z.x - p.x) Im z.y
// - (Re z.y - p.y) Im z.x (CM31; simd/quotients.rs:73-164).  A thread owns
// rows 4u .. 4u + 3, whose points are P0, conj(P0), P1, conj(P1) with
// P0 = H.at(j0), P1 = H.at(j0 + 2^(L-2)), j0 = bitrev_{L-2}(u) (H the half
// coset).  The 4 x n_accs denominators are inverted with one M31 inversion
// (Montgomery's trick over their norms; exact, so equal to each inverse).
constexpr int kMaxAccs = 8;
struct QuotAcc {
  const uint32_t* num[4];
  uint32_t shift;  // L - log size of the partial numerator
  qm31 A;
  cm31 prx, pix, pry, piy;
};
struct QuotAccs {
  QuotAcc a[kMaxAccs];
};
struct QuotDomain {
  cpoint init;             // H.at(0)
  cpoint step_pow[30];     // step * 2^b
  cpoint quarter;          // step * 2^(L-2)
  uint32_t L;
};

__device__ __forceinline__ cm31 quot_den(const QuotAcc& a, cpoint p) {
  return cm31_sub(cm31_mul(cm31_sub(a.prx, cm31{p.x, 0}), a.piy), cm31_mul(cm31_sub(a.pry, cm31{p.y, 0}), a.pix));
}

__global__ void __launch_bounds__(256) quotients_combine_kernel(QuotAccs t, uint32_t n_accs, QuotDomain d,
                                                                int accumulate, Col4 out) {
  const uint64_t n = 1ull << d.L;
  const uint64_t n_units = n >> 2;
  for (uint64_t u = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; u < n_units;
       u += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t j0 = d.L > 2 ? (__brevll(u) >> (64 - (d.L - 2))) : 0;
    cpoint p0 = d.init;
    for (uint32_t b = 0; b + 2 < d.L; b++)
      if ((j0 >> b) & 1) p0 = cpoint_add(p0, d.step_pow[b]);
    const cpoint p1 = cpoint_add(p0, d.quarter);
    const cpoint pts[4] = {p0, {p0.x, m31_neg(p0.y)}, p1, {p1.x, m31_neg(p1.y)}};
    const uint64_t i0 = u << 2;
    qm31 q[4] = {qm31_zero(), qm31_zero(), qm31_zero(), qm31_zero()};
    // prefix products of the norms for the shared inversion
    cm31 den[kMaxAccs][4];
    uint32_t pref[kMaxAccs * 4 + 1];
    pref[0] = 1;
    for (uint32_t z = 0; z < n_accs; z++)
#pragma unroll
      for (int r = 0; r < 4; r++) {
        den[z][r] = quot_den(t.a[z], pts[r]);
        const uint32_t nrm = m31_add(m31_sqr(den[z][r].a), m31_sqr(den[z][r].b));
        pref[z * 4 + r + 1] = m31_mul(pref[z * 4 + r], nrm);
      }
    uint32_t inv = m31_inv(pref[n_accs * 4]);
    for (int z = (int)n_accs - 1; z >= 0; z--) {
      const QuotAcc& a = t.a[z];
#pragma unroll
      for (int r = 3; r >= 0; r--) {
        const uint32_t k = (uint32_t)z * 4 + r;
        const uint32_t ninv = m31_mul(inv, pref[k]);  // 1 / norm_k
        const cm31 c = den[z][r];
        const uint32_t nrm = m31_add(m31_sqr(c.a), m31_sqr(c.b));
        inv = m31_mul(inv, nrm);
        const cm31 dinv = cm31_mul({c.a, m31_neg(c.b)}, {ninv, 0});
        const uint64_t j = lift_index(i0 + r, a.shift);
        const qm31 num{__ldg(a.num[0] + j), __ldg(a.num[1] + j), __ldg(a.num[2] + j), __ldg(a.num[3] + j)};
        const qm31 full = qm31_sub(qm31_add(qm31_zero(), num), qm31_mul_m31(a.A, pts[r].y));
        q[r] = qm31_add(q[r], qm31_mul_cm31(full, dinv));
      }
    }
#pragma unroll
    for (int r = 0; r < 4; r++) {
      qm31 v = q[r];
      const uint64_t i = i0 + r;
      if (accumulate) v = qm31_add(qm31{out.c[0][i], out.c[1][i], out.c[2][i], out.c[3][i]}, v);
      out.c[0][i] = v.a;
      out.c[1][i] = v.b;
      out.c[2][i] = v.c;
      out.c[3][i] = v.d;
    }
  }
}

// ------------------------------------------------------------ accumulate ---
__global__ void __launch_bounds__(256) accumulate_kernel(Col4 col, Col4R other, uint64_t n) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
#pragma unroll
    for (int k = 0; k < 4; k++) col.c[k][i] = m31_add(col.c[k][i], __ldg(other.c[k] + i));
  }
}

// --------------------------------------------------- generate_secure_powers
// out[k] = felt^k (QM31, 4 words each): thread k by square-and-multiply.
__global__ void __launch_bounds__(256) secure_powers_kernel(qm31 felt, uint32_t n, uint4* __restrict__ out) {
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    qm31 r = qm31_one(), b = felt;
    for (uint32_t e = k; e; e >>= 1) {
      if (e & 1) r = qm31_mul(r, b);
      b = qm31_mul(b, b);
    }
    out[k] = make_uint4(r.a, r.b, r.c, r.d);
  }
}

// ------------------------------------------- bit reversal of QM31 values ---
__global__ void bit_reverse_qm31_kernel(uint4* v, uint32_t log_n) {
  const uint64_t n = 1ull << log_n;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t j = __brevll(i) >> (64 - log_n);
    if (i < j) {
      const uint4 a = v[i];
      v[i] = v[j];
      v[j] = a;
    }
  }
}

unsigned grid_rows(uint64_t n, unsigned threads) {
  const uint64_t b = (n + threads - 1) / threads;
  return (unsigned)std::min<uint64_t>(std::max<uint64_t>(b, 1), 148ull * 32);
}

qm31 qm31_from_words(const uint32_t* w) { return {w[0], w[1], w[2], w[3]}; }
bool canonical4(const uint32_t* w) { return w[0] < M31_P && w[1] < M31_P && w[2] < M31_P && w[3] < M31_P; }

}  // namespace
}  // namespace stwo_b200

using namespace stwo_b200;

extern "C" int stwo_b200_accumulate_numerators(const uint32_t* const* d_cols, uint32_t n_cols, uint32_t log_size,
                                               const stwo_b200_sample_batch* batches, uint32_t n_batches,
                                               uint32_t* const* d_out, uint32_t* first_linear_term_out,
                                               void* stream, char* err, size_t err_len) {
  STWO_ARG_CHECK(n_batches == 0 || (batches && d_out && first_linear_term_out), "null argument");
  STWO_ARG_CHECK(log_size <= 30, "log size %u too large", log_size);
  cudaStream_t s = as_stream(stream);
  const uint64_t n = 1ull << log_size;
  for (uint32_t b = 0; b < n_batches; b++) {
    const stwo_b200_sample_batch& sb = batches[b];
    STWO_ARG_CHECK(sb.n_terms == 0 || sb.terms, "batch %u: null terms", b);
    STWO_ARG_CHECK(canonical4(sb.point) && canonical4(sb.point + 4), "batch %u: point not canonical", b);
    const qm31 zy = qm31_from_words(sb.point + 4);
    // core/constraints.rs:119-134: c = conj(z.y) - z.y, a = conj(v) - v,
    // b = v c - a z.y, each times the term's random coefficient
    const qm31 cz = qm31_sub(qm31_conj(zy), zy);
    STWO_ARG_CHECK(!qm31_eq(cz, qm31_zero()), "batch %u: the sample point equals its conjugate", b);
    std::vector<qm31> cs(sb.n_terms);
    qm31 a_sum = qm31_zero(), b_sum = qm31_zero();
    for (uint32_t k = 0; k < sb.n_terms; k++) {
      const stwo_b200_numerator_term& t = sb.terms[k];
      STWO_ARG_CHECK(t.column_index < n_cols && d_cols && d_cols[t.column_index], "batch %u term %u: bad column", b,
                     k);
      STWO_ARG_CHECK(canonical4(t.sample_value) && canonical4(t.random_coeff), "batch %u term %u: not canonical",
                     b, k);
      const qm31 v = qm31_from_words(t.sample_value), alpha = qm31_from_words(t.random_coeff);
      const qm31 a = qm31_sub(qm31_conj(v), v);
      const qm31 bb = qm31_sub(qm31_mul(v, cz), qm31_mul(a, zy));
      a_sum = qm31_add(a_sum, qm31_mul(alpha, a));
      b_sum = qm31_add(b_sum, qm31_mul(alpha, bb));
      cs[k] = qm31_mul(alpha, cz);
    }
    first_linear_term_out[4 * b] = a_sum.a;
    first_linear_term_out[4 * b + 1] = a_sum.b;
    first_linear_term_out[4 * b + 2] = a_sum.c;
    first_linear_term_out[4 * b + 3] = a_sum.d;
    Col4 out{{d_out[4 * b], d_out[4 * b + 1], d_out[4 * b + 2], d_out[4 * b + 3]}};
    for (int k = 0; k < 4; k++) STWO_ARG_CHECK(out.c[k], "batch %u: null output column", b);
    uint32_t k0 = 0;
    do {
      const uint32_t nt = std::min<uint32_t>(kNumTerms, sb.n_terms - k0);
      NumeratorTerms t;
      bool aligned = n % 4 == 0;
      for (uint32_t k = 0; k < nt; k++) {
        t.col[k] = d_cols[sb.terms[k0 + k].column_index];
        t.c[k] = cs[k0 + k];
        aligned = aligned && reinterpret_cast<uintptr_t>(t.col[k]) % 16 == 0;
      }
      const int acc = k0 > 0 ? 1 : 0;
      if (aligned)
        numerators_kernel<true><<<grid_rows(n / 4, 256), 256, 0, s>>>(t, nt, b_sum, n, acc, out);
      else
        numerators_kernel<false><<<grid_rows(n, 256), 256, 0, s>>>(t, nt, b_sum, n, acc, out);
      STWO_CHECK_LAUNCH();
      k0 += nt;
    } while (k0 < sb.n_terms);
  }
  return ok(err, err_len);
}

extern "C" int stwo_b200_lift_and_accumulate(const uint32_t* const* d_cols4, const uint32_t* log_sizes,
                                             uint32_t n_cols, uint32_t* const* d_out4, void* stream, char* err,
                                             size_t err_len) {
  STWO_ARG_CHECK(n_cols >= 1 && n_cols <= (uint32_t)kMaxLift, "1..%d columns", kMaxLift);
  STWO_ARG_CHECK(d_cols4 && log_sizes && d_out4, "null argument");
  const uint32_t L = log_sizes[n_cols - 1];
  STWO_ARG_CHECK(L <= 30 && log_sizes[0] >= 1, "log sizes out of range");
  LiftCols t;
  for (uint32_t k = 0; k < n_cols; k++) {
    STWO_ARG_CHECK(k == 0 || log_sizes[k] > log_sizes[k - 1], "log sizes must be strictly increasing");
    for (int c = 0; c < 4; c++) {
      t.c[k][c] = d_cols4[4 * k + c];
      STWO_ARG_CHECK(t.c[k][c], "null column %u", k);
    }
    t.shift[k] = L - log_sizes[k];
  }
  Col4 out{{d_out4[0], d_out4[1], d_out4[2], d_out4[3]}};
  const uint64_t n = 1ull << L;
  lift_accumulate_kernel<<<grid_rows(n, 256), 256, 0, as_stream(stream)>>>(t, n_cols, n, out);
  STWO_CHECK_LAUNCH();
  return ok(err, err_len);
}

extern "C" int stwo_b200_compute_quotients_and_combine(const stwo_b200_accumulated_numerators* accs,
                                                       uint32_t n_accs, uint32_t lifting_log_size,
                                                       uint32_t* const* d_out4, void* stream, char* err,
                                                       size_t err_len) {
  STWO_ARG_CHECK(n_accs == 0 || accs, "null accumulations");
  STWO_ARG_CHECK(d_out4 && d_out4[0] && d_out4[1] && d_out4[2] && d_out4[3], "null output");
  const uint32_t L = lifting_log_size;
  STWO_ARG_CHECK(L >= 2 && L <= 30, "lifting log size %u out of range [2, 30]", L);
  cudaStream_t s = as_stream(stream);
  Col4 out{{d_out4[0], d_out4[1], d_out4[2], d_out4[3]}};
  if (n_accs == 0) {
    for (int k = 0; k < 4; k++) STWO_CUDA_TRY(cudaMemsetAsync(out.c[k], 0, 4ull << L, s));
    return ok(err, err_len);
  }
  // CanonicCoset(L).circle_domain(): half coset of initial index 2^(31 - L - 1)
  // and step 2^(31 - (L - 1)) (core/poly/circle/canonic.rs:28-33).
  QuotDomain d;
  d.L = L;
  d.init = index_to_cpoint(1ull << (31 - (L + 1)));
  cpoint st = index_to_cpoint(1ull << (31 - (L - 1)));
  for (uint32_t b = 0; b < 30; b++) {
    d.step_pow[b] = st;
    if (b + 2 == L) d.quarter = st;
    st = cpoint_add(st, st);
  }
  if (L == 2) d.quarter = d.step_pow[0];
  for (uint32_t z0 = 0; z0 < n_accs; z0 += kMaxAccs) {
    const uint32_t nz = std::min<uint32_t>(kMaxAccs, n_accs - z0);
    QuotAccs t;
    for (uint32_t z = 0; z < nz; z++) {
      const stwo_b200_accumulated_numerators& a = accs[z0 + z];
      STWO_ARG_CHECK(a.log_size >= 1 && a.log_size <= L, "accumulation %u: log size %u outside [1, %u]", z0 + z,
                     a.log_size, L);
      STWO_ARG_CHECK(canonical4(a.sample_point) && canonical4(a.sample_point + 4) && canonical4(a.first_linear_term),
                     "accumulation %u: not canonical", z0 + z);
      for (int k = 0; k < 4; k++) {
        t.a[z].num[k] = a.d_partial[k];
        STWO_ARG_CHECK(a.d_partial[k], "accumulation %u: null column", z0 + z);
      }
      t.a[z].shift = L - a.log_size;
      t.a[z].A = qm31_from_words(a.first_linear_term);
      const uint32_t* p = a.sample_point;
      t.a[z].prx = {p[0], p[1]};
      t.a[z].pix = {p[2], p[3]};
      t.a[z].pry = {p[4], p[5]};
      t.a[z].piy = {p[6], p[7]};
    }
    quotients_combine_kernel<<<grid_rows(1ull << (L - 2), 256), 256, 0, s>>>(t, nz, d, z0 > 0 ? 1 : 0, out);
    STWO_CHECK_LAUNCH();
  }
  return ok(err, err_len);
}

extern "C" int stwo_b200_accumulate(uint32_t* const* d_col4, const uint32_t* const* d_other4, uint64_t len,
                                    void* stream, char* err, size_t err_len) {
  STWO_ARG_CHECK(d_col4 && d_other4, "null argument");
  if (len == 0) return ok(err, err_len);
  Col4 col{{d_col4[0], d_col4[1], d_col4[2], d_col4[3]}};
  Col4R other{{d_other4[0], d_other4[1], d_other4[2], d_other4[3]}};
  for (int k = 0; k < 4; k++) STWO_ARG_CHECK(col.c[k] && other.c[k], "null coordinate column %d", k);
  accumulate_kernel<<<grid_rows(len, 256), 256, 0, as_stream(stream)>>>(col, other, len);
  STWO_CHECK_LAUNCH();
  return ok(err, err_len);
}

extern "C" int stwo_b200_generate_secure_powers(const uint32_t* felt, uint32_t n_powers, uint32_t* d_out,
                                                void* stream, char* err, size_t err_len) {
  STWO_ARG_CHECK(felt && (n_powers == 0 || d_out), "null argument");
  STWO_ARG_CHECK(canonical4(felt), "felt not canonical");
  if (n_powers == 0) return ok(err, err_len);
  STWO_ARG_CHECK(reinterpret_cast<uintptr_t>(d_out) % 16 == 0, "output must be 16-byte aligned");
  secure_powers_kernel<<<grid_rows(n_powers, 256), 256, 0, as_stream(stream)>>>(
      qm31_from_words(felt), n_powers, reinterpret_cast<uint4*>(d_out));
  STWO_CHECK_LAUNCH();
  return ok(err, err_len);
}

extern "C" int stwo_b200_batch_eval_at_point(const uint32_t* const* d_coeffs, uint32_t n_polys, uint32_t log_size,
                                             const uint32_t* point, uint32_t* values_out, void* stream, char* err,
                                             size_t err_len) {
  STWO_ARG_CHECK(point && (n_polys == 0 || (d_coeffs && values_out)), "null argument");
  STWO_ARG_CHECK(log_size <= 30, "log size %u too large", log_size);
  STWO_ARG_CHECK(canonical4(point) && canonical4(point + 4), "point not canonical");
  if (n_polys == 0) return ok(err, err_len);
  cudaStream_t s = as_stream(stream);
  if (log_size == 0) {
    // A single coefficient is its own value, word for word (core/poly/utils.rs fold of one value).
    for (uint32_t p = 0; p < n_polys; p++) {
      STWO_CUDA_TRY(cudaMemcpyAsync(values_out + 4 * p, d_coeffs[p], 4, cudaMemcpyDeviceToHost, s));
      values_out[4 * p + 1] = values_out[4 * p + 2] = values_out[4 * p + 3] = 0;
    }
    STWO_CUDA_TRY(cudaStreamSynchronize(s));
    return ok(err, err_len);
  }
  const spoint z{qm31_from_words(point), qm31_from_words(point + 4)};
  const uint32_t lg = log_size, h = poly_eval_lo_bits(lg);
  const uint32_t n_chunk_polys = std::min<uint32_t>(n_polys, kMaxPolys);
  const size_t n_w = (1ull << h) + (1ull << (lg - h));
  const size_t words = n_w + (size_t)n_chunk_polys * poly_eval_chunks(lg) + n_polys;
  qm31* scratch = nullptr;
  STWO_CUDA_TRY(cudaMallocAsync(reinterpret_cast<void**>(&scratch), words * sizeof(qm31), s));
  qm31* w_lo = scratch;
  qm31* w_hi = scratch + (1ull << h);
  qm31* partial = scratch + n_w;
  qm31* vals = partial + (size_t)n_chunk_polys * poly_eval_chunks(lg);
  int rc = launch_eval_weights(z, lg, w_lo, w_hi, s, err, err_len);
  for (uint32_t p0 = 0; rc == 0 && p0 < n_polys; p0 += kMaxPolys) {
    const uint32_t np = std::min<uint32_t>(kMaxPolys, n_polys - p0);
    rc = launch_poly_eval(d_coeffs + p0, np, lg, w_lo, w_hi, partial, vals + p0, s, err, err_len);
  }
  if (rc == 0) {
    const cudaError_t e = cudaMemcpyAsync(values_out, vals, (size_t)n_polys * sizeof(qm31), cudaMemcpyDeviceToHost, s);
    if (e != cudaSuccess) rc = set_err(err, err_len, STWO_B200_ECUDA, "copy of the values: %s", cudaGetErrorString(e));
  }
  cudaFreeAsync(scratch, s);
  if (rc) return rc;
  STWO_CUDA_TRY(cudaStreamSynchronize(s));
  return ok(err, err_len);
}

extern "C" int stwo_b200_eval_at_point(const uint32_t* d_coeffs, uint32_t log_size, const uint32_t* point,
                                       uint32_t* value_out, void* stream, char* err, size_t err_len) {
  STWO_ARG_CHECK(d_coeffs, "null coefficients");
  return stwo_b200_batch_eval_at_point(&d_coeffs, 1, log_size, point, value_out, stream, err, err_len);
}

extern "C" int stwo_b200_grind(const uint8_t* digest, uint32_t pow_bits, int m31_channel, uint64_t* nonce_out,
                               void* stream, char* err, size_t err_len) {
  STWO_ARG_CHECK(digest && nonce_out, "null argument");
  STWO_ARG_CHECK(pow_bits <= 32, "pow_bits %u > 32 is not supported", pow_bits);
  cudaStream_t s = as_stream(stream);
  HostChannel ch(m31_channel != 0);
  uint32_t dw[8];
  std::memcpy(dw, digest, 32);
  ch.set_state(dw, 0);
  const Hash32 pre = ch.pow_prefixed(pow_bits);
  uint32_t pw[8];
  std::memcpy(pw, pre.data(), 32);
  uint32_t* d_found = nullptr;
  uint32_t* h_found = nullptr;
  STWO_CUDA_TRY(cudaMallocAsync(reinterpret_cast<void**>(&d_found), 4, s));
  int rc = STWO_B200_OK;
  cudaError_t e = cudaMallocHost(reinterpret_cast<void**>(&h_found), 4);
  if (e != cudaSuccess) rc = set_err(err, err_len, STWO_B200_ECUDA, "pinned flag: %s", cudaGetErrorString(e));
  // SimdBackend's order: for hi = 0, 1, ... the low words [0, 2^20), smallest
  // first (simd/grind.rs:20-96); one launch covers one hi.
  bool found = false;
  for (uint32_t hi = 0; rc == 0 && !found && hi < M31_P; hi++) {
    e = cudaMemsetAsync(d_found, 0xFF, 4, s);
    if (e == cudaSuccess) rc = launch_grind(pw, hi, 0, 1u << 20, pow_bits, m31_channel != 0, d_found, s, err, err_len);
    if (rc == 0 && e == cudaSuccess) e = cudaMemcpyAsync(h_found, d_found, 4, cudaMemcpyDeviceToHost, s);
    if (rc == 0 && e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) rc = set_err(err, err_len, STWO_B200_ECUDA, "grind: %s", cudaGetErrorString(e));
    if (rc == 0 && *h_found != 0xFFFFFFFFu) {
      *nonce_out = ((uint64_t)hi << 32) | *h_found;
      found = true;
    }
  }
  cudaFreeAsync(d_found, s);
  if (h_found) {
    cudaStreamSynchronize(s);
    cudaFreeHost(h_found);
  }
  if (rc) return rc;
  if (!found) return set_err(err, err_len, STWO_B200_ESTATE, "grind found no nonce");
  return ok(err, err_len);
}

extern "C" int stwo_b200_bit_reverse_secure_column(uint32_t* const* d_coords4, uint32_t log_size, void* stream,
                                                   char* err, size_t err_len) {
  STWO_ARG_CHECK(d_coords4, "null argument");
  const uint32_t logs[4] = {log_size, log_size, log_size, log_size};
  return stwo_b200_bit_reverse_columns(const_cast<const uint32_t* const*>(d_coords4), d_coords4, logs, 4, stream,
                                       err, err_len);
}

extern "C" int stwo_b200_bit_reverse_secure_field(uint32_t* d_values, uint32_t log_size, void* stream, char* err,
                                                  size_t err_len) {
  STWO_ARG_CHECK(d_values && reinterpret_cast<uintptr_t>(d_values) % 16 == 0, "values must be 16-byte aligned");
  STWO_ARG_CHECK(log_size <= 30, "log size %u too large", log_size);
  if (log_size == 0) return ok(err, err_len);
  bit_reverse_qm31_kernel<<<grid_rows(1ull << log_size, 256), 256, 0, as_stream(stream)>>>(
      reinterpret_cast<uint4*>(d_values), log_size);
  STWO_CHECK_LAUNCH();
  return ok(err, err_len);
}
