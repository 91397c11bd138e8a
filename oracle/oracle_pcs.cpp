// ORACLE — test infrastructure only.  CPU restatement of the trait methods
// stwo's generic prover calls beside the commit and FRI operations, in
// SimdBackend's order of operations, with flat C entry points for tests/:
//
//   QuotientOps::accumulate_numerators   prover/backend/simd/quotients.rs:34-71,124-134
//   QuotientOps::compute_quotients_and_combine
//                                        prover/backend/simd/quotients.rs:73-164
//   line coefficients                    core/constraints.rs:119-134,
//                                        core/pcs/quotients.rs:205-230
//   AccumulationOps::accumulate          prover/backend/simd/accumulation.rs:13-18
//   AccumulationOps::generate_secure_powers
//                                        prover/backend/cpu/accumulation.rs:16-24
//   AccumulationOps::lift_and_accumulate prover/backend/simd/accumulation.rs:45-80
//   PolyOps::eval_at_point               prover/backend/cpu/circle.rs:82-99
//   ColumnOps<SecureField>::bit_reverse_column
//                                        core/utils.rs:91-101
// (paths relative to the vendored stwo crate of the reference).
#include <cstring>
#include <stdexcept>
#include <vector>

#include "stwo_oracle.hpp"
#include "stwo_oracle_prove.hpp"

using namespace oracle;

namespace {

QM31 q_at(const uint32_t* const* c4, size_t i) { return QM31::from(c4[0][i], c4[1][i], c4[2][i], c4[3][i]); }
void q_set(uint32_t* const* c4, size_t i, QM31 v) {
  auto w = v.coords();
  for (int k = 0; k < 4; k++) c4[k][i] = w[k];
}
QM31 q_words(const uint32_t* w) { return QM31::from(w[0], w[1], w[2], w[3]); }
void put_words(uint32_t* w, QM31 v) {
  auto c = v.coords();
  for (int k = 0; k < 4; k++) w[k] = c[k];
}

// core/constraints.rs:119-134 (complex_conjugate_line_coeffs), times alpha.
void line_coeffs(const SPoint& z, QM31 value, QM31 alpha, QM31& a, QM31& b, QM31& c) {
  if (z.y == qconj(z.y)) throw std::runtime_error("Cannot evaluate a line with a single point");
  QM31 aa = qconj(value) - value;
  QM31 cc = qconj(z.y) - z.y;
  QM31 bb = value * cc - aa * z.y;
  a = alpha * aa;
  b = alpha * bb;
  c = alpha * cc;
}

// ((i >> (r + 1)) << 1) + (i & 1): index of row i of a column lifted by r
// (prover/backend/cpu/accumulation.rs:40, simd/utils.rs:40-70).
size_t lift(size_t i, uint32_t r) { return r == 0 ? i : ((i >> (r + 1)) << 1) + (i & 1); }

}  // namespace

extern "C" {

// One batch of accumulate_numerators: terms (column index, value, alpha) as
// idx[k], values[4k..], alphas[4k..]; point as 8 words.  out4: 4 columns of
// 2^log_n words; first_linear (4 words).
int oracle_accumulate_numerators(const uint32_t* const* cols, uint32_t n_cols, uint32_t log_n, const uint32_t* point,
                                 const uint32_t* idx, const uint32_t* values, const uint32_t* alphas,
                                 uint32_t n_terms, uint32_t** out4, uint32_t* first_linear) {
  try {
    SPoint z{q_words(point), q_words(point + 4)};
    std::vector<QM31> la(n_terms), lb(n_terms), lc(n_terms);
    for (uint32_t k = 0; k < n_terms; k++) {
      if (idx[k] >= n_cols) throw std::runtime_error("column index out of range");
      line_coeffs(z, q_words(values + 4 * k), q_words(alphas + 4 * k), la[k], lb[k], lc[k]);
    }
    size_t n = (size_t)1 << log_n;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)n; i++) {
      QM31 num = QM31::zero();
      for (uint32_t k = 0; k < n_terms; k++) num = num + (qmul_m31(lc[k], cols[idx[k]][i]) - lb[k]);
      q_set(out4, (size_t)i, num);
    }
    QM31 a = QM31::zero();
    for (auto& x : la) a = a + x;
    put_words(first_linear, a);
    return 0;
  } catch (const std::exception&) {
    return -1;
  }
}

// compute_quotients_and_combine: accumulation z has its point (8 words at
// points + 8z), partial numerator columns parts[4z..4z+3] of 2^logs[z] words
// and first linear term (4 words at firsts + 4z).
int oracle_compute_quotients_and_combine(const uint32_t* points, const uint32_t* const* parts, const uint32_t* logs,
                                         const uint32_t* firsts, uint32_t n_accs, uint32_t lifting_log,
                                         uint32_t** out4) {
  try {
    size_t n = (size_t)1 << lifting_log;
    Coset half = canonic_half_coset(lifting_log);
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)n; i++) {
      CPoint p = index_to_point(circle_domain_index_at(half, bit_reverse_index((uint64_t)i, lifting_log)));
      QM31 q = QM31::zero();
      for (uint32_t z = 0; z < n_accs; z++) {
        const uint32_t* pt = points + 8 * z;
        CM31 prx{pt[0], pt[1]}, pix{pt[2], pt[3]}, pry{pt[4], pt[5]}, piy{pt[6], pt[7]};
        CM31 den = (prx - CM31{p.x, 0}) * piy - (pry - CM31{p.y, 0}) * pix;
        CM31 dinv = cinv(den);
        size_t j = lift((size_t)i, lifting_log - logs[z]);
        QM31 lifted = q_at(parts + 4 * z, j);
        QM31 full = (QM31::zero() + lifted) - qmul_m31(q_words(firsts + 4 * z), p.y);
        q = q + QM31{full.x * dinv, full.y * dinv};
      }
      q_set(out4, (size_t)i, q);
    }
    return 0;
  } catch (const std::exception&) {
    return -1;
  }
}

// lift_and_accumulate (SimdBackend): prev = first; col_k[i] += lift(prev)[i].
// cols4[4k..4k+3] of 2^logs[k] words (strictly increasing); writes out4 (the
// size of the last).
int oracle_lift_and_accumulate(const uint32_t* const* cols4, const uint32_t* logs, uint32_t n_cols, uint32_t** out4) {
  if (n_cols == 0) return -1;
  for (uint32_t k = 1; k < n_cols; k++)
    if (logs[k] <= logs[k - 1]) return -1;
  std::vector<std::vector<uint32_t>> prev(4);
  size_t n0 = (size_t)1 << logs[0];
  for (int c = 0; c < 4; c++) prev[c].assign(cols4[c], cols4[c] + n0);
  for (uint32_t k = 1; k < n_cols; k++) {
    size_t n = (size_t)1 << logs[k];
    uint32_t r = logs[k] - logs[k - 1];
    std::vector<std::vector<uint32_t>> cur(4, std::vector<uint32_t>(n));
    for (size_t i = 0; i < n; i++) {
      size_t j = lift(i, r);
      for (int c = 0; c < 4; c++) cur[c][i] = add(cols4[4 * k + c][i], prev[c][j]);
    }
    prev.swap(cur);
  }
  size_t n = (size_t)1 << logs[n_cols - 1];
  for (int c = 0; c < 4; c++) std::memcpy(out4[c], prev[c].data(), n * 4);
  return 0;
}

// accumulate: col += other (4 coordinate columns of len words).
void oracle_accumulate(uint32_t** col4, const uint32_t* const* other4, size_t len) {
  for (size_t i = 0; i < len; i++)
    for (int c = 0; c < 4; c++) col4[c][i] = add(col4[c][i], other4[c][i]);
}

// generate_secure_powers: out[4k..4k+3] = felt^k, by the CPU scan.
void oracle_generate_secure_powers(const uint32_t* felt, uint32_t n, uint32_t* out) {
  QM31 f = q_words(felt), acc = QM31::one();
  for (uint32_t k = 0; k < n; k++) {
    put_words(out + 4 * k, acc);
    acc = acc * f;
  }
}

// eval_at_point at a secure point (8 words) of 2^log_n natural-order
// coefficients.
void oracle_eval_at_secure_point(const uint32_t* coeffs, uint32_t log_n, const uint32_t* point, uint32_t* out) {
  SPoint z{q_words(point), q_words(point + 4)};
  put_words(out, eval_at_point_q(coeffs, log_n, z));
}

}  // extern "C"
