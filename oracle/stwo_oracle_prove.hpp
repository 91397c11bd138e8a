// ORACLE — test infrastructure only: proof types of the Wide-Fibonacci prove
// restatement (core/pcs/quotients.rs:27-35, core/fri.rs:361-395).
#pragma once
#include "stwo_oracle.hpp"

namespace oracle {

struct SPoint { QM31 x, y; };  // CirclePoint<SecureField>
SPoint sadd(const SPoint& p, const SPoint& q);
QM31 double_x(QM31 x);
SPoint sdouble(const SPoint& p);
SPoint srepeated_double(SPoint p, uint32_t n);
QM31 qconj(QM31 a);
SPoint get_random_point(Channel& ch);
uint32_t coset_vanishing_m31(const Coset& coset, CPoint p);
QM31 coset_vanishing_q(const Coset& coset, SPoint p);
QM31 eval_at_point_q(const uint32_t* coeffs, uint32_t log_n, const SPoint& p);
std::vector<QM31> line_interpolate_ordered(std::vector<QM31> vals, const Coset& line_coset);

struct WideFibConfig {
  uint32_t log_n_rows = 4;
  uint32_t n_cols = 100;
  uint32_t log_blowup = 1;
  uint32_t pow_bits = 10;
  uint32_t n_queries = 3;
  uint32_t log_last_layer_degree_bound = 0;
  uint32_t line_fold_step = 1;
  bool m31_channel = false;
};

struct FriConfigO { uint32_t log_last_layer, log_blowup, n_queries, line_fold_step; };

struct FriLayerProofO {
  std::vector<QM31> fri_witness;
  std::vector<Hash> hash_witness;
  Hash commitment{};
};

struct Proof {
  WideFibConfig cfg;
  std::vector<Hash> commitments;
  std::vector<std::vector<std::vector<QM31>>> sampled_values;      // tree, column, sample
  std::vector<std::vector<Hash>> decommitments;                    // tree -> hash witness
  std::vector<std::vector<std::vector<uint32_t>>> queried_values;  // tree, column, query
  uint64_t proof_of_work = 0;
  FriLayerProofO fri_first;
  std::vector<FriLayerProofO> fri_inner;
  std::vector<QM31> last_layer_poly;  // ordered coefficients
  std::vector<size_t> query_positions; // not serialized (derived by the verifier)
};

// Intermediate values exposed to the parity tests.
struct ProveTrace {
  std::vector<std::vector<uint32_t>> composition_evals;  // 4 coords, eval domain
  std::vector<std::vector<uint32_t>> quotients;          // 4 coords, lifting domain
  std::vector<Hash> roots;
  SPoint oods;
};

void merkle_decommit(const std::vector<std::vector<Hash>>& layers_root_first, std::vector<size_t> queries,
                     const std::vector<const uint32_t*>& cols, const std::vector<uint32_t>& log_sizes,
                     std::vector<std::vector<uint32_t>>& queried_values, std::vector<Hash>& witness);
Proof prove_wide_fib(const WideFibConfig& cfg, const uint32_t* in_a, const uint32_t* in_b, ProveTrace* dbg);
std::vector<uint8_t> serialize(const Proof& p);
std::vector<uint8_t> fri_prove_seeded(const uint32_t* const coords[4], uint32_t log_n, const QM31* alphas,
                                      std::vector<size_t> queries, bool m31);
void verify_wide_fib(const uint8_t* data, size_t n, uint32_t log_n_rows, uint32_t n_cols, bool m31);

}  // namespace oracle
