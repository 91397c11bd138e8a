// ORACLE — test infrastructure only.  Flat C entry points over the CPU
// restatement, loaded by tests/ (ctypes), __graft_entry__.smoke() and the CPU
// baseline legs of bench.py.  Every function returns 0 on success and a
// negative value on error (message via oracle_last_error()).
#include "stwo_oracle.hpp"

#include <cstdio>
#include <string>
#ifdef _OPENMP
#include <omp.h>
#endif

using namespace oracle;

static thread_local std::string g_err;

template <class F>
static int guard(F&& f) {
  try {
    f();
    return 0;
  } catch (const std::exception& e) {
    g_err = e.what();
    return -1;
  }
}

extern "C" {

const char* oracle_last_error() { return g_err.c_str(); }

int oracle_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
  return omp_get_max_threads();
#else
  (void)n;
  return 1;
#endif
}

void oracle_blake2s(const uint8_t* data, size_t len, int m31, uint8_t* out) {
  Hash h = blake2s_hash(data, len, m31 != 0);
  std::memcpy(out, h.data(), 32);
}

// Coset point (x, y) for a CirclePointIndex.
void oracle_index_to_point(uint64_t index, uint32_t* xy) {
  CPoint p = index_to_point(index);
  xy[0] = p.x; xy[1] = p.y;
}

void oracle_bit_reverse(uint32_t* v, uint32_t log_n) { bit_reverse(v, log_n); }

// QM31 product and inverse (core/fields/qm31.rs:78-88, 125-133); CM31 values
// are the QM31 values with the upper half zero.
int oracle_qm31_mul(const uint32_t* a, const uint32_t* b, uint32_t* out) {
  return guard([&] {
    QM31 r = QM31::from(a[0], a[1], a[2], a[3]) * QM31::from(b[0], b[1], b[2], b[3]);
    out[0] = r.x.a; out[1] = r.x.b; out[2] = r.y.a; out[3] = r.y.b;
  });
}

int oracle_qm31_inv(const uint32_t* a, uint32_t* out) {
  return guard([&] {
    QM31 r = qinv(QM31::from(a[0], a[1], a[2], a[3]));
    out[0] = r.x.a; out[1] = r.x.b; out[2] = r.y.a; out[3] = r.y.b;
  });
}

// Twiddle tree of the coset (initial_index, log_size): 2^log_size words each.
int oracle_precompute_twiddles(uint64_t initial_index, uint32_t log_size, uint32_t* tw, uint32_t* itw) {
  return guard([&] {
    TwiddleTree t = precompute_twiddles(Coset::make(initial_index, log_size));
    std::memcpy(tw, t.tw.data(), t.tw.size() * 4);
    std::memcpy(itw, t.itw.data(), t.itw.size() * 4);
  });
}

// `half_initial_index` = the evaluation domain's half-coset initial index
// (CanonicCoset(n): 2^(31 - (n + 1))).
int oracle_interpolate(uint32_t* values, uint32_t log_n, uint64_t half_initial_index, const uint32_t* itw,
                       size_t itw_len) {
  return guard([&] { interpolate(values, log_n, Coset::make(half_initial_index, log_n ? log_n - 1 : 0), itw, itw_len); });
}

int oracle_interpolate_columns(uint32_t** cols, const uint32_t* log_sizes, uint32_t n_cols, const uint32_t* itw,
                               size_t itw_len) {
  return guard([&] {
#pragma omp parallel for schedule(dynamic, 1)
    for (long c = 0; c < (long)n_cols; c++)
      interpolate(cols[c], log_sizes[c], canonic_half_coset(log_sizes[c]), itw, itw_len);
  });
}

int oracle_evaluate(const uint32_t* coeffs, uint32_t log_n, uint32_t log_eval, uint64_t half_initial_index,
                    const uint32_t* tw, size_t tw_len, uint32_t* out) {
  return guard([&] { evaluate(coeffs, log_n, log_eval, Coset::make(half_initial_index, log_eval - 1), tw, tw_len, out); });
}

int oracle_evaluate_columns(const uint32_t* const* coeffs, const uint32_t* log_sizes, uint32_t n_cols,
                            uint32_t log_blowup, const uint32_t* tw, size_t tw_len, uint32_t** out) {
  return guard([&] {
#pragma omp parallel for schedule(dynamic, 1)
    for (long c = 0; c < (long)n_cols; c++) {
      uint32_t le = log_sizes[c] + log_blowup;
      evaluate(coeffs[c], log_sizes[c], le, canonic_half_coset(le), tw, tw_len, out[c]);
    }
  });
}

int oracle_eval_at_point_m31(const uint32_t* coeffs, uint32_t log_n, uint32_t x, uint32_t y, uint32_t* out) {
  return guard([&] { *out = eval_at_point_m31(coeffs, log_n, CPoint{x, y}); });
}

// Lifted Merkle: layers root first, concatenated (layer k has 2^k hashes).
// staged != 0: the leaves in SimdBackend's staged form (same hashes).
int oracle_merkle_build_layers(const uint32_t* const* cols, const uint32_t* log_sizes, uint32_t n_cols, uint32_t L,
                               int m31, int staged, uint8_t* layers_out) {
  return guard([&] {
    std::vector<const uint32_t*> c(cols, cols + n_cols);
    std::vector<uint32_t> l(log_sizes, log_sizes + n_cols);
    auto layers = build_merkle_layers(c, l, L, m31 != 0, staged != 0);
    size_t off = 0;
    for (auto& layer : layers) {
      std::memcpy(layers_out + off, layer.data(), layer.size() * 32);
      off += layer.size() * 32;
    }
  });
}

// Leaves of already length-sorted columns (MerkleOpsLifted::build_leaves).
int oracle_merkle_build_leaves(const uint32_t* const* cols, const uint32_t* log_sizes, uint32_t n_cols, uint32_t L,
                               int m31, uint8_t* out) {
  return guard([&] {
    std::vector<const uint32_t*> c(cols, cols + n_cols);
    std::vector<uint32_t> l(log_sizes, log_sizes + n_cols);
    auto leaves = build_leaves(c, l, L, m31 != 0);
    std::memcpy(out, leaves.data(), leaves.size() * 32);
  });
}

int oracle_merkle_next_layer(const uint8_t* prev, uint32_t log_prev, int m31, uint8_t* out) {
  return guard([&] {
    std::vector<Hash> p((size_t)1 << log_prev);
    std::memcpy(p.data(), prev, p.size() * 32);
    auto n = build_next_layer(p, m31 != 0);
    std::memcpy(out, n.data(), n.size() * 32);
  });
}

int oracle_commit_on_layer(uint32_t log_size, const uint8_t* prev, const uint32_t* const* cols, uint32_t n_cols,
                           int m31, uint8_t* out) {
  return guard([&] {
    std::vector<const uint32_t*> c(cols, cols + n_cols);
    auto r = commit_on_layer(log_size, (const Hash*)prev, c, m31 != 0);
    std::memcpy(out, r.data(), r.size() * 32);
  });
}

int oracle_fold_line(const uint32_t* const* in4, uint32_t log_m, const uint32_t* itw, size_t itw_len,
                     const uint32_t* alpha, uint32_t fold_step, uint32_t** out4) {
  return guard([&] {
    const uint32_t* in[4] = {in4[0], in4[1], in4[2], in4[3]};
    uint32_t* out[4] = {out4[0], out4[1], out4[2], out4[3]};
    fold_line(in, log_m, itw, itw_len, QM31::from(alpha[0], alpha[1], alpha[2], alpha[3]), fold_step, out);
  });
}

int oracle_fold_line_direct(const uint32_t* const* in4, uint64_t initial_index, uint32_t log_m, const uint32_t* alpha,
                            uint32_t** out4) {
  return guard([&] {
    const uint32_t* in[4] = {in4[0], in4[1], in4[2], in4[3]};
    uint32_t* out[4] = {out4[0], out4[1], out4[2], out4[3]};
    fold_line_direct(in, Coset::make(initial_index, log_m), QM31::from(alpha[0], alpha[1], alpha[2], alpha[3]), out);
  });
}

int oracle_fold_circle_into_line(uint32_t** dst4, const uint32_t* const* src4, uint64_t half_initial_index,
                                 uint32_t log_n, const uint32_t* itw, size_t itw_len, const uint32_t* alpha) {
  return guard([&] {
    const uint32_t* src[4] = {src4[0], src4[1], src4[2], src4[3]};
    uint32_t* dst[4] = {dst4[0], dst4[1], dst4[2], dst4[3]};
    fold_circle_into_line(dst, src, Coset::make(half_initial_index, log_n - 1), itw, itw_len,
                          QM31::from(alpha[0], alpha[1], alpha[2], alpha[3]));
  });
}

int oracle_fold_circle_into_line_direct(uint32_t** dst4, const uint32_t* const* src4, uint64_t half_initial_index,
                                        uint32_t log_n, const uint32_t* alpha) {
  return guard([&] {
    const uint32_t* src[4] = {src4[0], src4[1], src4[2], src4[3]};
    uint32_t* dst[4] = {dst4[0], dst4[1], dst4[2], dst4[3]};
    fold_circle_into_line_direct(dst, src, Coset::make(half_initial_index, log_n - 1),
                                 QM31::from(alpha[0], alpha[1], alpha[2], alpha[3]));
  });
}

int oracle_decompose(const uint32_t* const* in4, uint32_t log_n, uint32_t** out4, uint32_t* lambda) {
  return guard([&] {
    const uint32_t* in[4] = {in4[0], in4[1], in4[2], in4[3]};
    uint32_t* out[4] = {out4[0], out4[1], out4[2], out4[3]};
    auto l = decompose(in, log_n, out).coords();
    for (int k = 0; k < 4; k++) lambda[k] = l[k];
  });
}

// ---- channel (state passed as digest[32] + n_draws) ----
struct OracleChannelState { uint8_t digest[32]; uint32_t n_draws; int32_t m31; };

static Channel load(const OracleChannelState* s) {
  Channel c; std::memcpy(c.digest.data(), s->digest, 32); c.n_draws = s->n_draws; c.m31 = s->m31 != 0; return c;
}
static void store(const Channel& c, OracleChannelState* s) {
  std::memcpy(s->digest, c.digest.data(), 32); s->n_draws = c.n_draws;
}
void oracle_channel_mix_u32s(OracleChannelState* s, const uint32_t* d, size_t n) { Channel c = load(s); c.mix_u32s(d, n); store(c, s); }
void oracle_channel_mix_u64(OracleChannelState* s, uint64_t v) { Channel c = load(s); c.mix_u64(v); store(c, s); }
void oracle_channel_mix_felts(OracleChannelState* s, const uint32_t* f, size_t n) {
  Channel c = load(s);
  std::vector<QM31> v(n);
  for (size_t i = 0; i < n; i++) v[i] = QM31::from(f[4 * i], f[4 * i + 1], f[4 * i + 2], f[4 * i + 3]);
  c.mix_felts(v.data(), n); store(c, s);
}
void oracle_channel_mix_root(OracleChannelState* s, const uint8_t* root) {
  Channel c = load(s); Hash h; std::memcpy(h.data(), root, 32); c.mix_root(h); store(c, s);
}
void oracle_channel_draw_u32s(OracleChannelState* s, uint32_t* out8) {
  Channel c = load(s); auto w = c.draw_u32s(); std::memcpy(out8, w.data(), 32); store(c, s);
}
void oracle_channel_draw_secure_felts(OracleChannelState* s, size_t n, uint32_t* out) {
  Channel c = load(s);
  auto v = c.draw_secure_felts(n);
  for (size_t i = 0; i < n; i++) { auto k = v[i].coords(); std::memcpy(out + 4 * i, k.data(), 16); }
  store(c, s);
}
int oracle_channel_verify_pow(const OracleChannelState* s, uint32_t bits, uint64_t nonce) {
  return load(s).verify_pow_nonce(bits, nonce) ? 1 : 0;
}
uint64_t oracle_channel_grind(const OracleChannelState* s, uint32_t bits) { return load(s).grind(bits); }

}  // extern "C"

// ---- Wide-Fibonacci prove (Blake2s Merkle channel) ----
#include "stwo_oracle_prove.hpp"

struct OracleWideFibConfig {
  uint32_t log_n_rows, n_cols, log_blowup, pow_bits, n_queries, log_last_layer_degree_bound, line_fold_step;
  int32_t m31_channel;
};

static WideFibConfig to_cfg(const OracleWideFibConfig* c) {
  WideFibConfig w;
  w.log_n_rows = c->log_n_rows; w.n_cols = c->n_cols; w.log_blowup = c->log_blowup; w.pow_bits = c->pow_bits;
  w.n_queries = c->n_queries; w.log_last_layer_degree_bound = c->log_last_layer_degree_bound;
  w.line_fold_step = c->line_fold_step; w.m31_channel = c->m31_channel != 0;
  return w;
}

static std::vector<uint8_t> g_last_proof;
static ProveTrace g_last_trace;

// Proves; the serialized proof is kept until the next call (oracle_last_proof).
extern "C" int oracle_prove_wide_fib(const OracleWideFibConfig* cfg, const uint32_t* a, const uint32_t* b,
                                     size_t* proof_len) {
  return guard([&] {
    g_last_trace = ProveTrace{};
    Proof p = prove_wide_fib(to_cfg(cfg), a, b, &g_last_trace);
    g_last_proof = serialize(p);
    *proof_len = g_last_proof.size();
  });
}
extern "C" void oracle_last_proof(uint8_t* out) { std::memcpy(out, g_last_proof.data(), g_last_proof.size()); }
// FRI-heavy workload: alphas = log_n QM31 values (4 words each); the proof
// bytes are kept until the next call (oracle_last_proof).
extern "C" int oracle_fri_prove_seeded(const uint32_t* const* coords4, uint32_t log_n, const uint32_t* alphas,
                                       const uint64_t* queries, size_t n_queries, int m31, size_t* proof_len) {
  return guard([&] {
    std::vector<QM31> a(log_n);
    for (uint32_t k = 0; k < log_n; k++)
      a[k] = QM31::from(alphas[4 * k], alphas[4 * k + 1], alphas[4 * k + 2], alphas[4 * k + 3]);
    const uint32_t* c[4] = {coords4[0], coords4[1], coords4[2], coords4[3]};
    g_last_proof = fri_prove_seeded(c, log_n, a.data(), std::vector<size_t>(queries, queries + n_queries), m31 != 0);
    *proof_len = g_last_proof.size();
  });
}
// Intermediates of the last prove: which = 0 composition evals (coord k), 1 quotients (coord k).
extern "C" size_t oracle_last_intermediate(int which, int k, uint32_t* out) {
  const auto& v = which == 0 ? g_last_trace.composition_evals : g_last_trace.quotients;
  if (k < 0 || (size_t)k >= v.size()) return 0;
  if (out) std::memcpy(out, v[k].data(), v[k].size() * 4);
  return v[k].size();
}
extern "C" void oracle_last_roots(uint8_t* out) {
  for (size_t i = 0; i < g_last_trace.roots.size(); i++) std::memcpy(out + 32 * i, g_last_trace.roots[i].data(), 32);
}

// 0 = accepted; -1 = rejected (reason via oracle_last_error()).
extern "C" int oracle_verify_wide_fib(const uint8_t* proof, size_t len, uint32_t log_n_rows, uint32_t n_cols,
                                      int m31) {
  return guard([&] { verify_wide_fib(proof, len, log_n_rows, n_cols, m31 != 0); });
}
