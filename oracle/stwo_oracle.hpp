// ORACLE — test infrastructure only.
//
// A CPU restatement of stwo's SimdBackend semantics for the commit + FRI path
// (vendored stwo `crates/stwo/src`, paths below are relative to that crate).
// It is the bit-exactness checker for the B200 backend and the timed CPU
// baseline.  Only tests/, __graft_entry__.smoke() and bench.py's CPU legs may
// load it; the product path never does.
//
// Parity pins: Blake2s("a") KAT (core/vcs/blake2_hash.rs:134-139), channel KATs
// (core/channel/blake2s.rs:213-247), domain_line_twiddles slicing
// (core/poly/utils.rs:141-148), lifted leaf byte layouts
// (prover/vcs_lifted/prover.rs:247-275), FFT vs naive evaluation
// (prover/backend/simd/fft/ifft.rs:687-718, rfft.rs:717-746).
#pragma once
#include <cstdint>
#include <cstring>
#include <vector>
#include <array>
#include <string>
#include <algorithm>
#include <stdexcept>

namespace oracle {

// ---------------------------------------------------------------- M31 -------
// core/fields/m31.rs:13  P = 2^31 - 1.
constexpr uint32_t P = 2147483647u;

// Packed add / sub exactly as prover/backend/simd/m31.rs:150-162, 253-265:
// add = min(a+b, a+b-P), sub = min(a-b+P, a-b) on wrapping u32.  For inputs in
// [0, P] they coincide with the scalar partial_reduce forms (core/fields/m31.rs).
inline uint32_t add(uint32_t a, uint32_t b) {
  uint32_t c = a + b;
  uint32_t d = c - P;
  return c < d ? c : d;
}
inline uint32_t sub(uint32_t a, uint32_t b) {
  uint32_t c = a - b;
  uint32_t d = c + P;
  return d < c ? d : c;
}
// Scalar negation, core/fields/m31.rs (Neg): partial_reduce(P - a) -> neg(0) = 0.
inline uint32_t neg(uint32_t a) { uint32_t c = P - a; return c >= P ? c - P : c; }
// Packed negation, simd/m31.rs (Neg for PackedM31): P - a, so neg(0) = P.
inline uint32_t neg_packed(uint32_t a) { return P - a; }
// core/fields/m31.rs:58-60 M31::reduce for val in [0, P^2).
inline uint32_t reduce64(uint64_t v) {
  return (uint32_t)(((((v >> 31) + v + 1) >> 31) + v) & (uint64_t)P);
}
inline uint32_t mul(uint32_t a, uint32_t b) { return reduce64((uint64_t)a * b); }
inline uint32_t sqr(uint32_t a) { return mul(a, a); }
inline uint32_t pow(uint32_t a, uint64_t e) {
  uint32_t r = 1;
  while (e) { if (e & 1) r = mul(r, a); a = mul(a, a); e >>= 1; }
  return r;
}
inline uint32_t inv(uint32_t a) {
  if (a % P == 0) throw std::runtime_error("0 has no inverse");
  return pow(a, (uint64_t)P - 2);
}
// M31::from(u32) = reduce(u32) (core/fields/m31.rs From<u32>).
inline uint32_t from_u32(uint32_t v) { return reduce64(v); }

// ---------------------------------------------------------------- CM31 ------
// core/fields/cm31.rs: a + b i with i^2 = -1.
struct CM31 {
  uint32_t a = 0, b = 0;
  bool operator==(const CM31& o) const { return a == o.a && b == o.b; }
};
inline CM31 operator+(CM31 x, CM31 y) { return {add(x.a, y.a), add(x.b, y.b)}; }
inline CM31 operator-(CM31 x, CM31 y) { return {sub(x.a, y.a), sub(x.b, y.b)}; }
inline CM31 operator*(CM31 x, CM31 y) {  // cm31.rs:44-54
  return {sub(mul(x.a, y.a), mul(x.b, y.b)), add(mul(x.a, y.b), mul(x.b, y.a))};
}
inline CM31 cneg(CM31 x) { return {neg(x.a), neg(x.b)}; }
inline CM31 cinv(CM31 x) {  // cm31.rs FieldExpOps::inverse
  uint32_t d = inv(add(sqr(x.a), sqr(x.b)));
  return CM31{x.a, neg(x.b)} * CM31{d, 0};
}

// ---------------------------------------------------------------- QM31 ------
// core/fields/qm31.rs: (a + b i) + (c + d i) u with u^2 = 2 + i  (R = (2,1)).
struct QM31 {
  CM31 x, y;  // x + y u
  bool operator==(const QM31& o) const { return x == o.x && y == o.y; }
  bool operator!=(const QM31& o) const { return !(*this == o); }
  std::array<uint32_t, 4> coords() const { return {x.a, x.b, y.a, y.b}; }
  static QM31 from(uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
    return QM31{CM31{a, b}, CM31{c, d}};
  }
  static QM31 base(uint32_t a) { return from(a, 0, 0, 0); }
  static QM31 zero() { return from(0, 0, 0, 0); }
  static QM31 one() { return from(1, 0, 0, 0); }
  bool is_zero() const { return x.a == 0 && x.b == 0 && y.a == 0 && y.b == 0; }
};
constexpr CM31 QM31_R{2, 1};
inline QM31 operator+(QM31 p, QM31 q) { return {p.x + q.x, p.y + q.y}; }
inline QM31 operator-(QM31 p, QM31 q) { return {p.x - q.x, p.y - q.y}; }
inline QM31 operator*(QM31 p, QM31 q) {  // qm31.rs:78-88
  return {p.x * q.x + QM31_R * (p.y * q.y), p.x * q.y + p.y * q.x};
}
inline QM31 qmul_m31(QM31 p, uint32_t m) {
  return QM31::from(mul(p.x.a, m), mul(p.x.b, m), mul(p.y.a, m), mul(p.y.b, m));
}
inline QM31 qadd_m31(QM31 p, uint32_t m) { p.x.a = add(p.x.a, m); return p; }
inline QM31 qneg(QM31 p) { return {cneg(p.x), cneg(p.y)}; }
inline QM31 qsqr(QM31 p) { return p * p; }
inline QM31 qinv(QM31 p) {  // qm31.rs:125-133
  CM31 b2 = p.y * p.y;
  CM31 ib2{neg(b2.b), b2.a};
  CM31 denom = (p.x * p.x) - (b2 + b2 + ib2);
  CM31 di = cinv(denom);
  return {p.x * di, cneg(p.y) * di};
}
inline QM31 qpow(QM31 a, uint64_t e) {
  QM31 r = QM31::one();
  while (e) { if (e & 1) r = r * a; a = a * a; e >>= 1; }
  return r;
}

// -------------------------------------------------------------- circle -------
// core/circle.rs: points on x^2 + y^2 = 1, group law (x1x2 - y1y2, x1y2 + y1x2).
struct CPoint { uint32_t x = 1, y = 0; };
inline CPoint padd(CPoint p, CPoint q) {
  return {sub(mul(p.x, q.x), mul(p.y, q.y)), add(mul(p.x, q.y), mul(p.y, q.x))};
}
inline CPoint pdouble(CPoint p) { return padd(p, p); }
inline CPoint pconj(CPoint p) { return {p.x, neg(p.y)}; }
// core/circle.rs:202  M31_CIRCLE_GEN = (2, 1268011823), order 2^31.
constexpr CPoint CIRCLE_GEN{2u, 1268011823u};
constexpr uint32_t CIRCLE_LOG_ORDER = 31;
inline CPoint pmul(CPoint p, uint64_t s) {  // circle.rs:71-82 (double-and-add)
  CPoint r{1, 0};
  while (s) { if (s & 1) r = padd(r, p); p = pdouble(p); s >>= 1; }
  return r;
}
// CirclePointIndex arithmetic modulo 2^31 (circle.rs:219-282).
inline uint64_t idx_reduce(uint64_t i) { return i & ((1ull << 31) - 1); }
inline CPoint index_to_point(uint64_t i) { return pmul(CIRCLE_GEN, idx_reduce(i)); }
inline uint64_t subgroup_gen(uint32_t log_size) { return 1ull << (31 - log_size); }

// Coset = initial_index + <step> (circle.rs:284-413).
struct Coset {
  uint64_t initial_index = 0, step_size = 0;
  uint32_t log_size = 0;
  static Coset make(uint64_t initial_index, uint32_t log_size) {
    return Coset{idx_reduce(initial_index), subgroup_gen(log_size), log_size};
  }
  static Coset subgroup(uint32_t log_size) { return make(0, log_size); }
  static Coset odds(uint32_t log_size) { return make(subgroup_gen(log_size + 1), log_size); }
  static Coset half_odds(uint32_t log_size) { return make(subgroup_gen(log_size + 2), log_size); }
  size_t size() const { return (size_t)1 << log_size; }
  uint64_t index_at(uint64_t i) const { return idx_reduce(initial_index + idx_reduce(step_size * i)); }
  CPoint at(uint64_t i) const { return index_to_point(index_at(i)); }
  CPoint initial() const { return index_to_point(initial_index); }
  CPoint step() const { return index_to_point(step_size); }
  Coset dbl() const {
    return Coset{idx_reduce(initial_index * 2), idx_reduce(step_size * 2), log_size ? log_size - 1 : 0};
  }
  Coset repeated_double(uint32_t n) const { Coset c = *this; for (uint32_t i = 0; i < n; i++) c = c.dbl(); return c; }
  Coset conjugate() const {
    return Coset{idx_reduce((1ull << 31) - initial_index), idx_reduce((1ull << 31) - step_size), log_size};
  }
  bool operator==(const Coset& o) const {
    return initial_index == o.initial_index && step_size == o.step_size && log_size == o.log_size;
  }
  bool is_doubling_of(const Coset& o) const {
    return log_size <= o.log_size && *this == o.repeated_double(o.log_size - log_size);
  }
};

// CanonicCoset(n) (core/poly/circle/canonic.rs:28-48): coset = odds(n),
// circle_domain().half_coset = half_odds(n - 1).
inline Coset canonic_half_coset(uint32_t log_size) { return Coset::half_odds(log_size - 1); }

// CircleDomain point i (core/poly/circle/domain.rs:56-66): first half_coset,
// then its conjugate (negated indices).
inline uint64_t circle_domain_index_at(const Coset& half, uint64_t i) {
  if (i < half.size()) return half.index_at(i);
  return idx_reduce((1ull << 31) - half.index_at(i - half.size()));
}

// core/utils.rs:79-84
inline uint64_t bit_reverse_index(uint64_t i, uint32_t log_size) {
  if (log_size == 0) return i;
  uint64_t r = 0;
  for (uint32_t b = 0; b < log_size; b++) r |= ((i >> b) & 1ull) << (log_size - 1 - b);
  return r;
}
template <class T> void bit_reverse(T* v, uint32_t log_n) {  // core/utils.rs:91-101
  size_t n = (size_t)1 << log_n;
  for (size_t i = 0; i < n; i++) {
    size_t j = bit_reverse_index(i, log_n);
    if (j > i) std::swap(v[i], v[j]);
  }
}

// -------------------------------------------------------------- Blake2s ------
// Blake2s-256 (RFC 7693), the hash of crate blake2 = 0.10.6 used by
// core/vcs/blake2_hash.rs:84-94.  Written from the RFC.
struct Blake2s {
  static constexpr uint32_t IV[8] = {0x6A09E667u, 0xBB67AE85u, 0x3C6EF372u, 0xA54FF53Au,
                                      0x510E527Fu, 0x9B05688Cu, 0x1F83D9ABu, 0x5BE0CD19u};
  static constexpr uint8_t SIGMA[10][16] = {
      {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15},
      {14, 10, 4, 8, 9, 15, 13, 6, 1, 12, 0, 2, 11, 7, 5, 3},
      {11, 8, 12, 0, 5, 2, 15, 13, 10, 14, 3, 6, 7, 1, 9, 4},
      {7, 9, 3, 1, 13, 12, 11, 14, 2, 6, 5, 10, 4, 0, 15, 8},
      {9, 0, 5, 7, 2, 4, 10, 15, 14, 1, 11, 12, 6, 8, 3, 13},
      {2, 12, 6, 10, 0, 11, 8, 3, 4, 13, 7, 5, 15, 14, 1, 9},
      {12, 5, 1, 15, 14, 13, 4, 10, 0, 7, 6, 3, 9, 2, 8, 11},
      {13, 11, 7, 14, 12, 1, 3, 9, 5, 0, 15, 4, 8, 6, 2, 10},
      {6, 15, 14, 9, 11, 3, 0, 8, 12, 2, 13, 7, 1, 4, 10, 5},
      {10, 2, 8, 4, 7, 6, 1, 5, 15, 11, 9, 14, 3, 12, 13, 0}};
  static inline uint32_t rotr(uint32_t x, int n) { return (x >> n) | (x << (32 - n)); }
  static void compress(uint32_t h[8], const uint32_t m[16], uint64_t t, bool last) {
    uint32_t v[16];
    for (int i = 0; i < 8; i++) { v[i] = h[i]; v[i + 8] = IV[i]; }
    v[12] ^= (uint32_t)t;
    v[13] ^= (uint32_t)(t >> 32);
    if (last) v[14] = ~v[14];
    auto G = [&](int a, int b, int c, int d, uint32_t x, uint32_t y) {
      v[a] = v[a] + v[b] + x; v[d] = rotr(v[d] ^ v[a], 16);
      v[c] = v[c] + v[d];     v[b] = rotr(v[b] ^ v[c], 12);
      v[a] = v[a] + v[b] + y; v[d] = rotr(v[d] ^ v[a], 8);
      v[c] = v[c] + v[d];     v[b] = rotr(v[b] ^ v[c], 7);
    };
    for (int r = 0; r < 10; r++) {
      const uint8_t* s = SIGMA[r];
      G(0, 4, 8, 12, m[s[0]], m[s[1]]);
      G(1, 5, 9, 13, m[s[2]], m[s[3]]);
      G(2, 6, 10, 14, m[s[4]], m[s[5]]);
      G(3, 7, 11, 15, m[s[6]], m[s[7]]);
      G(0, 5, 10, 15, m[s[8]], m[s[9]]);
      G(1, 6, 11, 12, m[s[10]], m[s[11]]);
      G(2, 7, 8, 13, m[s[12]], m[s[13]]);
      G(3, 4, 9, 14, m[s[14]], m[s[15]]);
    }
    for (int i = 0; i < 8; i++) h[i] ^= v[i] ^ v[i + 8];
  }

  // Streaming state: buffers one block so the final block is compressed with
  // the last-block flag, like any RFC 7693 implementation.
  uint32_t h[8];
  uint8_t buf[64];
  size_t buflen = 0;
  uint64_t t = 0;
  Blake2s() { reset(); }
  void reset() {
    for (int i = 0; i < 8; i++) h[i] = IV[i];
    h[0] ^= 0x01010000u ^ 32u;  // digest length 32, no key, fanout/depth 1
    buflen = 0; t = 0;
  }
  void update(const void* data, size_t len) {
    const uint8_t* p = (const uint8_t*)data;
    while (len) {
      if (buflen == 64) {
        t += 64;
        uint32_t m[16]; std::memcpy(m, buf, 64);
        compress(h, m, t, false);
        buflen = 0;
      }
      size_t take = std::min(len, (size_t)(64 - buflen));
      std::memcpy(buf + buflen, p, take);
      buflen += take; p += take; len -= take;
    }
  }
  void update_u32(uint32_t w) { update(&w, 4); }
  std::array<uint8_t, 32> finalize() {
    t += buflen;
    std::memset(buf + buflen, 0, 64 - buflen);
    uint32_t m[16]; std::memcpy(m, buf, 64);
    compress(h, m, t, true);
    std::array<uint8_t, 32> out;
    std::memcpy(out.data(), h, 32);
    return out;
  }
};

using Hash = std::array<uint8_t, 32>;

// core/vcs/blake2_hash.rs:110-118: each LE u32 word reduced with M31::reduce.
inline Hash reduce_to_m31(Hash h) {
  for (int i = 0; i < 8; i++) {
    uint32_t w; std::memcpy(&w, h.data() + 4 * i, 4);
    w = reduce64(w);
    std::memcpy(h.data() + 4 * i, &w, 4);
  }
  return h;
}
inline Hash finalize_hash(Blake2s& s, bool m31_output) {
  Hash h = s.finalize();
  return m31_output ? reduce_to_m31(h) : h;
}
inline Hash blake2s_hash(const void* data, size_t len, bool m31_output = false) {
  Blake2s s; s.update(data, len); return finalize_hash(s, m31_output);
}

}  // namespace oracle

// ------------------------------------------------------ algorithm entry points
namespace oracle {

struct TwiddleTree {
  Coset root;
  std::vector<uint32_t> tw, itw;  // canonical values, CpuBackend layout
};
std::vector<uint32_t> slow_precompute_twiddles(Coset coset);
TwiddleTree precompute_twiddles(Coset root);
void batch_inverse(const uint32_t* in, uint32_t* out, size_t n);
const uint32_t* line_twiddles(const uint32_t* buf, size_t len, uint32_t line_log, uint32_t layer);

void interpolate(uint32_t* values, uint32_t log_n, const Coset& half, const uint32_t* itw, size_t itw_len);
void evaluate(const uint32_t* coeffs, uint32_t log_n, uint32_t log_eval, const Coset& half, const uint32_t* tw,
              size_t tw_len, uint32_t* out);
uint32_t eval_at_point_m31(const uint32_t* coeffs, uint32_t log_n, CPoint p);

std::vector<Hash> build_leaves(const std::vector<const uint32_t*>& cols, const std::vector<uint32_t>& log_sizes,
                               uint32_t L, bool m31);
std::vector<Hash> build_leaves_staged(const std::vector<const uint32_t*>& cols, const std::vector<uint32_t>& log_sizes,
                                      uint32_t L, bool m31);
std::vector<Hash> build_next_layer(const std::vector<Hash>& prev, bool m31);
// staged: the leaves in SimdBackend's staged form (build_leaves_staged)
std::vector<std::vector<Hash>> build_merkle_layers(std::vector<const uint32_t*> cols, std::vector<uint32_t> log_sizes,
                                                   uint32_t L, bool m31, bool staged = false);
std::vector<Hash> commit_on_layer(uint32_t log_size, const Hash* prev, const std::vector<const uint32_t*>& cols,
                                  bool m31);

void fold_line(const uint32_t* const in[4], uint32_t log_m, const uint32_t* itw, size_t itw_len, QM31 alpha,
               uint32_t fold_step, uint32_t* const out[4]);
void fold_line_direct(const uint32_t* const in[4], const Coset& line_coset, QM31 alpha, uint32_t* const out[4]);
void fold_circle_into_line(uint32_t* const dst[4], const uint32_t* const src[4], const Coset& half, const uint32_t* itw,
                           size_t itw_len, QM31 alpha);
void fold_circle_into_line_direct(uint32_t* const dst[4], const uint32_t* const src[4], const Coset& half,
                                  QM31 alpha);
QM31 decompose(const uint32_t* const in[4], uint32_t log_n, uint32_t* const out[4]);

struct Channel {
  Hash digest{};
  uint32_t n_draws = 0;
  bool m31 = false;
  void update_digest(const Hash& h);
  void mix_u32s(const uint32_t* data, size_t n);
  void mix_u64(uint64_t v);
  void mix_felts(const QM31* f, size_t n);
  std::array<uint32_t, 8> draw_u32s();
  std::array<uint32_t, 8> draw_base_felts();
  QM31 draw_secure_felt();
  std::vector<QM31> draw_secure_felts(size_t n);
  void mix_root(const Hash& root);
  Hash pow_prefixed(uint32_t n_bits) const;
  bool verify_pow_nonce(uint32_t n_bits, uint64_t nonce) const;
  uint64_t grind(uint32_t n_bits) const;
};

}  // namespace oracle
