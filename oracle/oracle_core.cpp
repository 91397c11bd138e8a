// ORACLE — test infrastructure only (see stwo_oracle.hpp).
//
// Twiddles, circle FFT, bit reversal, lifted / mixed-degree Blake2s Merkle,
// FRI folds and the Blake2s channel, restated from vendored stwo
// (`crates/stwo/src`, paths relative to that crate).
#include "stwo_oracle.hpp"

#include <cstdio>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace oracle {

// ------------------------------------------------------------ twiddles ------
// prover/backend/cpu/circle.rs:294-311 slow_precompute_twiddles: for each
// tower level, the x coordinates of the first half of the coset in bit-reversed
// order, then coset <- coset.double(); a trailing 1 pads to a power of two.
// SimdBackend (prover/backend/simd/circle.rs:449-486) stores the same values
// doubled; this oracle keeps them canonical.
std::vector<uint32_t> slow_precompute_twiddles(Coset coset) {
  std::vector<uint32_t> tw;
  tw.reserve(coset.size());
  uint32_t levels = coset.log_size;
  for (uint32_t l = 0; l < levels; l++) {
    size_t i0 = tw.size();
    size_t half = coset.size() / 2;
    CPoint cur = coset.initial();
    CPoint step = coset.step();
    for (size_t j = 0; j < half; j++) { tw.push_back(cur.x); cur = padd(cur, step); }
    // bit-reverse the level segment
    uint32_t lg = 0; while (((size_t)1 << lg) < half) lg++;
    bit_reverse(tw.data() + i0, lg);
    coset = coset.dbl();
  }
  tw.push_back(1);
  return tw;
}

void batch_inverse(const uint32_t* in, uint32_t* out, size_t n) {
  if (n == 0) return;
  std::vector<uint32_t> pre(n);
  uint32_t acc = 1;
  for (size_t i = 0; i < n; i++) { pre[i] = acc; acc = mul(acc, in[i]); }
  uint32_t ia = inv(acc);
  for (size_t i = n; i-- > 0;) { out[i] = mul(ia, pre[i]); ia = mul(ia, in[i]); }
}

TwiddleTree precompute_twiddles(Coset root) {
  TwiddleTree t;
  t.root = root;
  t.tw = slow_precompute_twiddles(root);
  t.itw.resize(t.tw.size());
  // Chunked batch inversion like cpu/circle.rs:252-281 (values identical).
  const size_t chunk = 4096;
  if (t.tw.size() < chunk) {
    for (size_t i = 0; i < t.tw.size(); i++) t.itw[i] = inv(t.tw[i]);
  } else {
#pragma omp parallel for schedule(static)
    for (long c = 0; c < (long)(t.tw.size() / chunk); c++)
      batch_inverse(t.tw.data() + c * chunk, t.itw.data() + c * chunk, chunk);
  }
  return t;
}

// core/poly/utils.rs:98-114: layer i (0 = largest) of a line domain of log size
// `line_log` is buf[len - 2^(line_log - i) .. len - 2^(line_log - i - 1)].
const uint32_t* line_twiddles(const uint32_t* buf, size_t len, uint32_t line_log, uint32_t layer) {
  size_t sz = (size_t)1 << (line_log - layer);
  if (sz > len) throw std::runtime_error("Not enough twiddles!");
  return buf + (len - sz);
}

// --------------------------------------------------------------- FFT --------
// core/fft.rs:5-21
static inline void butterfly(uint32_t& v0, uint32_t& v1, uint32_t t) {
  uint32_t tmp = mul(v1, t);
  v1 = sub(v0, tmp);
  v0 = add(v0, tmp);
}
static inline void ibutterfly(uint32_t& v0, uint32_t& v1, uint32_t t) {
  uint32_t tmp = v0;
  v0 = add(tmp, v1);
  v1 = mul(sub(tmp, v1), t);
}
// cpu/circle.rs:313-327
template <class F>
static void fft_layer_loop(uint32_t* v, uint32_t i, size_t h, uint32_t t, F bf) {
  for (size_t l = 0; l < ((size_t)1 << i); l++) {
    size_t i0 = (h << (i + 1)) + l, i1 = i0 + ((size_t)1 << i);
    bf(v[i0], v[i1], t);
  }
}
// cpu/circle.rs:332-354: circle layer twiddle h from line layer 1 pairs (x, y):
// [y, -y, -x, x].
static inline uint32_t circle_twiddle(const uint32_t* lt0, size_t h) {
  uint32_t base = lt0[(h >> 1) ^ 1];
  bool negate = ((h ^ (h >> 1)) & 1) != 0;
  return negate ? neg(base) : base;
}

// PolyOps::interpolate: prover/backend/cpu/circle.rs:28-80 (SimdBackend's
// prover/backend/simd/circle.rs:138-166 gives the same values; below log 5 it
// calls the CPU code).  `half` is the evaluation domain's half coset.
void interpolate(uint32_t* values, uint32_t log_n, const Coset& half, const uint32_t* itw, size_t itw_len) {
  if (log_n == 0) return;
  if (log_n == 1) {
    uint32_t y = half.initial().y;
    uint32_t n = 2;
    uint32_t yn_inv = inv(mul(y, n));
    uint32_t y_inv = mul(yn_inv, n);
    uint32_t n_inv = mul(yn_inv, y);
    ibutterfly(values[0], values[1], y_inv);
    values[0] = mul(values[0], n_inv);
    values[1] = mul(values[1], n_inv);
    return;
  }
  if (log_n == 2) {
    CPoint p = half.initial();
    uint32_t n = 4;
    uint32_t xyn_inv = inv(mul(mul(p.x, p.y), n));
    uint32_t x_inv = mul(mul(xyn_inv, p.y), n);
    uint32_t y_inv = mul(mul(xyn_inv, p.x), n);
    uint32_t n_inv = mul(mul(xyn_inv, p.x), p.y);
    uint32_t* v = values;
    ibutterfly(v[0], v[1], y_inv);
    ibutterfly(v[2], v[3], neg(y_inv));
    ibutterfly(v[0], v[2], x_inv);
    ibutterfly(v[1], v[3], x_inv);
    for (int i = 0; i < 4; i++) v[i] = mul(v[i], n_inv);
    return;
  }
  uint32_t line_log = log_n - 1;
  const uint32_t* lt0 = line_twiddles(itw, itw_len, line_log, 0);
  for (size_t h = 0; h < ((size_t)1 << (log_n - 1)); h++)
    fft_layer_loop(values, 0, h, circle_twiddle(lt0, h), ibutterfly);
  for (uint32_t layer = 0; layer < line_log; layer++) {
    const uint32_t* lt = line_twiddles(itw, itw_len, line_log, layer);
    for (size_t h = 0; h < ((size_t)1 << (line_log - 1 - layer)); h++)
      fft_layer_loop(values, layer + 1, h, lt[h], ibutterfly);
  }
  uint32_t inv_n = inv(from_u32((uint32_t)1 << log_n));
  for (size_t i = 0; i < ((size_t)1 << log_n); i++) values[i] = mul(values[i], inv_n);
}

// CPU evaluate on the full domain (cpu/circle.rs:199-250): zero-extended
// coefficients, all line layers top-down, then the circle layer.
static void evaluate_cpu(const uint32_t* coeffs, uint32_t log_n, uint32_t log_eval, const Coset& half,
                         const uint32_t* tw, size_t tw_len, uint32_t* out) {
  size_t N = (size_t)1 << log_eval;
  for (size_t i = 0; i < N; i++) out[i] = i < ((size_t)1 << log_n) ? coeffs[i] : 0;
  if (log_eval == 1) {
    butterfly(out[0], out[1], half.initial().y);
    return;
  }
  if (log_eval == 2) {
    CPoint p = half.initial();
    butterfly(out[0], out[2], p.x);
    butterfly(out[1], out[3], p.x);
    butterfly(out[0], out[1], p.y);
    butterfly(out[2], out[3], neg(p.y));
    return;
  }
  uint32_t line_log = log_eval - 1;
  for (uint32_t layer = line_log; layer-- > 0;) {
    const uint32_t* lt = line_twiddles(tw, tw_len, line_log, layer);
    for (size_t h = 0; h < ((size_t)1 << (line_log - 1 - layer)); h++)
      fft_layer_loop(out, layer + 1, h, lt[h], butterfly);
  }
  const uint32_t* lt0 = line_twiddles(tw, tw_len, line_log, 0);
  for (size_t h = 0; h < N / 2; h++) fft_layer_loop(out, 0, h, circle_twiddle(lt0, h), butterfly);
}

// PolyOps::evaluate_into for SimdBackend, prover/backend/simd/circle.rs:388-443:
// below MIN_FFT_LOG_SIZE (5) the CPU path; otherwise 2^(log_eval - log_n)
// subdomain FFTs of the coefficients, subdomain i using slice
// [i << (log_n - 2 - l), (i + 1) << (log_n - 2 - l)) of each big-domain line
// twiddle layer l.
void evaluate(const uint32_t* coeffs, uint32_t log_n, uint32_t log_eval, const Coset& half,
              const uint32_t* tw, size_t tw_len, uint32_t* out) {
  if (log_eval < log_n) throw std::runtime_error("Can only evaluate on larger domains");
  if (log_n < 5) { evaluate_cpu(coeffs, log_n, log_eval, half, tw, tw_len, out); return; }
  uint32_t big_line_log = log_eval - 1;
  size_t n = (size_t)1 << log_n;
  for (size_t sub = 0; sub < ((size_t)1 << (log_eval - log_n)); sub++) {
    uint32_t* buf = out + sub * n;
    std::memcpy(buf, coeffs, n * 4);
    // line layers l = log_n-2 .. 0 (fft layer l+1), top-down
    for (uint32_t l = log_n - 1; l-- > 0;) {
      const uint32_t* lt = line_twiddles(tw, tw_len, big_line_log, l) + (sub << (log_n - 2 - l));
      for (size_t h = 0; h < ((size_t)1 << (log_n - 2 - l)); h++) fft_layer_loop(buf, l + 1, h, lt[h], butterfly);
    }
    const uint32_t* lt0 = line_twiddles(tw, tw_len, big_line_log, 0) + (sub << (log_n - 2));
    for (size_t h = 0; h < n / 2; h++) fft_layer_loop(buf, 0, h, circle_twiddle(lt0, h), butterfly);
  }
}

// cpu/circle.rs:82-99 + core/poly/utils.rs:27-38: coefficient fold at a point
// with mappings [y, x, pi(x), ...] reversed (natural coefficient order).
uint32_t eval_at_point_m31(const uint32_t* coeffs, uint32_t log_n, CPoint p) {
  if (log_n == 0) return coeffs[0];
  std::vector<uint32_t> maps{p.y};
  uint32_t x = p.x;
  for (uint32_t i = 1; i < log_n; i++) { maps.push_back(x); x = sub(add(sqr(x), sqr(x)), 1); }
  std::reverse(maps.begin(), maps.end());
  // Recursive definition written directly (small sizes only).
  struct R {
    static uint32_t go(const uint32_t* v, size_t n, const uint32_t* f) {
      if (n == 1) return v[0];
      uint32_t l = go(v, n / 2, f + 1), r = go(v + n / 2, n / 2, f + 1);
      return add(l, mul(r, f[0]));
    }
  };
  return R::go(coeffs, (size_t)1 << log_n, maps.data());
}

// --------------------------------------------------------- Merkle (lifted) --
// core/vcs_lifted/blake2_merkle.rs + prover/backend/cpu/merkle_lifted.rs:44-85.
static inline uint64_t lift_index(uint64_t i, uint32_t r) {
  return r == 0 ? i : ((i >> (r + 1)) << 1) + (i & 1);
}

std::vector<Hash> build_leaves(const std::vector<const uint32_t*>& cols, const std::vector<uint32_t>& log_sizes,
                               uint32_t L, bool m31) {
  if (cols.empty()) return {blake2s_hash(nullptr, 0, m31)};
  for (size_t c = 0; c + 1 < cols.size(); c++)
    if (log_sizes[c] > log_sizes[c + 1]) throw std::runtime_error("columns must be sorted by length");
  if (log_sizes[0] < 1) throw std::runtime_error("A column must be of length >= 2.");
  if (log_sizes.back() > L) throw std::runtime_error("lifting_log_size below max column size");
  size_t n = (size_t)1 << L;
  std::vector<Hash> out(n);
#pragma omp parallel for schedule(static)
  for (long long i = 0; i < (long long)n; i++) {
    Blake2s s;
    for (size_t c = 0; c < cols.size(); c++) s.update_u32(cols[c][lift_index((uint64_t)i, L - log_sizes[c])]);
    out[i] = finalize_hash(s, m31);
  }
  return out;
}

// SimdBackend's form of the same leaves (prover/backend/simd/blake2s_lifted.rs
// :42-160): message block b (columns [16b, 16b + 16) of the sorted list) is
// compressed at the size of its largest column, 2^S chaining values, each
// starting from the previous block's value at lift_index(i, S - S_prev)
// (lift_index(lift_index(i, a), b) == lift_index(i, a + b)); the last block
// runs at L with the final flag.  Fewer compressions than build_leaves when
// the columns differ in size; the same hashes.
std::vector<Hash> build_leaves_staged(const std::vector<const uint32_t*>& cols, const std::vector<uint32_t>& log_sizes,
                                      uint32_t L, bool m31) {
  if (cols.empty()) return {blake2s_hash(nullptr, 0, m31)};
  for (size_t c = 0; c + 1 < cols.size(); c++)
    if (log_sizes[c] > log_sizes[c + 1]) throw std::runtime_error("columns must be sorted by length");
  if (log_sizes[0] < 1) throw std::runtime_error("A column must be of length >= 2.");
  if (log_sizes.back() > L) throw std::runtime_error("lifting_log_size below max column size");
  using State = std::array<uint32_t, 8>;
  const size_t n_cols = cols.size(), n_blocks = (n_cols + 15) / 16;
  State init;
  {
    Blake2s b;
    std::memcpy(init.data(), b.h, 32);
  }
  std::vector<State> prev, next;
  uint32_t prev_log = 0;
  for (size_t blk = 0; blk < n_blocks; blk++) {
    const bool last = blk + 1 == n_blocks;
    const uint32_t S = last ? L : log_sizes[std::min(16 * blk + 15, n_cols - 1)];
    const uint64_t t = last ? 4 * (uint64_t)n_cols : 64 * (uint64_t)(blk + 1);
    next.assign((size_t)1 << S, State{});
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < (long long)next.size(); i++) {
      State h = blk == 0 ? init : prev[lift_index((uint64_t)i, S - prev_log)];
      uint32_t m[16];
      for (size_t k = 0; k < 16; k++) {
        const size_t c = 16 * blk + k;
        m[k] = c < n_cols ? cols[c][lift_index((uint64_t)i, S - log_sizes[c])] : 0u;
      }
      Blake2s::compress(h.data(), m, t, last);
      next[i] = h;
    }
    std::swap(prev, next);
    prev_log = S;
  }
  std::vector<Hash> out(prev.size());
#pragma omp parallel for schedule(static)
  for (long long i = 0; i < (long long)out.size(); i++) {
    std::memcpy(out[i].data(), prev[i].data(), 32);
    if (m31) out[i] = reduce_to_m31(out[i]);
  }
  return out;
}

std::vector<Hash> build_next_layer(const std::vector<Hash>& prev, bool m31) {
  size_t n = prev.size() / 2;
  std::vector<Hash> out(n);
#pragma omp parallel for schedule(static)
  for (long long i = 0; i < (long long)n; i++) {
    Blake2s s;
    s.update(prev[2 * i].data(), 32);
    s.update(prev[2 * i + 1].data(), 32);
    out[i] = finalize_hash(s, m31);
  }
  return out;
}

// prover/vcs_lifted/ops.rs:29-45 build_merkle_layers: stable sort by length,
// leaves, then lifting_log_size node layers; returned root first.
std::vector<std::vector<Hash>> build_merkle_layers(std::vector<const uint32_t*> cols, std::vector<uint32_t> log_sizes,
                                                   uint32_t L, bool m31, bool staged) {
  if (cols.empty()) return {build_leaves({}, {}, L, m31)};
  std::vector<size_t> order(cols.size());
  for (size_t i = 0; i < order.size(); i++) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return log_sizes[a] < log_sizes[b]; });
  std::vector<const uint32_t*> sc;
  std::vector<uint32_t> sl;
  for (size_t i : order) { sc.push_back(cols[i]); sl.push_back(log_sizes[i]); }
  std::vector<std::vector<Hash>> layers;
  layers.push_back(staged ? build_leaves_staged(sc, sl, L, m31) : build_leaves(sc, sl, L, m31));
  for (uint32_t i = 0; i < L; i++) layers.push_back(build_next_layer(layers.back(), m31));
  std::reverse(layers.begin(), layers.end());
  return layers;
}

// ------------------------------------------------- Merkle (mixed degree) ----
// prover/backend/cpu/blake2s.rs:13-26 + core/vcs/blake2_merkle.rs:17-38.
std::vector<Hash> commit_on_layer(uint32_t log_size, const Hash* prev, const std::vector<const uint32_t*>& cols,
                                  bool m31) {
  size_t n = (size_t)1 << log_size;
  std::vector<Hash> out(n);
#pragma omp parallel for schedule(static)
  for (long long i = 0; i < (long long)n; i++) {
    Blake2s s;
    if (prev) { s.update(prev[2 * i].data(), 32); s.update(prev[2 * i + 1].data(), 32); }
    for (auto c : cols) s.update_u32(c[i]);
    out[i] = finalize_hash(s, m31);
  }
  return out;
}

// ----------------------------------------------------------------- FRI ------
// prover/backend/cpu/fri.rs:67-92 fold_line_cpu, with x^{-1} taken from the
// twiddle tree like prover/backend/simd/fri.rs:32-122 (same values).
void fold_line(const uint32_t* const in[4], uint32_t log_m, const uint32_t* itw, size_t itw_len, QM31 alpha,
               uint32_t fold_step, uint32_t* const out[4]) {
  if (fold_step < 1 || fold_step > log_m) throw std::runtime_error("bad fold_step");
  std::vector<QM31> cur((size_t)1 << log_m);
  for (size_t i = 0; i < cur.size(); i++) cur[i] = QM31::from(in[0][i], in[1][i], in[2][i], in[3][i]);
  QM31 a = alpha;
  for (uint32_t s = 0; s < fold_step; s++) {
    uint32_t lg = log_m - s;
    const uint32_t* it = line_twiddles(itw, itw_len, lg, 0);
    std::vector<QM31> nxt(cur.size() / 2);
    for (size_t i = 0; i < nxt.size(); i++) {
      QM31 fx = cur[2 * i], fnx = cur[2 * i + 1];
      QM31 f0 = fx + fnx;
      QM31 f1 = qmul_m31(fx - fnx, it[i]);
      nxt[i] = f0 + a * f1;
    }
    cur.swap(nxt);
    a = a * a;
  }
  for (size_t i = 0; i < cur.size(); i++) {
    auto c = cur[i].coords();
    for (int k = 0; k < 4; k++) out[k][i] = c[k];
  }
}

// Direct form with domain points (cpu/fri.rs:67-92), for checking the tree form.
void fold_line_direct(const uint32_t* const in[4], const Coset& line_coset, QM31 alpha, uint32_t* const out[4]) {
  uint32_t lg = line_coset.log_size;
  for (size_t i = 0; i < ((size_t)1 << (lg - 1)); i++) {
    uint32_t x = line_coset.at(bit_reverse_index(i << 1, lg)).x;
    QM31 fx = QM31::from(in[0][2 * i], in[1][2 * i], in[2][2 * i], in[3][2 * i]);
    QM31 fnx = QM31::from(in[0][2 * i + 1], in[1][2 * i + 1], in[2][2 * i + 1], in[3][2 * i + 1]);
    QM31 r = (fx + fnx) + alpha * qmul_m31(fx - fnx, inv(x));
    auto c = r.coords();
    for (int k = 0; k < 4; k++) out[k][i] = c[k];
  }
}

void fold_circle_into_line_direct(uint32_t* const dst[4], const uint32_t* const src[4], const Coset& half,
                                  QM31 alpha) {
  uint32_t log_n = half.log_size + 1;
  QM31 a2 = alpha * alpha;
  for (size_t i = 0; i < ((size_t)1 << (log_n - 1)); i++) {
    uint64_t pi = circle_domain_index_at(half, bit_reverse_index(i << 1, log_n));
    uint32_t yinv = inv(index_to_point(pi).y);
    QM31 fp = QM31::from(src[0][2 * i], src[1][2 * i], src[2][2 * i], src[3][2 * i]);
    QM31 fnp = QM31::from(src[0][2 * i + 1], src[1][2 * i + 1], src[2][2 * i + 1], src[3][2 * i + 1]);
    QM31 fprime = (fp + fnp) + alpha * qmul_m31(fp - fnp, yinv);
    QM31 d = QM31::from(dst[0][i], dst[1][i], dst[2][i], dst[3][i]);
    auto c = (d * a2 + fprime).coords();
    for (int k = 0; k < 4; k++) dst[k][i] = c[k];
  }
}

// prover/backend/cpu/fri.rs:95-123 fold_circle_into_line_cpu; y^{-1} of the
// circle domain point bit_reverse(2i) equals the circle-layer inverse twiddle
// derived from line layer 0 of the tree (simd/fri.rs:124-172).
void fold_circle_into_line(uint32_t* const dst[4], const uint32_t* const src[4], const Coset& half, const uint32_t* itw,
                           size_t itw_len, QM31 alpha) {
  uint32_t log_n = half.log_size + 1;
  // simd/fri.rs:130-140: up to log 4 the CPU form with domain points (the
  // circle-from-line derivation needs a line layer of >= 2 twiddles).
  if (log_n <= 4) { fold_circle_into_line_direct(dst, src, half, alpha); return; }
  QM31 a2 = alpha * alpha;
  const uint32_t* lt0 = line_twiddles(itw, itw_len, log_n - 1, 0);
  for (size_t i = 0; i < ((size_t)1 << (log_n - 1)); i++) {
    uint32_t yinv = circle_twiddle(lt0, i);
    QM31 fp = QM31::from(src[0][2 * i], src[1][2 * i], src[2][2 * i], src[3][2 * i]);
    QM31 fnp = QM31::from(src[0][2 * i + 1], src[1][2 * i + 1], src[2][2 * i + 1], src[3][2 * i + 1]);
    QM31 f0 = fp + fnp;
    QM31 f1 = qmul_m31(fp - fnp, yinv);
    QM31 fprime = f0 + alpha * f1;
    QM31 d = QM31::from(dst[0][i], dst[1][i], dst[2][i], dst[3][i]);
    QM31 r = d * a2 + fprime;
    auto c = r.coords();
    for (int k = 0; k < 4; k++) dst[k][i] = c[k];
  }
}

// prover/backend/simd/fri.rs:174-195 decompose + :265-296 coefficient, on
// 16-lane packed vectors: the coefficient adds vectors [0, (n/16)/2) and
// subtracts vectors [(n/16)/2, n/16) (so n < 16 gives lambda = 0 and n = 16
// gives -sum/16); g subtracts lambda on vectors [0, ceil(n/16)/2) and adds it
// on the rest.
QM31 decompose(const uint32_t* const in[4], uint32_t log_n, uint32_t* const out[4]) {
  size_t n = (size_t)1 << log_n;
  size_t range = n / 16, half_a = range / 2;
  uint32_t s[4] = {0, 0, 0, 0};
  for (int k = 0; k < 4; k++) {
    for (size_t i = 0; i < 16 * half_a; i++) s[k] = add(s[k], in[k][i]);
    for (size_t i = 16 * half_a; i < 16 * range; i++) s[k] = sub(s[k], in[k][i]);
  }
  QM31 lambda = qmul_m31(QM31::from(s[0], s[1], s[2], s[3]), inv((uint32_t)n));
  size_t half_range = ((n + 15) / 16) / 2;
  for (size_t i = 0; i < n; i++) {
    QM31 v = QM31::from(in[0][i], in[1][i], in[2][i], in[3][i]);
    QM31 r = (i / 16 < half_range) ? v - lambda : v + lambda;
    auto c = r.coords();
    for (int k = 0; k < 4; k++) out[k][i] = c[k];
  }
  return lambda;
}

// ------------------------------------------------------------- channel ------
// core/channel/blake2s.rs:25-141.
void Channel::update_digest(const Hash& h) { digest = h; n_draws = 0; }
void Channel::mix_u32s(const uint32_t* data, size_t n) {
  Blake2s s; s.update(digest.data(), 32);
  for (size_t i = 0; i < n; i++) s.update_u32(data[i]);
  update_digest(finalize_hash(s, m31));
}
void Channel::mix_u64(uint64_t v) { uint32_t w[2] = {(uint32_t)v, (uint32_t)(v >> 32)}; mix_u32s(w, 2); }
void Channel::mix_felts(const QM31* f, size_t n) {
  Blake2s s; s.update(digest.data(), 32);
  for (size_t i = 0; i < n; i++) for (uint32_t c : f[i].coords()) s.update_u32(c);
  update_digest(finalize_hash(s, m31));
}
std::array<uint32_t, 8> Channel::draw_u32s() {
  uint8_t in[37];
  std::memcpy(in, digest.data(), 32);
  std::memcpy(in + 32, &n_draws, 4);
  in[36] = 0;
  n_draws++;
  Hash h = blake2s_hash(in, 37, m31);
  std::array<uint32_t, 8> w;
  std::memcpy(w.data(), h.data(), 32);
  return w;
}
std::array<uint32_t, 8> Channel::draw_base_felts() {
  for (;;) {
    auto w = draw_u32s();
    bool ok = true;
    for (uint32_t x : w) ok = ok && x < 2 * P;
    if (ok) { for (auto& x : w) x = reduce64(x); return w; }
  }
}
QM31 Channel::draw_secure_felt() { auto f = draw_base_felts(); return QM31::from(f[0], f[1], f[2], f[3]); }
std::vector<QM31> Channel::draw_secure_felts(size_t n) {
  std::vector<QM31> out;
  std::vector<uint32_t> pool;
  size_t pos = 0;
  while (out.size() < n) {
    if (pool.size() - pos < 4) {
      auto f = draw_base_felts();
      pool.erase(pool.begin(), pool.begin() + pos); pos = 0;
      pool.insert(pool.end(), f.begin(), f.end());
      continue;
    }
    out.push_back(QM31::from(pool[pos], pool[pos + 1], pool[pos + 2], pool[pos + 3]));
    pos += 4;
  }
  return out;
}
void Channel::mix_root(const Hash& root) {  // core/vcs_lifted/blake2_merkle.rs:49-56
  Blake2s s; s.update(digest.data(), 32); s.update(root.data(), 32);
  update_digest(finalize_hash(s, m31));
}
Hash Channel::pow_prefixed(uint32_t n_bits) const {
  Blake2s s;
  uint32_t prefix = 0x12345678u;
  uint8_t zeros[12] = {0};
  s.update(&prefix, 4); s.update(zeros, 12); s.update(digest.data(), 32); s.update(&n_bits, 4);
  return finalize_hash(s, m31);
}
static inline uint32_t trailing_zeros_128(const Hash& h) {
  uint32_t tz = 0;
  for (int i = 0; i < 16; i++) {
    if (h[i] == 0) { tz += 8; continue; }
    return tz + (uint32_t)__builtin_ctz(h[i]);
  }
  return 128;
}
bool Channel::verify_pow_nonce(uint32_t n_bits, uint64_t nonce) const {
  Hash pre = pow_prefixed(n_bits);
  Blake2s s; s.update(pre.data(), 32); s.update(&nonce, 8);
  return trailing_zeros_128(finalize_hash(s, m31)) >= n_bits;
}
// prover/backend/simd/grind.rs:25-60, 98-138: the smallest nonce
// (hi << 32) | low with low < 2^GRIND_LOW_BITS (20), searched hi-major; a hit
// needs trailing_zeros(first digest word) >= n_bits (n_bits <= 32).
uint64_t Channel::grind(uint32_t n_bits) const {
  if (n_bits > 32) throw std::runtime_error("pow_bits > 32 is not supported");
  Hash pre = pow_prefixed(n_bits);
  for (uint64_t hi = 0;; hi++) {
    for (uint64_t low = 0; low < (1ull << 20); low++) {
      uint64_t nonce = (hi << 32) | low;
      Blake2s s; s.update(pre.data(), 32); s.update(&nonce, 8);
      Hash h = finalize_hash(s, m31);
      uint32_t w0; std::memcpy(&w0, h.data(), 4);
      uint32_t tz = w0 == 0 ? 32 : (uint32_t)__builtin_ctz(w0);
      if (tz >= n_bits) return nonce;
    }
  }
}

}  // namespace oracle
