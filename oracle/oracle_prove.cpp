// ORACLE — test infrastructure only (see stwo_oracle.hpp).
//
// Restatement of stwo's prove flow for the Wide-Fibonacci AIR on the Blake2s
// Merkle channel, SimdBackend semantics:
//   trace gen            examples/src/wide_fibonacci/mod.rs:27-50
//   commitment scheme    crates/stwo/src/prover/pcs/mod.rs:374-386,512-803
//   composition          constraint-framework/src/prover/component_prover.rs:29-160,
//                        crates/stwo/src/prover/air/accumulation.rs (powers, finalize)
//   prove                crates/stwo/src/prover/mod.rs:41-138
//   quotients            crates/stwo/src/prover/pcs/quotient_ops.rs:81-233,
//                        prover/backend/simd/quotients.rs:34-164,
//                        core/pcs/quotients.rs:223-276, core/constraints.rs:119-134
//   FRI                  crates/stwo/src/prover/fri.rs:133-488, core/fri.rs:31-80
//   queries / decommit   core/queries.rs:11-58, prover/vcs_lifted/prover.rs:58-196,
//                        core/pcs/utils.rs:195-213
// and the canonical byte serialization of the resulting proof (struct field
// order of core/pcs/quotients.rs:27-35, core/fri.rs:361-395).
#include <map>

#include "stwo_oracle.hpp"
#include "stwo_oracle_prove.hpp"

namespace oracle {

// ------------------------------------------------------- secure points ------
SPoint sadd(const SPoint& p, const SPoint& q) { return {p.x * q.x - p.y * q.y, p.x * q.y + p.y * q.x}; }
QM31 double_x(QM31 x) { QM31 s = x * x; return (s + s) - QM31::one(); }
SPoint sdouble(const SPoint& p) { return sadd(p, p); }
SPoint srepeated_double(SPoint p, uint32_t n) { for (uint32_t i = 0; i < n; i++) p = sdouble(p); return p; }
QM31 qconj(QM31 a) { return {a.x, cneg(a.y)}; }  // core/fields/mod.rs:413-415

// core/circle.rs:169-181
SPoint get_random_point(Channel& ch) {
  QM31 t = ch.draw_secure_felt();
  QM31 t2 = t * t;
  QM31 inv1 = qinv(t2 + QM31::one());
  return {(QM31::one() + qneg(t2)) * inv1, (t + t) * inv1};
}

// core/constraints.rs:12-34 on an M31 point.
uint32_t coset_vanishing_m31(const Coset& coset, CPoint p) {
  // p - coset.initial + step_size.half().to_point()
  CPoint init = coset.initial();
  CPoint shifted = padd(p, pconj(init));
  shifted = padd(shifted, index_to_point(coset.step_size >> 1));
  uint32_t x = shifted.x;
  for (uint32_t i = 1; i < coset.log_size; i++) x = sub(add(sqr(x), sqr(x)), 1);
  return x;
}
QM31 coset_vanishing_q(const Coset& coset, SPoint p) {
  CPoint init = coset.initial();
  CPoint h = index_to_point(coset.step_size >> 1);
  SPoint minus_init{QM31::base(init.x), QM31::base(neg(init.y))};
  SPoint hh{QM31::base(h.x), QM31::base(h.y)};
  SPoint s = sadd(sadd(p, minus_init), hh);
  QM31 x = s.x;
  for (uint32_t i = 1; i < coset.log_size; i++) x = double_x(x);
  return x;
}

// Polynomial value at a secure point from natural-order coefficients
// (prover/backend/cpu/circle.rs:82-99 with core/poly/utils.rs:27-70).
QM31 eval_at_point_q(const uint32_t* coeffs, uint32_t log_n, const SPoint& p) {
  if (log_n == 0) return QM31::base(coeffs[0]);
  std::vector<QM31> maps{p.y};
  QM31 x = p.x;
  for (uint32_t i = 1; i < log_n; i++) { maps.push_back(x); x = double_x(x); }
  std::reverse(maps.begin(), maps.end());
  // fold(values, factors) = fold(lhs, factors[1:]) + fold(rhs, factors[1:]) * factors[0];
  // evaluated bottom-up: level j combines pairs at distance 2^(log_n-1-j)... with
  // factor maps[log_n - 1 - level].
  size_t n = (size_t)1 << log_n;
  std::vector<QM31> cur(n / 2);
  const QM31& f_last = maps[log_n - 1];
  for (size_t i = 0; i < n / 2; i++)
    cur[i] = QM31::base(coeffs[2 * i]) + qmul_m31(f_last, coeffs[2 * i + 1]);
  for (int lv = (int)log_n - 2; lv >= 0; lv--) {
    size_t m = cur.size() / 2;
    for (size_t i = 0; i < m; i++) cur[i] = cur[2 * i] + cur[2 * i + 1] * maps[lv];
    cur.resize(m);
  }
  return cur[0];
}

// core/poly/line.rs / prover/line.rs:54-99: interpolate a size-n line
// evaluation (bit-reversed) into ordered coefficients.
std::vector<QM31> line_interpolate_ordered(std::vector<QM31> vals, const Coset& line_coset) {
  size_t n = vals.size();
  uint32_t lg = 0; while (((size_t)1 << lg) < n) lg++;
  bit_reverse(vals.data(), lg);
  Coset dom = line_coset;
  while (dom.size() > 1) {
    size_t sz = dom.size();
    for (size_t c = 0; c < n; c += sz) {
      for (size_t i = 0; i < sz / 2; i++) {
        uint32_t xinv = inv(dom.at(i).x);
        QM31 l = vals[c + i], r = vals[c + i + sz / 2];
        vals[c + i] = l + r;
        vals[c + i + sz / 2] = qmul_m31(l - r, xinv);
      }
    }
    dom = dom.dbl();
  }
  uint32_t ninv = inv(from_u32((uint32_t)n));
  for (auto& v : vals) v = qmul_m31(v, ninv);
  bit_reverse(vals.data(), lg);  // into_ordered_coefficients
  return vals;
}

// ------------------------------------------------------- Merkle decommit ----
// prover/vcs_lifted/prover.rs:58-196.
void merkle_decommit(const std::vector<std::vector<Hash>>& layers_root_first, std::vector<size_t> queries,
                     const std::vector<const uint32_t*>& cols, const std::vector<uint32_t>& log_sizes,
                     std::vector<std::vector<uint32_t>>& queried_values, std::vector<Hash>& witness) {
  size_t max_log = layers_root_first.size() - 1;
  queried_values.clear();
  for (size_t c = 0; c < cols.size(); c++) {
    size_t shift = max_log - log_sizes[c];
    std::vector<uint32_t> v;
    for (size_t pos : queries) v.push_back(cols[c][((pos >> (shift + 1)) << 1) + (pos & 1)]);
    queried_values.push_back(v);
  }
  queries.erase(std::unique(queries.begin(), queries.end()), queries.end());
  std::vector<size_t> prev = queries;
  for (size_t layer_log = max_log; layer_log-- > 0;) {
    const auto& children = layers_root_first[layer_log + 1];
    std::vector<size_t> cur;
    for (size_t i = 0; i < prev.size();) {
      size_t first = prev[i];
      bool pair = (i + 1 < prev.size()) && ((first ^ 1) == prev[i + 1]);
      if (!pair) witness.push_back(children[first ^ 1]);
      cur.push_back(first >> 1);
      i += pair ? 2 : 1;
    }
    prev = cur;
  }
}

// prover/fri.rs:459-488
static void decommit_positions_and_witness(const std::vector<std::vector<uint32_t>>& coords4,
                                           const std::vector<size_t>& queries, uint32_t fold_step,
                                           std::vector<size_t>& positions, std::vector<QM31>& witness) {
  for (size_t i = 0; i < queries.size();) {
    size_t j = i;
    while (j < queries.size() && (queries[j] >> fold_step) == (queries[i] >> fold_step)) j++;
    size_t start = (queries[i] >> fold_step) << fold_step;
    size_t qi = i;
    for (size_t pos = start; pos < start + ((size_t)1 << fold_step); pos++) {
      positions.push_back(pos);
      QM31 e = QM31::from(coords4[0][pos], coords4[1][pos], coords4[2][pos], coords4[3][pos]);
      if (qi < j && queries[qi] == pos) qi++;
      else witness.push_back(e);
    }
    i = j;
  }
}

static std::vector<size_t> fold_queries(const std::vector<size_t>& q, uint32_t n) {
  std::vector<size_t> r;
  for (size_t p : q) { size_t f = p >> n; if (r.empty() || r.back() != f) r.push_back(f); }
  return r;
}

// ------------------------------------------------------------- tree ---------
struct Tree {
  std::vector<std::vector<uint32_t>> coeffs;  // natural order
  std::vector<std::vector<uint32_t>> evals;   // bit-reversed evaluations
  std::vector<uint32_t> eval_logs;
  std::vector<std::vector<Hash>> layers;      // root first
  Hash root() const { return layers[0][0]; }
};

static Tree commit_polys(std::vector<std::vector<uint32_t>> coeffs, uint32_t log_blowup, const TwiddleTree& tw,
                         bool m31) {
  Tree t;
  t.coeffs = std::move(coeffs);
  size_t n = t.coeffs.size();
  t.evals.resize(n);
  t.eval_logs.resize(n);
  uint32_t max_log = 0;
#pragma omp parallel for schedule(dynamic, 1)
  for (long c = 0; c < (long)n; c++) {
    uint32_t lg = 0; while (((size_t)1 << lg) < t.coeffs[c].size()) lg++;
    uint32_t le = lg + log_blowup;
    t.evals[c].resize((size_t)1 << le);
    evaluate(t.coeffs[c].data(), lg, le, canonic_half_coset(le), tw.tw.data(), tw.tw.size(), t.evals[c].data());
    t.eval_logs[c] = le;
  }
  for (uint32_t l : t.eval_logs) max_log = std::max(max_log, l);
  std::vector<const uint32_t*> ptrs;
  for (auto& e : t.evals) ptrs.push_back(e.data());
  t.layers = build_merkle_layers(ptrs, t.eval_logs, max_log, m31);
  return t;
}

// ------------------------------------------------------------ prover --------
Proof prove_wide_fib(const WideFibConfig& cfg, const uint32_t* in_a, const uint32_t* in_b, ProveTrace* dbg) {
  const uint32_t log_n = cfg.log_n_rows, N = cfg.n_cols, blowup = cfg.log_blowup;
  const bool m31 = cfg.m31_channel;
  if (N < 3) throw std::runtime_error("Wide-Fibonacci needs at least 3 columns");
  Proof proof;
  proof.cfg = cfg;
  Channel ch;
  ch.m31 = m31;
  // Twiddles of CanonicCoset(log_n + 1 + blowup).half_coset (harness :119-123).
  TwiddleTree tw = precompute_twiddles(canonic_half_coset(log_n + 1 + blowup));

  // Tree 0: empty preprocessed trace.
  Tree t0;
  t0.layers = build_merkle_layers({}, {}, 0, m31);
  ch.mix_root(t0.root());

  // Tree 1: the trace (evaluations in bit-reversed order; rows are independent).
  size_t rows = (size_t)1 << log_n;
  std::vector<std::vector<uint32_t>> trace(N, std::vector<uint32_t>(rows));
#pragma omp parallel for schedule(static)
  for (long r = 0; r < (long)rows; r++) {
    uint32_t a = in_a[r], b = in_b[r];
    trace[0][r] = a;
    trace[1][r] = b;
    for (uint32_t c = 2; c < N; c++) {
      uint32_t nb = add(sqr(a), sqr(b));
      a = b; b = nb;
      trace[c][r] = b;
    }
  }
#pragma omp parallel for schedule(dynamic, 1)
  for (long c = 0; c < (long)N; c++)
    interpolate(trace[c].data(), log_n, canonic_half_coset(log_n), tw.itw.data(), tw.itw.size());
  Tree t1 = commit_polys(std::move(trace), blowup, tw, m31);
  ch.mix_root(t1.root());

  // Composition (prover/mod.rs:57-76).
  QM31 random_coeff = ch.draw_secure_felt();
  const uint32_t eval_log = log_n + 1;  // max_constraint_log_degree_bound
  const uint32_t n_cons = N - 2;
  std::vector<std::vector<uint32_t>> ext;  // trace on CanonicCoset(eval_log)
  const std::vector<std::vector<uint32_t>>* tev = &t1.evals;
  if (eval_log != log_n + blowup) {
    TwiddleTree tw2 = precompute_twiddles(canonic_half_coset(eval_log));
    ext.resize(N);
#pragma omp parallel for schedule(dynamic, 1)
    for (long c = 0; c < (long)N; c++) {
      ext[c].resize((size_t)1 << eval_log);
      evaluate(t1.coeffs[c].data(), log_n, eval_log, canonic_half_coset(eval_log), tw2.tw.data(), tw2.tw.size(),
               ext[c].data());
    }
    tev = &ext;
  }
  // random_coeff_powers = [1, a, ..., a^(n-1)] reversed (accumulation.rs, component_prover.rs:91-94).
  std::vector<QM31> pw(n_cons);
  {
    QM31 acc = QM31::one();
    for (uint32_t k = 0; k < n_cons; k++) { pw[k] = acc; acc = acc * random_coeff; }
    std::reverse(pw.begin(), pw.end());
  }
  // denom_inv[j] = coset_vanishing(trace coset, eval_domain.at(j))^-1, bit-reversed.
  uint32_t log_expand = eval_log - log_n;
  std::vector<uint32_t> denom_inv((size_t)1 << log_expand);
  {
    Coset trace_coset = Coset::odds(log_n);  // CanonicCoset(log_n).coset
    Coset half = canonic_half_coset(eval_log);
    for (size_t j = 0; j < denom_inv.size(); j++) {
      CPoint pt = index_to_point(circle_domain_index_at(half, j));
      denom_inv[j] = inv(coset_vanishing_m31(trace_coset, pt));
    }
    bit_reverse(denom_inv.data(), log_expand);
  }
  size_t eval_n = (size_t)1 << eval_log;
  std::vector<std::vector<uint32_t>> comp(4, std::vector<uint32_t>(eval_n));
#pragma omp parallel for schedule(static)
  for (long i = 0; i < (long)eval_n; i++) {
    QM31 row = QM31::zero();
    for (uint32_t k = 0; k < n_cons; k++) {
      uint32_t a = (*tev)[k][i], b = (*tev)[k + 1][i], c = (*tev)[k + 2][i];
      uint32_t cons = sub(c, add(sqr(a), sqr(b)));
      row = row + qmul_m31(pw[k], cons);
    }
    QM31 v = QM31::zero() + qmul_m31(row, denom_inv[(size_t)i >> log_n]);
    auto co = v.coords();
    for (int k = 0; k < 4; k++) comp[k][i] = co[k];
  }
  if (dbg) dbg->composition_evals = comp;
  // finalize: interpolate each coordinate on CanonicCoset(eval_log).
  TwiddleTree twc = precompute_twiddles(canonic_half_coset(eval_log));
  for (int k = 0; k < 4; k++)
    interpolate(comp[k].data(), eval_log, canonic_half_coset(eval_log), twc.itw.data(), twc.itw.size());
  // split_at_mid: left = first half of the coefficients, right = second half.
  std::vector<std::vector<uint32_t>> comp_polys;
  for (int half = 0; half < 2; half++)
    for (int k = 0; k < 4; k++)
      comp_polys.emplace_back(comp[k].begin() + (half ? eval_n / 2 : 0), comp[k].begin() + (half ? eval_n : eval_n / 2));
  Tree t2 = commit_polys(std::move(comp_polys), blowup, tw, m31);
  ch.mix_root(t2.root());

  // OODS (prover/mod.rs:80-116).
  SPoint oods = get_random_point(ch);
  uint32_t lifting = (uint32_t)t2.layers.size() - 1;
  uint32_t max_log_degree_bound = lifting - blowup;
  // Sampled values: trace columns and composition columns at the OODS point.
  std::vector<const Tree*> trees{&t0, &t1, &t2};
  proof.sampled_values.resize(3);
  for (size_t t = 1; t < 3; t++) {
    const Tree& tr = *trees[t];
    proof.sampled_values[t].resize(tr.coeffs.size());
#pragma omp parallel for schedule(dynamic, 1)
    for (long c = 0; c < (long)tr.coeffs.size(); c++) {
      uint32_t lg = 0; while (((size_t)1 << lg) < tr.coeffs[c].size()) lg++;
      SPoint pt = srepeated_double(oods, lifting - tr.eval_logs[c]);
      proof.sampled_values[t][c] = {eval_at_point_q(tr.coeffs[c].data(), lg, pt)};
    }
  }
  {
    std::vector<QM31> flat;
    for (auto& tr : proof.sampled_values) for (auto& col : tr) for (auto& v : col) flat.push_back(v);
    ch.mix_felts(flat.data(), flat.size());
  }

  // Quotients (pcs/mod.rs:112-118, quotient_ops.rs:134-233).
  QM31 qcoeff = ch.draw_secure_felt();
  // Every column of this AIR has exactly one sample (the OODS point) and all
  // columns share the lifting log size, so there is one batch: columns in tree
  // order with random powers qcoeff^k.
  std::vector<const uint32_t*> qcols;
  std::vector<QM31> qvals;
  for (size_t t = 1; t < 3; t++)
    for (size_t c = 0; c < trees[t]->evals.size(); c++) {
      if (trees[t]->eval_logs[c] != lifting) throw std::runtime_error("uneven column sizes unsupported here");
      qcols.push_back(trees[t]->evals[c].data());
      qvals.push_back(proof.sampled_values[t][c][0]);
    }
  std::vector<QM31> la(qcols.size()), lb(qcols.size()), lc(qcols.size());
  {
    QM31 pk = QM31::one();
    for (size_t i = 0; i < qcols.size(); i++) {
      // core/constraints.rs:119-134
      QM31 v = qvals[i];
      QM31 a = qconj(v) - v;
      QM31 c = qconj(oods.y) - oods.y;
      QM31 b = v * c - a * oods.y;
      la[i] = pk * a; lb[i] = pk * b; lc[i] = pk * c;
      pk = pk * qcoeff;
    }
  }
  QM31 A = QM31::zero();
  for (auto& a : la) A = A + a;
  size_t L = (size_t)1 << lifting;
  std::vector<std::vector<uint32_t>> quot(4, std::vector<uint32_t>(L));
  {
    Coset half = canonic_half_coset(lifting);
    CM31 prx = oods.x.x, pix = oods.x.y, pry = oods.y.x, piy = oods.y.y;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)L; i++) {
      CPoint p = index_to_point(circle_domain_index_at(half, bit_reverse_index((uint64_t)i, lifting)));
      QM31 num = QM31::zero();
      for (size_t k = 0; k < qcols.size(); k++) num = num + (qmul_m31(lc[k], qcols[k][i]) - lb[k]);
      QM31 full = num - qmul_m31(A, p.y);
      CM31 den = (prx - CM31{p.x, 0}) * piy - (pry - CM31{p.y, 0}) * pix;
      CM31 dinv = cinv(den);
      QM31 q = QM31::zero() + QM31{full.x * dinv, full.y * dinv};
      auto co = q.coords();
      for (int k = 0; k < 4; k++) quot[k][i] = co[k];
    }
  }
  if (dbg) dbg->quotients = quot;

  // FRI commit (prover/fri.rs:133-291).
  FriConfigO fc{cfg.log_last_layer_degree_bound, blowup, cfg.n_queries, cfg.line_fold_step};
  struct Layer { std::vector<std::vector<uint32_t>> coords; std::vector<std::vector<Hash>> layers; uint32_t fold_step; };
  Layer first;
  first.coords = quot;
  {
    std::vector<const uint32_t*> p4{first.coords[0].data(), first.coords[1].data(), first.coords[2].data(), first.coords[3].data()};
    first.layers = build_merkle_layers(p4, {lifting, lifting, lifting, lifting}, lifting, m31);
  }
  ch.mix_root(first.layers[0][0]);
  QM31 alpha = ch.draw_secure_felt();
  uint32_t cur_log = lifting - 1;
  std::vector<std::vector<uint32_t>> cur(4, std::vector<uint32_t>((size_t)1 << cur_log, 0));
  {
    uint32_t* d[4] = {cur[0].data(), cur[1].data(), cur[2].data(), cur[3].data()};
    const uint32_t* s[4] = {quot[0].data(), quot[1].data(), quot[2].data(), quot[3].data()};
    fold_circle_into_line(d, s, canonic_half_coset(lifting), tw.itw.data(), tw.itw.size(), alpha);
  }
  const uint32_t last_log = fc.log_last_layer + fc.log_blowup;
  std::vector<Layer> inner;
  auto commit_inner = [&](uint32_t fold_step) {
    Layer l;
    l.coords = cur;
    std::vector<const uint32_t*> p4{l.coords[0].data(), l.coords[1].data(), l.coords[2].data(), l.coords[3].data()};
    l.layers = build_merkle_layers(p4, {cur_log, cur_log, cur_log, cur_log}, cur_log, m31);
    l.fold_step = fold_step;
    ch.mix_root(l.layers[0][0]);
    QM31 a = ch.draw_secure_felt();
    std::vector<std::vector<uint32_t>> nxt(4, std::vector<uint32_t>((size_t)1 << (cur_log - fold_step)));
    const uint32_t* in[4] = {cur[0].data(), cur[1].data(), cur[2].data(), cur[3].data()};
    uint32_t* out[4] = {nxt[0].data(), nxt[1].data(), nxt[2].data(), nxt[3].data()};
    fold_line(in, cur_log, tw.itw.data(), tw.itw.size(), a, fold_step, out);
    cur.swap(nxt);
    cur_log -= fold_step;
    inner.push_back(std::move(l));
  };
  if (cur_log != last_log) {
    while (cur_log > last_log + fc.line_fold_step) commit_inner(fc.line_fold_step);
    commit_inner(cur_log - last_log);
  }
  // Last layer (prover/fri.rs:274-291): the line domain is the first inner
  // layer domain doubled down to the last layer size.
  {
    std::vector<QM31> vals((size_t)1 << cur_log);
    for (size_t i = 0; i < vals.size(); i++) vals[i] = QM31::from(cur[0][i], cur[1][i], cur[2][i], cur[3][i]);
    Coset dom = canonic_half_coset(lifting).repeated_double(lifting - 1 - cur_log);
    auto coeffs = line_interpolate_ordered(vals, dom);
    size_t bound = (size_t)1 << fc.log_last_layer;
    for (size_t i = bound; i < coeffs.size(); i++)
      if (!coeffs[i].is_zero()) throw std::runtime_error("invalid degree");
    coeffs.resize(bound);
    proof.last_layer_poly = coeffs;  // ordered; stored bit-reversed when serialized
    ch.mix_felts(coeffs.data(), coeffs.size());
  }

  // Proof of work (pcs/mod.rs:140-142).
  proof.proof_of_work = ch.grind(cfg.pow_bits);
  ch.mix_u64(proof.proof_of_work);

  // Queries (prover/fri.rs:294-306, core/queries.rs:11-58).
  std::vector<size_t> raw;
  {
    size_t mask = ((size_t)1 << lifting) - 1;
    while (raw.size() < cfg.n_queries) {
      auto w = ch.draw_u32s();
      for (uint32_t x : w) { if (raw.size() < cfg.n_queries) raw.push_back(x & mask); }
    }
  }
  std::vector<size_t> queries = raw;
  std::sort(queries.begin(), queries.end());
  queries.erase(std::unique(queries.begin(), queries.end()), queries.end());
  proof.query_positions = queries;

  // FRI decommit.
  auto decommit_layer = [&](const Layer& l, const std::vector<size_t>& q, uint32_t fold_step, FriLayerProofO& out) {
    std::vector<size_t> pos;
    decommit_positions_and_witness(l.coords, q, fold_step, pos, out.fri_witness);
    std::vector<std::vector<uint32_t>> qv;
    uint32_t lg = (uint32_t)l.layers.size() - 1;
    std::vector<const uint32_t*> p4{l.coords[0].data(), l.coords[1].data(), l.coords[2].data(), l.coords[3].data()};
    merkle_decommit(l.layers, pos, p4, {lg, lg, lg, lg}, qv, out.hash_witness);
    out.commitment = l.layers[0][0];
  };
  decommit_layer(first, queries, 1, proof.fri_first);
  std::vector<size_t> lq = fold_queries(queries, 1);
  for (auto& l : inner) {
    FriLayerProofO lp;
    decommit_layer(l, lq, l.fold_step, lp);
    proof.fri_inner.push_back(lp);
    lq = fold_queries(lq, l.fold_step);
  }

  // Tree decommitments (pcs/mod.rs:159-313).
  proof.commitments = {t0.root(), t1.root(), t2.root()};
  proof.queried_values.resize(3);
  proof.decommitments.resize(3);
  for (size_t t = 0; t < 3; t++) {
    const Tree& tr = *trees[t];
    uint32_t tree_log = (uint32_t)tr.layers.size() - 1;
    std::vector<size_t> tq;
    if (tree_log != 0) {
      for (size_t p : queries) {
        if (lifting < tree_log) tq.push_back(((p >> 1) << (tree_log - lifting + 1)) + (p & 1));
        else tq.push_back(((p >> (lifting - tree_log + 1)) << 1) + (p & 1));
      }
    }
    std::vector<const uint32_t*> ptrs;
    for (auto& e : tr.evals) ptrs.push_back(e.data());
    merkle_decommit(tr.layers, tq, ptrs, tr.eval_logs, proof.queried_values[t], proof.decommitments[t]);
  }

  // Sanity check (prover/mod.rs:123-138): composition OODS value from the
  // split halves equals the constraint quotient evaluated at the OODS point.
  {
    auto& cm = proof.sampled_values[2];
    QM31 left = QM31::zero(), right = QM31::zero();
    const QM31 basis[4] = {QM31::one(), QM31::from(0, 1, 0, 0), QM31::from(0, 0, 1, 0), QM31::from(0, 0, 0, 1)};
    for (int k = 0; k < 4; k++) { left = left + cm[k][0] * basis[k]; right = right + cm[4 + k][0] * basis[k]; }
    QM31 comp_oods = left + srepeated_double(oods, max_log_degree_bound - 1).x * right;
    QM31 acc = QM31::zero();
    QM31 dinv = qinv(coset_vanishing_q(Coset::odds(max_log_degree_bound), oods));
    auto& tv = proof.sampled_values[1];
    for (uint32_t k = 0; k < n_cons; k++) {
      QM31 a = tv[k][0], b = tv[k + 1][0], c = tv[k + 2][0];
      acc = acc * random_coeff + (c - (a * a + b * b)) * dinv;
    }
    if (acc != comp_oods) throw std::runtime_error("ConstraintsNotSatisfied");
  }
  if (dbg) {
    dbg->roots = proof.commitments;
    dbg->oods = oods;
  }
  return proof;
}

// --------------------------------------------------------- serializer -------
static void put_u32(std::vector<uint8_t>& o, uint32_t v) { for (int i = 0; i < 4; i++) o.push_back((v >> (8 * i)) & 0xFF); }
static void put_u64(std::vector<uint8_t>& o, uint64_t v) { for (int i = 0; i < 8; i++) o.push_back((v >> (8 * i)) & 0xFF); }
static void put_q(std::vector<uint8_t>& o, const QM31& q) { for (uint32_t c : q.coords()) put_u32(o, c); }
static void put_h(std::vector<uint8_t>& o, const Hash& h) { o.insert(o.end(), h.begin(), h.end()); }
// FriLayerProof field order (core/fri.rs:361-395).
static void put_fri_layer(std::vector<uint8_t>& o, const FriLayerProofO& l) {
  put_u64(o, l.fri_witness.size());
  for (auto& q : l.fri_witness) put_q(o, q);
  put_u64(o, l.hash_witness.size());
  for (auto& h : l.hash_witness) put_h(o, h);
  put_h(o, l.commitment);
}

std::vector<uint8_t> serialize(const Proof& p) {
  std::vector<uint8_t> o;
  const char magic[8] = {'S', 'T', 'W', 'O', 'P', 'R', 'F', '1'};
  o.insert(o.end(), magic, magic + 8);
  // config: pow_bits, fri (log_blowup, log_last_layer, n_queries, line_fold_step), lifting (None)
  put_u32(o, p.cfg.pow_bits);
  put_u32(o, p.cfg.log_blowup);
  put_u32(o, p.cfg.log_last_layer_degree_bound);
  put_u64(o, p.cfg.n_queries);
  put_u32(o, p.cfg.line_fold_step);
  o.push_back(0);  // lifting_log_size: None
  put_u64(o, p.commitments.size());
  for (auto& h : p.commitments) put_h(o, h);
  put_u64(o, p.sampled_values.size());
  for (auto& t : p.sampled_values) {
    put_u64(o, t.size());
    for (auto& c : t) { put_u64(o, c.size()); for (auto& v : c) put_q(o, v); }
  }
  put_u64(o, p.decommitments.size());
  for (auto& d : p.decommitments) { put_u64(o, d.size()); for (auto& h : d) put_h(o, h); }
  put_u64(o, p.queried_values.size());
  for (auto& t : p.queried_values) {
    put_u64(o, t.size());
    for (auto& c : t) { put_u64(o, c.size()); for (uint32_t v : c) put_u32(o, v); }
  }
  put_u64(o, p.proof_of_work);
  auto layer = [&](const FriLayerProofO& l) { put_fri_layer(o, l); };
  layer(p.fri_first);
  put_u64(o, p.fri_inner.size());
  for (auto& l : p.fri_inner) layer(l);
  // LinePoly: coefficients in bit-reversed storage order (core/poly/line.rs:115-170).
  std::vector<QM31> lp = p.last_layer_poly;
  uint32_t lg = 0; while (((size_t)1 << lg) < lp.size()) lg++;
  bit_reverse(lp.data(), lg);
  put_u64(o, lp.size());
  for (auto& q : lp) put_q(o, q);
  return o;
}

// FRI-heavy workload: FriProver::commit (prover/fri.rs:133-291) of one secure
// column on CanonicCoset(log_n) with the folding alphas supplied instead of
// drawn from a channel: circle-to-line fold, then line folds by 2 down to a
// single value (a last layer of log size 0), a lifted Blake2s tree for every
// layer folded from; then the decommitment of the sorted, distinct query
// positions (prover/fri.rs:294-350, 459-488).  Serialized as the FriProof part
// of serialize(): first layer, inner layers, last-layer polynomial (here the
// one folded value, its own interpolant).
std::vector<uint8_t> fri_prove_seeded(const uint32_t* const coords[4], uint32_t log_n, const QM31* alphas,
                                      std::vector<size_t> queries, bool m31) {
  if (log_n < 2 || log_n > 28) throw std::runtime_error("log_n out of range");
  std::sort(queries.begin(), queries.end());
  queries.erase(std::unique(queries.begin(), queries.end()), queries.end());
  for (size_t q : queries)
    if (q >> log_n) throw std::runtime_error("query out of range");
  TwiddleTree tw = precompute_twiddles(canonic_half_coset(log_n + 1));
  struct Layer { std::vector<std::vector<uint32_t>> coords; std::vector<std::vector<Hash>> layers; };
  const size_t n = (size_t)1 << log_n;
  Layer first;
  for (int k = 0; k < 4; k++) first.coords.emplace_back(coords[k], coords[k] + n);
  {
    std::vector<const uint32_t*> p4{first.coords[0].data(), first.coords[1].data(), first.coords[2].data(),
                                    first.coords[3].data()};
    first.layers = build_merkle_layers(p4, {log_n, log_n, log_n, log_n}, log_n, m31);
  }
  uint32_t cur_log = log_n - 1;
  std::vector<std::vector<uint32_t>> cur(4, std::vector<uint32_t>((size_t)1 << cur_log, 0));
  {
    uint32_t* d[4] = {cur[0].data(), cur[1].data(), cur[2].data(), cur[3].data()};
    const uint32_t* s[4] = {coords[0], coords[1], coords[2], coords[3]};
    fold_circle_into_line(d, s, canonic_half_coset(log_n), tw.itw.data(), tw.itw.size(), alphas[0]);
  }
  std::vector<Layer> inner;
  for (uint32_t k = 1; cur_log >= 1; k++) {
    Layer l;
    l.coords = cur;
    std::vector<const uint32_t*> p4{l.coords[0].data(), l.coords[1].data(), l.coords[2].data(), l.coords[3].data()};
    l.layers = build_merkle_layers(p4, {cur_log, cur_log, cur_log, cur_log}, cur_log, m31);
    std::vector<std::vector<uint32_t>> nxt(4, std::vector<uint32_t>((size_t)1 << (cur_log - 1)));
    const uint32_t* in[4] = {cur[0].data(), cur[1].data(), cur[2].data(), cur[3].data()};
    uint32_t* out[4] = {nxt[0].data(), nxt[1].data(), nxt[2].data(), nxt[3].data()};
    fold_line(in, cur_log, tw.itw.data(), tw.itw.size(), alphas[k], 1, out);
    cur.swap(nxt);
    cur_log -= 1;
    inner.push_back(std::move(l));
  }
  const QM31 last = QM31::from(cur[0][0], cur[1][0], cur[2][0], cur[3][0]);
  auto decommit = [&](const Layer& l, const std::vector<size_t>& q) {
    FriLayerProofO out;
    std::vector<size_t> pos;
    decommit_positions_and_witness(l.coords, q, 1, pos, out.fri_witness);
    std::vector<std::vector<uint32_t>> qv;
    uint32_t lg = (uint32_t)l.layers.size() - 1;
    std::vector<const uint32_t*> p4{l.coords[0].data(), l.coords[1].data(), l.coords[2].data(), l.coords[3].data()};
    merkle_decommit(l.layers, pos, p4, {lg, lg, lg, lg}, qv, out.hash_witness);
    out.commitment = l.layers[0][0];
    return out;
  };
  std::vector<uint8_t> o;
  put_fri_layer(o, decommit(first, queries));
  put_u64(o, inner.size());
  std::vector<size_t> lq = fold_queries(queries, 1);
  for (auto& l : inner) {
    put_fri_layer(o, decommit(l, lq));
    lq = fold_queries(lq, 1);
  }
  put_u64(o, 1);
  put_q(o, last);
  return o;
}

}  // namespace oracle
