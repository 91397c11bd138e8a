// ORACLE — test infrastructure only (see stwo_oracle.hpp).
//
// Verifier restatement for Wide-Fibonacci proofs in the canonical byte
// serialization (oracle_prove.cpp::serialize):
//   verify / verify_ex          crates/stwo/src/core/verifier.rs:16-100
//   CommitmentSchemeVerifier     core/pcs/verifier.rs:43-129
//   fri_answers                  core/pcs/quotients.rs:120-214
//   FriVerifier                  core/fri.rs:94-256, 420-560, 690-760
//   MerkleVerifierLifted::verify core/vcs_lifted/verifier.rs:54-180
#include <map>

#include "stwo_oracle_prove.hpp"

namespace oracle {

namespace {

struct Reader {
  const uint8_t* p;
  size_t n, off = 0;
  void need(size_t k) {
    if (off + k > n) throw std::runtime_error("InvalidStructure: truncated proof");
  }
  uint8_t u8() { need(1); return p[off++]; }
  uint32_t u32() { need(4); uint32_t v; std::memcpy(&v, p + off, 4); off += 4; return v; }
  uint64_t u64() { need(8); uint64_t v; std::memcpy(&v, p + off, 8); off += 8; return v; }
  uint64_t len(uint64_t limit) {
    uint64_t v = u64();
    if (v > limit) throw std::runtime_error("InvalidStructure: length field out of range");
    return v;
  }
  QM31 q() { uint32_t a = u32(), b = u32(), c = u32(), d = u32(); return QM31::from(a, b, c, d); }
  Hash h() { need(32); Hash r; std::memcpy(r.data(), p + off, 32); off += 32; return r; }
};

Proof deserialize(const uint8_t* data, size_t n) {
  Reader r{data, n};
  const char magic[8] = {'S', 'T', 'W', 'O', 'P', 'R', 'F', '1'};
  r.need(8);
  if (std::memcmp(data, magic, 8) != 0) throw std::runtime_error("InvalidStructure: bad magic");
  r.off = 8;
  Proof p;
  p.cfg.pow_bits = r.u32();
  p.cfg.log_blowup = r.u32();
  p.cfg.log_last_layer_degree_bound = r.u32();
  p.cfg.n_queries = (uint32_t)r.u64();
  p.cfg.line_fold_step = r.u32();
  if (r.u8() != 0) throw std::runtime_error("InvalidStructure: lifting_log_size must be None");
  const uint64_t BIG = 1ull << 24;
  p.commitments.resize(r.len(64));
  for (auto& h : p.commitments) h = r.h();
  p.sampled_values.resize(r.len(64));
  for (auto& t : p.sampled_values) {
    t.resize(r.len(BIG));
    for (auto& c : t) { c.resize(r.len(64)); for (auto& v : c) v = r.q(); }
  }
  p.decommitments.resize(r.len(64));
  for (auto& d : p.decommitments) { d.resize(r.len(BIG)); for (auto& h : d) h = r.h(); }
  p.queried_values.resize(r.len(64));
  for (auto& t : p.queried_values) {
    t.resize(r.len(BIG));
    for (auto& c : t) { c.resize(r.len(BIG)); for (auto& v : c) v = r.u32(); }
  }
  p.proof_of_work = r.u64();
  auto layer = [&](FriLayerProofO& l) {
    l.fri_witness.resize(r.len(BIG));
    for (auto& q : l.fri_witness) q = r.q();
    l.hash_witness.resize(r.len(BIG));
    for (auto& h : l.hash_witness) h = r.h();
    l.commitment = r.h();
  };
  layer(p.fri_first);
  p.fri_inner.resize(r.len(64));
  for (auto& l : p.fri_inner) layer(l);
  std::vector<QM31> lp(r.len(1 << 12));
  for (auto& q : lp) q = r.q();
  uint32_t lg = 0; while (((size_t)1 << lg) < lp.size()) lg++;
  if (!lp.empty() && ((size_t)1 << lg) != lp.size()) throw std::runtime_error("InvalidStructure: last layer size");
  bit_reverse(lp.data(), lg);
  p.last_layer_poly = lp;
  if (r.off != n) throw std::runtime_error("InvalidStructure: trailing bytes");
  return p;
}

// core/vcs_lifted/verifier.rs:96-180
void merkle_verify(const Hash& root, const std::vector<uint32_t>& col_logs, uint32_t height,
                   const std::vector<size_t>& positions, const std::vector<std::vector<uint32_t>>& values,
                   const std::vector<Hash>& witness, bool m31) {
  if (height == 0) return;
  if (values.size() != col_logs.size()) throw std::runtime_error("Merkle: column count mismatch");
  for (auto& v : values)
    if (v.size() != positions.size()) throw std::runtime_error("Merkle: value count mismatch");
  std::vector<size_t> order(col_logs.size());
  for (size_t i = 0; i < order.size(); i++) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return col_logs[a] < col_logs[b]; });
  std::vector<std::pair<size_t, Hash>> prev;
  for (size_t i = 0; i < positions.size(); i++) {
    if (i > 0 && positions[i] == positions[i - 1]) continue;
    Blake2s s;
    for (size_t c : order) s.update_u32(values[c][i]);
    prev.push_back({positions[i], finalize_hash(s, m31)});
  }
  size_t wi = 0;
  for (uint32_t l = 0; l < height; l++) {
    std::vector<std::pair<size_t, Hash>> cur;
    for (size_t i = 0; i < prev.size();) {
      bool pair = (i + 1 < prev.size()) && ((prev[i].first ^ 1) == prev[i + 1].first);
      Hash left, right;
      if (pair) {
        left = prev[i].second; right = prev[i + 1].second;
      } else {
        if (wi >= witness.size()) throw std::runtime_error("Merkle: WitnessTooShort");
        if (prev[i].first & 1) { left = witness[wi++]; right = prev[i].second; }
        else { left = prev[i].second; right = witness[wi++]; }
      }
      Blake2s s; s.update(left.data(), 32); s.update(right.data(), 32);
      cur.push_back({prev[i].first >> 1, finalize_hash(s, m31)});
      i += pair ? 2 : 1;
    }
    prev = cur;
  }
  if (wi != witness.size()) throw std::runtime_error("Merkle: WitnessTooLong");
  if (prev.size() != 1 || prev[0].second != root) throw std::runtime_error("Merkle: RootMismatch");
}

QM31 qfrom_partial(const QM31* e) {
  const QM31 basis[4] = {QM31::one(), QM31::from(0, 1, 0, 0), QM31::from(0, 0, 1, 0), QM31::from(0, 0, 0, 1)};
  QM31 r = QM31::zero();
  for (int k = 0; k < 4; k++) r = r + e[k] * basis[k];
  return r;
}

struct Subsets {
  std::vector<size_t> positions;
  std::vector<std::vector<QM31>> evals;
  std::vector<size_t> initial_bitrev;  // bit_reverse_index(subset_start, log_domain)
};

// core/fri.rs:560-610
Subsets rebuild(const std::vector<size_t>& queries, uint32_t log_domain, const std::vector<QM31>& qevals,
                const std::vector<QM31>& witness, uint32_t fold_step, const char* what) {
  Subsets s;
  size_t qi = 0, wi = 0;
  for (size_t i = 0; i < queries.size();) {
    size_t j = i;
    while (j < queries.size() && (queries[j] >> fold_step) == (queries[i] >> fold_step)) j++;
    size_t start = (queries[i] >> fold_step) << fold_step;
    std::vector<QM31> ev;
    size_t k = i;
    for (size_t pos = start; pos < start + ((size_t)1 << fold_step); pos++) {
      s.positions.push_back(pos);
      if (k < j && queries[k] == pos) { ev.push_back(qevals[qi++]); k++; }
      else {
        if (wi >= witness.size()) throw std::runtime_error(std::string(what) + "EvaluationsInvalid");
        ev.push_back(witness[wi++]);
      }
    }
    s.evals.push_back(ev);
    s.initial_bitrev.push_back(bit_reverse_index(start, log_domain));
    i = j;
  }
  if (wi != witness.size()) throw std::runtime_error(std::string(what) + "EvaluationsInvalid");
  return s;
}

void merkle_verify_coords(const FriLayerProofO& lp, uint32_t log_size, const Subsets& s, bool m31,
                          const char* what) {
  std::vector<std::vector<uint32_t>> vals(4);
  for (auto& ev : s.evals)
    for (auto& q : ev) { auto c = q.coords(); for (int k = 0; k < 4; k++) vals[k].push_back(c[k]); }
  try {
    merkle_verify(lp.commitment, {log_size, log_size, log_size, log_size}, log_size, s.positions, vals,
                  lp.hash_witness, m31);
  } catch (const std::exception& e) {
    throw std::runtime_error(std::string(what) + "CommitmentInvalid: " + e.what());
  }
}

}  // namespace

// Throws with the VerificationError name when the proof is rejected.
void verify_wide_fib(const uint8_t* data, size_t n, uint32_t log_n_rows, uint32_t n_cols, bool m31) {
  Proof p = deserialize(data, n);
  const uint32_t blowup = p.cfg.log_blowup;
  if (p.commitments.size() != 3 || p.sampled_values.size() != 3 || p.decommitments.size() != 3 ||
      p.queried_values.size() != 3)
    throw std::runtime_error("InvalidStructure: expected 3 trees");
  if (p.sampled_values[0].size() != 0 || p.sampled_values[1].size() != n_cols || p.sampled_values[2].size() != 8)
    throw std::runtime_error("InvalidStructure: sampled values shape");
  for (size_t t = 1; t < 3; t++)
    for (auto& c : p.sampled_values[t])
      if (c.size() != 1) throw std::runtime_error("InvalidStructure: one sample per column");
  Channel ch;
  ch.m31 = m31;
  // Harness: commit trees 0 and 1 (sizes from the AIR).
  ch.mix_root(p.commitments[0]);
  ch.mix_root(p.commitments[1]);
  // verify_ex
  const uint32_t composition_log_degree_bound = log_n_rows + 1;
  const uint32_t split_bound = composition_log_degree_bound - 1;
  const uint32_t lifting = split_bound + blowup;
  const uint32_t max_log_degree_bound = lifting - blowup;
  QM31 random_coeff = ch.draw_secure_felt();
  ch.mix_root(p.commitments[2]);
  SPoint oods = get_random_point(ch);
  // OODS consistency.
  {
    QM31 left[4], right[4];
    for (int k = 0; k < 4; k++) { left[k] = p.sampled_values[2][k][0]; right[k] = p.sampled_values[2][4 + k][0]; }
    QM31 comp = qfrom_partial(left) + srepeated_double(oods, max_log_degree_bound - 1).x * qfrom_partial(right);
    QM31 dinv = qinv(coset_vanishing_q(Coset::odds(max_log_degree_bound), oods));
    QM31 acc = QM31::zero();
    auto& tv = p.sampled_values[1];
    for (uint32_t k = 0; k + 2 < n_cols; k++)
      acc = acc * random_coeff + (tv[k + 2][0] - (tv[k][0] * tv[k][0] + tv[k + 1][0] * tv[k + 1][0])) * dinv;
    if (acc != comp) throw std::runtime_error("OodsNotMatching");
  }
  // verify_values
  {
    std::vector<QM31> flat;
    for (auto& t : p.sampled_values) for (auto& c : t) for (auto& v : c) flat.push_back(v);
    ch.mix_felts(flat.data(), flat.size());
  }
  QM31 qcoeff = ch.draw_secure_felt();
  // FriVerifier::commit (column bound = lifting - blowup).
  ch.mix_root(p.fri_first.commitment);
  QM31 alpha0 = ch.draw_secure_felt();
  uint32_t layer_bound = max_log_degree_bound - 1;
  std::vector<QM31> alphas;
  std::vector<uint32_t> steps, layer_logs;
  for (size_t i = 0; i < p.fri_inner.size(); i++) {
    ch.mix_root(p.fri_inner[i].commitment);
    bool last = i + 1 == p.fri_inner.size();
    uint32_t step = p.cfg.line_fold_step;
    if (last) {
      if (layer_bound < p.cfg.log_last_layer_degree_bound) throw std::runtime_error("InvalidNumFriLayers");
      step = layer_bound - p.cfg.log_last_layer_degree_bound;
      if (step < 1 || step > p.cfg.line_fold_step) throw std::runtime_error("InvalidNumFriLayers");
    }
    layer_logs.push_back(layer_bound + blowup);
    alphas.push_back(ch.draw_secure_felt());
    steps.push_back(step);
    if (layer_bound < step) throw std::runtime_error("InvalidNumFriLayers");
    layer_bound -= step;
  }
  if (layer_bound != p.cfg.log_last_layer_degree_bound) throw std::runtime_error("InvalidNumFriLayers");
  if (p.last_layer_poly.size() > ((size_t)1 << p.cfg.log_last_layer_degree_bound))
    throw std::runtime_error("LastLayerDegreeInvalid");
  ch.mix_felts(p.last_layer_poly.data(), p.last_layer_poly.size());
  if (!ch.verify_pow_nonce(p.cfg.pow_bits, p.proof_of_work)) throw std::runtime_error("ProofOfWork");
  ch.mix_u64(p.proof_of_work);
  std::vector<size_t> queries;
  {
    size_t mask = ((size_t)1 << lifting) - 1;
    while (queries.size() < p.cfg.n_queries) {
      auto w = ch.draw_u32s();
      for (uint32_t x : w) if (queries.size() < p.cfg.n_queries) queries.push_back(x & mask);
    }
    std::sort(queries.begin(), queries.end());
    queries.erase(std::unique(queries.begin(), queries.end()), queries.end());
  }
  // Tree decommitments.
  std::vector<std::vector<uint32_t>> tree_logs{{}, std::vector<uint32_t>(n_cols, log_n_rows + blowup),
                                               std::vector<uint32_t>(8, max_log_degree_bound + blowup)};
  for (size_t t = 0; t < 3; t++) {
    uint32_t height = 0;
    for (uint32_t l : tree_logs[t]) height = std::max(height, l);
    std::vector<size_t> tq;
    if (height != 0)
      for (size_t pos : queries) tq.push_back(((pos >> (lifting - height + 1)) << 1) + (pos & 1));
    if (height == 0 && (!p.queried_values[t].empty() || !p.decommitments[t].empty()))
      throw std::runtime_error("InvalidStructure: empty tree with values");
    merkle_verify(p.commitments[t], tree_logs[t], height, tq, p.queried_values[t], p.decommitments[t], m31);
  }
  // fri_answers (one sample per column, all at the lifting size).
  std::vector<QM31> answers;
  {
    std::vector<QM31> la, lb, lc;
    QM31 pk = QM31::one();
    std::vector<const std::vector<uint32_t>*> cols;
    for (size_t t = 1; t < 3; t++)
      for (size_t c = 0; c < p.sampled_values[t].size(); c++) {
        QM31 v = p.sampled_values[t][c][0];
        QM31 a = qconj(v) - v, cc = qconj(oods.y) - oods.y, b = v * cc - a * oods.y;
        la.push_back(pk * a); lb.push_back(pk * b); lc.push_back(pk * cc);
        pk = pk * qcoeff;
        cols.push_back(&p.queried_values[t][c]);
      }
    Coset half = canonic_half_coset(lifting);
    CM31 prx = oods.x.x, pix = oods.x.y, pry = oods.y.x, piy = oods.y.y;
    for (size_t qi = 0; qi < queries.size(); qi++) {
      CPoint dp = index_to_point(circle_domain_index_at(half, bit_reverse_index(queries[qi], lifting)));
      QM31 num = QM31::zero();
      for (size_t k = 0; k < cols.size(); k++) {
        QM31 value = qmul_m31(lc[k], (*cols[k])[qi]);
        num = num + (value - (qmul_m31(la[k], dp.y) + lb[k]));
      }
      CM31 den = (prx - CM31{dp.x, 0}) * piy - (pry - CM31{dp.y, 0}) * pix;
      CM31 di = cinv(den);
      answers.push_back(QM31::zero() + QM31{num.x * di, num.y * di});
    }
  }
  // FRI decommit.
  Subsets s0 = rebuild(queries, lifting, answers, p.fri_first.fri_witness, 1, "FirstLayer");
  merkle_verify_coords(p.fri_first, lifting, s0, m31, "FirstLayer");
  // fold_circle on each 2-point subset (core/fri.rs:645-664, 731-756).
  std::vector<QM31> evals;
  {
    Coset half = canonic_half_coset(lifting);
    QM31 a2 = alpha0 * alpha0;
    for (size_t i = 0; i < s0.evals.size(); i++) {
      uint64_t init = circle_domain_index_at(half, s0.initial_bitrev[i]);
      // fold domain = CircleDomain(Coset::new(init, 0)): point 0 = init.
      CPoint pt = index_to_point(init);
      QM31 f0 = s0.evals[i][0] + s0.evals[i][1];
      QM31 f1 = qmul_m31(s0.evals[i][0] - s0.evals[i][1], inv(pt.y));
      QM31 fp = alpha0 * f1 + f0;
      evals.push_back(QM31::zero() * a2 + fp);
    }
  }
  std::vector<size_t> lq;
  for (size_t q : queries) { size_t f = q >> 1; if (lq.empty() || lq.back() != f) lq.push_back(f); }
  Coset line_dom = canonic_half_coset(lifting);  // LineDomain(half_odds(lifting - 1))
  for (size_t i = 0; i < p.fri_inner.size(); i++) {
    uint32_t lg = layer_logs[i];
    if (line_dom.log_size != lg) throw std::runtime_error("InvalidNumFriLayers");
    std::string what = "InnerLayer" + std::to_string(i);
    Subsets s = rebuild(lq, lg, evals, p.fri_inner[i].fri_witness, steps[i], what.c_str());
    merkle_verify_coords(p.fri_inner[i], lg, s, m31, what.c_str());
    std::vector<QM31> nxt;
    for (size_t j = 0; j < s.evals.size(); j++) {
      uint64_t init = line_dom.index_at(s.initial_bitrev[j]);
      Coset fd = Coset::make(init, steps[i]);
      std::vector<QM31> ev = s.evals[j];
      QM31 fa = alphas[i];
      for (uint32_t st = 0; st < steps[i]; st++) {
        uint32_t n2 = fd.log_size;
        for (size_t k = 0; k < ((size_t)1 << (n2)); k += 2) {
          uint32_t x = fd.at(bit_reverse_index(k, n2)).x;
          QM31 f0 = ev[k] + ev[k + 1], f1 = qmul_m31(ev[k] - ev[k + 1], inv(x));
          ev[k >> 1] = f0 + fa * f1;
        }
        fa = fa * fa;
        fd = fd.dbl();
      }
      nxt.push_back(ev[0]);
    }
    evals = nxt;
    std::vector<size_t> fq;
    for (size_t q : lq) { size_t f = q >> steps[i]; if (fq.empty() || fq.back() != f) fq.push_back(f); }
    lq = fq;
    line_dom = line_dom.repeated_double(steps[i]);
  }
  // Last layer.
  for (size_t i = 0; i < lq.size(); i++) {
    uint32_t x = line_dom.at(bit_reverse_index(lq[i], line_dom.log_size)).x;
    // LinePoly::eval_at_point: fold over doublings of x (core/poly/line.rs).
    std::vector<QM31> c = p.last_layer_poly;  // ordered
    uint32_t lg = 0; while (((size_t)1 << lg) < c.size()) lg++;
    QM31 v;
    if (c.empty()) v = QM31::zero();
    else {
      std::vector<QM31> br = c;
      bit_reverse(br.data(), lg);
      // fold(coeffs in bit-reversed storage, [x, pi(x), pi^2(x), ...]): factor 0
      // splits the top halves (core/poly/line.rs:138-145, core/poly/utils.rs:27-38).
      std::vector<uint32_t> maps;
      uint32_t xx = x;
      for (uint32_t k = 0; k < lg; k++) { maps.push_back(xx); xx = sub(add(sqr(xx), sqr(xx)), 1); }
      std::vector<QM31> cur = br;
      for (int lv = (int)lg - 1; lv >= 0; lv--) {
        std::vector<QM31> nx(cur.size() / 2);
        for (size_t k = 0; k < nx.size(); k++) nx[k] = cur[2 * k] + qmul_m31(cur[2 * k + 1], maps[lv]);
        cur = nx;
      }
      v = cur[0];
    }
    if (evals[i] != v) throw std::runtime_error("LastLayerEvaluationsInvalid");
  }
}

}  // namespace oracle
