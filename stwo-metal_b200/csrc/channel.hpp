// Host-side Fiat-Shamir channel of the B200 prover: Blake2s-256 (RFC 7693)
// and stwo's Blake2s channel (crates/stwo/src/core/channel/blake2s.rs:25-141),
// with the M31-output variant (core/vcs/blake2_hash.rs:110-118).  The channel
// is a few hundred bytes of hashing per proof, so it stays on the host and
// serialises only the Fiat-Shamir points of the device pipeline.
#pragma once
#include <array>
#include <cstdint>
#include <cstring>
#include <vector>

#include "field.cuh"

namespace stwo_b200 {

using Hash32 = std::array<uint8_t, 32>;

class HostBlake2s {
 public:
  HostBlake2s() { reset(); }
  void reset() {
    static const uint32_t iv[8] = {0x6A09E667u, 0xBB67AE85u, 0x3C6EF372u, 0xA54FF53Au,
                                   0x510E527Fu, 0x9B05688Cu, 0x1F83D9ABu, 0x5BE0CD19u};
    std::memcpy(h_, iv, 32);
    h_[0] ^= 0x01010020u;
    len_ = 0;
    total_ = 0;
  }
  void update(const void* data, size_t n) {
    const uint8_t* p = static_cast<const uint8_t*>(data);
    while (n) {
      if (len_ == 64) {
        total_ += 64;
        compress(false);
        len_ = 0;
      }
      size_t k = n < 64 - len_ ? n : 64 - len_;
      std::memcpy(buf_ + len_, p, k);
      len_ += k;
      p += k;
      n -= k;
    }
  }
  void update_u32(uint32_t w) { update(&w, 4); }
  Hash32 finalize(bool m31_output) {
    total_ += len_;
    std::memset(buf_ + len_, 0, 64 - len_);
    compress(true);
    Hash32 out;
    for (int i = 0; i < 8; i++) {
      uint32_t w = m31_output ? m31_reduce_u32(h_[i]) : h_[i];
      std::memcpy(out.data() + 4 * i, &w, 4);
    }
    return out;
  }

 private:
  static uint32_t rotr(uint32_t x, int n) { return (x >> n) | (x << (32 - n)); }
  void compress(bool last) {
    static const uint8_t S[10][16] = {
        {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15}, {14, 10, 4, 8, 9, 15, 13, 6, 1, 12, 0, 2, 11, 7, 5, 3},
        {11, 8, 12, 0, 5, 2, 15, 13, 10, 14, 3, 6, 7, 1, 9, 4}, {7, 9, 3, 1, 13, 12, 11, 14, 2, 6, 5, 10, 4, 0, 15, 8},
        {9, 0, 5, 7, 2, 4, 10, 15, 14, 1, 11, 12, 6, 8, 3, 13}, {2, 12, 6, 10, 0, 11, 8, 3, 4, 13, 7, 5, 15, 14, 1, 9},
        {12, 5, 1, 15, 14, 13, 4, 10, 0, 7, 6, 3, 9, 2, 8, 11}, {13, 11, 7, 14, 12, 1, 3, 9, 5, 0, 15, 4, 8, 6, 2, 10},
        {6, 15, 14, 9, 11, 3, 0, 8, 12, 2, 13, 7, 1, 4, 10, 5}, {10, 2, 8, 4, 7, 6, 1, 5, 15, 11, 9, 14, 3, 12, 13, 0}};
    static const uint32_t iv[8] = {0x6A09E667u, 0xBB67AE85u, 0x3C6EF372u, 0xA54FF53Au,
                                   0x510E527Fu, 0x9B05688Cu, 0x1F83D9ABu, 0x5BE0CD19u};
    uint32_t m[16], v[16];
    std::memcpy(m, buf_, 64);
    for (int i = 0; i < 8; i++) {
      v[i] = h_[i];
      v[i + 8] = iv[i];
    }
    v[12] ^= (uint32_t)total_;
    v[13] ^= (uint32_t)(total_ >> 32);
    if (last) v[14] = ~v[14];
    auto g = [&](int a, int b, int c, int d, uint32_t x, uint32_t y) {
      v[a] = v[a] + v[b] + x;
      v[d] = rotr(v[d] ^ v[a], 16);
      v[c] = v[c] + v[d];
      v[b] = rotr(v[b] ^ v[c], 12);
      v[a] = v[a] + v[b] + y;
      v[d] = rotr(v[d] ^ v[a], 8);
      v[c] = v[c] + v[d];
      v[b] = rotr(v[b] ^ v[c], 7);
    };
    for (int r = 0; r < 10; r++) {
      const uint8_t* s = S[r];
      g(0, 4, 8, 12, m[s[0]], m[s[1]]);
      g(1, 5, 9, 13, m[s[2]], m[s[3]]);
      g(2, 6, 10, 14, m[s[4]], m[s[5]]);
      g(3, 7, 11, 15, m[s[6]], m[s[7]]);
      g(0, 5, 10, 15, m[s[8]], m[s[9]]);
      g(1, 6, 11, 12, m[s[10]], m[s[11]]);
      g(2, 7, 8, 13, m[s[12]], m[s[13]]);
      g(3, 4, 9, 14, m[s[14]], m[s[15]]);
    }
    for (int i = 0; i < 8; i++) h_[i] ^= v[i] ^ v[i + 8];
  }
  uint32_t h_[8];
  uint8_t buf_[64];
  size_t len_;
  uint64_t total_;
};

class HostChannel {
 public:
  explicit HostChannel(bool m31_output) : m31_(m31_output) { digest_.fill(0); }
  const Hash32& digest() const { return digest_; }
  // Adopts a channel state computed elsewhere (the device channel).
  void set_state(const uint32_t digest[8], uint32_t n_draws) {
    std::memcpy(digest_.data(), digest, 32);
    n_draws_ = n_draws;
  }
  uint32_t n_draws() const { return n_draws_; }
  bool m31() const { return m31_; }

  void mix_root(const Hash32& root) {  // core/vcs_lifted/blake2_merkle.rs:49-56
    HostBlake2s s;
    s.update(digest_.data(), 32);
    s.update(root.data(), 32);
    set(s.finalize(m31_));
  }
  void mix_u32s(const uint32_t* w, size_t n) {
    HostBlake2s s;
    s.update(digest_.data(), 32);
    for (size_t i = 0; i < n; i++) s.update_u32(w[i]);
    set(s.finalize(m31_));
  }
  void mix_u64(uint64_t v) {
    uint32_t w[2] = {(uint32_t)v, (uint32_t)(v >> 32)};
    mix_u32s(w, 2);
  }
  void mix_felts(const qm31* f, size_t n) {
    HostBlake2s s;
    s.update(digest_.data(), 32);
    for (size_t i = 0; i < n; i++) {
      s.update_u32(f[i].a);
      s.update_u32(f[i].b);
      s.update_u32(f[i].c);
      s.update_u32(f[i].d);
    }
    set(s.finalize(m31_));
  }
  std::array<uint32_t, 8> draw_u32s() {
    uint8_t in[37];
    std::memcpy(in, digest_.data(), 32);
    std::memcpy(in + 32, &n_draws_, 4);
    in[36] = 0;
    n_draws_++;
    HostBlake2s s;
    s.update(in, 37);
    Hash32 h = s.finalize(m31_);
    std::array<uint32_t, 8> w;
    std::memcpy(w.data(), h.data(), 32);
    return w;
  }
  qm31 draw_secure_felt() {
    for (;;) {
      auto w = draw_u32s();
      bool ok = true;
      for (uint32_t x : w) ok = ok && x < 2 * M31_P;
      if (ok) return {m31_reduce_u32(w[0]), m31_reduce_u32(w[1]), m31_reduce_u32(w[2]), m31_reduce_u32(w[3])};
    }
  }
  // H(POW_PREFIX, [0; 12], digest, n_bits) (core/channel/blake2s.rs:124-132).
  Hash32 pow_prefixed(uint32_t n_bits) const {
    HostBlake2s s;
    uint32_t prefix = 0x12345678u;
    uint8_t zeros[12] = {0};
    s.update(&prefix, 4);
    s.update(zeros, 12);
    s.update(digest_.data(), 32);
    s.update(&n_bits, 4);
    return s.finalize(m31_);
  }

 private:
  void set(const Hash32& h) {
    digest_ = h;
    n_draws_ = 0;
  }
  Hash32 digest_;
  uint32_t n_draws_ = 0;
  bool m31_;
};

}  // namespace stwo_b200
