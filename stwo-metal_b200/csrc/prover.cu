// The B200 Wide-Fibonacci prover: stwo's prove flow (crates/stwo/src/prover/mod.rs:41-138)
// for the Wide-Fibonacci AIR (examples/src/wide_fibonacci/mod.rs:27-101) over the
// Blake2s Merkle channel, with every column-sized step on the device:
//   trace generation, interpolate / evaluate (fft.cu), lifted Merkle commits
//   (merkle.cu), the composition polynomial, OODS sampling, FRI quotients, the
//   FRI folds (fri.cu), proof-of-work grinding and the decommitment gathers.
// The host keeps the Fiat-Shamir channel and assembles the proof; it waits on
// the device only where the transcript needs a device value (roots, sampled
// values, the last FRI layer, the nonce, the decommitted values).
// Device buffers are allocated once per prover (resident between proofs).
#include <cuda_runtime.h>

#include <algorithm>
#include <memory>
#include <string>
#include <vector>

#include "blake2s.cuh"
#include "channel.hpp"
#include "common.cuh"
#include "fft.hpp"
#include "field.cuh"
#include "pcs.hpp"
#include "rowops.cuh"
#include "stream.cuh"

namespace stwo_b200 {

int build_leaves_impl(const uint32_t* const* d_cols, const uint32_t* log_sizes, uint32_t n_cols, uint32_t L,
                      int m31, uint8_t* d_leaves, uint8_t* const* layer_ws, cudaStream_t s, char* err,
                      size_t err_len);
int build_node_layers_impl(const uint8_t* in, uint32_t in_log, uint32_t stop_log, int m31,
                           uint8_t* const* outs_by_log, cudaStream_t s, char* err, size_t err_len);

// ----------------------------------------------------------------- kernels --

// One thread per row: col[i+2] = col[i]^2 + col[i+1]^2 (wide_fibonacci/mod.rs:27-50).
// `rows` rows from a/b; column c of the trace at cols + c * stride.
__global__ void wide_fib_trace_kernel(const uint32_t* __restrict__ a, const uint32_t* __restrict__ b,
                                      uint32_t* __restrict__ cols, uint32_t n_cols, uint64_t rows, uint64_t stride) {
  for (uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r < rows; r += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t x = __ldg(a + r), y = __ldg(b + r);
    cols[r] = x;
    cols[stride + r] = y;
    for (uint32_t c = 2; c < n_cols; c++) {
      uint32_t z = m31_add(m31_sqr(x), m31_sqr(y));
      cols[(uint64_t)c * stride + r] = z;
      x = y;
      y = z;
    }
  }
}

// Composition evaluation at every point of the evaluation domain
// (constraint-framework/src/prover/component_prover.rs:91-160): for constraint
// k (0-based) c_{k+2} - (c_k^2 + c_{k+1}^2) weighted by powers[k] (already
// reversed), times the vanishing inverse of the point's trace-coset class.
// Four consecutive points per thread: 16-byte loads keep four times the bytes
// in flight per load, which this memory-latency-bound loop needs.
// n_points % 4 == 0, columns 16-byte aligned.  The streaming form
// composition_tma_kernel takes every domain of at least one 512-row tile.
__global__ void __launch_bounds__(256) composition4_kernel(const uint32_t* __restrict__ evals, uint64_t col_stride,
                                                          uint32_t n_cons, const qm31* __restrict__ powers,
                                                          const uint32_t* __restrict__ denom_inv, uint32_t log_n,
                                                          uint64_t n_points, uint32_t* __restrict__ out) {
  const uint64_t n4 = n_points >> 2;
  for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q < n4; q += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t i = q << 2;
    const uint4 a = ldg4(evals + i), b = ldg4(evals + col_stride + i);
    uint32_t sa[4], sb[4];
#pragma unroll
    for (int r = 0; r < 4; r++) {
      sa[r] = m31_sqr(u4get(a, r));
      sb[r] = m31_sqr(u4get(b, r));
    }
    acc4 row[4];
#pragma unroll
    for (int r = 0; r < 4; r++) row[r] = {0, 0, 0, 0};
    uint32_t k = 0;
    for (; k + 6 <= n_cons; k += 6) {
      uint4 cv[6];
#pragma unroll
      for (int u = 0; u < 6; u++) cv[u] = ldg4(evals + (uint64_t)(k + u + 2) * col_stride + i);
#pragma unroll
      for (int u = 0; u < 6; u++) {
        const qm31 pw = powers[k + u];
#pragma unroll
        for (int r = 0; r < 4; r++) {
          const uint32_t c = u4get(cv[u], r);
          acc4_mad(row[r], pw, m31_sub(c, m31_add(sa[r], sb[r])));
          sa[r] = sb[r];
          sb[r] = m31_sqr(c);
        }
        if (u == 2 || u == 5) {
#pragma unroll
          for (int r = 0; r < 4; r++) acc4_fold(row[r]);
        }
      }
    }
    for (; k < n_cons; k++) {  // remainder: fold after every term
      const uint4 cv = ldg4(evals + (uint64_t)(k + 2) * col_stride + i);
      const qm31 pw = powers[k];
#pragma unroll
      for (int r = 0; r < 4; r++) {
        const uint32_t c = u4get(cv, r);
        acc4_mad(row[r], pw, m31_sub(c, m31_add(sa[r], sb[r])));
        acc4_fold(row[r]);
        sa[r] = sb[r];
        sb[r] = m31_sqr(c);
      }
    }
    qm31 v[4];
#pragma unroll
    for (int r = 0; r < 4; r++) v[r] = qm31_mul_m31(acc4_reduce(row[r]), __ldg(denom_inv + ((i + r) >> log_n)));
    *reinterpret_cast<uint4*>(out + i) = make_uint4(v[0].a, v[1].a, v[2].a, v[3].a);
    *reinterpret_cast<uint4*>(out + n_points + i) = make_uint4(v[0].b, v[1].b, v[2].b, v[3].b);
    *reinterpret_cast<uint4*>(out + 2 * n_points + i) = make_uint4(v[0].c, v[1].c, v[2].c, v[3].c);
    *reinterpret_cast<uint4*>(out + 3 * n_points + i) = make_uint4(v[0].d, v[1].d, v[2].d, v[3].d);
  }
}

// OODS sampling for every polynomial of one size: the block stages the
// weights w_j of a 1024-index chunk in shared memory, then each warp takes one
// polynomial at a time and reduces its chunk (coalesced loads, 8 in flight per
// lane) to one partial sum per (polynomial, chunk).  Sums are exact field sums,
// so the grouping does not change the result.
constexpr uint32_t kOodsChunk = 1024;
__global__ void __launch_bounds__(256) oods_eval_kernel(PolyTable t, uint32_t n_polys, uint32_t log_n, uint32_t h,
                                                       const qm31* __restrict__ w_lo, const qm31* __restrict__ w_hi,
                                                       qm31* __restrict__ partial) {
  __shared__ uint4 ws[kOodsChunk];
  const uint64_t n = 1ull << log_n;
  const uint32_t chunk = n < kOodsChunk ? (uint32_t)n : kOodsChunk;
  const uint64_t j0 = (uint64_t)blockIdx.x * chunk;
  const uint64_t lo_mask = (1ull << h) - 1;
  // A chunk inside one w_hi bucket (chunk <= 2^h, both powers of two): the
  // inner sums take w_lo alone and each partial is multiplied by the bucket's
  // w_hi once, an exact rewrite of the same sum.
  const bool one_bucket = chunk <= (1ull << h);
  for (uint32_t k = threadIdx.x; k < chunk; k += blockDim.x) {
    const uint64_t j = j0 + k;
    const qm31 w = one_bucket ? w_lo[j & lo_mask] : qm31_mul(w_hi[j >> h], w_lo[j & lo_mask]);
    ws[k] = make_uint4(w.a, w.b, w.c, w.d);
  }
  const qm31 wh = one_bucket ? w_hi[j0 >> h] : qm31_one();
  __syncthreads();
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t n_warps = blockDim.x >> 5;
  // blockIdx.y picks a group of polynomials: smaller blocks, so that the grid
  // spans several waves instead of one full wave and a nearly empty second.
  const uint32_t per_group = (n_polys + gridDim.y - 1) / gridDim.y;
  const uint32_t p_end = min(n_polys, (blockIdx.y + 1) * per_group);
  for (uint32_t p = blockIdx.y * per_group + warp; p < p_end; p += n_warps) {
    const uint32_t* __restrict__ col = t.p[p] + j0;
    acc4 s{0, 0, 0, 0};
    if (chunk == kOodsChunk) {
#pragma unroll 1
      for (uint32_t b = 0; b < kOodsChunk; b += 512) {
        uint32_t v[16];  // 16 loads in flight per lane
#pragma unroll
        for (int u = 0; u < 16; u++) v[u] = __ldg(col + b + u * 32 + lane);
#pragma unroll
        for (int u = 0; u < 16; u++) {
          const uint4 w = ws[b + u * 32 + lane];
          acc4_mad(s, qm31{w.x, w.y, w.z, w.w}, v[u]);
          if (u % 4 == 3) acc4_fold(s);
        }
      }
    } else {
      for (uint32_t k = lane; k < chunk; k += 32) {
        const uint4 w = ws[k];
        acc4_mad(s, qm31{w.x, w.y, w.z, w.w}, __ldg(col + k));
        acc4_fold(s);
      }
    }
    qm31 v = acc4_reduce(s);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const qm31 u = {__shfl_xor_sync(0xffffffffu, v.a, o), __shfl_xor_sync(0xffffffffu, v.b, o),
                      __shfl_xor_sync(0xffffffffu, v.c, o), __shfl_xor_sync(0xffffffffu, v.d, o)};
      v = qm31_add(v, u);
    }
    if (lane == 0) partial[(uint64_t)p * gridDim.x + blockIdx.x] = one_bucket ? qm31_mul(v, wh) : v;
  }
}

// out[p] = sum of partial[p][0 .. n_chunks); one block per polynomial.
__global__ void __launch_bounds__(256) oods_reduce_kernel(const qm31* __restrict__ partial, uint32_t n_chunks,
                                                         qm31* __restrict__ out) {
  __shared__ qm31 red[256];
  const uint32_t p = blockIdx.x;
  qm31 s = qm31_zero();
  for (uint32_t c = threadIdx.x; c < n_chunks; c += blockDim.x) s = qm31_add(s, partial[(uint64_t)p * n_chunks + c]);
  red[threadIdx.x] = s;
  __syncthreads();
  for (uint32_t k = blockDim.x / 2; k > 0; k >>= 1) {
    if (threadIdx.x < k) red[threadIdx.x] = qm31_add(red[threadIdx.x], red[threadIdx.x + k]);
    __syncthreads();
  }
  if (threadIdx.x == 0) out[p] = red[0];
}

// OODS sampling of polynomials whose index splits as bucket b (the bits above
// kEvalLoBits) and position e < 1024: sum_j c_j w_j = sum_b w_hi[b] sum_e
// c_(1024 b + e) w_lo[e].  Each warp takes one unit (a polynomial and
// kEvalUnitBuckets consecutive buckets) and keeps the next bucket's 16-byte
// loads in flight while it multiplies the current one; a lane reads 4
// consecutive coefficients per load.  The block stages w_lo once,
// component-major, so the 4 weights of a lane's coefficients are one
// conflict-free 16-byte shared load per component.  Per bucket a lane
// reduces its sum, multiplies it by w_hi[b] and adds it to its unit total;
// the warp reduces the totals once per unit into
// partial[p * units_per_poly + unit].  The 4 wide multiply-adds per
// coefficient bound it (about 80 us of the multiply-add pipe for 108 x 2^20
// coefficients), above the HBM time of the reads.
constexpr uint32_t kEvalLoBits = 10;
constexpr uint32_t kEvalUnitBuckets = 8;
__global__ void __launch_bounds__(256, 2) poly_eval_bucket_kernel(PolyTable t, uint32_t n_polys, uint32_t units_per_poly,
                                                                  const qm31* __restrict__ w_lo,
                                                                  const qm31* __restrict__ w_hi,
                                                                  qm31* __restrict__ partial) {
  __shared__ uint4 wc[4][256];  // wc[k][q]: component k of w_lo[4q .. 4q+3]
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t unit = blockIdx.x * 8 + warp;
  const bool active = unit < n_polys * units_per_poly;
  const uint32_t p = active ? unit / units_per_poly : 0, u = unit - p * units_per_poly;
  const uint32_t b0 = u * kEvalUnitBuckets;
  const uint32_t* __restrict__ col = t.p[p] + ((size_t)b0 << kEvalLoBits) + 4 * lane;
  uint4 cur[8], nxt[8];
  if (active) {
#pragma unroll
    for (int k = 0; k < 8; k++) cur[k] = ldg4(col + 128 * k);
  }
  {
    const qm31 a = w_lo[4 * threadIdx.x], b = w_lo[4 * threadIdx.x + 1], c = w_lo[4 * threadIdx.x + 2],
               d = w_lo[4 * threadIdx.x + 3];
    wc[0][threadIdx.x] = make_uint4(a.a, b.a, c.a, d.a);
    wc[1][threadIdx.x] = make_uint4(a.b, b.b, c.b, d.b);
    wc[2][threadIdx.x] = make_uint4(a.c, b.c, c.c, d.c);
    wc[3][threadIdx.x] = make_uint4(a.d, b.d, c.d, d.d);
  }
  __syncthreads();
  if (!active) return;  // no block barrier follows
  qm31 tot = qm31_zero();
#pragma unroll 1
  for (uint32_t bi = 0; bi < kEvalUnitBuckets; bi++) {
    if (bi + 1 < kEvalUnitBuckets) {
#pragma unroll
      for (int k = 0; k < 8; k++) nxt[k] = ldg4(col + ((size_t)(bi + 1) << kEvalLoBits) + 128 * k);
    }
    acc4 s{0, 0, 0, 0};
#pragma unroll
    for (int k = 0; k < 8; k++) {
      const uint32_t q = 32 * k + lane;
      const uint4 x = cur[k];
      const uint4 wa = wc[0][q], wb = wc[1][q], wcc = wc[2][q], wd = wc[3][q];
      s.a += (uint64_t)wa.x * x.x + (uint64_t)wa.y * x.y + (uint64_t)wa.z * x.z + (uint64_t)wa.w * x.w;
      s.b += (uint64_t)wb.x * x.x + (uint64_t)wb.y * x.y + (uint64_t)wb.z * x.z + (uint64_t)wb.w * x.w;
      s.c += (uint64_t)wcc.x * x.x + (uint64_t)wcc.y * x.y + (uint64_t)wcc.z * x.z + (uint64_t)wcc.w * x.w;
      s.d += (uint64_t)wd.x * x.x + (uint64_t)wd.y * x.y + (uint64_t)wd.z * x.z + (uint64_t)wd.w * x.w;
      acc4_fold(s);
    }
    tot = qm31_add(tot, qm31_mul(acc4_reduce(s), w_hi[b0 + bi]));
#pragma unroll
    for (int k = 0; k < 8; k++) cur[k] = nxt[k];
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const qm31 v = {__shfl_xor_sync(0xffffffffu, tot.a, o), __shfl_xor_sync(0xffffffffu, tot.b, o),
                    __shfl_xor_sync(0xffffffffu, tot.c, o), __shfl_xor_sync(0xffffffffu, tot.d, o)};
    tot = qm31_add(tot, v);
  }
  if (lane == 0) partial[unit] = tot;
}

uint32_t poly_eval_chunks(uint32_t lg) { return lg > 10 ? 1u << (lg - 10) : 1u; }  // kOodsChunk indices each
// kEvalLoBits wherever the bucketed form applies (at least kEvalUnitBuckets
// buckets per polynomial and a w_hi table of at most 2^14 entries).
uint32_t poly_eval_lo_bits(uint32_t lg) { return lg >= 13 && lg <= 24 ? kEvalLoBits : lg / 2; }

int launch_poly_eval(const uint32_t* const* polys, uint32_t n_polys, uint32_t lg, const qm31* d_w_lo,
                     const qm31* d_w_hi, qm31* d_partial, qm31* d_out, cudaStream_t s, char* err, size_t err_len) {
  STWO_ARG_CHECK(n_polys >= 1 && n_polys <= (uint32_t)kMaxPolys && lg <= 30, "poly eval: bad shape");
  PolyTable pt;
  for (uint32_t c = 0; c < n_polys; c++) pt.p[c] = polys[c];
  const uint32_t h = poly_eval_lo_bits(lg);
  if (h == kEvalLoBits) {
    // 2^(lg - h) >= kEvalUnitBuckets buckets of 1024 indices per polynomial
    const uint32_t units_per_poly = (1u << (lg - h)) / kEvalUnitBuckets;
    const uint32_t units = n_polys * units_per_poly;
    poly_eval_bucket_kernel<<<(units + 7) / 8, 256, 0, s>>>(pt, n_polys, units_per_poly, d_w_lo, d_w_hi, d_partial);
    STWO_CHECK_LAUNCH();
    oods_reduce_kernel<<<n_polys, 256, 0, s>>>(d_partial, units_per_poly, d_out);
    STWO_CHECK_LAUNCH();
    return STWO_B200_OK;
  }
  const uint32_t chunks = poly_eval_chunks(lg);
  // about 4 waves of 148 SMs x 6 resident blocks, at least 8 polynomials (one per warp) per group
  const uint32_t groups = std::max(1u, std::min({8u, (4u * 148u * 6u + chunks - 1) / chunks, n_polys / 8u}));
  oods_eval_kernel<<<dim3(chunks, groups), 256, 0, s>>>(pt, n_polys, lg, h, d_w_lo, d_w_hi, d_partial);
  STWO_CHECK_LAUNCH();
  oods_reduce_kernel<<<n_polys, 256, 0, s>>>(d_partial, chunks, d_out);
  STWO_CHECK_LAUNCH();
  return STWO_B200_OK;
}

// FRI quotient of one sample batch (all columns sampled at point z, same
// size): q(p) = [c * sum_k alpha^k f_k(p) - B - A * p.y] / den(p), den(p) =
// (Re z.x - p.x) Im z.y - (Re z.y - p.y) Im z.x in CM31.  Equal, value for
// value, to the line-coefficient form of prover/backend/simd/quotients.rs:34-164
// with core/constraints.rs:119-134 coefficients.
// Per-proof constants of the quotient rows (they depend on the OODS point
// and the sampled values): written in device memory by fs_quotient_kernel.
struct QuotientDyn {
  qm31 c, A, B;
  cm31 prx, pix, pry, piy;
};
struct QuotientParams {
  cpoint init;           // first point of the half coset
  cpoint step_pow[31];   // step * 2^b
  uint32_t log_size;     // lifting domain
  cpoint tile_pts[256];  // m * step * 2^(log_size - tile bits), m < rows/4 (quotient_tma_kernel)
};

// FRI quotients, 4 consecutive rows per thread: 16-byte column loads and one
// shared inversion for the four denominators (their norms are inverted
// together with Montgomery's trick; exact, so equal to four cm31_inv).
// n % 4 == 0, columns 16-byte aligned.  The streaming form quotient_tma_kernel
// takes every domain of at least two 512-row tiles.
__device__ __forceinline__ cpoint quotient_point(const QuotientParams& q, uint64_t i) {
  const uint64_t n = 1ull << q.log_size, half = n >> 1;
  const uint64_t j = __brevll(i) >> (64 - q.log_size);
  const uint64_t jj = j < half ? j : j - half;
  cpoint pt = q.init;
  for (uint32_t b = 0; b + 1 < q.log_size; b++)
    if ((jj >> b) & 1) pt = cpoint_add(pt, q.step_pow[b]);
  if (j >= half) pt.y = m31_neg(pt.y);
  return pt;
}

__global__ void __launch_bounds__(256) quotient4_kernel(QuotientParams q, PolyTable cols, uint32_t n_cols,
                                                       const qm31* __restrict__ alpha_pows,
                                                       const QuotientDyn* __restrict__ dyn,
                                                       uint32_t* __restrict__ out) {
  const QuotientDyn& qd = *dyn;  // read at the epilogue, through the read-only cache
  const uint64_t n = 1ull << q.log_size;
  const uint64_t n4 = n >> 2;
  for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < n4; t += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t i = t << 2;
    acc4 s4[4];
#pragma unroll
    for (int r = 0; r < 4; r++) s4[r] = {0, 0, 0, 0};
    uint32_t k = 0;
    for (; k + 6 <= n_cols; k += 6) {
      uint4 fv[6];
#pragma unroll
      for (int u = 0; u < 6; u++) fv[u] = ldg4(cols.p[k + u] + i);
#pragma unroll
      for (int u = 0; u < 6; u++) {
        const qm31 ap = alpha_pows[k + u];
#pragma unroll
        for (int r = 0; r < 4; r++) acc4_mad(s4[r], ap, u4get(fv[u], r));
        if (u == 2 || u == 5) {
#pragma unroll
          for (int r = 0; r < 4; r++) acc4_fold(s4[r]);
        }
      }
    }
    for (; k < n_cols; k++) {  // remainder: fold after every term
      const uint4 fv = ldg4(cols.p[k] + i);
      const qm31 ap = alpha_pows[k];
#pragma unroll
      for (int r = 0; r < 4; r++) {
        acc4_mad(s4[r], ap, u4get(fv, r));
        acc4_fold(s4[r]);
      }
    }
    qm31 full[4];
    cm31 den[4];
    uint32_t norm[4];
#pragma unroll
    for (int r = 0; r < 4; r++) {
      const cpoint pt = quotient_point(q, i + r);
      const qm31 num = qm31_sub(qm31_mul(qd.c, acc4_reduce(s4[r])), qd.B);
      full[r] = qm31_sub(num, qm31_mul_m31(qd.A, pt.y));
      den[r] = cm31_sub(cm31_mul(cm31_sub(qd.prx, cm31{pt.x, 0}), qd.piy),
                        cm31_mul(cm31_sub(qd.pry, cm31{pt.y, 0}), qd.pix));
      norm[r] = m31_add(m31_sqr(den[r].a), m31_sqr(den[r].b));
    }
    // Montgomery batch inversion of the four norms.
    const uint32_t p01 = m31_mul(norm[0], norm[1]);
    const uint32_t p012 = m31_mul(p01, norm[2]);
    uint32_t inv = m31_inv(m31_mul(p012, norm[3]));
    uint32_t ninv[4];
    ninv[3] = m31_mul(inv, p012);
    inv = m31_mul(inv, norm[3]);
    ninv[2] = m31_mul(inv, p01);
    inv = m31_mul(inv, norm[2]);
    ninv[1] = m31_mul(inv, norm[0]);
    ninv[0] = m31_mul(inv, norm[1]);
    qm31 v[4];
#pragma unroll
    for (int r = 0; r < 4; r++) {
      const cm31 di = cm31_mul({den[r].a, m31_neg(den[r].b)}, {ninv[r], 0});
      v[r] = qm31_mul_cm31(full[r], di);
    }
    *reinterpret_cast<uint4*>(out + i) = make_uint4(v[0].a, v[1].a, v[2].a, v[3].a);
    *reinterpret_cast<uint4*>(out + n + i) = make_uint4(v[0].b, v[1].b, v[2].b, v[3].b);
    *reinterpret_cast<uint4*>(out + 2 * n + i) = make_uint4(v[0].c, v[1].c, v[2].c, v[3].c);
    *reinterpret_cast<uint4*>(out + 3 * n + i) = make_uint4(v[0].d, v[1].d, v[2].d, v[3].d);
  }
}

// ---- TMA column-streaming versions ----
// A block owns kStreamRows consecutive rows; consumer thread t owns rows 4t ..
// 4t+3.  Columns arrive kStreamG at a time through the shared-memory stages of
// ColumnPipe (cp.async.bulk issued by a producer warp, full/empty mbarriers),
// so the DRAM reads of the next groups overlap the arithmetic of the current
// one and no block barrier is taken per group.  Same arithmetic per point as
// composition4_kernel / quotient4_kernel.
constexpr int kStreamTileBits = 9, kStreamRows = 1 << kStreamTileBits, kStreamG = 6, kStreamS = 3;
static_assert(kStreamG == 6, "the fold positions of the streaming kernels assume 6-column groups");
constexpr int kStreamThreads = kStreamRows / 4;      // consumers: four rows per thread
constexpr int kStreamBlock = kStreamThreads + 32;    // plus the producer warp
using StreamPipe = ColumnPipe<kStreamG, kStreamS, kStreamRows, kStreamThreads>;
constexpr int kPipeBarWords = 2 * kStreamS + (kStreamS * kPipeHeaderWords + 1 + 1) / 2;  // uint64 slots
constexpr uint32_t kStreamErrWord = 8;  // word of the prover's flag buffer set by a timed-out stage
constexpr size_t kStreamRing = (size_t)kStreamS * kStreamG * kStreamRows * sizeof(uint32_t);
constexpr uint32_t kStreamMaxW = 1024;  // QM31 weights staged in shared memory
constexpr size_t kStreamSmem = kStreamRing + kStreamMaxW * sizeof(uint4);

__device__ __forceinline__ void stage_weights(uint4* sw, const qm31* __restrict__ w, uint32_t n) {
  for (uint32_t k = threadIdx.x; k < n; k += blockDim.x) sw[k] = make_uint4(w[k].a, w[k].b, w[k].c, w[k].d);
}

__global__ void __launch_bounds__(kStreamBlock) composition_tma_kernel(
    const uint32_t* __restrict__ evals, uint64_t col_stride, uint32_t n_cons, const qm31* __restrict__ powers,
    const uint32_t* __restrict__ denom_inv, uint32_t log_n, uint64_t n_points, uint32_t* __restrict__ out,
    uint32_t* err, uint32_t spin) {
  extern __shared__ __align__(128) uint32_t smem[];
  __shared__ uint64_t bars[kPipeBarWords];
  uint4* sw = reinterpret_cast<uint4*>(smem + kStreamRing / sizeof(uint32_t));
  const uint32_t t4 = threadIdx.x * 4;
  auto col = [evals, col_stride](uint32_t c) { return evals + (uint64_t)c * col_stride; };
  StreamPipe pipe(smem, bars, n_cons + 2, (uint32_t)(n_points / kStreamRows), spin);
  stage_weights(sw, powers, n_cons);
  __syncthreads();  // the last block barrier: the producer warp leaves the loop below
  if (threadIdx.x >= kStreamThreads) {
    if (threadIdx.x == kStreamThreads) pipe.produce(col, [](uint32_t, uint32_t*) {}, err);
    return;
  }
  for (uint32_t t = 0; t < pipe.my_tiles; t++) {
    uint32_t sa[4] = {0, 0, 0, 0}, sb[4] = {0, 0, 0, 0};
    acc4 row[4];
#pragma unroll
    for (int r = 0; r < 4; r++) row[r] = {0, 0, 0, 0};
    // Constraint k = c - 2 of column c = 6g + j: folding after j = 3 in even
    // groups and after j = 1 and j = 5 in odd ones leaves at most four
    // products between folds.
    for (uint32_t g = 0; g < pipe.n_groups; g++) {
      const uint32_t gg = t * pipe.n_groups + g;
      if (!pipe.wait(gg, err)) return;
      const uint32_t nc = pipe.cols_in(g);
#pragma unroll
      for (int j = 0; j < kStreamG; j++) {
        if ((uint32_t)j < nc) {
          const uint32_t c = g * kStreamG + j;
          const uint4 v = *reinterpret_cast<const uint4*>(pipe.seg(gg, j) + t4);
          if (c >= 2) {
            const uint4 pw4 = sw[c - 2];
            const qm31 pw{pw4.x, pw4.y, pw4.z, pw4.w};
#pragma unroll
            for (int r = 0; r < 4; r++) {
              const uint32_t x = u4get(v, r);
              acc4_mad(row[r], pw, m31_sub(x, m31_add(sa[r], sb[r])));
              sa[r] = sb[r];
              sb[r] = m31_sqr(x);
            }
          } else {
#pragma unroll
            for (int r = 0; r < 4; r++) {
              sa[r] = sb[r];
              sb[r] = m31_sqr(u4get(v, r));
            }
          }
        }
        if ((g & 1) ? (j == 1 || j == 5) : (j == 3)) {
#pragma unroll
          for (int r = 0; r < 4; r++) acc4_fold(row[r]);
        }
      }
      pipe.release(gg);
    }
    const uint64_t i = pipe.tile_row0(t) + t4;
    qm31 v[4];
#pragma unroll
    for (int r = 0; r < 4; r++) v[r] = qm31_mul_m31(acc4_reduce(row[r]), __ldg(denom_inv + ((i + r) >> log_n)));
    *reinterpret_cast<uint4*>(out + i) = make_uint4(v[0].a, v[1].a, v[2].a, v[3].a);
    *reinterpret_cast<uint4*>(out + n_points + i) = make_uint4(v[0].b, v[1].b, v[2].b, v[3].b);
    *reinterpret_cast<uint4*>(out + 2 * n_points + i) = make_uint4(v[0].c, v[1].c, v[2].c, v[3].c);
    *reinterpret_cast<uint4*>(out + 3 * n_points + i) = make_uint4(v[0].d, v[1].d, v[2].d, v[3].d);
  }
}

// Rows 4t .. 4t+3 of a tile (R = 2^b rows, t < R/4): with r0 a multiple of
// R, the bit-reversed positions are j(r0 + 4t + e) = J0 + bitrev_{b-2}(t) *
// 2^(log-b) + bitrev2(e) * 2^(log-2).  e = 0, 2 lie below the half (jj = J0 +
// bitrev_{b-2}(t) * 2^(log-b) and that + 2^(log-2)); e = 1, 3 are their
// conjugates in the upper half.  So the two points are B +
// tile_pts[bitrev_{b-2}(t)] and that + step * 2^(log-2), B = init + J0 * step.
__global__ void __launch_bounds__(kStreamBlock) quotient_tma_kernel(QuotientParams q, PolyTable cols,
                                                                   uint32_t n_cols,
                                                                   const qm31* __restrict__ alpha_pows,
                                                                   const QuotientDyn* __restrict__ dyn,
                                                                   uint32_t* __restrict__ out, uint32_t* err,
                                                                   uint32_t spin) {
  const QuotientDyn& qd = *dyn;  // read at the epilogue, through the read-only cache
  extern __shared__ __align__(128) uint32_t smem[];
  __shared__ uint64_t bars[kPipeBarWords];
  uint4* sw = reinterpret_cast<uint4*>(smem + kStreamRing / sizeof(uint32_t));
  const uint64_t n = 1ull << q.log_size;
  const uint32_t t4 = threadIdx.x * 4;
  const PolyTable* tab = &cols;
  auto col = [tab](uint32_t c) { return tab->p[c]; };
  StreamPipe pipe(smem, bars, n_cols, (uint32_t)(n / kStreamRows), spin);
  stage_weights(sw, alpha_pows, n_cols);
  __syncthreads();  // the last block barrier: the producer warp leaves the loop below
  if (threadIdx.x >= kStreamThreads) {
    if (threadIdx.x == kStreamThreads) {
      // Tile header: B = init + J0 * step, J0 the bit-reversed first row.
      const QuotientParams* qp = &q;
      pipe.produce(col,
                   [qp, &pipe](uint32_t t, uint32_t* h) {
                     const uint64_t J0 = __brevll(pipe.tile_row0(t)) >> (64 - qp->log_size);
                     cpoint b = qp->init;
                     for (uint32_t k = 0; k + 1 < qp->log_size; k++)
                       if ((J0 >> k) & 1) b = cpoint_add(b, qp->step_pow[k]);
                     h[0] = b.x;
                     h[1] = b.y;
                   },
                   err);
    }
    return;
  }
  for (uint32_t t = 0; t < pipe.my_tiles; t++) {
    const uint64_t r0 = pipe.tile_row0(t);
    cpoint base{0, 0};
    acc4 s4[4];
#pragma unroll
    for (int r = 0; r < 4; r++) s4[r] = {0, 0, 0, 0};
    for (uint32_t g = 0; g < pipe.n_groups; g++) {
      const uint32_t gg = t * pipe.n_groups + g;
      if (!pipe.wait(gg, err)) return;
      if (g == 0) {  // header of the tile, valid while this stage is held
        const uint32_t* h = pipe.head(gg);
        base = cpoint{h[0], h[1]};
      }
      const uint32_t nc = pipe.cols_in(g);
#pragma unroll
      for (int j = 0; j < kStreamG; j++) {
        if ((uint32_t)j < nc) {
          const uint32_t c = g * kStreamG + j;
          const uint4 v = *reinterpret_cast<const uint4*>(pipe.seg(gg, j) + t4);
          const uint4 a4 = sw[c];
          const qm31 ap{a4.x, a4.y, a4.z, a4.w};
#pragma unroll
          for (int r = 0; r < 4; r++) acc4_mad(s4[r], ap, u4get(v, r));
        }
        if ((g & 1) ? (j == 1 || j == 5) : (j == 3)) {  // at most four products between folds
#pragma unroll
          for (int r = 0; r < 4; r++) acc4_fold(s4[r]);
        }
      }
      pipe.release(gg);
    }
    const cpoint p0 = cpoint_add(base, q.tile_pts[__brev(threadIdx.x) >> (32 - (kStreamTileBits - 2))]);
    const cpoint p2 = cpoint_add(p0, q.step_pow[q.log_size - 2]);
    const uint32_t xs[4] = {p0.x, p0.x, p2.x, p2.x};
    const uint32_t ys[4] = {p0.y, m31_neg(p0.y), p2.y, m31_neg(p2.y)};
    qm31 full[4];
    cm31 den[4];
    uint32_t norm[4];
#pragma unroll
    for (int r = 0; r < 4; r++) {
      const qm31 num = qm31_sub(qm31_mul(qd.c, acc4_reduce(s4[r])), qd.B);
      full[r] = qm31_sub(num, qm31_mul_m31(qd.A, ys[r]));
      den[r] = cm31_sub(cm31_mul(cm31_sub(qd.prx, cm31{xs[r], 0}), qd.piy),
                        cm31_mul(cm31_sub(qd.pry, cm31{ys[r], 0}), qd.pix));
      norm[r] = m31_add(m31_sqr(den[r].a), m31_sqr(den[r].b));
    }
    // Montgomery batch inversion of the four norms.
    const uint32_t p01 = m31_mul(norm[0], norm[1]);
    const uint32_t p012 = m31_mul(p01, norm[2]);
    uint32_t inv = m31_inv(m31_mul(p012, norm[3]));
    uint32_t ninv[4];
    ninv[3] = m31_mul(inv, p012);
    inv = m31_mul(inv, norm[3]);
    ninv[2] = m31_mul(inv, p01);
    inv = m31_mul(inv, norm[2]);
    ninv[1] = m31_mul(inv, norm[0]);
    ninv[0] = m31_mul(inv, norm[1]);
    qm31 v[4];
#pragma unroll
    for (int r = 0; r < 4; r++)
      v[r] = qm31_mul_cm31(full[r], cm31_mul({den[r].a, m31_neg(den[r].b)}, {ninv[r], 0}));
    const uint64_t i = r0 + t4;
    *reinterpret_cast<uint4*>(out + i) = make_uint4(v[0].a, v[1].a, v[2].a, v[3].a);
    *reinterpret_cast<uint4*>(out + n + i) = make_uint4(v[0].b, v[1].b, v[2].b, v[3].b);
    *reinterpret_cast<uint4*>(out + 2 * n + i) = make_uint4(v[0].c, v[1].c, v[2].c, v[3].c);
    *reinterpret_cast<uint4*>(out + 3 * n + i) = make_uint4(v[0].d, v[1].d, v[2].d, v[3].d);
  }
}

// Proof-of-work search over nonces (hi << 32) | (low_base + t)
// (prover/backend/simd/grind.rs:62-96): a hit needs trailing_zeros(word 0 of
// Blake2s(prefixed_digest || LE64(nonce))) >= bits; the smallest hit wins.
struct Digest8 {
  uint32_t w[8];
};
constexpr uint32_t kGrindBatch = 1u << 16;  // nonces per grind launch of the prover
__global__ void grind_kernel(Digest8 pre, uint32_t hi, uint32_t low_base, uint32_t bits, int m31,
                             uint32_t* __restrict__ found) {
  uint32_t low = low_base + blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t m[16];
#pragma unroll
  for (int k = 0; k < 8; k++) m[k] = pre.w[k];
  m[8] = low;
  m[9] = hi;
#pragma unroll
  for (int k = 10; k < 16; k++) m[k] = 0;
  uint32_t h[8];
  blake2s_init(h);
  blake2s_compress(h, m, 40, true);
  uint32_t w0 = m31 ? m31_reduce_u32(h[0]) : h[0];
  uint32_t tz = w0 == 0 ? 32u : (uint32_t)__ffs(w0) - 1;
  if (tz >= bits) atomicMin(found, low);
}

// Nonces (hi << 32) | (low_base + t), t < count (a multiple of 256): the
// smallest hit is atomicMin'ed into *d_found (which the caller sets to
// 0xFFFFFFFF first).
int launch_grind(const uint32_t pre[8], uint32_t hi, uint32_t low_base, uint32_t count, uint32_t bits, int m31,
                 uint32_t* d_found, cudaStream_t s, char* err, size_t err_len) {
  STWO_ARG_CHECK(count % 256 == 0 && count > 0, "grind batch must be a positive multiple of 256");
  Digest8 d;
  for (int k = 0; k < 8; k++) d.w[k] = pre[k];
  grind_kernel<<<count / 256, 256, 0, s>>>(d, hi, low_base, bits, m31, d_found);
  STWO_CHECK_LAUNCH();
  return STWO_B200_OK;
}

__global__ void gather_kernel(const uint64_t* __restrict__ addrs, uint32_t n, uint32_t* __restrict__ out) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = *reinterpret_cast<const uint32_t*>(addrs[i]);
}
// 32-byte hashes at 32-byte aligned addresses (Merkle tree nodes).
__global__ void gather_hashes_kernel(const uint64_t* __restrict__ addrs, uint32_t n, uint4* __restrict__ out) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    const uint4* p = reinterpret_cast<const uint4*>(addrs[i]);
    out[2 * i] = p[0];
    out[2 * i + 1] = p[1];
  }
}

// ---- device-side Fiat-Shamir steps of the FRI commit ----
// The channel state lives in device memory so the FRI layer loop (commit a
// layer, mix its root, draw the folding alpha, fold) is enqueued without host
// round trips (core/channel/blake2s.rs:25-120, core/vcs_lifted/blake2_merkle.rs:49-56).
struct DevChannel {
  uint32_t digest[8];
  uint32_t n_draws;
  uint32_t m31;
  uint32_t error;  // set when a secure-felt draw exhausted its retry bound
  uint32_t pad;
};

__device__ void dev_finalize(uint32_t h[8], bool m31) {
  if (m31)
    for (int k = 0; k < 8; k++) h[k] = m31_reduce_u32(h[k]);
}

// digest <- H(digest || root) (core/vcs_lifted/blake2_merkle.rs:49-56); one thread.
__device__ void dev_chan_mix_root(DevChannel* ch, const uint32_t* root) {
  uint32_t m[16];
  for (int k = 0; k < 8; k++) m[k] = ch->digest[k];
  for (int k = 0; k < 8; k++) m[8 + k] = root[k];
  uint32_t h[8];
  blake2s_init(h);
  blake2s_compress_lat(h, m, 64, true);
  dev_finalize(h, ch->m31 != 0);
  for (int k = 0; k < 8; k++) ch->digest[k] = h[k];
  ch->n_draws = 0;
}

// draw_secure_felt (core/channel/blake2s.rs:72-120): draw_base_felts retries
// until all 8 words are below 2P (probability of a retry ~2^-28 per draw);
// bounded, with an error flag instead of a hang.  One thread.
__device__ qm31 dev_chan_draw_felt(DevChannel* ch) {
  uint32_t m[16], h[8];
  uint32_t n_draws = ch->n_draws;
  for (int attempt = 0; attempt < 64; attempt++) {
    for (int k = 0; k < 8; k++) m[k] = ch->digest[k];
    m[8] = n_draws;
    for (int k = 9; k < 16; k++) m[k] = 0;
    n_draws++;
    blake2s_init(h);
    blake2s_compress_lat(h, m, 37, true);
    dev_finalize(h, ch->m31 != 0);
    bool okw = true;
    for (int k = 0; k < 8; k++) okw = okw && h[k] < 2 * M31_P;
    if (okw) {
      ch->n_draws = n_draws;
      return {m31_reduce_u32(h[0]), m31_reduce_u32(h[1]), m31_reduce_u32(h[2]), m31_reduce_u32(h[3])};
    }
  }
  ch->error = 1;
  ch->n_draws = n_draws;
  return qm31_zero();
}

// digest <- H(digest || LE32 coordinates of n QM31 values) (core/channel/
// blake2s.rs:54-64).  The digest and the values are staged by the block as
// 16-word message blocks in s_words (zero padded, 8 + 4 n words); thread 0
// then chains the compressions, reading each block from shared memory.
constexpr uint32_t kMixWordsCap = (8 + 4 * kMaxPolys + 15) & ~15u;
__device__ void stage_mix_words(const DevChannel* ch, const qm31* __restrict__ f, uint32_t n, uint32_t* s_words) {
  const uint32_t total = 8 + 4 * n, padded = (total + 15) & ~15u;
  const uint32_t* fw = reinterpret_cast<const uint32_t*>(f);  // a, b, c, d of each value in order
  for (uint32_t w = threadIdx.x; w < padded; w += blockDim.x)
    s_words[w] = w < 8 ? ch->digest[w] : (w < total ? fw[w - 8] : 0u);
}
__device__ void dev_chan_mix_staged(DevChannel* ch, const uint32_t* s_words, uint32_t n) {
  const uint32_t total_words = 8 + 4 * n;
  const uint32_t blocks = (total_words + 15) / 16;
  uint32_t h[8], m[16];
  blake2s_init(h);
  for (uint32_t bk = 0; bk < blocks; bk++) {
#pragma unroll
    for (int k = 0; k < 16; k++) m[k] = s_words[bk * 16 + k];
    const bool last = bk + 1 == blocks;
    blake2s_compress_lat(h, m, last ? 4 * total_words : 64 * (bk + 1), last);
  }
  dev_finalize(h, ch->m31 != 0);
  for (int k = 0; k < 8; k++) ch->digest[k] = h[k];
  ch->n_draws = 0;
}

// The end of the FRI commit on the device channel (prover/fri.rs:274-291,
// pcs/mod.rs:140-142), so that the first proof-of-work batch runs without a
// host round trip: the last layer's 2^last_log evaluations (4 coordinate
// columns) -> coefficients as LineEvaluation::interpolate computes them
// (bit reversal, the line IFFT with the inverse x-coordinates xi, in the
// order the host walks them, times 1/n, bit reversal into coefficient
// order); the first 2^bound_log are mixed into a copy of the channel, and
// pow[0..8) receives H(POW_PREFIX, [0; 12], digest, n_bits)
// (core/channel/blake2s.rs:124-132); pow[8] = 1 when a higher coefficient is
// nonzero.  The channel itself is left at its end-of-commit state, which the
// host downloads to replay the transcript.  One thread.
constexpr uint32_t kFinishMaxLast = 64;
__global__ void fri_finish_kernel(const DevChannel* __restrict__ ch, const uint32_t* __restrict__ last,
                                  uint32_t last_log, uint32_t bound_log, const uint32_t* __restrict__ xi,
                                  uint32_t n_inv, uint32_t pow_bits, uint32_t* __restrict__ pow) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const uint32_t n = 1u << last_log;
  qm31 v[kFinishMaxLast];
  for (uint32_t i = 0; i < n; i++) {
    const uint32_t j = last_log ? __brev(i) >> (32 - last_log) : 0u;
    v[j] = {last[i], last[n + i], last[2 * n + i], last[3 * n + i]};
  }
  uint32_t off = 0;
  for (uint32_t lg = last_log; lg >= 1; lg--) {
    const uint32_t sz = 1u << lg;
    for (uint32_t c0 = 0; c0 < n; c0 += sz)
      for (uint32_t i = 0; i < sz / 2; i++) {
        const qm31 l = v[c0 + i], r = v[c0 + i + sz / 2];
        v[c0 + i] = qm31_add(l, r);
        v[c0 + i + sz / 2] = qm31_mul_m31(qm31_sub(l, r), xi[off + i]);
      }
    off += sz / 2;
  }
  for (uint32_t i = 0; i < n; i++) v[i] = qm31_mul_m31(v[i], n_inv);
  for (uint32_t i = 0; i < n; i++) {
    const uint32_t j = last_log ? __brev(i) >> (32 - last_log) : 0u;
    if (j > i) {
      const qm31 t = v[i];
      v[i] = v[j];
      v[j] = t;
    }
  }
  uint32_t bad = 0;
  for (uint32_t i = 1u << bound_log; i < n; i++) bad |= !qm31_eq(v[i], qm31_zero());
  // mix_felts on a copy of the digest: digest || a, b, c, d of each coefficient
  const uint32_t nb = 1u << bound_log, total = 8 + 4 * nb, blocks = (total + 15) / 16;
  auto word = [&](uint32_t w) -> uint32_t {
    if (w < 8) return ch->digest[w];
    if (w >= total) return 0u;
    const qm31 x = v[(w - 8) >> 2];
    const uint32_t k = (w - 8) & 3;
    return k == 0 ? x.a : k == 1 ? x.b : k == 2 ? x.c : x.d;
  };
  uint32_t h[8], m[16];
  blake2s_init(h);
  for (uint32_t bk = 0; bk < blocks; bk++) {
    for (int k = 0; k < 16; k++) m[k] = word(bk * 16 + k);
    const bool fin = bk + 1 == blocks;
    blake2s_compress_lat(h, m, fin ? 4 * total : 64 * (bk + 1), fin);
  }
  dev_finalize(h, ch->m31 != 0);
  m[0] = 0x12345678u;
  m[1] = m[2] = m[3] = 0;
  for (int k = 0; k < 8; k++) m[4 + k] = h[k];
  m[12] = pow_bits;
  m[13] = m[14] = m[15] = 0;
  uint32_t p[8];
  blake2s_init(p);
  blake2s_compress_lat(p, m, 52, true);
  dev_finalize(p, ch->m31 != 0);
  for (int k = 0; k < 8; k++) pow[k] = p[k];
  pow[8] = bad;
}
// grind_kernel with the prefixed digest read from device memory.
__global__ void grind_dev_kernel(const uint32_t* __restrict__ pre, uint32_t hi, uint32_t low_base, uint32_t bits,
                                 int m31, uint32_t* __restrict__ found) {
  uint32_t low = low_base + blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t m[16];
#pragma unroll
  for (int k = 0; k < 8; k++) m[k] = __ldg(pre + k);
  m[8] = low;
  m[9] = hi;
#pragma unroll
  for (int k = 10; k < 16; k++) m[k] = 0;
  uint32_t h[8];
  blake2s_init(h);
  blake2s_compress(h, m, 40, true);
  uint32_t w0 = m31 ? m31_reduce_u32(h[0]) : h[0];
  uint32_t tz = w0 == 0 ? 32u : (uint32_t)__ffs(w0) - 1;
  if (tz >= bits) atomicMin(found, low);
}

// The channel state in registers, for the one-CTA kernels that run several
// Fiat-Shamir steps: loaded once, where its latency overlaps the tree work,
// and stored once.  Same steps as dev_chan_mix_root / dev_chan_draw_felt.
struct ChanRegs {
  uint32_t digest[8];
  uint32_t n_draws, m31, error;
};
__device__ __forceinline__ void chan_load(const DevChannel* ch, ChanRegs& c) {
#pragma unroll
  for (int k = 0; k < 8; k++) c.digest[k] = ch->digest[k];
  c.n_draws = ch->n_draws;
  c.m31 = ch->m31;
  c.error = ch->error;
}
__device__ __forceinline__ void chan_store(DevChannel* ch, const ChanRegs& c) {
#pragma unroll
  for (int k = 0; k < 8; k++) ch->digest[k] = c.digest[k];
  ch->n_draws = c.n_draws;
  ch->error = c.error;
}
__device__ __forceinline__ void chan_mix_root(ChanRegs& c, const uint32_t root[8]) {
  uint32_t m[16], h[8];
#pragma unroll
  for (int k = 0; k < 8; k++) {
    m[k] = c.digest[k];
    m[8 + k] = root[k];
  }
  blake2s_init(h);
  blake2s_compress_lat(h, m, 64, true);
  dev_finalize(h, c.m31 != 0);
#pragma unroll
  for (int k = 0; k < 8; k++) c.digest[k] = h[k];
  c.n_draws = 0;
}
__device__ __forceinline__ qm31 chan_draw_felt(ChanRegs& c) {
  uint32_t m[16], h[8];
  for (int attempt = 0; attempt < 64; attempt++) {
#pragma unroll
    for (int k = 0; k < 8; k++) m[k] = c.digest[k];
    m[8] = c.n_draws;
#pragma unroll
    for (int k = 9; k < 16; k++) m[k] = 0;
    c.n_draws++;
    blake2s_init(h);
    blake2s_compress_lat(h, m, 37, true);
    dev_finalize(h, c.m31 != 0);
    bool okw = true;
#pragma unroll
    for (int k = 0; k < 8; k++) okw = okw && h[k] < 2 * M31_P;
    if (okw) return {m31_reduce_u32(h[0]), m31_reduce_u32(h[1]), m31_reduce_u32(h[2]), m31_reduce_u32(h[3])};
  }
  c.error = 1;
  return qm31_zero();
}

__device__ qm31 qm31_pow_u32(qm31 x, uint32_t e) {
  qm31 r = qm31_one();
  while (e) {
    if (e & 1) r = qm31_mul(r, x);
    x = qm31_mul(x, x);
    e >>= 1;
  }
  return r;
}

// ---- device-side Fiat-Shamir steps before the FRI commit ----
// Each mixes one commitment into the device channel, draws the next random
// value and derives what the following kernels read, so the prover enqueues
// the whole commit-to-FRI sequence without a host round trip.  The host
// replays the transcript from the downloaded roots and values afterwards.
// FsOut holds the drawn values for that replay.
struct FsOut {
  qm31 random_coeff;  // composition (prover/mod.rs:57-63)
  qm31 oods_t;        // OODS point parameter (core/circle.rs get_random_point)
  qm31 oods_x, oods_y;
  qm31 quotient_coeff;  // pcs/mod.rs:112
};

// Trace root -> composition random coefficient and its reversed powers
// pw[n_cons - 1 - k] = coeff^k.
__global__ void fs_composition_kernel(DevChannel* ch, const uint8_t* root, uint32_t n_cons, qm31* __restrict__ pw,
                                      FsOut* out) {
  __shared__ qm31 s_rc;
  if (threadIdx.x == 0) {
    dev_chan_mix_root(ch, reinterpret_cast<const uint32_t*>(root));
    s_rc = dev_chan_draw_felt(ch);
    out->random_coeff = s_rc;
  }
  __syncthreads();
  for (uint32_t k = threadIdx.x; k < n_cons; k += blockDim.x) pw[n_cons - 1 - k] = qm31_pow_u32(s_rc, k);
}

// Weight tables of oods_eval_kernel from the fold factors f[0..lg) (shared
// memory, written before a block barrier): w_lo[t] = prod over set bits b of t
// of f[b] (t < 2^h), w_hi[t] = prod over set bits b of t of f[h + b].  Built by
// doubling, one product per entry: entries [2^b, 2^(b+1)) are entries
// [0, 2^b) times f[b], a block barrier per bit.  The products are canonical
// field values, so the order of the factors does not change the words.  All
// threads of the block call it.
__device__ void build_eval_weights(const qm31* f, uint32_t lg, uint32_t h, qm31* __restrict__ w_lo,
                                   qm31* __restrict__ w_hi) {
  const uint32_t hi_bits = lg - h;
  if (threadIdx.x == 0) {
    w_lo[0] = qm31_one();
    w_hi[0] = qm31_one();
  }
  __syncthreads();
  const uint32_t rounds = h > hi_bits ? h : hi_bits;
  for (uint32_t b = 0; b < rounds; b++) {
    for (uint32_t t = threadIdx.x; t < (1u << b); t += blockDim.x) {
      if (b < h) w_lo[(1u << b) + t] = qm31_mul(w_lo[t], f[b]);
      if (b < hi_bits) w_hi[(1u << b) + t] = qm31_mul(w_hi[t], f[h + b]);
    }
    __syncthreads();
  }
}

// Composition root -> OODS point ((1 - t^2) / (1 + t^2), 2t / (1 + t^2)), its
// fold factors f = [y, x, pi(x), ...] and the weight tables of
// oods_eval_kernel (w_lo over f[0..h), w_hi over f[h..lg)).
__global__ void fs_oods_kernel(DevChannel* ch, const uint8_t* root, uint32_t lg, uint32_t h, qm31* __restrict__ w_lo,
                               qm31* __restrict__ w_hi, FsOut* out) {
  __shared__ qm31 f[32];
  if (threadIdx.x == 0) {
    dev_chan_mix_root(ch, reinterpret_cast<const uint32_t*>(root));
    const qm31 t = dev_chan_draw_felt(ch);
    const qm31 t2s = qm31_mul(t, t);
    const qm31 inv1 = qm31_inv(qm31_add(t2s, qm31_one()));
    const qm31 x = qm31_mul(qm31_add(qm31_one(), qm31_neg(t2s)), inv1);
    const qm31 y = qm31_mul(qm31_add(t, t), inv1);
    out->oods_t = t;
    out->oods_x = x;
    out->oods_y = y;
    f[0] = y;
    qm31 xx = x;
    for (uint32_t b = 1; b < lg; b++) {
      f[b] = xx;
      xx = qm31_double_x(xx);
    }
  }
  __syncthreads();
  build_eval_weights(f, lg, h, w_lo, w_hi);
}

// The weight tables of oods_eval_kernel for an explicit point z
// (PolyOps::batch_eval_at_point): f = [y, x, pi(x), ...] of z, then as above.
__global__ void eval_weights_kernel(spoint z, uint32_t lg, uint32_t h, qm31* __restrict__ w_lo,
                                    qm31* __restrict__ w_hi) {
  __shared__ qm31 f[32];
  if (threadIdx.x == 0) {
    f[0] = z.y;
    qm31 xx = z.x;
    for (uint32_t b = 1; b < lg; b++) {
      f[b] = xx;
      xx = qm31_double_x(xx);
    }
  }
  __syncthreads();
  build_eval_weights(f, lg, h, w_lo, w_hi);
}

int launch_eval_weights(const spoint& z, uint32_t lg, qm31* d_w_lo, qm31* d_w_hi, cudaStream_t s, char* err,
                        size_t err_len) {
  eval_weights_kernel<<<1, 1024, 0, s>>>(z, lg, poly_eval_lo_bits(lg), d_w_lo, d_w_hi);
  STWO_CHECK_LAUNCH();
  return STWO_B200_OK;
}


// Sampled values -> quotient random coefficient q, its powers ap[k] = q^k and
// the row constants (pcs/quotient_ops.rs:134-233 in the form of
// quotient4_kernel): c = conj(y) - y, A = sum q^k (conj(v_k) - v_k),
// B = sum q^k (v_k c - (conj(v_k) - v_k) y) over the nq sampled values.
constexpr int kFsThreads = 256;
__global__ void __launch_bounds__(kFsThreads) fs_quotient_kernel(DevChannel* ch, const qm31* __restrict__ vals,
                                                                 uint32_t nq, qm31* __restrict__ ap, QuotientDyn* dyn,
                                                                 FsOut* out) {
  __shared__ qm31 s_q;
  __shared__ qm31 sa[kFsThreads], sb[kFsThreads];
  __shared__ __align__(16) uint32_t s_words[kMixWordsCap];
  stage_mix_words(ch, vals, nq, s_words);
  __syncthreads();
  if (threadIdx.x == 0) {
    dev_chan_mix_staged(ch, s_words, nq);
    s_q = dev_chan_draw_felt(ch);
    out->quotient_coeff = s_q;
  }
  __syncthreads();
  const qm31 x = out->oods_x, y = out->oods_y;
  const qm31 cz = qm31_sub(qm31_conj(y), y);
  qm31 A = qm31_zero(), B = qm31_zero();
  for (uint32_t k = threadIdx.x; k < nq; k += blockDim.x) {
    const qm31 pk = qm31_pow_u32(s_q, k);
    const qm31 v = vals[k];
    const qm31 a = qm31_sub(qm31_conj(v), v);
    const qm31 b = qm31_sub(qm31_mul(v, cz), qm31_mul(a, y));
    A = qm31_add(A, qm31_mul(pk, a));
    B = qm31_add(B, qm31_mul(pk, b));
    ap[k] = pk;
  }
  sa[threadIdx.x] = A;
  sb[threadIdx.x] = B;
  __syncthreads();
  for (uint32_t o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      sa[threadIdx.x] = qm31_add(sa[threadIdx.x], sa[threadIdx.x + o]);
      sb[threadIdx.x] = qm31_add(sb[threadIdx.x], sb[threadIdx.x + o]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    QuotientDyn d;
    d.c = cz;
    d.A = sa[0];
    d.B = sb[0];
    d.prx = {x.a, x.b};
    d.pix = {x.c, x.d};
    d.pry = {y.a, y.b};
    d.piy = {y.c, y.d};
    *dyn = d;
  }
}

// Lifted leaf of one FRI layer element: Blake2s of its 4 coordinates (16
// bytes), the leaf of a tree over 4 equal-length columns
// (prover/backend/cpu/merkle_lifted.rs:44-78).
__device__ __forceinline__ void fri_leaf_store(uint8_t* leaves, uint64_t i, const qm31& v, bool m31) {
  uint32_t m[16];
  m[0] = v.a;
  m[1] = v.b;
  m[2] = v.c;
  m[3] = v.d;
#pragma unroll
  for (int k = 4; k < 16; k++) m[k] = 0;
  uint32_t h[8];
  blake2s_init(h);
  blake2s_compress(h, m, 16, true);
  dev_finalize(h, m31);
  uint4* g = reinterpret_cast<uint4*>(leaves + i * 32);
  g[0] = make_uint4(h[0], h[1], h[2], h[3]);
  g[1] = make_uint4(h[4], h[5], h[6], h[7]);
}

// Folds of more than 2^kFoldPairLog outputs take two outputs per thread (wide
// loads; several waves of blocks either way); smaller ones, which are on the
// latency-bound FRI chain, keep one output (and one leaf hash) per thread.
constexpr uint32_t kFoldPairLog = 16;
__host__ __device__ constexpr uint64_t fold_threads(uint32_t log_out) {
  return log_out > kFoldPairLog ? 1ull << (log_out - 1) : 1ull << log_out;
}

// fold_line with alpha read from device memory (prover/backend/cpu/fri.rs:67-92).
// When `leaves` is not null the fold also writes the leaf hashes of the next
// layer's tree (its Merkle leaf layer), saving a launch and a re-read.
__global__ void fold_line_dev_kernel(const uint32_t* __restrict__ in, uint32_t log_m, uint32_t fold_step,
                                     const qm31* __restrict__ d_alpha, const uint32_t* __restrict__ itw,
                                     uint64_t tw_len, uint32_t* __restrict__ out, uint8_t* __restrict__ leaves,
                                     int m31) {
  const uint64_t n_in = 1ull << log_m;
  const uint64_t n_out = n_in >> fold_step;
  qm31 a0 = *d_alpha;
  if (fold_step == 1 && log_m - 1 > kFoldPairLog && reinterpret_cast<uintptr_t>(in) % 16 == 0 &&
      reinterpret_cast<uintptr_t>(out) % 8 == 0) {
    // two outputs per thread: one 16-byte load per input coordinate, one
    // 8-byte twiddle load and one 8-byte store per output coordinate
    const uint32_t* lt = itw + (tw_len - (1ull << log_m));
    for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < (n_out >> 1);
         k += (uint64_t)gridDim.x * blockDim.x) {
      uint4 w[4];
#pragma unroll
      for (int c = 0; c < 4; c++) w[c] = __ldg(reinterpret_cast<const uint4*>(in + c * n_in) + k);
      const uint2 t = __ldg(reinterpret_cast<const uint2*>(lt) + k);
      const qm31 f0x{w[0].x, w[1].x, w[2].x, w[3].x}, f0n{w[0].y, w[1].y, w[2].y, w[3].y};
      const qm31 f1x{w[0].z, w[1].z, w[2].z, w[3].z}, f1n{w[0].w, w[1].w, w[2].w, w[3].w};
      const qm31 v0 = qm31_add(qm31_add(f0x, f0n), qm31_mul(a0, qm31_mul_m31(qm31_sub(f0x, f0n), t.x)));
      const qm31 v1 = qm31_add(qm31_add(f1x, f1n), qm31_mul(a0, qm31_mul_m31(qm31_sub(f1x, f1n), t.y)));
      reinterpret_cast<uint2*>(out)[k] = make_uint2(v0.a, v1.a);
      reinterpret_cast<uint2*>(out + n_out)[k] = make_uint2(v0.b, v1.b);
      reinterpret_cast<uint2*>(out + 2 * n_out)[k] = make_uint2(v0.c, v1.c);
      reinterpret_cast<uint2*>(out + 3 * n_out)[k] = make_uint2(v0.d, v1.d);
      if (leaves) {
        fri_leaf_store(leaves, 2 * k, v0, m31 != 0);
        fri_leaf_store(leaves, 2 * k + 1, v1, m31 != 0);
      }
    }
    return;
  }
  if (fold_step == 1) {
    const uint32_t* lt = itw + (tw_len - (1ull << log_m));
    for (uint64_t o = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; o < n_out;
         o += (uint64_t)gridDim.x * blockDim.x) {
      qm31 fx = {__ldg(in + 2 * o), __ldg(in + n_in + 2 * o), __ldg(in + 2 * n_in + 2 * o), __ldg(in + 3 * n_in + 2 * o)};
      qm31 fnx = {__ldg(in + 2 * o + 1), __ldg(in + n_in + 2 * o + 1), __ldg(in + 2 * n_in + 2 * o + 1),
                  __ldg(in + 3 * n_in + 2 * o + 1)};
      qm31 v = qm31_add(qm31_add(fx, fnx), qm31_mul(a0, qm31_mul_m31(qm31_sub(fx, fnx), __ldg(lt + o))));
      out[o] = v.a;
      out[n_out + o] = v.b;
      out[2 * n_out + o] = v.c;
      out[3 * n_out + o] = v.d;
      if (leaves) fri_leaf_store(leaves, o, v, m31 != 0);
    }
    return;
  }
  for (uint64_t o = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; o < n_out; o += (uint64_t)gridDim.x * blockDim.x) {
    qm31 v[1 << 6];
    const uint32_t w = 1u << fold_step;
    for (uint32_t j = 0; j < w; j++) {
      uint64_t i = o * w + j;
      v[j] = {__ldg(in + i), __ldg(in + n_in + i), __ldg(in + 2 * n_in + i), __ldg(in + 3 * n_in + i)};
    }
    qm31 a = a0;
    for (uint32_t st = 0; st < fold_step; st++) {
      const uint32_t* lt = itw + (tw_len - (1ull << (log_m - st)));
      uint32_t pairs = w >> (st + 1);
      for (uint32_t j = 0; j < pairs; j++) {
        qm31 fx = v[2 * j], fnx = v[2 * j + 1];
        qm31 f0 = qm31_add(fx, fnx);
        qm31 f1 = qm31_mul_m31(qm31_sub(fx, fnx), __ldg(lt + o * pairs + j));
        v[j] = qm31_add(f0, qm31_mul(a, f1));
      }
      a = qm31_mul(a, a);
    }
    out[o] = v[0].a;
    out[n_out + o] = v[0].b;
    out[2 * n_out + o] = v[0].c;
    out[3 * n_out + o] = v[0].d;
    if (leaves) fri_leaf_store(leaves, o, v[0], m31 != 0);
  }
}

// First FRI layer: dst = 0 * alpha^2 + fold(src) = fold(src) (prover/fri.rs:74-85
// with a zero line evaluation), alpha from device memory; log_n > 4.
struct Src4 {
  const uint32_t* c[4];  // the four coordinate columns
};
__global__ void fold_circle_first_dev_kernel(Src4 src, uint32_t log_n, const qm31* __restrict__ d_alpha,
                                             const uint32_t* __restrict__ itw, uint64_t tw_len,
                                             uint32_t* __restrict__ dst, uint8_t* __restrict__ leaves, int m31) {
  const uint64_t n_in = 1ull << log_n, n_out = n_in >> 1;
  const uint32_t* lt0 = itw + (tw_len - (1ull << (log_n - 1)));
  qm31 alpha = *d_alpha;
  bool vec = log_n - 1 > kFoldPairLog && reinterpret_cast<uintptr_t>(dst) % 8 == 0;
  for (int c = 0; c < 4; c++) vec = vec && reinterpret_cast<uintptr_t>(src.c[c]) % 16 == 0;
  if (vec) {
    // two outputs per thread: one 16-byte load per source coordinate, one
    // 8-byte store per output coordinate
    for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < (n_out >> 1);
         k += (uint64_t)gridDim.x * blockDim.x) {
      uint4 w[4];
#pragma unroll
      for (int c = 0; c < 4; c++) w[c] = __ldg(reinterpret_cast<const uint4*>(src.c[c]) + k);
      const uint32_t b = __ldg(lt0 + (k ^ 1));  // circle twiddles of outputs 2k, 2k + 1: [b, -b] or [-b, b]
      const uint32_t y0 = (k & 1) ? m31_neg(b) : b, y1 = (k & 1) ? b : m31_neg(b);
      const qm31 p0{w[0].x, w[1].x, w[2].x, w[3].x}, n0{w[0].y, w[1].y, w[2].y, w[3].y};
      const qm31 p1{w[0].z, w[1].z, w[2].z, w[3].z}, n1{w[0].w, w[1].w, w[2].w, w[3].w};
      const qm31 v0 = qm31_add(qm31_zero(), qm31_add(qm31_add(p0, n0), qm31_mul(alpha, qm31_mul_m31(qm31_sub(p0, n0), y0))));
      const qm31 v1 = qm31_add(qm31_zero(), qm31_add(qm31_add(p1, n1), qm31_mul(alpha, qm31_mul_m31(qm31_sub(p1, n1), y1))));
      reinterpret_cast<uint2*>(dst)[k] = make_uint2(v0.a, v1.a);
      reinterpret_cast<uint2*>(dst + n_out)[k] = make_uint2(v0.b, v1.b);
      reinterpret_cast<uint2*>(dst + 2 * n_out)[k] = make_uint2(v0.c, v1.c);
      reinterpret_cast<uint2*>(dst + 3 * n_out)[k] = make_uint2(v0.d, v1.d);
      if (leaves) {
        fri_leaf_store(leaves, 2 * k, v0, m31 != 0);
        fri_leaf_store(leaves, 2 * k + 1, v1, m31 != 0);
      }
    }
    return;
  }
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n_out; i += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t b = __ldg(lt0 + ((i >> 1) ^ 1));
    uint32_t yinv = ((i ^ (i >> 1)) & 1) ? m31_neg(b) : b;
    qm31 fp = {__ldg(src.c[0] + 2 * i), __ldg(src.c[1] + 2 * i), __ldg(src.c[2] + 2 * i), __ldg(src.c[3] + 2 * i)};
    qm31 fnp = {__ldg(src.c[0] + 2 * i + 1), __ldg(src.c[1] + 2 * i + 1), __ldg(src.c[2] + 2 * i + 1),
                __ldg(src.c[3] + 2 * i + 1)};
    qm31 f0 = qm31_add(fp, fnp);
    qm31 f1 = qm31_mul_m31(qm31_sub(fp, fnp), yinv);
    qm31 v = qm31_add(qm31_zero(), qm31_add(f0, qm31_mul(alpha, f1)));
    dst[i] = v.a;
    dst[n_out + i] = v.b;
    dst[2 * n_out + i] = v.c;
    dst[3 * n_out + i] = v.d;
    if (leaves) fri_leaf_store(leaves, i, v, m31 != 0);
  }
}

// ---- fused FRI tail ----
// The small FRI layers (log size <= kFriTailLog) are latency-bound: at most
// a few hundred compressions each, spread over leaf, node, channel and fold
// launches.  One CTA runs all of them back to back: per layer it hashes the
// lifted leaves (4 equal columns, prover/backend/cpu/merkle_lifted.rs:44-78),
// every node level to the root with the levels in shared memory (and in the
// tree buffer, for decommitment), mixes the root and draws alpha on the device
// channel, and folds into the next layer (prover/backend/cpu/fri.rs:67-92).
// Data written inside the kernel is read back with plain loads, never through
// the read-only path.  Layers up to log 9 (512 threads): one SM's hash
// throughput still keeps up there, while a log-10 layer already cost more in
// the one CTA than its separate grid launches.
constexpr uint32_t kFriTailLog = 9;
constexpr int kFriTailMaxLayers = 32;
constexpr int kFriTailThreads = 1 << kFriTailLog;  // one thread per leaf of the largest tail layer
constexpr size_t kFriTailSmem = (size_t)3 << (kFriTailLog + 4);  // 2^L + 2^(L-1) hashes of 32 bytes
struct FriTail {
  uint32_t* coords[kFriTailMaxLayers];  // 4 x 2^log_size
  uint8_t* tree[kFriTailMaxLayers];     // MerkleTree base: layer k at ((1 << k) - 1) * 32
  uint32_t log_size[kFriTailMaxLayers];
  uint32_t fold_step[kFriTailMaxLayers];
  uint32_t* last;  // destination of the last fold
  uint32_t n_layers;
  uint32_t m31;
};

__device__ __forceinline__ void put_hash(uint8_t* layer, uint4* smem, uint32_t i, const uint32_t h[8]) {
  const uint4 a = make_uint4(h[0], h[1], h[2], h[3]);
  const uint4 b = make_uint4(h[4], h[5], h[6], h[7]);
  uint4* g = reinterpret_cast<uint4*>(layer + (size_t)i * 32);
  g[0] = a;
  g[1] = b;
  smem[2 * i] = a;
  smem[2 * i + 1] = b;
}

// Node levels lg-1 .. 0 of a tree whose level lg (2^lg hashes) is in shared
// memory at `src`; every level also goes to the tree buffer.  Returns the
// buffer that holds the root.  Called by all threads of the block.
__device__ const uint4* tree_levels_smem(uint8_t* base, uint32_t lg, uint4* src, uint4* dst, bool m31) {
  for (int d = (int)lg - 1; d >= 0; d--) {
    const uint32_t np = 1u << d;
    for (uint32_t p = threadIdx.x; p < np; p += blockDim.x) {
      uint32_t m[16];
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const uint4 w = src[4 * p + q];
        m[4 * q] = w.x;
        m[4 * q + 1] = w.y;
        m[4 * q + 2] = w.z;
        m[4 * q + 3] = w.w;
      }
      uint32_t h[8];
      blake2s_init(h);
      blake2s_compress_lat(h, m, 64, true);
      dev_finalize(h, m31);
      put_hash(base + ((size_t)np - 1) * 32, dst, p, h);
    }
    __syncthreads();
    uint4* tmp = src;
    src = dst;
    dst = tmp;
  }
  return src;
}

// Top of one FRI layer tree and its Fiat-Shamir step: hashes levels
// top_log-1 .. 0 from tree level top_log (2^top_log hashes in global memory,
// top_log <= kFriTailLog), then mixes the root and draws alpha.
__global__ void __launch_bounds__(kFriTailThreads, 1) tree_top_channel_kernel(uint8_t* base, uint32_t top_log,
                                                                              DevChannel* ch, qm31* alpha,
                                                                              int m31) {
  extern __shared__ uint4 tail_smem[];
  uint4* ping = tail_smem;
  uint4* pong = tail_smem + (2u << kFriTailLog);
  const bool m31b = m31 != 0;
  const uint4* src = ping;
  ChanRegs cr;
  if (threadIdx.x == 0) chan_load(ch, cr);  // used after the tree levels
  if (top_log == 0) {
    if (threadIdx.x == 0) {
      const uint4* r = reinterpret_cast<const uint4*>(base);
      ping[0] = r[0];
      ping[1] = r[1];
    }
    __syncthreads();
  } else {
    const uint32_t np = 1u << (top_log - 1);
    const uint4* in = reinterpret_cast<const uint4*>(base + (((size_t)1 << top_log) - 1) * 32);
    for (uint32_t p = threadIdx.x; p < np; p += blockDim.x) {
      uint32_t m[16];
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const uint4 w = __ldg(in + 4 * p + q);
        m[4 * q] = w.x;
        m[4 * q + 1] = w.y;
        m[4 * q + 2] = w.z;
        m[4 * q + 3] = w.w;
      }
      uint32_t h[8];
      blake2s_init(h);
      blake2s_compress_lat(h, m, 64, true);
      dev_finalize(h, m31b);
      put_hash(base + ((size_t)np - 1) * 32, ping, p, h);
    }
    __syncthreads();
    src = tree_levels_smem(base, top_log - 1, ping, pong, m31b);
  }
  if (threadIdx.x == 0) {
    const uint4 a = src[0], b = src[1];
    const uint32_t root[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
    chan_mix_root(cr, root);
    *alpha = chan_draw_felt(cr);
    chan_store(ch, cr);
  }
}

__global__ void __launch_bounds__(kFriTailThreads, 1) fri_tail_kernel(FriTail t, DevChannel* ch, qm31* alphas,
                                                                      const uint32_t* __restrict__ itw,
                                                                      uint64_t tw_len) {
  extern __shared__ uint4 tail_smem[];  // ping: 2^kFriTailLog hashes, pong: 2^(kFriTailLog-1)
  __shared__ qm31 s_alpha;
  uint4* ping = tail_smem;
  uint4* pong = tail_smem + (2u << kFriTailLog);
  const uint32_t tid = threadIdx.x;
  const bool m31 = t.m31 != 0;
  ChanRegs cr;
  if (tid == 0) chan_load(ch, cr);
  for (uint32_t li = 0; li < t.n_layers; li++) {
    const uint32_t L = t.log_size[li];
    const uint32_t n = 1u << L;
    const uint32_t* c = t.coords[li];
    uint8_t* base = t.tree[li];
    for (uint32_t i = tid; i < n; i += kFriTailThreads) {
      uint32_t m[16];
      m[0] = c[i];
      m[1] = c[n + i];
      m[2] = c[2 * n + i];
      m[3] = c[3 * n + i];
#pragma unroll
      for (int k = 4; k < 16; k++) m[k] = 0;
      uint32_t h[8];
      blake2s_init(h);
      blake2s_compress_lat(h, m, 16, true);
      dev_finalize(h, m31);
      put_hash(base + ((size_t)n - 1) * 32, ping, i, h);
    }
    __syncthreads();
    const uint4* src = tree_levels_smem(base, L, ping, pong, m31);
    if (tid == 0) {
      const uint4 a = src[0], b = src[1];
      const uint32_t root[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
      chan_mix_root(cr, root);
      const qm31 alpha = chan_draw_felt(cr);
      alphas[li] = alpha;
      s_alpha = alpha;
      if (li + 1 == t.n_layers) chan_store(ch, cr);
    }
    __syncthreads();
    const qm31 a0 = s_alpha;
    const uint32_t fs = t.fold_step[li];
    const uint32_t n_out = n >> fs;
    uint32_t* out = li + 1 < t.n_layers ? t.coords[li + 1] : t.last;
    if (fs == 1) {
      const uint32_t* lt = itw + (tw_len - (1ull << L));
      for (uint32_t o = tid; o < n_out; o += kFriTailThreads) {
        const qm31 fx = {c[2 * o], c[n + 2 * o], c[2 * n + 2 * o], c[3 * n + 2 * o]};
        const qm31 fnx = {c[2 * o + 1], c[n + 2 * o + 1], c[2 * n + 2 * o + 1], c[3 * n + 2 * o + 1]};
        const qm31 v = qm31_add(qm31_add(fx, fnx), qm31_mul(a0, qm31_mul_m31(qm31_sub(fx, fnx), __ldg(lt + o))));
        out[o] = v.a;
        out[n_out + o] = v.b;
        out[2 * n_out + o] = v.c;
        out[3 * n_out + o] = v.d;
      }
    }
    for (uint32_t o = tid; fs > 1 && o < n_out; o += kFriTailThreads) {
      qm31 v[1 << 6];
      const uint32_t w = 1u << fs;
      for (uint32_t j = 0; j < w; j++) {
        const uint32_t i = o * w + j;
        v[j] = {c[i], c[n + i], c[2 * n + i], c[3 * n + i]};
      }
      qm31 a = a0;
      for (uint32_t st = 0; st < fs; st++) {
        const uint32_t* lt = itw + (tw_len - (1ull << (L - st)));
        const uint32_t pairs = w >> (st + 1);
        for (uint32_t j = 0; j < pairs; j++) {
          const qm31 fx = v[2 * j], fnx = v[2 * j + 1];
          const qm31 f0 = qm31_add(fx, fnx);
          const qm31 f1 = qm31_mul_m31(qm31_sub(fx, fnx), __ldg(lt + o * pairs + j));
          v[j] = qm31_add(f0, qm31_mul(a, f1));
        }
        a = qm31_mul(a, a);
      }
      out[o] = v[0].a;
      out[n_out + o] = v[0].b;
      out[2 * n_out + o] = v[0].c;
      out[3 * n_out + o] = v[0].d;
    }
    __syncthreads();
  }
}

// Persistent grid of the column-streaming kernels: as many blocks as are
// resident at once (occupancy of this kernel with its shared memory), never
// more blocks than tiles.
template <typename K>
static unsigned stream_grid(K kernel, size_t smem, uint32_t n_tiles) {
  int dev = 0, sms = 148, per_sm = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kStreamBlock, smem);
  const uint32_t resident = (uint32_t)std::max(1, sms) * (uint32_t)std::max(1, per_sm);
  return std::max(1u, std::min(n_tiles, resident));
}

static unsigned grid1d(uint64_t n, unsigned threads) {
  uint64_t b = (n + threads - 1) / threads;
  return (unsigned)std::min<uint64_t>(std::max<uint64_t>(b, 1), 148ull * 32);
}

// ------------------------------------------------------------- host side ----

struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
};

struct MerkleTree {  // lifted tree layers in one buffer, root first
  uint8_t* base = nullptr;
  uint32_t L = 0;
  uint8_t* layer(uint32_t k) const { return base + (((size_t)1 << k) - 1) * 32; }
  static size_t bytes_for(uint32_t L) { return (((size_t)2 << L) - 1) * 32; }
};

struct FriLayerBuf {
  uint32_t log_size;
  uint32_t* coords;  // 4 x 2^log_size
  MerkleTree tree;
  uint32_t fold_step;
};

struct GatherPlan {
  std::vector<uint64_t> addrs;
  size_t add_word(const void* p) {
    addrs.push_back(reinterpret_cast<uint64_t>(p));
    return addrs.size() - 1;
  }
  size_t add_hash(const uint8_t* p) {
    size_t first = addrs.size();
    for (int k = 0; k < 8; k++) addrs.push_back(reinterpret_cast<uint64_t>(p + 4 * k));
    return first;
  }
};

// Witness node (layer log, index) list of a lifted Merkle decommitment in
// proof order (prover/vcs_lifted/prover.rs:114-185), into `out`.  The level
// lists live in two per-thread buffers that keep their capacity between
// calls: a proof runs this for about two dozen trees of ~20 levels.
static void witness_nodes_into(const std::vector<size_t>& queries, uint32_t L,
                               std::vector<std::pair<uint32_t, size_t>>& out) {
  out.clear();
  thread_local std::vector<size_t> prev, cur;
  prev.assign(queries.begin(), queries.end());
  prev.erase(std::unique(prev.begin(), prev.end()), prev.end());
  for (uint32_t layer_log = L; layer_log-- > 0;) {
    cur.clear();
    for (size_t i = 0; i < prev.size();) {
      size_t first = prev[i];
      bool pair = (i + 1 < prev.size()) && ((first ^ 1) == prev[i + 1]);
      if (!pair) out.push_back({layer_log + 1, first ^ 1});
      cur.push_back(first >> 1);
      i += pair ? 2 : 1;
    }
    prev.swap(cur);
  }
}

static std::vector<std::pair<uint32_t, size_t>> witness_nodes(const std::vector<size_t>& queries, uint32_t L) {
  std::vector<std::pair<uint32_t, size_t>> out;
  witness_nodes_into(queries, L, out);
  return out;
}

// Decommitment plans of one proof: an FRI layer (positions of the folded
// subsets, their value and witness-node slots in the gather) and a trace
// tree (queried values column-major, witness nodes).
struct FriDecommit {
  std::vector<size_t> positions;  // subset positions
  std::vector<uint8_t> is_query;
  std::vector<size_t> value_slot;  // 4 words per position
  std::vector<std::pair<uint32_t, size_t>> nodes;
  std::vector<size_t> node_slot;
};
struct TreeDecommit {
  std::vector<size_t> value_slot;  // column-major: col * n_q + qi
  std::vector<std::pair<uint32_t, size_t>> nodes;
  std::vector<size_t> node_slot;
};

// Little-endian proof encoding: integers are appended as their in-memory
// bytes, which on this (little-endian) host are the little-endian bytes.
static_assert(__BYTE_ORDER__ == __ORDER_LITTLE_ENDIAN__, "the proof encoding copies little-endian integers");
struct ProofOut {
  std::vector<uint8_t> bytes;
  void raw(const void* p, size_t n) {
    const size_t at = bytes.size();
    bytes.resize(at + n);
    std::memcpy(bytes.data() + at, p, n);
  }
  void u32(uint32_t v) { raw(&v, 4); }
  void u64(uint64_t v) { raw(&v, 8); }
  void q(const qm31& x) {
    const uint32_t w[4] = {x.a, x.b, x.c, x.d};
    raw(w, 16);
  }
  void h(const uint8_t* p) { raw(p, 32); }
};

// Phases timed with CUDA events when timing is enabled
// (stwo_b200_prover_phase_times).
enum Phase {
  kTraceGen, kTraceInterpolate, kTraceEvaluate, kTraceMerkle, kComposition, kCompInterpolate, kCompEvaluate,
  kCompMerkle, kOodsSampling, kQuotients, kFriMerkle, kFriFold, kGrind, kDecommit, kNumPhases
};

class WideFibProver {
 public:
  bool timing = false;
  // Polls a consumer of the column-streaming kernels makes before a stage
  // wait gives up (stwo_b200_prover_set_stream_spin).
  uint32_t stream_spin = kStreamSpin;
  std::vector<cudaEvent_t> ev_pool;
  std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> marks;
  size_t ev_used = 0;
  double phase_ms[kNumPhases] = {0};
  uint32_t proofs_timed = 0;

  cudaEvent_t next_event() {
    if (ev_used == ev_pool.size()) {
      cudaEvent_t e;
      cudaEventCreate(&e);
      ev_pool.push_back(e);
    }
    return ev_pool[ev_used++];
  }
  // Opens phase `ph` at the current point of the stream; closes the previous.
  int open_phase = -1;
  cudaEvent_t open_event = nullptr;
  void phase(int ph) {
    if (!timing) return;
    if (capture_slot >= 0) {  // inside a graph capture: an event-record node
      cudaEvent_t e = graph_events[graph_ev_next++];
      cudaEventRecordWithFlags(e, s, cudaEventRecordExternal);
      graph_phase_seq[capture_slot].push_back({ph, e});
      return;
    }
    cudaEvent_t e = next_event();
    cudaEventRecord(e, s);
    apply_phase(ph, e);
  }
  void apply_phase(int ph, cudaEvent_t e) {
    if (open_phase >= 0) marks.push_back({open_phase, {open_event, e}});
    open_phase = ph;
    open_event = e;
  }
  void finish_timing() {
    if (!timing) return;
    phase(-1);
    cudaStreamSynchronize(s);
    for (auto& m : marks) {
      float ms = 0;
      cudaEventElapsedTime(&ms, m.second.first, m.second.second);
      phase_ms[m.first] += ms;
    }
    marks.clear();
    ev_used = 0;
    open_phase = -1;
    proofs_timed++;
  }
  stwo_b200_wide_fib_config cfg;
  uint32_t log_n = 0, N = 0, blowup = 0, eval_log = 0, L1 = 0, L2 = 0, lift = 0, tree_log = 0;
  cudaStream_t s = nullptr;  // the prover's own stream (none in measure mode)

  uint32_t *d_tw = nullptr, *d_itw = nullptr;
  uint32_t* d_coeffs = nullptr;   // N x 2^log_n (trace, then coefficients)
  uint32_t* d_evals = nullptr;    // N x 2^L1
  uint32_t* d_ext = nullptr;      // N x 2^eval_log when eval_log != L1
  MerkleTree t1, t2, tq;
  uint32_t* d_comp = nullptr;     // 4 x 2^eval_log (evals, then coefficients)
  uint32_t* d_comp_lde = nullptr; // 8 x 2^L2
  uint32_t* d_quot = nullptr;     // 4 x 2^lift
  std::vector<FriLayerBuf> fri;   // inner layers
  uint32_t* d_last = nullptr;     // 4 x 2^last_log
  // Device finish of the FRI commit (fri_finish_kernel) for last layers of up
  // to kFinishMaxLast values: its proof-of-work prefix and flag, and the
  // inverse x-coordinates of the last layer's line IFFT.
  bool dev_finish = false;
  uint32_t* d_pow = nullptr;
  uint32_t* d_last_xi = nullptr;
  uint32_t last_n_inv = 0;
  qm31* d_small = nullptr;        // powers / weights / partials / alpha powers
  uint32_t* d_denom = nullptr;
  FsOut* d_fs = nullptr;         // values drawn by the device Fiat-Shamir steps
  QuotientDyn* d_qdyn = nullptr;  // per-proof quotient row constants
  uint32_t* d_found = nullptr;
  DevChannel* d_chan = nullptr;
  qm31* d_alphas = nullptr;       // folding alphas of the FRI layers
  uint64_t* d_gather_addr = nullptr;
  uint32_t* d_gather_out = nullptr;
  size_t gather_cap = 0;
  size_t last_proof_bytes = 1u << 16;  // capacity reserved for the next proof's bytes
  // host decommitment plan, reused from proof to proof
  GatherPlan gplan;
  std::vector<FriDecommit> fri_dec_buf;
  TreeDecommit td_buf[2];
  std::vector<size_t> lq_buf, nq_buf, tq_buf;
  std::vector<uint32_t> words_buf;
  qm31* d_oods_partial = nullptr;  // OODS partial sums (polynomials x chunks)
  qm31* h_pinned = nullptr;       // staging for small uploads / downloads
  DevChannel* h_chan = nullptr;   // staging of the device channel state (own region: the
                                  // quotient upload from h_pinned may still be in flight)
  size_t h_pinned_bytes = 0;
  uint8_t* h_tx = nullptr;          // pre-FRI transcript download: roots 1-2, FsOut, sampled values
  size_t h_tx_bytes = 0;
  cudaEvent_t ev_tx = nullptr;      // recorded after that download
  std::vector<void*> allocs;

  // The prover enqueues on its own non-blocking stream `s` (so the FRI commit
  // can be a captured CUDA graph), ordered after and before the caller's
  // stream `user_s` with events.
  cudaStream_t user_s = nullptr;
  cudaEvent_t ev_in = nullptr, ev_out = nullptr;
  // Host-input proofs: the two input columns are copied in kHostChunks row
  // chunks on the copy stream `cs` into d_in (allocated on first use), and
  // each chunk's trace rows are generated as soon as it lands.  Four chunks:
  // with sixteen the per-copy overhead outweighed the overlap.
  static constexpr uint32_t kHostChunks = 4;
  uint32_t* d_in = nullptr;
  cudaStream_t cs = nullptr;
  cudaEvent_t ev_chunk[kHostChunks] = {};
  const uint32_t* h_src_a = nullptr;  // set for the duration of a host-input proof
  const uint32_t* h_src_b = nullptr;
  // FRI commit graphs, [timing off, timing on], captured on first use.
  cudaGraphExec_t fri_exec[2] = {nullptr, nullptr};
  uint64_t fri_graph_launches[2] = {0, 0};
  std::vector<std::pair<int, cudaEvent_t>> graph_phase_seq[2];
  std::vector<cudaEvent_t> graph_events;  // created before a capture, owned
  size_t graph_ev_next = 0;
  int capture_slot = -1;

  ~WideFibProver() {
    if (s) cudaStreamSynchronize(s);
    for (int k = 0; k < 2; k++)
      if (fri_exec[k]) cudaGraphExecDestroy(fri_exec[k]);
    for (cudaEvent_t e : graph_events) cudaEventDestroy(e);
    if (ev_in) cudaEventDestroy(ev_in);
    if (ev_out) cudaEventDestroy(ev_out);
    if (ev_tx) cudaEventDestroy(ev_tx);
    for (cudaEvent_t e : ev_chunk)
      if (e) cudaEventDestroy(e);
    if (cs) {
      cudaStreamSynchronize(cs);
      cudaStreamDestroy(cs);
    }
    for (cudaEvent_t e : ev_pool) cudaEventDestroy(e);
    for (void* p : allocs) cudaFree(p);  // empty in measure mode
    if (h_pinned) cudaFreeHost(h_pinned);
    if (h_tx) cudaFreeHost(h_tx);
    if (h_chan) cudaFreeHost(h_chan);
    if (s) cudaStreamDestroy(s);
  }

  // measure: run init's allocation arithmetic only (no device work), for the
  // footprint query; allocated_bytes sums every device allocation.
  bool measure = false;
  size_t allocated_bytes = 0;
  uint32_t N_cap = 0;  // columns the buffers hold; a proof may use 3..N_cap

  int alloc(void** p, size_t bytes, char* err, size_t err_len) {
    allocated_bytes += std::max<size_t>(bytes, 16);
    if (measure) {
      *p = reinterpret_cast<void*>(uintptr_t{256});  // never dereferenced
      return 0;
    }
    STWO_CUDA_TRY(cudaMalloc(p, std::max<size_t>(bytes, 16)));
    allocs.push_back(*p);
    return 0;
  }

  int init(const stwo_b200_wide_fib_config& c, cudaStream_t stream, char* err, size_t err_len) {
    cfg = c;
    user_s = stream;
    if (!measure) {
      STWO_CUDA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
      STWO_CUDA_TRY(cudaEventCreateWithFlags(&ev_in, cudaEventDisableTiming));
      STWO_CUDA_TRY(cudaEventCreateWithFlags(&ev_out, cudaEventDisableTiming));
      STWO_CUDA_TRY(cudaEventCreateWithFlags(&ev_tx, cudaEventDisableTiming));
      STWO_CUDA_TRY(
          cudaFuncSetAttribute(fri_tail_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kFriTailSmem));
      STWO_CUDA_TRY(cudaFuncSetAttribute(tree_top_channel_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)kFriTailSmem));
      STWO_CUDA_TRY(
          cudaFuncSetAttribute(composition_tma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kStreamSmem));
      STWO_CUDA_TRY(
          cudaFuncSetAttribute(quotient_tma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kStreamSmem));
    }
    log_n = c.log_n_rows;
    N = N_cap = c.n_cols;
    blowup = c.log_blowup;
    STWO_ARG_CHECK(N >= 3 && N <= kMaxPolys - 8, "n_cols %u out of range [3, %d]", N, kMaxPolys - 8);
    STWO_ARG_CHECK(log_n >= 4 && log_n + blowup <= 28, "log_n_rows %u / log_blowup %u out of range", log_n, blowup);
    STWO_ARG_CHECK(blowup >= 1 && blowup <= 16, "log_blowup %u out of range", blowup);
    STWO_ARG_CHECK(c.line_fold_step >= 1 && c.line_fold_step <= 6, "line_fold_step %u unsupported", c.line_fold_step);
    STWO_ARG_CHECK(c.pow_bits <= 32, "pow_bits > 32 is not supported");
    STWO_ARG_CHECK(c.n_queries >= 1 && c.n_queries <= 4096, "n_queries %u out of range", c.n_queries);
    STWO_ARG_CHECK(c.log_last_layer_degree_bound <= 10, "log_last_layer_degree_bound out of range");
    eval_log = log_n + 1;           // max_constraint_log_degree_bound of Wide-Fibonacci
    L1 = log_n + blowup;            // trace tree
    L2 = eval_log - 1 + blowup;     // composition tree (lifting size)
    lift = L2;
    STWO_ARG_CHECK(L1 <= lift, "trace tree larger than the lifting domain");
    STWO_ARG_CHECK(lift - 1 >= c.log_last_layer_degree_bound + blowup, "domain too small for the FRI config");
    tree_log = log_n + blowup;      // twiddles of CanonicCoset(log_n + 1 + blowup).half_coset
    int rc;
    if ((rc = alloc((void**)&d_tw, 4ull << tree_log, err, err_len))) return rc;
    if ((rc = alloc((void**)&d_itw, 4ull << tree_log, err, err_len))) return rc;
    // CanonicCoset(tree_log + 1).half_coset = half_odds(tree_log): initial index 2^(31 - (tree_log + 2)).
    if (!measure) {
      rc = stwo_b200_precompute_twiddles(1ull << (31 - (tree_log + 2)), tree_log, d_tw, d_itw, s, err, err_len);
      if (rc) return rc;
    }
    if ((rc = alloc((void**)&d_coeffs, (4ull * N) << log_n, err, err_len))) return rc;
    if ((rc = alloc((void**)&d_evals, (4ull * N) << L1, err, err_len))) return rc;
    if (eval_log != L1 && (rc = alloc((void**)&d_ext, (4ull * N) << eval_log, err, err_len))) return rc;
    t1.L = L1;
    if ((rc = alloc((void**)&t1.base, MerkleTree::bytes_for(L1), err, err_len))) return rc;
    t2.L = L2;
    if ((rc = alloc((void**)&t2.base, MerkleTree::bytes_for(L2), err, err_len))) return rc;
    tq.L = lift;
    if ((rc = alloc((void**)&tq.base, MerkleTree::bytes_for(lift), err, err_len))) return rc;
    if ((rc = alloc((void**)&d_comp, 16ull << eval_log, err, err_len))) return rc;
    if ((rc = alloc((void**)&d_comp_lde, 32ull << L2, err, err_len))) return rc;
    if ((rc = alloc((void**)&d_quot, 16ull << lift, err, err_len))) return rc;
    // FRI inner layers (prover/fri.rs:188-262).
    uint32_t last_log = c.log_last_layer_degree_bound + blowup;
    uint32_t cur = lift - 1;
    if (cur != last_log) {
      while (cur > last_log + c.line_fold_step) {
        fri.push_back({cur, nullptr, {}, c.line_fold_step});
        cur -= c.line_fold_step;
      }
      fri.push_back({cur, nullptr, {}, cur - last_log});
      cur = last_log;
    }
    // the first inner layer receives the circle fold; the others the line folds
    for (auto& l : fri) {
      if ((rc = alloc((void**)&l.coords, 16ull << l.log_size, err, err_len))) return rc;
      l.tree.L = l.log_size;
      if ((rc = alloc((void**)&l.tree.base, MerkleTree::bytes_for(l.log_size), err, err_len))) return rc;
    }
    if ((rc = alloc((void**)&d_last, 16ull << last_log, err, err_len))) return rc;
    dev_finish = (1u << last_log) <= kFinishMaxLast;
    if ((rc = alloc((void**)&d_pow, 64, err, err_len))) return rc;
    if ((rc = alloc((void**)&d_last_xi, 4u << last_log, err, err_len))) return rc;
    size_t small_q = std::max<size_t>(4096, 2 * (1u << 12) + (size_t)kMaxPolys * 1024);
    if ((rc = alloc((void**)&d_small, small_q * sizeof(qm31), err, err_len))) return rc;
    // OODS partial sums: one per (polynomial, 1024-index chunk)
    const size_t oods_chunks = log_n > 10 ? (size_t)1 << (log_n - 10) : 1;
    if ((rc = alloc((void**)&d_oods_partial, (size_t)(N + 8) * oods_chunks * sizeof(qm31), err, err_len))) return rc;
    if ((rc = alloc((void**)&d_denom, 4ull << (eval_log - log_n), err, err_len))) return rc;
    if ((rc = alloc((void**)&d_found, 64, err, err_len))) return rc;
    if ((rc = alloc((void**)&d_chan, sizeof(DevChannel), err, err_len))) return rc;
    if ((rc = alloc((void**)&d_alphas, (fri.size() + 2) * sizeof(qm31), err, err_len))) return rc;
    if ((rc = alloc((void**)&d_fs, sizeof(FsOut), err, err_len))) return rc;
    if ((rc = alloc((void**)&d_qdyn, sizeof(QuotientDyn), err, err_len))) return rc;
    h_pinned_bytes = std::max<size_t>(small_q * sizeof(qm31), (16ull << last_log) + 65536);
    if (measure) return 0;
    STWO_CUDA_TRY(cudaMallocHost((void**)&h_pinned, h_pinned_bytes));
    STWO_CUDA_TRY(cudaMallocHost((void**)&h_chan, sizeof(DevChannel)));
    h_tx_bytes = 64 + sizeof(FsOut) + (size_t)(N + 8) * sizeof(qm31) + 16;  // + the stream error word
    STWO_CUDA_TRY(cudaMallocHost((void**)&h_tx, h_tx_bytes));
    {
      // Vanishing inverses of the 2^(eval_log - log_n) trace-coset classes,
      // bit-reversed (a function of the sizes only).
      const uint32_t log_expand = eval_log - log_n;
      uint32_t* dn = reinterpret_cast<uint32_t*>(h_pinned);
      for (uint32_t j = 0; j < (1u << log_expand); j++) {
        // eval_domain.at(j): half coset of CanonicCoset(eval_log)
        uint64_t init = 1ull << (31 - (eval_log + 1)), step = 1ull << (31 - (eval_log - 1));
        uint64_t half = 1ull << (eval_log - 1);
        uint64_t idx =
            j < half ? (init + step * j) : ((1ull << 31) - ((init + step * (j - half)) & ((1ull << 31) - 1)));
        cpoint p = index_to_cpoint(idx);
        // coset_vanishing(CanonicCoset(log_n).coset, p) (core/constraints.rs:12-34)
        uint64_t cinit = 1ull << (31 - (log_n + 1)), cstep = 1ull << (31 - log_n);
        cpoint ci = index_to_cpoint(cinit);
        cpoint sh = cpoint_add(cpoint_add(p, cpoint{ci.x, m31_neg(ci.y)}), index_to_cpoint(cstep >> 1));
        uint32_t x = sh.x;
        for (uint32_t i = 1; i < log_n; i++) x = m31_sub(m31_add(m31_sqr(x), m31_sqr(x)), 1);
        dn[bitrev32(j, log_expand)] = m31_inv(x);
      }
      STWO_CUDA_TRY(cudaMemcpyAsync(d_denom, dn, 4ull << log_expand, cudaMemcpyHostToDevice, s));
    }
    if (dev_finish) {
      // The inverse x-coordinates of the last layer's line IFFT, in the order
      // the host interpolation after the FRI commit walks them (line domain:
      // the half coset of CanonicCoset(lift) doubled down to last_log).
      const uint32_t last_log = c.log_last_layer_degree_bound + blowup;
      uint32_t* xi = reinterpret_cast<uint32_t*>(h_pinned) + 4096;
      uint64_t dinit = (1ull << (31 - (lift + 1))) << (lift - 1 - last_log);
      uint64_t dstep = 1ull << (31 - last_log);
      uint32_t off = 0;
      for (uint32_t lg = last_log; lg >= 1; lg--) {
        for (uint64_t i = 0; i < (1ull << (lg - 1)); i++) xi[off + i] = m31_inv(index_to_cpoint(dinit + dstep * i).x);
        off += 1u << (lg - 1);
        dinit = (dinit * 2) & ((1ull << 31) - 1);
        dstep = (dstep * 2) & ((1ull << 31) - 1);
      }
      last_n_inv = m31_inv(m31_reduce_u32(1u << last_log));
      if (off) STWO_CUDA_TRY(cudaMemcpyAsync(d_last_xi, xi, 4ull * off, cudaMemcpyHostToDevice, s));
    }
    STWO_CUDA_TRY(cudaStreamSynchronize(s));
    return 0;
  }

  int ensure_gather(size_t n, char* err, size_t err_len) {
    if (n <= gather_cap) return 0;
    int rc;
    size_t cap = std::max<size_t>(n, 4096);
    if ((rc = alloc((void**)&d_gather_addr, cap * 8, err, err_len))) return rc;
    if ((rc = alloc((void**)&d_gather_out, cap * 4, err, err_len))) return rc;
    gather_cap = cap;
    return 0;
  }

  // One FRI layer tree from its leaf level L: grid-wide node launches down to
  // 2^kFriTailLog hashes, then one CTA for the top levels (latency-bound, a
  // few hundred compressions), the root mix and the alpha draw on the device
  // channel.
  int fri_tree_top(const MerkleTree& t, uint32_t L, qm31* alpha, char* err, size_t err_len) {
    const uint32_t top = std::min<uint32_t>(L, kFriTailLog);
    if (L > top) {
      std::vector<uint8_t*> outs(L);
      for (uint32_t k = 0; k < L; k++) outs[k] = t.layer(k);
      int rc = build_node_layers_impl(t.layer(L), L, top, cfg.m31_channel, outs.data(), s, err, err_len);
      if (rc) return rc;
    }
    tree_top_channel_kernel<<<1, kFriTailThreads, kFriTailSmem, s>>>(t.base, top, d_chan, alpha, cfg.m31_channel);
    STWO_CHECK_LAUNCH();
    return 0;
  }

  // FRI commit (prover/fri.rs:133-291) on the device channel: the circle
  // layer tree, the first fold, every line layer's tree top, alpha draw and
  // fold, then the fused tail.  Launch parameters depend only on the
  // configuration and the buffers allocated at init, so the sequence is
  // captured once as a CUDA graph and replayed.
  int enqueue_fri(char* err, size_t err_len) {
    const bool m31 = cfg.m31_channel != 0;
    int rc;
    {
      std::vector<uint32_t*> q4(4);
      for (int k = 0; k < 4; k++) q4[k] = d_quot + ((uint64_t)k << lift);
      phase(kFriMerkle);
      if ((rc = build_leaves_impl(q4.data(), std::vector<uint32_t>(4, lift).data(), 4, lift, m31, tq.layer(lift),
                                  nullptr, s, err, err_len)))
        return rc;
      if ((rc = fri_tree_top(tq, lift, d_alphas, err, err_len))) return rc;
    }
    size_t tail0 = fri.size();  // first layer of the fused tail
    while (tail0 > 0 && fri[tail0 - 1].log_size <= kFriTailLog) tail0--;
    {
      phase(kFriFold);
      uint32_t* dst = fri.empty() ? d_last : fri[0].coords;
      uint8_t* leaves = tail0 > 0 ? fri[0].tree.layer(fri[0].log_size) : nullptr;
      if (lift <= 4) return set_err(err, err_len, STWO_B200_EARG, "lifting domain too small");
      const Src4 q4{{d_quot, d_quot + (1ull << lift), d_quot + (2ull << lift), d_quot + (3ull << lift)}};
      fold_circle_first_dev_kernel<<<grid1d(fold_threads(lift - 1), 256), 256, 0, s>>>(
          q4, lift, d_alphas, d_itw, 1ull << tree_log, dst, leaves, m31 ? 1 : 0);
      STWO_CHECK_LAUNCH();
    }
    for (size_t li = 0; li < tail0; li++) {
      FriLayerBuf& l = fri[li];
      phase(kFriMerkle);  // leaves were hashed by the fold that produced this layer
      if ((rc = fri_tree_top(l.tree, l.log_size, d_alphas + li + 1, err, err_len))) return rc;
      phase(kFriFold);
      uint32_t* nxt = (li + 1 < fri.size()) ? fri[li + 1].coords : d_last;
      uint8_t* leaves = li + 1 < tail0 ? fri[li + 1].tree.layer(fri[li + 1].log_size) : nullptr;
      uint32_t nlog = l.log_size - l.fold_step;
      const uint64_t threads = l.fold_step == 1 ? fold_threads(nlog) : 1ull << nlog;
      fold_line_dev_kernel<<<grid1d(threads, 256), 256, 0, s>>>(l.coords, l.log_size, l.fold_step,
                                                                       d_alphas + li + 1, d_itw, 1ull << tree_log, nxt,
                                                                       leaves, m31 ? 1 : 0);
      STWO_CHECK_LAUNCH();
    }
    if (tail0 < fri.size()) {
      phase(kFriMerkle);
      FriTail t;
      t.n_layers = (uint32_t)(fri.size() - tail0);
      STWO_ARG_CHECK(t.n_layers <= (uint32_t)kFriTailMaxLayers, "too many FRI layers");
      for (uint32_t k = 0; k < t.n_layers; k++) {
        const FriLayerBuf& l = fri[tail0 + k];
        t.coords[k] = l.coords;
        t.tree[k] = l.tree.base;
        t.log_size[k] = l.log_size;
        t.fold_step[k] = l.fold_step;
      }
      t.last = d_last;
      t.m31 = m31 ? 1u : 0u;
      fri_tail_kernel<<<1, kFriTailThreads, kFriTailSmem, s>>>(t, d_chan, d_alphas + tail0 + 1, d_itw, 1ull << tree_log);
      STWO_CHECK_LAUNCH();
    }
    return 0;
  }

  int run_fri(char* err, size_t err_len) {
    const int k = timing ? 1 : 0;
    if (!fri_exec[k]) {
      const uint64_t before = g_kernel_launches.load();
      graph_phase_seq[k].clear();
      if (timing) {
        const size_t need = graph_ev_next + 2 * fri.size() + 8;  // phase() calls in enqueue_fri
        while (graph_events.size() < need) {
          cudaEvent_t e;
          STWO_CUDA_TRY(cudaEventCreate(&e));
          graph_events.push_back(e);
        }
      }
      STWO_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
      capture_slot = k;
      int rc = enqueue_fri(err, err_len);
      capture_slot = -1;
      cudaGraph_t g = nullptr;
      cudaError_t ce = cudaStreamEndCapture(s, &g);
      const uint64_t n = g_kernel_launches.load() - before;
      g_kernel_launches.fetch_sub(n);  // nothing ran during capture
      if (rc) {
        if (g) cudaGraphDestroy(g);
        return rc;
      }
      if (ce != cudaSuccess) return set_err(err, err_len, STWO_B200_ECUDA, "FRI graph capture: %s", cudaGetErrorString(ce));
      ce = cudaGraphInstantiate(&fri_exec[k], g, 0);
      cudaGraphDestroy(g);
      if (ce != cudaSuccess) {
        fri_exec[k] = nullptr;
        return set_err(err, err_len, STWO_B200_ECUDA, "FRI graph instantiate: %s", cudaGetErrorString(ce));
      }
      fri_graph_launches[k] = n;
    }
    STWO_CUDA_TRY(cudaGraphLaunch(fri_exec[k], s));
    g_kernel_launches.fetch_add(fri_graph_launches[k]);
    if (timing)
      for (auto& pe : graph_phase_seq[k]) apply_phase(pe.first, pe.second);
    return 0;
  }

  int download_root(const MerkleTree& t, Hash32& root, char* err, size_t err_len) {
    STWO_CUDA_TRY(cudaMemcpyAsync(h_pinned, t.layer(0), 32, cudaMemcpyDeviceToHost, s));
    STWO_CUDA_TRY(cudaStreamSynchronize(s));
    std::memcpy(root.data(), h_pinned, 32);
    return 0;
  }

  int commit_columns(uint32_t* const* cols, const std::vector<uint32_t>& logs, MerkleTree& t, char* err,
                     size_t err_len) {
    std::vector<uint8_t*> layers(t.L + 1);
    for (uint32_t k = 0; k <= t.L; k++) layers[k] = t.layer(k);
    return stwo_b200_merkle_build_layers(const_cast<const uint32_t* const*>(cols), logs.data(), (uint32_t)logs.size(),
                                         t.L, cfg.m31_channel, layers.data(), s, err, err_len);
  }

  int prove(const uint32_t* d_a, const uint32_t* d_b, ProofOut& out, char* err, size_t err_len,
            uint32_t n_cols = 0) {
    STWO_ARG_CHECK(n_cols == 0 || (n_cols >= 3 && n_cols <= N_cap), "n_cols %u out of range [3, %u]", n_cols, N_cap);
    N = n_cols ? n_cols : N_cap;
    STWO_CUDA_TRY(cudaEventRecord(ev_in, user_s));
    STWO_CUDA_TRY(cudaStreamWaitEvent(s, ev_in, 0));
    const int rc = prove_body(d_a, d_b, out, err, err_len);
    cudaEventRecord(ev_out, s);
    cudaStreamWaitEvent(user_s, ev_out, 0);
    return rc;
  }
  // The same proof from host input columns (pinned memory overlaps the copy
  // with the trace generation; pageable memory works, copied synchronously).
  int prove_host(const uint32_t* h_a, const uint32_t* h_b, ProofOut& out, char* err, size_t err_len) {
    const uint64_t rows = 1ull << log_n;
    if (!d_in) {
      int rc;
      if ((rc = alloc((void**)&d_in, 8ull << log_n, err, err_len))) return rc;
      STWO_CUDA_TRY(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
      for (cudaEvent_t& e : ev_chunk) STWO_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    h_src_a = h_a;
    h_src_b = h_b;
    const int rc = prove(d_in, d_in + rows, out, err, err_len);
    h_src_a = h_src_b = nullptr;
    return rc;
  }
  int prove_body(const uint32_t* d_a, const uint32_t* d_b, ProofOut& out, char* err, size_t err_len);
};

int WideFibProver::prove_body(const uint32_t* d_a, const uint32_t* d_b, ProofOut& out, char* err, size_t err_len) {
  const bool m31 = cfg.m31_channel != 0;
  HostChannel ch(m31);
  int rc;
  const uint64_t rows = 1ull << log_n;
  STWO_CUDA_TRY(cudaMemsetAsync(d_found + kStreamErrWord, 0, 4, s));
  // ---- tree 0: empty preprocessed trace -> Blake2s("") ----
  Hash32 root0;
  {
    HostBlake2s e;
    root0 = e.finalize(m31);
  }
  ch.mix_root(root0);
  // The device channel carries the transcript from here to the end of the
  // FRI commit; the host replays it after one download.
  {
    DevChannel* hc = h_chan;
    std::memset(hc, 0, sizeof(DevChannel));
    std::memcpy(hc->digest, ch.digest().data(), 32);
    hc->n_draws = ch.n_draws();
    hc->m31 = m31 ? 1 : 0;
    STWO_CUDA_TRY(cudaMemcpyAsync(d_chan, hc, sizeof(DevChannel), cudaMemcpyHostToDevice, s));
  }

  // ---- tree 1: trace ----
  std::vector<uint32_t*> coeff_ptrs(N), eval_ptrs(N);
  std::vector<uint32_t> logs_n(N, log_n), logs_1(N, L1);
  for (uint32_t c = 0; c < N; c++) {
    coeff_ptrs[c] = d_coeffs + (uint64_t)c * rows;
    eval_ptrs[c] = d_evals + ((uint64_t)c << L1);
  }
  // With host inputs and a split interpolation, the first pass runs chunk by
  // chunk as each chunk's trace rows are generated (its tiles are
  // consecutive rows), under the copies of the later chunks.
  const std::vector<uint32_t> ifft_split = fft_split(log_n);
  const bool chunked_ifft = h_src_a && ifft_split.size() >= 2 && ((rows / kHostChunks) >> ifft_split[0]) >= 1 &&
                            (rows / kHostChunks) % (1ull << ifft_split[0]) == 0;
  phase(kTraceGen);
  if (h_src_a) {
    // Host inputs: chunk k's copies (copy stream, ordered after the caller's
    // stream) gate chunk k's trace rows on the prover's stream.
    const uint64_t chunk = rows / kHostChunks;  // rows >= 16
    STWO_CUDA_TRY(cudaStreamWaitEvent(cs, ev_in, 0));
    for (uint32_t k = 0; k < kHostChunks; k++) {
      const uint64_t off = k * chunk;
      STWO_CUDA_TRY(cudaMemcpyAsync(const_cast<uint32_t*>(d_a) + off, h_src_a + off, 4 * chunk, cudaMemcpyHostToDevice,
                                    cs));
      STWO_CUDA_TRY(cudaMemcpyAsync(const_cast<uint32_t*>(d_b) + off, h_src_b + off, 4 * chunk, cudaMemcpyHostToDevice,
                                    cs));
      STWO_CUDA_TRY(cudaEventRecord(ev_chunk[k], cs));
      STWO_CUDA_TRY(cudaStreamWaitEvent(s, ev_chunk[k], 0));
      wide_fib_trace_kernel<<<grid1d(chunk, 256), 256, 0, s>>>(d_a + off, d_b + off, d_coeffs + off, N, chunk, rows);
      STWO_CHECK_LAUNCH();
      if (chunked_ifft && (rc = interpolate_pass(coeff_ptrs.data(), N, log_n, ifft_split, 0, off, off + chunk, d_itw,
                                                 tree_log, s, err, err_len)))
        return rc;
    }
  } else {
    wide_fib_trace_kernel<<<grid1d(rows, 256), 256, 0, s>>>(d_a, d_b, d_coeffs, N, rows, rows);
    STWO_CHECK_LAUNCH();
  }
  // Interpolation passes before the last (the first one already ran per
  // chunk when chunked); the last one runs with the evaluation, fused with its
  // first pass where the split allows (interpolate_evaluate).
  const uint32_t n_ifft = (uint32_t)ifft_split.size();
  phase(kTraceInterpolate);
  for (uint32_t pi = chunked_ifft ? 1 : 0; pi + 1 < n_ifft; pi++)
    if ((rc = interpolate_pass(coeff_ptrs.data(), N, log_n, ifft_split, pi, 0, rows, d_itw, tree_log, s, err,
                               err_len)))
      return rc;
  phase(kTraceEvaluate);
  if ((rc = interpolate_evaluate(coeff_ptrs.data(), eval_ptrs.data(), N, log_n, blowup, ifft_split, n_ifft - 1, d_itw,
                                 d_tw, tree_log, s, err, err_len)))
    return rc;
  phase(kTraceMerkle);
  if ((rc = commit_columns(eval_ptrs.data(), logs_1, t1, err, err_len))) return rc;
  // ---- composition (prover/mod.rs:57-77) ----
  const uint32_t n_cons = N - 2;
  phase(kComposition);
  fs_composition_kernel<<<1, 128, 0, s>>>(d_chan, t1.layer(0), n_cons, d_small, d_fs);
  STWO_CHECK_LAUNCH();
  const uint32_t* comp_src = d_evals;
  uint64_t comp_stride = 1ull << L1;
  if (eval_log != L1) {
    std::vector<uint32_t*> ext_ptrs(N);
    for (uint32_t c = 0; c < N; c++) ext_ptrs[c] = d_ext + ((uint64_t)c << eval_log);
    if ((rc = stwo_b200_evaluate_polynomials(const_cast<const uint32_t* const*>(coeff_ptrs.data()), logs_n.data(), N,
                                             eval_log - log_n, ext_ptrs.data(), d_tw, tree_log, s, err, err_len)))
      return rc;
    comp_src = d_ext;
    comp_stride = 1ull << eval_log;
  }
  const uint64_t n_eval = 1ull << eval_log;
  if (n_eval % kStreamRows == 0 && n_cons <= kStreamMaxW && comp_stride % 4 == 0 &&
      reinterpret_cast<uintptr_t>(comp_src) % 16 == 0)
    composition_tma_kernel<<<stream_grid(composition_tma_kernel, kStreamRing + n_cons * sizeof(uint4),
                                         (uint32_t)(n_eval / kStreamRows)),
                             kStreamBlock, kStreamRing + n_cons * sizeof(uint4), s>>>(
        comp_src, comp_stride, n_cons, d_small, d_denom, log_n, n_eval, d_comp, d_found + kStreamErrWord,
        stream_spin);
  else if (n_eval % 4 == 0 && comp_stride % 4 == 0 && reinterpret_cast<uintptr_t>(comp_src) % 16 == 0)
    composition4_kernel<<<grid1d(n_eval / 4, 256), 256, 0, s>>>(comp_src, comp_stride, n_cons, d_small, d_denom,
                                                                log_n, n_eval, d_comp);
  else  // the prover's own buffers are pool-allocated (256-byte aligned) and log_n >= 4
    return set_err(err, err_len, STWO_B200_ESTATE, "composition: unaligned evaluation buffer");
  STWO_CHECK_LAUNCH();
  std::vector<uint32_t*> comp_cols(4);
  std::vector<uint32_t> logs_e(4, eval_log);
  for (int k = 0; k < 4; k++) comp_cols[k] = d_comp + ((uint64_t)k << eval_log);
  phase(kCompInterpolate);
  if ((rc = stwo_b200_interpolate_columns(comp_cols.data(), logs_e.data(), nullptr, 4, d_itw, tree_log, s, err,
                                          err_len)))
    return rc;
  phase(kCompEvaluate);
  // split_at_mid (natural coefficient order): left = first half, right = second half.
  std::vector<uint32_t*> split(8), lde(8);
  std::vector<uint32_t> logs_h(8, eval_log - 1), logs_2(8, L2);
  for (int k = 0; k < 4; k++) {
    split[k] = comp_cols[k];
    split[4 + k] = comp_cols[k] + (n_eval >> 1);
  }
  for (int k = 0; k < 8; k++) lde[k] = d_comp_lde + ((uint64_t)k << L2);
  if ((rc = stwo_b200_evaluate_polynomials(const_cast<const uint32_t* const*>(split.data()), logs_h.data(), 8, blowup,
                                           lde.data(), d_tw, tree_log, s, err, err_len)))
    return rc;
  phase(kCompMerkle);
  if ((rc = commit_columns(lde.data(), logs_2, t2, err, err_len))) return rc;

  // ---- OODS point and sampled values (prover/mod.rs:80-119, pcs/mod.rs:512-689) ----
  const uint32_t max_log_degree_bound = lift - blowup;
  const uint32_t np = N + 8;
  qm31* d_vals = nullptr;
  {
    // Every column is committed at the lifting size, so all 108 polynomials
    // (log_n coefficients each) are sampled at the OODS point itself.
    STWO_ARG_CHECK(L1 == lift && eval_log - 1 == log_n, "sampling assumes one column size");
    STWO_ARG_CHECK(log_n <= 31, "log size too large for the fold factors");
    const uint32_t lg = log_n, h = poly_eval_lo_bits(lg);
    size_t n_w = (1u << h) + (1u << (lg - h));
    phase(kOodsSampling);
    fs_oods_kernel<<<1, 1024, 0, s>>>(d_chan, t2.layer(0), lg, h, d_small, d_small + (1u << h), d_fs);
    STWO_CHECK_LAUNCH();
    std::vector<const uint32_t*> polys(coeff_ptrs.begin(), coeff_ptrs.begin() + N);
    for (int k = 0; k < 8; k++) polys.push_back(split[k]);
    d_vals = d_small + n_w;
    if ((rc = launch_poly_eval(polys.data(), np, lg, d_small, d_small + (1u << h), d_oods_partial, d_vals, s, err,
                               err_len)))
      return rc;
  }

  // ---- FRI quotients (pcs/mod.rs:112-118, quotient_ops.rs:134-233) ----
  {
    const uint32_t nq = np;
    QuotientParams qp;
    phase(kQuotients);
    qm31* d_ap = d_vals + np;  // after the sampled values, which the host downloads later
    fs_quotient_kernel<<<1, kFsThreads, 0, s>>>(d_chan, d_vals, nq, d_ap, d_qdyn, d_fs);
    STWO_CHECK_LAUNCH();
    qp.log_size = lift;
    qp.init = index_to_cpoint(1ull << (31 - (lift + 1)));
    cpoint st = index_to_cpoint(1ull << (31 - (lift - 1)));
    for (int b = 0; b < 31; b++) {
      qp.step_pow[b] = st;
      st = cpoint_add(st, st);
    }
    PolyTable cols;
    for (uint32_t c = 0; c < N; c++) cols.p[c] = eval_ptrs[c];
    for (int k = 0; k < 8; k++) cols.p[N + k] = lde[k];
    bool aligned = lift >= 2;
    for (uint32_t c = 0; c < nq; c++) aligned = aligned && reinterpret_cast<uintptr_t>(cols.p[c]) % 16 == 0;
    if (aligned && lift >= (uint32_t)kStreamTileBits + 1 && nq <= kStreamMaxW) {
      cpoint g = qp.step_pow[lift - kStreamTileBits], acc = {1, 0};
      for (int m = 0; m < kStreamRows / 4; m++) {
        qp.tile_pts[m] = acc;
        acc = cpoint_add(acc, g);
      }
      quotient_tma_kernel<<<stream_grid(quotient_tma_kernel, kStreamRing + nq * sizeof(uint4),
                                        (uint32_t)((1ull << lift) / kStreamRows)),
                            kStreamBlock, kStreamRing + nq * sizeof(uint4), s>>>(
          qp, cols, nq, d_ap, d_qdyn, d_quot, d_found + kStreamErrWord, stream_spin);
    } else if (aligned) {
      quotient4_kernel<<<grid1d(1ull << (lift - 2), 256), 256, 0, s>>>(qp, cols, nq, d_ap, d_qdyn, d_quot);
    } else {  // pool-allocated columns are 256-byte aligned and lift >= 5
      return set_err(err, err_len, STWO_B200_ESTATE, "quotients: unaligned column buffer");
    }
    STWO_CHECK_LAUNCH();
  }

  // ---- FRI commit (prover/fri.rs:133-291) ----
  // The layer loop runs on the device: commit, mix root / draw alpha on the
  // device channel, fold.  The host replays the transcript afterwards from the
  // downloaded roots and checks the device alphas against its own.
  std::vector<Hash32> fri_roots(1 + fri.size());
  const uint32_t last_log = cfg.log_last_layer_degree_bound + blowup;
  // Download of the pre-FRI transcript values, so that the host replays
  // them while the device runs the FRI commit.
  STWO_CUDA_TRY(cudaMemcpyAsync(h_tx, t1.layer(0), 32, cudaMemcpyDeviceToHost, s));
  STWO_CUDA_TRY(cudaMemcpyAsync(h_tx + 32, t2.layer(0), 32, cudaMemcpyDeviceToHost, s));
  STWO_CUDA_TRY(cudaMemcpyAsync(h_tx + 64, d_fs, sizeof(FsOut), cudaMemcpyDeviceToHost, s));
  STWO_CUDA_TRY(cudaMemcpyAsync(h_tx + 64 + sizeof(FsOut), d_vals, np * sizeof(qm31), cudaMemcpyDeviceToHost, s));
  const size_t tx_flag_off = 64 + sizeof(FsOut) + np * sizeof(qm31);
  STWO_CUDA_TRY(cudaMemcpyAsync(h_tx + tx_flag_off, d_found + kStreamErrWord, 4, cudaMemcpyDeviceToHost, s));
  STWO_CUDA_TRY(cudaEventRecord(ev_tx, s));
  if ((rc = run_fri(err, err_len))) return rc;
  if (dev_finish) {
    // the last layer, the proof-of-work prefix and the first grind batch,
    // queued behind the FRI commit; the host checks the prefix against its
    // own and continues the search from the second batch when this one
    // finds no nonce
    fri_finish_kernel<<<1, 32, 0, s>>>(d_chan, d_last, last_log, cfg.log_last_layer_degree_bound, d_last_xi,
                                       last_n_inv, cfg.pow_bits, d_pow);
    STWO_CHECK_LAUNCH();
    STWO_CUDA_TRY(cudaMemsetAsync(d_found, 0xFF, 4, s));
    grind_dev_kernel<<<kGrindBatch / 256, 256, 0, s>>>(d_pow, 0, 0, cfg.pow_bits, m31, d_found);
    STWO_CHECK_LAUNCH();
  }
  Hash32 root1, root2;
  std::vector<qm31> sampled(np);
  {
    STWO_CUDA_TRY(cudaEventSynchronize(ev_tx));
    FsOut fs;
    std::memcpy(root1.data(), h_tx, 32);
    std::memcpy(root2.data(), h_tx + 32, 32);
    std::memcpy(&fs, h_tx + 64, sizeof(FsOut));
    std::memcpy(sampled.data(), h_tx + 64 + sizeof(FsOut), np * sizeof(qm31));
    auto fail = [&](int code, const char* what) {
      cudaStreamSynchronize(s);
      return set_err(err, err_len, code, "%s", what);
    };
    // A timed-out composition stream leaves partial rows behind: report it
    // before any check of the values built on them.
    if (*reinterpret_cast<const uint32_t*>(h_tx + tx_flag_off))
      return fail(STWO_B200_ETIMEOUT, "column stream: a bulk copy did not complete in time");
    ch.mix_root(root1);
    const qm31 random_coeff = ch.draw_secure_felt();
    if (!qm31_eq(random_coeff, fs.random_coeff))
      return fail(STWO_B200_ESTATE, "device and host channels diverged at the composition coefficient");
    ch.mix_root(root2);
    spoint oods;
    {
      const qm31 t = ch.draw_secure_felt();
      const qm31 t2s = qm31_mul(t, t);
      const qm31 inv1 = qm31_inv(qm31_add(t2s, qm31_one()));
      oods = {qm31_mul(qm31_add(qm31_one(), qm31_neg(t2s)), inv1), qm31_mul(qm31_add(t, t), inv1)};
      if (!qm31_eq(t, fs.oods_t) || !qm31_eq(oods.x, fs.oods_x) || !qm31_eq(oods.y, fs.oods_y))
        return fail(STWO_B200_ESTATE, "device and host channels diverged at the OODS point");
    }
    ch.mix_felts(sampled.data(), sampled.size());
    if (!qm31_eq(ch.draw_secure_felt(), fs.quotient_coeff))
      return fail(STWO_B200_ESTATE, "device and host channels diverged at the quotient coefficient");
    // Sanity check (prover/mod.rs:123-138): the composition value rebuilt
    // from the split halves equals the constraint quotient at the OODS point.
    {
      const qm31 basis[4] = {qm31_one(), {0, 1, 0, 0}, {0, 0, 1, 0}, {0, 0, 0, 1}};
      qm31 left = qm31_zero(), right = qm31_zero();
      for (int k = 0; k < 4; k++) {
        left = qm31_add(left, qm31_mul(sampled[N + k], basis[k]));
        right = qm31_add(right, qm31_mul(sampled[N + 4 + k], basis[k]));
      }
      qm31 comp = qm31_add(left, qm31_mul(spoint_repeated_double(oods, max_log_degree_bound - 1).x, right));
      // coset_vanishing(CanonicCoset(max_log_degree_bound).coset, oods)
      uint64_t cinit = 1ull << (31 - (max_log_degree_bound + 1)), cstep = 1ull << (31 - max_log_degree_bound);
      cpoint ci = index_to_cpoint(cinit), hs = index_to_cpoint(cstep >> 1);
      spoint sp = spoint_add(spoint_add(oods, {qm31_from_m31(ci.x), qm31_from_m31(m31_neg(ci.y))}),
                             {qm31_from_m31(hs.x), qm31_from_m31(hs.y)});
      qm31 vx = sp.x;
      for (uint32_t i = 1; i < max_log_degree_bound; i++) vx = qm31_double_x(vx);
      qm31 dinv = qm31_inv(vx);
      qm31 acc = qm31_zero();
      for (uint32_t k = 0; k < n_cons; k++) {
        qm31 a = sampled[k], b = sampled[k + 1], c = sampled[k + 2];
        qm31 cons = qm31_sub(c, qm31_add(qm31_mul(a, a), qm31_mul(b, b)));
        acc = qm31_add(qm31_mul(acc, random_coeff), qm31_mul(cons, dinv));
      }
      if (!qm31_eq(acc, comp))
        return fail(STWO_B200_ESTATE, "ConstraintsNotSatisfied: composition OODS mismatch");
    }
  }
  // One download after the FRI commit: roots, device alphas, channel state,
  // error flags and the last layer.  The host continues from the device
  // channel's state (last layer, proof of work) and replays the transcript
  // to check the device alphas while the first grind batch runs.
  const uint64_t n_last = 1ull << last_log;
  HostChannel dev_ch(m31);
  const uint8_t* hp = reinterpret_cast<const uint8_t*>(h_pinned);
  size_t alpha_off = 0, chan_off = 0, flag_off = 0, last_off = 0, pow_off = 0;
  uint32_t fri_end_digest[8];
  uint32_t fri_end_draws = 0;
  std::vector<qm31> dev_alphas;
  {
    uint8_t* hpw = reinterpret_cast<uint8_t*>(h_pinned);
    size_t off = 0;
    STWO_CUDA_TRY(cudaMemcpyAsync(hpw + off, tq.layer(0), 32, cudaMemcpyDeviceToHost, s));
    off += 32;
    for (auto& l : fri) {
      STWO_CUDA_TRY(cudaMemcpyAsync(hpw + off, l.tree.layer(0), 32, cudaMemcpyDeviceToHost, s));
      off += 32;
    }
    alpha_off = off;
    STWO_CUDA_TRY(cudaMemcpyAsync(hpw + off, d_alphas, (fri.size() + 1) * sizeof(qm31), cudaMemcpyDeviceToHost, s));
    off += (fri.size() + 1) * sizeof(qm31);
    chan_off = off;
    STWO_CUDA_TRY(cudaMemcpyAsync(hpw + off, d_chan, sizeof(DevChannel), cudaMemcpyDeviceToHost, s));
    off += sizeof(DevChannel);
    flag_off = off;
    STWO_CUDA_TRY(cudaMemcpyAsync(hpw + off, d_found + kStreamErrWord, 4, cudaMemcpyDeviceToHost, s));
    off += 16;
    if (dev_finish) {
      pow_off = off;
      STWO_CUDA_TRY(cudaMemcpyAsync(hpw + off, d_pow, 36, cudaMemcpyDeviceToHost, s));
      STWO_CUDA_TRY(cudaMemcpyAsync(hpw + off + 48, d_found, 4, cudaMemcpyDeviceToHost, s));
      off += 64;
    }
    last_off = off;
    STWO_ARG_CHECK(off + 16 * n_last <= h_pinned_bytes, "pinned staging too small for the last layer");
    STWO_CUDA_TRY(cudaMemcpyAsync(hpw + off, d_last, 16 * n_last, cudaMemcpyDeviceToHost, s));
    STWO_CUDA_TRY(cudaStreamSynchronize(s));
    const DevChannel* dc = reinterpret_cast<const DevChannel*>(hp + chan_off);
    // A timed-out stream leaves the transcript built on partial rows, so its
    // flag is reported first.
    if (*reinterpret_cast<const uint32_t*>(hp + flag_off))
      return set_err(err, err_len, STWO_B200_ETIMEOUT, "column stream: a bulk copy did not complete in time");
    if (dc->error) return set_err(err, err_len, STWO_B200_ESTATE, "device channel: draw retry bound exhausted");
    dev_ch.set_state(dc->digest, dc->n_draws);
    std::memcpy(fri_end_digest, dc->digest, 32);
    fri_end_draws = dc->n_draws;
    for (size_t i = 0; i < fri_roots.size(); i++) std::memcpy(fri_roots[i].data(), hp + 32 * i, 32);
    dev_alphas.resize(fri_roots.size());
    std::memcpy(dev_alphas.data(), hp + alpha_off, fri_roots.size() * sizeof(qm31));
  }
  // Last layer (prover/fri.rs:274-291).
  std::vector<qm31> last_coeffs;
  {
    const uint32_t* hv = reinterpret_cast<const uint32_t*>(hp + last_off);
    std::vector<qm31> v(n_last);
    for (uint64_t i = 0; i < n_last; i++) v[i] = {hv[i], hv[n_last + i], hv[2 * n_last + i], hv[3 * n_last + i]};
    // LineEvaluation::interpolate (prover/line.rs:54-99): bit-reverse, line IFFT, 1/n.
    for (uint64_t i = 0; i < n_last; i++) {
      uint64_t j = bitrev32((uint32_t)i, last_log);
      if (j > i) std::swap(v[i], v[j]);
    }
    // line domain: half coset of CanonicCoset(lift) doubled down to last_log
    uint64_t dinit = (1ull << (31 - (lift + 1))) << (lift - 1 - last_log);
    uint64_t dstep = 1ull << (31 - last_log);
    for (uint32_t lg = last_log; lg >= 1; lg--) {
      uint64_t sz = 1ull << lg;
      for (uint64_t c0 = 0; c0 < n_last; c0 += sz)
        for (uint64_t i = 0; i < sz / 2; i++) {
          uint32_t xi = m31_inv(index_to_cpoint(dinit + dstep * i).x);
          qm31 l = v[c0 + i], r = v[c0 + i + sz / 2];
          v[c0 + i] = qm31_add(l, r);
          v[c0 + i + sz / 2] = qm31_mul_m31(qm31_sub(l, r), xi);
        }
      dinit = (dinit * 2) & ((1ull << 31) - 1);
      dstep = (dstep * 2) & ((1ull << 31) - 1);
    }
    uint32_t ninv = m31_inv(m31_reduce_u32((uint32_t)n_last));
    for (auto& x : v) x = qm31_mul_m31(x, ninv);
    for (uint64_t i = 0; i < n_last; i++) {  // into ordered coefficients
      uint64_t j = bitrev32((uint32_t)i, last_log);
      if (j > i) std::swap(v[i], v[j]);
    }
    size_t bound = 1ull << cfg.log_last_layer_degree_bound;
    for (size_t i = bound; i < v.size(); i++)
      if (!qm31_eq(v[i], qm31_zero())) return set_err(err, err_len, STWO_B200_ESTATE, "invalid degree");
    v.resize(bound);
    last_coeffs = v;
    dev_ch.mix_felts(last_coeffs.data(), last_coeffs.size());
  }

  // ---- proof of work (pcs/mod.rs:140-142) ----
  uint64_t nonce = 0;
  phase(kGrind);
  // Host replay of the FRI transcript: every device alpha and the channel
  // state at the end of the commit.  It runs while the first host-launched
  // grind batch runs or, when the device's batch found the nonce, while the
  // decommit gather runs.
  bool replayed = false;
  auto replay_fri = [&]() -> int {
    replayed = true;
    for (size_t i = 0; i < fri_roots.size(); i++) {
      ch.mix_root(fri_roots[i]);
      if (!qm31_eq(ch.draw_secure_felt(), dev_alphas[i])) {
        cudaStreamSynchronize(s);
        return set_err(err, err_len, STWO_B200_ESTATE, "device and host channels diverged at FRI layer %zu", i);
      }
    }
    if (std::memcmp(ch.digest().data(), fri_end_digest, 32) != 0 || ch.n_draws() != fri_end_draws) {
      cudaStreamSynchronize(s);
      return set_err(err, err_len, STWO_B200_ESTATE, "device and host channel states differ after FRI");
    }
    return 0;
  };
  {
    Hash32 pre = dev_ch.pow_prefixed(cfg.pow_bits);
    Digest8 d;
    std::memcpy(d.w, pre.data(), 32);
    bool found = false;
    uint32_t base0 = 0;
    if (dev_finish) {
      // the device's prefix and first batch (fri_finish_kernel, grind_dev_kernel)
      const uint32_t* pw = reinterpret_cast<const uint32_t*>(hp + pow_off);
      if (std::memcmp(pw, pre.data(), 32) != 0)
        return set_err(err, err_len, STWO_B200_ESTATE, "device and host channels diverged at the proof of work");
      if (pw[12] != 0xFFFFFFFFu) {
        nonce = pw[12];
        found = true;
      } else {
        base0 = kGrindBatch;
      }
    }
    for (uint32_t hi = 0; !found; hi++) {
      for (uint32_t base = hi == 0 ? base0 : 0; base < (1u << 20) && !found; base += kGrindBatch) {
        STWO_CUDA_TRY(cudaMemsetAsync(d_found, 0xFF, 4, s));
        if ((rc = launch_grind(d.w, hi, base, kGrindBatch, cfg.pow_bits, m31, d_found, s, err, err_len))) return rc;
        uint32_t* hf = reinterpret_cast<uint32_t*>(h_pinned) + (h_pinned_bytes / 4 - 1);
        STWO_CUDA_TRY(cudaMemcpyAsync(hf, d_found, 4, cudaMemcpyDeviceToHost, s));
        if (!replayed && (rc = replay_fri())) return rc;
        STWO_CUDA_TRY(cudaStreamSynchronize(s));
        if (*hf != 0xFFFFFFFFu) {
          nonce = ((uint64_t)hi << 32) | *hf;
          found = true;
        }
      }
      if (hi == 0x7ffffffeu && !found) return set_err(err, err_len, STWO_B200_ESTATE, "grind found no nonce");
    }
  }
  dev_ch.mix_u64(nonce);

  // ---- queries (core/queries.rs:11-58) ----
  std::vector<size_t> queries;
  {
    size_t mask = ((size_t)1 << lift) - 1;
    while (queries.size() < cfg.n_queries) {
      auto w = dev_ch.draw_u32s();
      for (uint32_t x : w)
        if (queries.size() < cfg.n_queries) queries.push_back(x & mask);
    }
    std::sort(queries.begin(), queries.end());
    queries.erase(std::unique(queries.begin(), queries.end()), queries.end());
  }

  // ---- decommitments: one gather of every needed word ----
  phase(kDecommit);
  // The plan's vectors are prover members, cleared here: they keep their
  // capacity from one proof to the next.
  GatherPlan& g = gplan;
  g.addrs.clear();
  auto plan_fri = [&](FriDecommit& d, const uint32_t* coords, uint32_t log_size, const MerkleTree& tree,
                      const std::vector<size_t>& q, uint32_t fold_step) {
    d.positions.clear();
    d.is_query.clear();
    d.value_slot.clear();
    d.node_slot.clear();
    for (size_t i = 0; i < q.size();) {
      size_t j = i;
      while (j < q.size() && (q[j] >> fold_step) == (q[i] >> fold_step)) j++;
      size_t start = (q[i] >> fold_step) << fold_step;
      size_t k = i;
      for (size_t pos = start; pos < start + ((size_t)1 << fold_step); pos++) {
        bool isq = k < j && q[k] == pos;
        if (isq) k++;
        d.positions.push_back(pos);
        d.is_query.push_back(isq ? 1 : 0);
        size_t slot = g.add_word(coords + pos);
        for (int c = 1; c < 4; c++) g.add_word(coords + ((uint64_t)c << log_size) + pos);
        d.value_slot.push_back(slot);
      }
      i = j;
    }
    witness_nodes_into(d.positions, tree.L, d.nodes);
    for (auto& nd : d.nodes) d.node_slot.push_back(g.add_hash(tree.layer(nd.first) + nd.second * 32));
  };
  std::vector<FriDecommit>& fri_dec = fri_dec_buf;
  fri_dec.resize(fri.size() + 1);
  plan_fri(fri_dec[0], d_quot, lift, tq, queries, 1);
  {
    std::vector<size_t>& lq = lq_buf;
    std::vector<size_t>& nq = nq_buf;
    lq.clear();
    for (size_t q : queries)
      if (lq.empty() || lq.back() != (q >> 1)) lq.push_back(q >> 1);
    for (size_t li = 0; li < fri.size(); li++) {
      const auto& l = fri[li];
      plan_fri(fri_dec[li + 1], l.coords, l.log_size, l.tree, lq, l.fold_step);
      nq.clear();
      for (size_t q : lq)
        if (nq.empty() || nq.back() != (q >> l.fold_step)) nq.push_back(q >> l.fold_step);
      lq.swap(nq);
    }
  }
  // trees 1 and 2 at the lifting size: queried values and witness nodes
  auto plan_tree = [&](TreeDecommit& d, const std::vector<uint32_t*>& cols, uint32_t log_size,
                       const MerkleTree& tree) {
    d.value_slot.clear();
    d.node_slot.clear();
    // prepare_query_positions_for_tree (core/pcs/utils.rs:195-213) and the
    // lifted read index (prover/vcs_lifted/prover.rs:83-109)
    std::vector<size_t>& tqs = tq_buf;
    tqs.clear();
    for (size_t p : queries) tqs.push_back(((p >> (lift - tree.L + 1)) << 1) + (p & 1));
    const size_t shift = tree.L - log_size;
    for (size_t c = 0; c < cols.size(); c++)
      for (size_t p : tqs) d.value_slot.push_back(g.add_word(cols[c] + (((p >> (shift + 1)) << 1) + (p & 1))));
    witness_nodes_into(tqs, tree.L, d.nodes);
    for (auto& nd : d.nodes) d.node_slot.push_back(g.add_hash(tree.layer(nd.first) + nd.second * 32));
  };
  TreeDecommit& td1 = td_buf[0];
  TreeDecommit& td2 = td_buf[1];
  plan_tree(td1, eval_ptrs, L1, t1);
  plan_tree(td2, lde, L2, t2);
  if ((rc = ensure_gather(g.addrs.size(), err, err_len))) return rc;
  {
    size_t n = g.addrs.size();
    std::vector<uint32_t>& words = words_buf;
    words.resize(n);
    // upload addresses through the pinned staging buffer in chunks
    size_t chunk = h_pinned_bytes / 8;
    for (size_t off = 0; off < n; off += chunk) {
      size_t m = std::min(chunk, n - off);
      std::memcpy(h_pinned, g.addrs.data() + off, m * 8);
      STWO_CUDA_TRY(cudaMemcpyAsync(d_gather_addr + off, h_pinned, m * 8, cudaMemcpyHostToDevice, s));
      // the staging buffer is reused by the next chunk only; the gather and
      // the download below are ordered after the upload on the stream
      if (off + m < n) STWO_CUDA_TRY(cudaStreamSynchronize(s));
    }
    gather_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(d_gather_addr, (uint32_t)n, d_gather_out);
    STWO_CHECK_LAUNCH();
    if (!replayed && (rc = replay_fri())) return rc;
    size_t wchunk = h_pinned_bytes / 4;
    for (size_t off = 0; off < n; off += wchunk) {
      size_t m = std::min(wchunk, n - off);
      STWO_CUDA_TRY(cudaMemcpyAsync(h_pinned, d_gather_out + off, m * 4, cudaMemcpyDeviceToHost, s));
      STWO_CUDA_TRY(cudaStreamSynchronize(s));
      std::memcpy(words.data() + off, h_pinned, m * 4);
    }
    // ---- serialize (canonical layout, struct field order of
    // core/pcs/quotients.rs:27-35 and core/fri.rs:361-395) ----
    auto hash_at = [&](size_t slot, ProofOut& o) { o.h(reinterpret_cast<const uint8_t*>(words.data() + slot)); };
    const char magic[8] = {'S', 'T', 'W', 'O', 'P', 'R', 'F', '1'};
    if (out.bytes.capacity() < last_proof_bytes) out.bytes.reserve(last_proof_bytes);
    out.bytes.assign(magic, magic + 8);
    out.u32(cfg.pow_bits);
    out.u32(cfg.log_blowup);
    out.u32(cfg.log_last_layer_degree_bound);
    out.u64(cfg.n_queries);
    out.u32(cfg.line_fold_step);
    out.bytes.push_back(0);  // lifting_log_size: None
    out.u64(3);
    out.h(root0.data());
    out.h(root1.data());
    out.h(root2.data());
    // sampled values: tree 0 (no columns), tree 1 (N), tree 2 (8)
    out.u64(3);
    out.u64(0);
    out.u64(N);
    for (uint32_t c = 0; c < N; c++) {
      out.u64(1);
      out.q(sampled[c]);
    }
    out.u64(8);
    for (int k = 0; k < 8; k++) {
      out.u64(1);
      out.q(sampled[N + k]);
    }
    // decommitments
    out.u64(3);
    out.u64(0);
    out.u64(td1.nodes.size());
    for (size_t s2 : td1.node_slot) hash_at(s2, out);
    out.u64(td2.nodes.size());
    for (size_t s2 : td2.node_slot) hash_at(s2, out);
    // queried values
    const size_t nq = queries.size();
    out.u64(3);
    out.u64(0);
    out.u64(N);
    for (uint32_t c = 0; c < N; c++) {
      out.u64(nq);
      for (size_t qi = 0; qi < nq; qi++) out.u32(words[td1.value_slot[c * nq + qi]]);
    }
    out.u64(8);
    for (int c = 0; c < 8; c++) {
      out.u64(nq);
      for (size_t qi = 0; qi < nq; qi++) out.u32(words[td2.value_slot[c * nq + qi]]);
    }
    out.u64(nonce);
    auto fri_layer = [&](const FriDecommit& d, const Hash32& root) {
      size_t n_w = 0;
      for (bool b : d.is_query) n_w += b ? 0 : 1;
      out.u64(n_w);
      for (size_t i = 0; i < d.positions.size(); i++)
        if (!d.is_query[i]) {
          size_t sl = d.value_slot[i];
          out.q({words[sl], words[sl + 1], words[sl + 2], words[sl + 3]});
        }
      out.u64(d.nodes.size());
      for (size_t s2 : d.node_slot) hash_at(s2, out);
      out.h(root.data());
    };
    fri_layer(fri_dec[0], fri_roots[0]);
    out.u64(fri.size());
    for (size_t li = 0; li < fri.size(); li++) fri_layer(fri_dec[li + 1], fri_roots[li + 1]);
    // last layer poly: bit-reversed storage order
    std::vector<qm31> lp = last_coeffs;
    uint32_t lg = 0;
    while (((size_t)1 << lg) < lp.size()) lg++;
    for (size_t i = 0; i < lp.size(); i++) {
      size_t j = bitrev32((uint32_t)i, lg);
      if (j > i) std::swap(lp[i], lp[j]);
    }
    out.u64(lp.size());
    for (auto& x : lp) out.q(x);
  }
  last_proof_bytes = std::max(last_proof_bytes, out.bytes.size());
  finish_timing();
  return 0;
}

// ---- FRI-heavy path: FriProver commit + decommit with given alphas ----
// One secure column on CanonicCoset(log_n) (4 coordinate columns): lifted
// Blake2s tree of the circle layer, circle-to-line fold, then per line layer
// its tree and a fold by 2, down to one value; then the decommitment of the
// query positions (prover/fri.rs:133-350; alphas supplied instead of drawn).
// Output: the FriProof bytes (first layer, inner layers, last-layer value) in
// the proof's canonical layout.  All buffers are allocated once per size.
struct SeededFriProver {
  uint32_t n = 0, tree_log = 0;
  int m31 = 0;
  const uint32_t* itw = nullptr;
  cudaStream_t user_s = nullptr, s = nullptr;
  cudaEvent_t ev_in = nullptr, ev_out = nullptr;
  // The alphas are given, so no layer waits for another layer's root: the
  // node levels of each tree run on side streams, forked from the fold chain
  // when the tree's leaves are written and joined at the end of the commit.
  static constexpr int kSide = 4;
  cudaStream_t side[kSide] = {nullptr, nullptr, nullptr, nullptr};
  std::vector<cudaEvent_t> ev_fork;  // one per tree, plus one per side stream for the join
  std::vector<uint32_t*> line;   // line[k]: 4 x 2^(n-1-k) words, k = 0..n-1 (line[n-1]: the last value)
  std::vector<MerkleTree> trees;  // trees[0]: circle layer (L = n); trees[k]: line[k-1] (L = n-k)
  std::vector<void*> allocs;
  qm31* d_alphas = nullptr;  // the folding alphas (uploaded per call; read by the fold kernels)
  qm31* h_alphas = nullptr;  // pinned staging of the alphas
  uint64_t* d_gather_addr = nullptr;
  uint8_t* d_gather_out = nullptr;
  size_t gather_cap = 0;     // entries (words or hashes)
  uint8_t* h_stage = nullptr;  // pinned: addresses (8 B / entry), then gathered bytes (32 B / entry)
  // the commit sequence, captured once per input column set
  cudaGraphExec_t exec = nullptr;
  const void* key[4] = {nullptr, nullptr, nullptr, nullptr};
  uint64_t graph_launches = 0;

  ~SeededFriProver() {
    if (s) cudaStreamSynchronize(s);
    if (exec) cudaGraphExecDestroy(exec);
    if (h_stage) cudaFreeHost(h_stage);
    if (h_alphas) cudaFreeHost(h_alphas);
    for (void* p : allocs) cudaFree(p);
    if (ev_in) cudaEventDestroy(ev_in);
    if (ev_out) cudaEventDestroy(ev_out);
    for (cudaEvent_t e : ev_fork) cudaEventDestroy(e);
    for (cudaStream_t x : side)
      if (x) cudaStreamDestroy(x);
    if (s) cudaStreamDestroy(s);
  }
  int alloc(void** p, size_t bytes, char* err, size_t err_len) {
    STWO_CUDA_TRY(cudaMalloc(p, std::max<size_t>(bytes, 16)));
    allocs.push_back(*p);
    return 0;
  }
  int init(uint32_t log_n, int m31_output, const uint32_t* d_itw, uint32_t tree_log_size, cudaStream_t stream,
           char* err, size_t err_len) {
    STWO_ARG_CHECK(log_n >= 2 && log_n <= 28, "log_size %u out of range [2, 28]", log_n);
    STWO_ARG_CHECK(d_itw && log_n - 1 <= tree_log_size, "twiddle tree (log %u) too small", tree_log_size);
    n = log_n;
    m31 = m31_output;
    itw = d_itw;
    tree_log = tree_log_size;
    user_s = stream;
    STWO_CUDA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    STWO_CUDA_TRY(cudaEventCreateWithFlags(&ev_in, cudaEventDisableTiming));
    STWO_CUDA_TRY(cudaEventCreateWithFlags(&ev_out, cudaEventDisableTiming));
    for (cudaStream_t& x : side) STWO_CUDA_TRY(cudaStreamCreateWithFlags(&x, cudaStreamNonBlocking));
    ev_fork.resize(n + kSide);
    for (cudaEvent_t& e : ev_fork) STWO_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    int rc;
    line.resize(n);
    for (uint32_t k = 0; k < n; k++)
      if ((rc = alloc((void**)&line[k], 16ull << (n - 1 - k), err, err_len))) return rc;
    trees.resize(n);
    for (uint32_t k = 0; k < n; k++) {
      trees[k].L = n - k;
      if ((rc = alloc((void**)&trees[k].base, MerkleTree::bytes_for(n - k), err, err_len))) return rc;
    }
    if ((rc = alloc((void**)&d_alphas, n * sizeof(qm31), err, err_len))) return rc;
    STWO_CUDA_TRY(cudaMallocHost((void**)&h_alphas, n * sizeof(qm31)));
    return 0;
  }
  static std::vector<uint32_t*> cols4(uint32_t* base, uint32_t log_size) {
    std::vector<uint32_t*> c(4);
    for (int k = 0; k < 4; k++) c[k] = base + ((uint64_t)k << log_size);
    return c;
  }
  std::vector<uint8_t*> layer_ptrs(const MerkleTree& t) const {
    std::vector<uint8_t*> l(t.L + 1);
    for (uint32_t k = 0; k <= t.L; k++) l[k] = t.layer(k);
    return l;
  }

  // Commit with the fused device kernels (log size >= 5): leaves of the circle
  // layer, then per layer the node levels and a fold that reads its alpha from
  // device memory and hashes the next layer's leaves.
  int enqueue_commit(const uint32_t* const* d_coords, char* err, size_t err_len) {
    int rc;
    const uint32_t lg[4] = {n, n, n, n};
    // node levels of tree k (leaves at level L, written on `s`) on a side stream
    auto nodes_on_side = [&](uint32_t k, uint32_t L) -> int {
      cudaStream_t x = side[1 + (k - 1) % (kSide - 1)];  // side[0] carries the circle layer's tree
      STWO_CUDA_TRY(cudaEventRecord(ev_fork[k], s));
      STWO_CUDA_TRY(cudaStreamWaitEvent(x, ev_fork[k], 0));
      auto lk = layer_ptrs(trees[k]);
      return build_node_layers_impl(trees[k].layer(L), L, 0, m31, lk.data(), x, err, err_len);
    };
    {
      // the circle layer's whole tree reads only the input columns: it runs
      // beside the fold chain from the start
      cudaStream_t x = side[0];
      STWO_CUDA_TRY(cudaEventRecord(ev_fork[0], s));
      STWO_CUDA_TRY(cudaStreamWaitEvent(x, ev_fork[0], 0));
      if ((rc = build_leaves_impl(d_coords, lg, 4, n, m31, trees[0].layer(n), nullptr, x, err, err_len))) return rc;
      auto l0 = layer_ptrs(trees[0]);
      if ((rc = build_node_layers_impl(trees[0].layer(n), n, 0, m31, l0.data(), x, err, err_len))) return rc;
    }
    const Src4 src{{d_coords[0], d_coords[1], d_coords[2], d_coords[3]}};
    fold_circle_first_dev_kernel<<<grid1d(fold_threads(n - 1), 256), 256, 0, s>>>(
        src, n, d_alphas, itw, 1ull << tree_log, line[0], trees[1].layer(n - 1), m31);
    STWO_CHECK_LAUNCH();
    for (uint32_t k = 1; k < n; k++) {
      const uint32_t L = n - k;  // log size of line[k-1]
      if ((rc = nodes_on_side(k, L))) return rc;
      uint8_t* next_leaves = k + 1 < n ? trees[k + 1].layer(L - 1) : nullptr;
      fold_line_dev_kernel<<<grid1d(fold_threads(L - 1), 256), 256, 0, s>>>(line[k - 1], L, 1, d_alphas + k, itw,
                                                                         1ull << tree_log, line[k], next_leaves, m31);
      STWO_CHECK_LAUNCH();
    }
    for (int j = 0; j < kSide; j++) {  // join
      STWO_CUDA_TRY(cudaEventRecord(ev_fork[n + j], side[j]));
      STWO_CUDA_TRY(cudaStreamWaitEvent(s, ev_fork[n + j], 0));
    }
    return 0;
  }

  // Small columns: the stand-alone FriOps and Merkle entry points.
  int enqueue_commit_small(const uint32_t* const* d_coords, const uint32_t* alphas, char* err, size_t err_len) {
    int rc;
    const uint32_t lg[4] = {n, n, n, n};
    auto l0 = layer_ptrs(trees[0]);
    if ((rc = stwo_b200_merkle_build_layers(d_coords, lg, 4, n, m31, l0.data(), s, err, err_len))) return rc;
    STWO_CUDA_TRY(cudaMemsetAsync(line[0], 0, 16ull << (n - 1), s));  // fold_circle_into_line accumulates
    auto c0 = cols4(line[0], n - 1);
    if ((rc = stwo_b200_fold_circle_into_line(c0.data(), d_coords, n, 1ull << (31 - (n + 1)), alphas, itw, tree_log,
                                              s, err, err_len)))
      return rc;
    for (uint32_t k = 1; k < n; k++) {
      const uint32_t L = n - k;
      auto cur = cols4(line[k - 1], L);
      auto nxt = cols4(line[k], L - 1);
      const uint32_t ll[4] = {L, L, L, L};
      auto lk = layer_ptrs(trees[k]);
      if ((rc = stwo_b200_merkle_build_layers(const_cast<const uint32_t* const*>(cur.data()), ll, 4, L, m31,
                                              lk.data(), s, err, err_len)))
        return rc;
      if ((rc = stwo_b200_fold_line(const_cast<const uint32_t* const*>(cur.data()), L, alphas + 4 * k, 1, itw,
                                    tree_log, nxt.data(), s, err, err_len)))
        return rc;
    }
    return 0;
  }

  int prove(const uint32_t* const* d_coords, const uint32_t* alphas, const uint64_t* queries_in, uint32_t n_q,
            ProofOut& out, char* err, size_t err_len) {
    std::vector<size_t> queries(queries_in, queries_in + n_q);
    for (uint32_t i = 0; i < n_q; i++) {
      STWO_ARG_CHECK(queries[i] >> n == 0, "query %zu out of range", queries[i]);
      STWO_ARG_CHECK(i == 0 || queries[i] > queries[i - 1], "queries must be sorted and distinct");
    }
    STWO_CUDA_TRY(cudaEventRecord(ev_in, user_s));
    STWO_CUDA_TRY(cudaStreamWaitEvent(s, ev_in, 0));
    int rc;
    // ---- commit (prover/fri.rs:133-291) ----
    if (n >= 5) {
      std::memcpy(h_alphas, alphas, n * sizeof(qm31));
      STWO_CUDA_TRY(cudaMemcpyAsync(d_alphas, h_alphas, n * sizeof(qm31), cudaMemcpyHostToDevice, s));
      const bool same = exec && std::equal(d_coords, d_coords + 4, key);
      if (!same) {
        if (exec) cudaGraphExecDestroy(exec);
        exec = nullptr;
        const uint64_t before = g_kernel_launches.load();
        STWO_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        rc = enqueue_commit(d_coords, err, err_len);
        cudaGraph_t g = nullptr;
        const cudaError_t ce = cudaStreamEndCapture(s, &g);
        const uint64_t launched = g_kernel_launches.load() - before;
        g_kernel_launches.fetch_sub(launched);  // nothing ran during capture
        if (rc) {
          if (g) cudaGraphDestroy(g);
          return rc;
        }
        if (ce != cudaSuccess)
          return set_err(err, err_len, STWO_B200_ECUDA, "FRI graph capture: %s", cudaGetErrorString(ce));
        const cudaError_t ie = cudaGraphInstantiate(&exec, g, 0);
        cudaGraphDestroy(g);
        if (ie != cudaSuccess) {
          exec = nullptr;
          return set_err(err, err_len, STWO_B200_ECUDA, "FRI graph instantiate: %s", cudaGetErrorString(ie));
        }
        std::copy(d_coords, d_coords + 4, key);
        graph_launches = launched;
      }
      STWO_CUDA_TRY(cudaGraphLaunch(exec, s));
      g_kernel_launches.fetch_add(graph_launches);
    } else if ((rc = enqueue_commit_small(d_coords, alphas, err, err_len))) {
      return rc;
    }
    // ---- decommit (prover/fri.rs:294-350, 459-488): one gather ----
    // word entries (queried-pair values, 4 coordinates each) first, then hash
    // entries (Merkle witness nodes and roots).
    std::vector<uint64_t> word_addr, hash_addr;
    word_addr.reserve((size_t)n * 4 * 2 * n_q + 4);
    hash_addr.reserve((size_t)n * (n + 2) * n_q + n);
    struct LayerPlan {
      std::vector<bool> is_query;
      std::vector<size_t> value_slot, node_slot;
    };
    auto plan = [&](const uint32_t* const* c4, const MerkleTree& t, const std::vector<size_t>& q) {
      LayerPlan d;
      std::vector<size_t> positions;
      for (size_t i = 0; i < q.size();) {
        size_t j = i;
        while (j < q.size() && (q[j] >> 1) == (q[i] >> 1)) j++;
        const size_t start = (q[i] >> 1) << 1;
        size_t k = i;
        for (size_t pos = start; pos < start + 2; pos++) {
          const bool isq = k < j && q[k] == pos;
          if (isq) k++;
          positions.push_back(pos);
          d.is_query.push_back(isq);
          d.value_slot.push_back(word_addr.size());
          for (int c = 0; c < 4; c++) word_addr.push_back(reinterpret_cast<uint64_t>(c4[c] + pos));
        }
        i = j;
      }
      for (auto& nd : witness_nodes(positions, t.L)) {
        d.node_slot.push_back(hash_addr.size());
        hash_addr.push_back(reinterpret_cast<uint64_t>(t.layer(nd.first) + nd.second * 32));
      }
      return d;
    };
    std::vector<LayerPlan> plans;
    plans.push_back(plan(d_coords, trees[0], queries));
    std::vector<size_t> lq;
    for (size_t q : queries)
      if (lq.empty() || lq.back() != (q >> 1)) lq.push_back(q >> 1);
    for (uint32_t k = 1; k < n; k++) {
      auto cur = cols4(line[k - 1], n - k);
      plans.push_back(plan(cur.data(), trees[k], lq));
      std::vector<size_t> nq;
      for (size_t q : lq)
        if (nq.empty() || nq.back() != (q >> 1)) nq.push_back(q >> 1);
      lq = nq;
    }
    const size_t last_slot = word_addr.size();
    for (int c = 0; c < 4; c++) word_addr.push_back(reinterpret_cast<uint64_t>(line[n - 1] + c));
    std::vector<size_t> root_slot(n);
    for (uint32_t k = 0; k < n; k++) {
      root_slot[k] = hash_addr.size();
      hash_addr.push_back(reinterpret_cast<uint64_t>(trees[k].layer(0)));
    }
    const size_t nw = word_addr.size(), nh = hash_addr.size(), total = nw + nh;
    if (total > gather_cap) {
      const size_t cap = std::max<size_t>(total * 2, 4096);
      if ((rc = alloc((void**)&d_gather_addr, cap * 8, err, err_len))) return rc;
      if ((rc = alloc((void**)&d_gather_out, cap * 32, err, err_len))) return rc;
      if (h_stage) cudaFreeHost(h_stage);
      h_stage = nullptr;
      STWO_CUDA_TRY(cudaMallocHost((void**)&h_stage, cap * 40));
      gather_cap = cap;
    }
    uint64_t* h_addr = reinterpret_cast<uint64_t*>(h_stage);
    std::memcpy(h_addr, word_addr.data(), nw * 8);
    std::memcpy(h_addr + nw, hash_addr.data(), nh * 8);
    STWO_CUDA_TRY(cudaMemcpyAsync(d_gather_addr, h_addr, total * 8, cudaMemcpyHostToDevice, s));
    uint32_t* d_words = reinterpret_cast<uint32_t*>(d_gather_out);
    uint4* d_hashes = reinterpret_cast<uint4*>(d_gather_out + ((nw * 4 + 31) / 32) * 32);
    gather_kernel<<<(unsigned)((nw + 255) / 256), 256, 0, s>>>(d_gather_addr, (uint32_t)nw, d_words);
    STWO_CHECK_LAUNCH();
    gather_hashes_kernel<<<(unsigned)((nh + 255) / 256), 256, 0, s>>>(d_gather_addr + nw, (uint32_t)nh, d_hashes);
    STWO_CHECK_LAUNCH();
    uint8_t* h_out = h_stage + gather_cap * 8;
    const size_t out_bytes = ((nw * 4 + 31) / 32) * 32 + nh * 32;
    STWO_CUDA_TRY(cudaMemcpyAsync(h_out, d_gather_out, out_bytes, cudaMemcpyDeviceToHost, s));
    STWO_CUDA_TRY(cudaStreamSynchronize(s));
    const uint32_t* words = reinterpret_cast<const uint32_t*>(h_out);
    const uint8_t* hashes = h_out + ((nw * 4 + 31) / 32) * 32;
    // ---- serialize: FriLayerProof order of core/fri.rs:361-395 ----
    out.bytes.reserve(out.bytes.size() + nw * 4 + nh * 32 + 64 * n);
    auto layer = [&](const LayerPlan& d, size_t rs) {
      size_t n_w = 0;
      for (bool b : d.is_query) n_w += b ? 0 : 1;
      out.u64(n_w);
      for (size_t i = 0; i < d.is_query.size(); i++)
        if (!d.is_query[i]) {
          const size_t sl = d.value_slot[i];
          out.q({words[sl], words[sl + 1], words[sl + 2], words[sl + 3]});
        }
      out.u64(d.node_slot.size());
      for (size_t sl : d.node_slot) out.h(hashes + 32 * sl);
      out.h(hashes + 32 * rs);
    };
    layer(plans[0], root_slot[0]);
    out.u64(n - 1);
    for (uint32_t k = 1; k < n; k++) layer(plans[k], root_slot[k]);
    out.u64(1);
    out.q({words[last_slot], words[last_slot + 1], words[last_slot + 2], words[last_slot + 3]});
    cudaEventRecord(ev_out, s);
    cudaStreamWaitEvent(user_s, ev_out, 0);
    return 0;
  }
};

}  // namespace stwo_b200

using namespace stwo_b200;

struct stwo_b200_prover {
  std::unique_ptr<WideFibProver> impl;
};

extern "C" int stwo_b200_prover_create(const stwo_b200_wide_fib_config* cfg, stwo_b200_prover** out, void* stream,
                                       char* err, size_t err_len) {
  STWO_ARG_CHECK(cfg && out, "null argument");
  *out = nullptr;
  auto p = std::make_unique<stwo_b200_prover>();
  p->impl = std::make_unique<WideFibProver>();
  int rc = p->impl->init(*cfg, as_stream(stream), err, err_len);
  if (rc) return rc;
  *out = p.release();
  return ok(err, err_len);
}

extern "C" int stwo_b200_prover_destroy(stwo_b200_prover* p, char* err, size_t err_len) {
  if (p) {
    cudaStreamSynchronize(p->impl->s);
    delete p;
  }
  return ok(err, err_len);
}

extern "C" int stwo_b200_prover_set_timing(stwo_b200_prover* p, int enable, char* err, size_t err_len) {
  STWO_ARG_CHECK(p, "null prover");
  p->impl->timing = enable != 0;
  for (double& x : p->impl->phase_ms) x = 0;
  p->impl->proofs_timed = 0;
  return ok(err, err_len);
}

extern "C" int stwo_b200_prover_set_stream_spin(stwo_b200_prover* p, uint32_t polls, char* err, size_t err_len) {
  STWO_ARG_CHECK(p, "null prover");
  p->impl->stream_spin = polls;
  return ok(err, err_len);
}

extern "C" int stwo_b200_prover_phase_times(stwo_b200_prover* p, double* ms_out, uint32_t n, uint32_t* proofs,
                                            char* err, size_t err_len) {
  STWO_ARG_CHECK(p && ms_out, "null argument");
  for (uint32_t i = 0; i < n && i < (uint32_t)kNumPhases; i++) ms_out[i] = p->impl->phase_ms[i];
  if (proofs) *proofs = p->impl->proofs_timed;
  return ok(err, err_len);
}

extern "C" int stwo_b200_prover_footprint(const stwo_b200_wide_fib_config* cfg, size_t* device_bytes, char* err,
                                          size_t err_len) {
  STWO_ARG_CHECK(cfg && device_bytes, "null argument");
  WideFibProver m;
  m.measure = true;
  int rc = m.init(*cfg, nullptr, err, err_len);
  if (rc) return rc;
  // + the decommitment gather buffers sized at the first proof
  *device_bytes = m.allocated_bytes + ((size_t)4 << 20);
  return ok(err, err_len);
}

extern "C" int stwo_b200_prove_wide_fib_cols(stwo_b200_prover* p, uint32_t n_cols, const uint32_t* d_a,
                                             const uint32_t* d_b, uint8_t* proof_out, size_t proof_cap,
                                             size_t* proof_len, char* err, size_t err_len) {
  STWO_ARG_CHECK(p && d_a && d_b && proof_len, "null argument");
  ProofOut out;
  int rc = p->impl->prove(d_a, d_b, out, err, err_len, n_cols);
  if (rc) return rc;
  *proof_len = out.bytes.size();
  if (proof_out) {
    STWO_ARG_CHECK(proof_cap >= out.bytes.size(), "proof buffer too small (%zu < %zu)", proof_cap, out.bytes.size());
    std::memcpy(proof_out, out.bytes.data(), out.bytes.size());
  }
  return ok(err, err_len);
}

extern "C" int stwo_b200_prove_wide_fib(stwo_b200_prover* p, const uint32_t* d_a, const uint32_t* d_b,
                                        uint8_t* proof_out, size_t proof_cap, size_t* proof_len, char* err,
                                        size_t err_len) {
  STWO_ARG_CHECK(p && d_a && d_b && proof_len, "null argument");
  ProofOut out;
  int rc = p->impl->prove(d_a, d_b, out, err, err_len);
  if (rc) return rc;
  *proof_len = out.bytes.size();
  if (proof_out) {
    STWO_ARG_CHECK(proof_cap >= out.bytes.size(), "proof buffer too small (%zu < %zu)", proof_cap, out.bytes.size());
    std::memcpy(proof_out, out.bytes.data(), out.bytes.size());
  }
  return ok(err, err_len);
}

extern "C" int stwo_b200_prove_wide_fib_host(stwo_b200_prover* p, const uint32_t* h_a, const uint32_t* h_b,
                                             uint8_t* proof_out, size_t proof_cap, size_t* proof_len, char* err,
                                             size_t err_len) {
  STWO_ARG_CHECK(p && h_a && h_b && proof_len, "null argument");
  ProofOut out;
  int rc = p->impl->prove_host(h_a, h_b, out, err, err_len);
  if (rc) return rc;
  *proof_len = out.bytes.size();
  if (proof_out) {
    STWO_ARG_CHECK(proof_cap >= out.bytes.size(), "proof buffer too small (%zu < %zu)", proof_cap, out.bytes.size());
    std::memcpy(proof_out, out.bytes.data(), out.bytes.size());
  }
  return ok(err, err_len);
}

struct stwo_b200_fri_prover {
  std::unique_ptr<SeededFriProver> impl;
};

extern "C" int stwo_b200_fri_prover_create(uint32_t log_size, int m31_output, const uint32_t* d_itwiddles,
                                           uint32_t tree_log_size, void* stream, stwo_b200_fri_prover** out,
                                           char* err, size_t err_len) {
  STWO_ARG_CHECK(out, "null argument");
  *out = nullptr;
  auto p = std::make_unique<stwo_b200_fri_prover>();
  p->impl = std::make_unique<SeededFriProver>();
  int rc = p->impl->init(log_size, m31_output, d_itwiddles, tree_log_size, as_stream(stream), err, err_len);
  if (rc) return rc;
  *out = p.release();
  return ok(err, err_len);
}

extern "C" int stwo_b200_fri_prover_destroy(stwo_b200_fri_prover* p, char* err, size_t err_len) {
  delete p;
  return ok(err, err_len);
}

extern "C" int stwo_b200_fri_prove_seeded(stwo_b200_fri_prover* p, const uint32_t* const* d_coords4,
                                          const uint32_t* alphas, const uint64_t* queries, uint32_t n_queries,
                                          uint8_t* proof_out, size_t proof_cap, size_t* proof_len, char* err,
                                          size_t err_len) {
  STWO_ARG_CHECK(p && d_coords4 && alphas && proof_len && (queries || n_queries == 0), "null argument");
  STWO_ARG_CHECK(n_queries >= 1, "at least one query");
  ProofOut out;
  int rc = p->impl->prove(d_coords4, alphas, queries, n_queries, out, err, err_len);
  if (rc) return rc;
  *proof_len = out.bytes.size();
  if (proof_out) {
    STWO_ARG_CHECK(proof_cap >= out.bytes.size(), "proof buffer too small (%zu < %zu)", proof_cap, out.bytes.size());
    std::memcpy(proof_out, out.bytes.data(), out.bytes.size());
  }
  return ok(err, err_len);
}
