// Circle FFT (PolyOps::interpolate / evaluate) and bit reversal for sm_100a.
//
// A transform of n butterfly layers runs as 1-3 passes.  A pass covers the
// consecutive layers [layer0, layer0 + T) on tiles of 2^T rows x 2^C columns
// held in shared memory: row r, column c of tile (hi, lo) is element
//   g = hi * 2^(layer0 + T) + r * 2^layer0 + lo * 2^C + c,
// so a tile row is 2^C contiguous words (C = 3: one 32-byte sector) and every
// butterfly of the pass stays inside the tile.  Inside the tile, layers run in
// register stages of up to 4 (radix-16 per thread); stages exchange through
// shared memory.  Butterflies and layer order follow
// crates/stwo/src/prover/backend/cpu/circle.rs:28-80,199-250 (fft_layer_loop
// :313-327): IFFT layer 0 (circle) upward, then x n^-1; RFFT top layer down to
// the circle layer.  Twiddles are read from the tree tail exactly as
// core/poly/utils.rs:98-114 slices it; circle-layer twiddles are derived from
// line layer 1 as [y, -y, -x, x] (cpu/circle.rs:332-354).
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <vector>

#include "common.cuh"
#include "fft.hpp"
#include "field.cuh"
#include "stream.cuh"

namespace stwo_b200 {

// A column table passed by value: up to kFftMaxCols (src, dst) pairs per launch.
constexpr int kFftMaxCols = 256;
struct FftCols {
  const uint32_t* src[kFftMaxCols];
  uint32_t* dst[kFftMaxCols];
};

struct FftPass {
  const uint32_t* tree;  // twiddle (or inverse twiddle) tree
  uint64_t tree_len;
  uint64_t src_mask;   // element g reads src[g & src_mask] ...
  uint64_t src_len;    // ... when (g & src_mask) < src_len, else 0
  uint32_t log_domain; // N: log size of the domain the twiddles belong to
  uint32_t layer0, T, C;
  uint32_t scale;      // outputs are multiplied by `scale` when != 1
  uint32_t vec_io;     // 16-byte global loads/stores are legal for this launch
  uint32_t cpb;        // columns per block: tiles of the same position share staged twiddles
  uint32_t n_cols;     // columns in this launch
  uint32_t natural = 0;  // the source is in natural order: the contiguous first pass gathers src[rev_N(i)]
  uint32_t tile0 = 0;    // tile positions of this launch start here (a launch over part of a pass)
};


// Circle-layer twiddle for butterfly h, from line layer 1 (x, y pairs).
__device__ __forceinline__ uint32_t circle_tw(const uint32_t* lt0, uint64_t h) {
  uint32_t b = __ldg(lt0 + ((h >> 1) ^ 1));
  return ((h ^ (h >> 1)) & 1) ? m31_neg(b) : b;
}

__device__ __forceinline__ void ibfly(uint32_t& a, uint32_t& b, uint32_t t) {
  uint32_t s = m31_add(a, b);
  b = m31_mul(m31_sub(a, b), t);
  a = s;
}
__device__ __forceinline__ void bfly(uint32_t& a, uint32_t& b, uint32_t t) {
  uint32_t m = m31_mul(b, t);
  b = m31_sub(a, m);
  a = m31_add(a, m);
}

// Butterflies with the twiddle stored doubled (t2 = 2t < 2^32): the 64-bit
// product b * t2 has (b t) >> 31 as its high word and 2 (b t mod 2^31) as its
// low word, so the reduction needs one shift instead of a mask and a funnel
// shift.  Same (lo, hi) pair, hence the same result, as m31_mul(b, t).
__device__ __forceinline__ uint32_t m31_mul_tw2(uint32_t b, uint32_t t2) {
  const uint64_t x = (uint64_t)b * t2;
  return m31_add((uint32_t)x >> 1, (uint32_t)(x >> 32));
}
__device__ __forceinline__ void ibfly2(uint32_t& a, uint32_t& b, uint32_t t2) {
  uint32_t s = m31_add(a, b);
  b = m31_mul_tw2(m31_sub(a, b), t2);
  a = s;
}
__device__ __forceinline__ void bfly2(uint32_t& a, uint32_t& b, uint32_t t2) {
  uint32_t m = m31_mul_tw2(b, t2);
  b = m31_sub(a, m);
  a = m31_add(a, m);
}

__host__ __device__ constexpr uint32_t tile_stride_words(uint32_t e) { return e + (e >> 4) + 1; }
__host__ __device__ constexpr uint32_t smem_off(uint32_t e) { return e + (e >> 4); }

// Threads per block of a pass: one radix-16 group per thread, 32..256.
__host__ __device__ constexpr int fft_threads(int T, int C, int CPB) {
  return ((CPB << (T + C)) >> 4) >= 256 ? 256
         : ((CPB << (T + C)) >> 4) >= 128 ? 128
         : ((CPB << (T + C)) >> 4) >= 64  ? 64
                                          : 32;
}

// One register stage over tile row bits [S0, S0 + RS) of CPB tiles.  Tile
// shape and stage position are compile-time, so the 2^RS shared-memory
// offsets of a group are immediates: for disjoint bit sets,
// smem_off(ebase | J) = smem_off(ebase) + smem_off(J).  Twiddles come from the
// per-position table `tws`: layer lam (relative to layer0) at offset
// 2^T - 2^(T - lam), indexed by row >> (lam + 1).
template <bool INV, int T, int C, int CPB, int NT, int RS, int S0>
__device__ __forceinline__ void tile_stage(uint32_t* __restrict__ sm, const uint32_t* __restrict__ tws,
                                           uint32_t n_tiles) {
  constexpr uint32_t E = 1u << (T + C);
  constexpr uint32_t STRIDE = tile_stride_words(E);
  constexpr int LG = T + C - RS;
  constexpr uint32_t GROUPS = (uint32_t)CPB << LG;
  constexpr int ITERS = (int)((GROUPS + NT - 1) / NT);
#pragma unroll
  for (int it = 0; it < ITERS; it++) {
    const uint32_t q = threadIdx.x + (uint32_t)it * NT;
    if ((GROUPS % NT) != 0 && q >= GROUPS) break;
    const uint32_t tile = q >> LG;
    if (CPB > 1 && tile >= n_tiles) break;
    const uint32_t qq = q & ((1u << LG) - 1);
    const uint32_t c = qq & ((1u << C) - 1);
    const uint32_t rest = qq >> C;
    const uint32_t low = rest & ((1u << S0) - 1);
    const uint32_t high = rest >> S0;
    const uint32_t ebase = (((high << (S0 + RS)) | low) << C) | c;
    uint32_t* __restrict__ g = sm + tile * STRIDE + smem_off(ebase);
    uint32_t v[1 << RS];
#pragma unroll
    for (int j = 0; j < (1 << RS); j++) v[j] = g[smem_off((uint32_t)j << (S0 + C))];
#pragma unroll
    for (int kk = 0; kk < RS; kk++) {
      const int k = INV ? kk : (RS - 1 - kk);
      // Butterfly (j, j | 2^k) uses twiddle (high << (RS-1-k)) + (j >> (k+1)):
      // 2^(RS-1-k) distinct values per group.
      const uint32_t* tl = tws + ((1u << T) - (1u << (T - (S0 + k)))) + (high << (RS - 1 - k));
      uint32_t t[1 << (RS - 1)];
#pragma unroll
      for (int m = 0; m < (1 << (RS - 1 - k)); m++) t[m] = tl[m];
#pragma unroll
      for (int j = 0; j < (1 << RS); j++) {
        if (j & (1 << k)) continue;
        if (INV)
          ibfly(v[j], v[j | (1 << k)], t[j >> (k + 1)]);
        else
          bfly(v[j], v[j | (1 << k)], t[j >> (k + 1)]);
      }
    }
#pragma unroll
    for (int j = 0; j < (1 << RS); j++) g[smem_off((uint32_t)j << (S0 + C))] = v[j];
  }
}

// IFFT stages bottom-up from S0; RFFT stages top-down from TOP.
template <int T, int C, int CPB, int NT, int S0>
__device__ __forceinline__ void inv_stages(uint32_t* sm, const uint32_t* tws, uint32_t n_tiles) {
  constexpr int RS = (T - S0) < 4 ? (T - S0) : 4;
  tile_stage<true, T, C, CPB, NT, RS, S0>(sm, tws, n_tiles);
  __syncthreads();
  if constexpr (S0 + RS < T) inv_stages<T, C, CPB, NT, S0 + RS>(sm, tws, n_tiles);
}
template <int T, int C, int CPB, int NT, int TOP>
__device__ __forceinline__ void fwd_stages(uint32_t* sm, const uint32_t* tws, uint32_t n_tiles) {
  constexpr int RS = TOP < 4 ? TOP : 4;
  tile_stage<false, T, C, CPB, NT, RS, TOP - RS>(sm, tws, n_tiles);
  __syncthreads();
  if constexpr (TOP - RS > 0) fwd_stages<T, C, CPB, NT, TOP - RS>(sm, tws, n_tiles);
}

template <bool INV, int T, int C, int CPB, int NT>
__global__ void __launch_bounds__(NT, 1024 / NT) fft_pass_kernel(FftPass p, FftCols cols) {
  constexpr uint32_t E = 1u << (T + C);
  constexpr uint32_t STRIDE = tile_stride_words(E);
  constexpr uint32_t CMASK = (1u << C) - 1;
  extern __shared__ uint32_t smem[];
  const uint32_t L0 = p.layer0;
  const uint32_t col0 = blockIdx.y * CPB;
  const uint32_t n_tiles = CPB == 1 ? 1u : min((uint32_t)CPB, p.n_cols - col0);
  uint32_t* __restrict__ sm = smem;
  uint32_t* __restrict__ tws = smem + CPB * STRIDE;
  const uint64_t tile = (uint64_t)p.tile0 + blockIdx.x;
  const uint32_t lo_bits = L0 - C;  // L0 >= C
  const uint64_t lo = tile & ((1ull << lo_bits) - 1);
  const uint64_t hi = tile >> lo_bits;
  const uint64_t base = (hi << (L0 + T)) | (lo << C);

  // Stage the twiddles of this tile position: layer lam needs 2^(T-1-lam)
  // consecutive entries starting at hi << (T-1-lam) of tree layer L0 + lam.
#pragma unroll
  for (int lam = 0; lam < T; lam++) {
    constexpr uint32_t one = 1;
    const uint32_t cnt = one << (T - 1 - lam);
    const uint32_t off = (one << T) - (one << (T - lam));
    const uint64_t h0 = hi << (T - 1 - lam);
    const uint32_t layer = L0 + lam;
    if (layer == 0) {
      const uint32_t* lt0 = p.tree + (p.tree_len - (1ull << (p.log_domain - 1)));
      for (uint32_t i = threadIdx.x; i < cnt; i += NT) tws[off + i] = circle_tw(lt0, h0 + i);
    } else {
      const uint32_t* lt = p.tree + (p.tree_len - (1ull << (p.log_domain - layer))) + h0;
      for (uint32_t i = threadIdx.x; i < cnt; i += NT) tws[off + i] = __ldg(lt + i);
    }
  }

  // Load the tiles; rows of 2^C >= 4 words (or contiguous tiles) use 16-byte loads.
  for (uint32_t cc = 0; cc < n_tiles; cc++) {
    const uint32_t* __restrict__ src = cols.src[col0 + cc];
    uint32_t* tsm = sm + cc * STRIDE;
    if (C == 0 && p.natural) {
      // Natural-order source (first pass, L0 = 0): element e of tile position
      // hi is src[rev_T(e) * 2^(N-T) + rev_{N-T}(hi)], the bit reversal of
      // ColumnOps::bit_reverse_column done by the loads.
      const uint32_t sh = p.log_domain - T;
      const uint64_t rh = sh ? __brevll(hi) >> (64 - sh) : 0;
      for (uint32_t e = threadIdx.x; e < E; e += NT)
        tsm[smem_off(e)] = __ldg(src + (((uint64_t)(__brev(e) >> (32 - T)) << sh) | rh));
    } else if (p.vec_io) {
#pragma unroll 4
      for (uint32_t e = threadIdx.x * 4; e < E; e += NT * 4) {
        const uint64_t g = base + ((uint64_t)(e >> C) << L0) + (e & CMASK);
        const uint64_t gi = g & p.src_mask;
        const uint4 w = gi < p.src_len ? __ldg(reinterpret_cast<const uint4*>(src + gi)) : make_uint4(0, 0, 0, 0);
        uint32_t* d = tsm + smem_off(e);  // e % 4 == 0: the four words share one padding group
        d[0] = w.x;
        d[1] = w.y;
        d[2] = w.z;
        d[3] = w.w;
      }
    } else {
      for (uint32_t e = threadIdx.x; e < E; e += NT) {
        const uint64_t g = base + ((uint64_t)(e >> C) << L0) + (e & CMASK);
        const uint64_t gi = g & p.src_mask;
        tsm[smem_off(e)] = gi < p.src_len ? __ldg(src + gi) : 0u;
      }
    }
  }
  __syncthreads();

  if constexpr (INV)
    inv_stages<T, C, CPB, NT, 0>(sm, tws, n_tiles);
  else
    fwd_stages<T, C, CPB, NT, T>(sm, tws, n_tiles);

  const uint32_t scale = p.scale;
  for (uint32_t cc = 0; cc < n_tiles; cc++) {
    uint32_t* __restrict__ dst = cols.dst[col0 + cc];
    const uint32_t* tsm = sm + cc * STRIDE;
    if (p.vec_io) {
#pragma unroll 4
      for (uint32_t e = threadIdx.x * 4; e < E; e += NT * 4) {
        const uint64_t g = base + ((uint64_t)(e >> C) << L0) + (e & CMASK);
        const uint32_t* d = tsm + smem_off(e);
        uint4 w = make_uint4(d[0], d[1], d[2], d[3]);
        if (scale != 1u) {
          w.x = m31_mul(w.x, scale);
          w.y = m31_mul(w.y, scale);
          w.z = m31_mul(w.z, scale);
          w.w = m31_mul(w.w, scale);
        }
        *reinterpret_cast<uint4*>(dst + g) = w;
      }
    } else {
      for (uint32_t e = threadIdx.x; e < E; e += NT) {
        const uint64_t g = base + ((uint64_t)(e >> C) << L0) + (e & CMASK);
        const uint32_t v = tsm[smem_off(e)];
        dst[g] = scale != 1u ? m31_mul(v, scale) : v;
      }
    }
  }
}

// Transforms of log size <= 2 follow the special cases of
// cpu/circle.rs:35-59 (interpolate) and :215-235 (evaluate); they need the
// domain's first point (x, y) and run on one thread.
struct SmallCols {
  const uint32_t* src[kFftMaxCols];
  uint32_t* dst[kFftMaxCols];
  uint32_t x[kFftMaxCols], y[kFftMaxCols];
  uint32_t log_src[kFftMaxCols], log_dst[kFftMaxCols];
};

__global__ void small_fft_kernel(SmallCols t, uint32_t n, int inverse) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t v[4] = {0, 0, 0, 0};
  uint32_t ls = t.log_src[i], ld = t.log_dst[i];
  for (uint32_t k = 0; k < (1u << ls); k++) v[k] = t.src[i][k];
  uint32_t x = t.x[i], y = t.y[i];
  if (inverse) {
    if (ld == 1) {
      uint32_t yn_inv = m31_inv(m31_mul(y, 2));
      uint32_t y_inv = m31_mul(yn_inv, 2), n_inv = m31_mul(yn_inv, y);
      ibfly(v[0], v[1], y_inv);
      v[0] = m31_mul(v[0], n_inv);
      v[1] = m31_mul(v[1], n_inv);
    } else {
      uint32_t xyn_inv = m31_inv(m31_mul(m31_mul(x, y), 4));
      uint32_t x_inv = m31_mul(m31_mul(xyn_inv, y), 4);
      uint32_t y_inv = m31_mul(m31_mul(xyn_inv, x), 4);
      uint32_t n_inv = m31_mul(m31_mul(xyn_inv, x), y);
      ibfly(v[0], v[1], y_inv);
      ibfly(v[2], v[3], m31_neg(y_inv));
      ibfly(v[0], v[2], x_inv);
      ibfly(v[1], v[3], x_inv);
      for (int k = 0; k < 4; k++) v[k] = m31_mul(v[k], n_inv);
    }
  } else {
    if (ld == 1) {
      bfly(v[0], v[1], y);
    } else {
      bfly(v[0], v[2], x);
      bfly(v[1], v[3], x);
      bfly(v[0], v[1], y);
      bfly(v[2], v[3], m31_neg(y));
    }
  }
  for (uint32_t k = 0; k < (1u << ld); k++) t.dst[i][k] = v[k];
}

// In-place bit reversal: thread i swaps i <-> rev(i) when i < rev(i).
__global__ void bit_reverse_kernel(uint32_t* v, uint32_t log_n) {
  uint64_t n = 1ull << log_n;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t j = __brevll(i) >> (64 - log_n);
    if (i < j) {
      uint32_t a = v[i], b = v[j];
      v[i] = b;
      v[j] = a;
    }
  }
}

// Integer-issue ceiling of the butterfly (no reference counterpart): every
// thread applies `iters` rounds of 5 layers x 16 forward butterflies (bfly2,
// the pass kernels' arithmetic) to 32 values held in registers, with one
// doubled twiddle per layer.  butterflies / elapsed time is the rate the FFT
// passes are measured against; no memory traffic, no twiddle loads.
__global__ void __launch_bounds__(256) butterfly_probe_kernel(uint32_t iters, uint32_t* out) {
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t v[32];
#pragma unroll
  for (int j = 0; j < 32; j++) v[j] = (tid * 32u + (uint32_t)j) & M31_P;  // < 2^31, so <= P
  uint32_t t2[5];
#pragma unroll
  for (int k = 0; k < 5; k++) t2[k] = ((tid * 5u + (uint32_t)k + 1u) % M31_P) << 1;  // 2t with t < P
  for (uint32_t it = 0; it < iters; it++) {
#pragma unroll
    for (int k = 0; k < 5; k++) {
#pragma unroll
      for (int j = 0; j < 32; j++)
        if (!(j & (1 << k))) bfly2(v[j], v[j | (1 << k)], t2[k]);
    }
  }
  uint32_t x = 0;
#pragma unroll
  for (int j = 0; j < 32; j++) x ^= v[j];
  if (x == 0x12345678u) out[0] = x;  // keeps the chain live
}

// Bit reversal of up to kFftMaxCols columns of one size in one launch
// (blockIdx.y = column): out of place (dst[brev(i)] = src[i], coalesced
// reads), or in place by pairwise swaps when dst == src.
__global__ void bit_reverse_cols_kernel(FftCols t, uint32_t log_n) {
  const uint64_t n = 1ull << log_n;
  const uint32_t* __restrict__ src = t.src[blockIdx.y];
  uint32_t* dst = t.dst[blockIdx.y];
  const bool in_place = src == dst;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t j = __brevll(i) >> (64 - log_n);
    if (!in_place) {
      dst[j] = src[i];
    } else if (i < j) {
      const uint32_t a = dst[i], b = dst[j];
      dst[i] = b;
      dst[j] = a;
    }
  }
}

// ---------------------------------------------------------------- host ----

struct PassPlan {
  uint32_t layer0, T, C;
};

// Pass plans: per transform size n, the layer counts of its passes, low
// layers first (the first pass is contiguous, C = 0; the others strided,
// C = 3).  A plan set with stwo_b200_fft_set_plan (the autotuner's choice)
// overrides the default split.
static std::mutex g_plan_mu;
static std::vector<uint32_t> g_plan_override[31];

static bool plan_is_valid(uint32_t n, const uint32_t* t, uint32_t k) {
  if (n == 0 || n > 30 || k == 0 || k > 4) return false;
  uint32_t sum = 0;
  for (uint32_t i = 0; i < k; i++) {
    if (t[i] < 1 || t[i] > 12) return false;
    sum += t[i];
  }
  // strided passes need layer0 >= C = 3
  return sum == n && (k == 1 || t[0] >= 3);
}

// Default: passes of <= 12 layers, two up to 23 layers, three above.  From
// 16 to 19 layers the first pass takes 10 (the 10-layer warp kernel), and at
// 22 the split is [12, 10] (a 12-layer warp-group pass, then a 10-layer warp
// pass), the splits the autotuner picks for them.
static std::vector<uint32_t> default_split(uint32_t n) {
  if (n <= 12) return {n};
  if (n >= 16 && n <= 19) return {10, n - 10};
  if (n == 22) return {12, 10};
  uint32_t parts = n <= 23 ? 2 : 3;
  std::vector<uint32_t> t;
  uint32_t rest = n;
  for (uint32_t i = 0; i < parts; i++) {
    uint32_t x = (rest + (parts - i) - 1) / (parts - i);
    t.push_back(x);
    rest -= x;
  }
  return t;
}

static std::vector<uint32_t> split_for(uint32_t n) {
  {
    std::lock_guard<std::mutex> g(g_plan_mu);
    if (n <= 30 && !g_plan_override[n].empty()) return g_plan_override[n];
  }
  return default_split(n);
}

static std::vector<PassPlan> plan_passes(uint32_t n) {
  std::vector<PassPlan> plan;
  uint32_t l0 = 0;
  for (uint32_t t : split_for(n)) {
    plan.push_back({l0, t, l0 == 0 ? 0u : 3u});
    l0 += t;
  }
  return plan;
}

static uint32_t host_pow2_inv(uint32_t log_n) { return m31_inv(m31_reduce_u32(1u << log_n)); }

// Domain first point for CanonicCoset-like half cosets (host).
static void index_point(uint64_t idx, uint32_t& x, uint32_t& y) {
  uint32_t gx = 2, gy = 1268011823u;
  x = 1;
  y = 0;
  idx &= (1ull << 31) - 1;
  for (int b = 0; b < 31; b++) {
    if ((idx >> b) & 1) {
      uint32_t nx = m31_sub(m31_mul(x, gx), m31_mul(y, gy));
      uint32_t ny = m31_add(m31_mul(x, gy), m31_mul(y, gx));
      x = nx;
      y = ny;
    }
    uint32_t dx = m31_sub(m31_mul(gx, gx), m31_mul(gy, gy));
    uint32_t dy = m31_add(m31_mul(gx, gy), m31_mul(gy, gx));
    gx = dx;
    gy = dy;
  }
}

// ---- 1024-point passes (T = 10) with 32 values per thread ----
// A thread holds 32 words of one tile column.  Layers 0..4 (row bits 0..4)
// run with them held lane-major (v[j] = row 32 b + j for the thread's 32-row
// block b); layers 5..9 with them held row-major (v[j] = row 32 j + b).  The
// contiguous pass gives a warp one column (b = lane) and exchanges the two
// layouts through a warp-private staged tile, so a warp needs no block
// barrier once the block's twiddles are staged; the strided pass spreads the
// 8 columns of its tile over the lanes and exchanges through the block.
// Butterflies, twiddle indices (row >> (lam+1) of tree layer layer0 + lam)
// and layer order are those of fft_stage.
constexpr int kWarpCols = 8;                  // warps (columns) per block of the contiguous pass

// Layers 0..4 on v[j] = row 32 b + j.
template <bool INV>
__device__ __forceinline__ void warp_phase_lo(uint32_t (&v)[32], const uint32_t* __restrict__ tws, uint32_t b) {
#pragma unroll
  for (int kk = 0; kk < 5; kk++) {
    const int lam = INV ? kk : 4 - kk;
    // row >> (lam + 1) = (b << (4 - lam)) + (j >> (lam + 1))
    const uint32_t* tl = tws + (1024u - (1024u >> lam)) + (b << (4 - lam));
    uint32_t t[16];
#pragma unroll
    for (int m = 0; m < (1 << (4 - lam)); m++) t[m] = tl[m];
#pragma unroll
    for (int j = 0; j < 32; j++) {
      if (j & (1 << lam)) continue;
      if (INV)
        ibfly2(v[j], v[j | (1 << lam)], t[j >> (lam + 1)]);
      else
        bfly2(v[j], v[j | (1 << lam)], t[j >> (lam + 1)]);
    }
  }
}

// Layers 5..9 on v[j] = row 32 j + b: row >> (lam + 1) = j >> (lam - 4),
// the same twiddle for every thread.
template <bool INV>
__device__ __forceinline__ void warp_phase_hi(uint32_t (&v)[32], const uint32_t* __restrict__ tws) {
#pragma unroll
  for (int kk = 0; kk < 5; kk++) {
    const int k = INV ? kk : 4 - kk;  // bit of j
    const uint32_t* tl = tws + (1024u - (1024u >> (5 + k)));
    uint32_t t[16];
#pragma unroll
    for (int m = 0; m < (1 << (4 - k)); m++) t[m] = tl[m];
#pragma unroll
    for (int j = 0; j < 32; j++) {
      if (j & (1 << k)) continue;
      if (INV)
        ibfly2(v[j], v[j | (1 << k)], t[j >> (k + 1)]);
      else
        bfly2(v[j], v[j | (1 << k)], t[j >> (k + 1)]);
    }
  }
}

// Layers 5..T-1 on v[j] = row 32 j + b (see warp_phase_hi), T = 6..10.  Below
// 10 layers each butterfly reads its twiddle from shared memory directly.
template <bool INV, int T>
__device__ __forceinline__ void warp_phase_hi_short(uint32_t (&v)[32], const uint32_t* __restrict__ tws) {
  if constexpr (T == 10) {
    warp_phase_hi<INV>(v, tws);
    return;
  }
  constexpr int NK = T - 5;
#pragma unroll
  for (int kk = 0; kk < NK; kk++) {
    const int k = INV ? kk : NK - 1 - kk;  // bit of j
    const uint32_t* tl = tws + (1024u - (1024u >> (5 + k)));
#pragma unroll
    for (int j = 0; j < 32; j++) {
      if (j & (1 << k)) continue;
      const uint32_t t = tl[j >> (k + 1)];
      if (INV)
        ibfly2(v[j], v[j | (1 << k)], t);
      else
        bfly2(v[j], v[j | (1 << k)], t);
    }
  }
}
// Stages the 1023 twiddles of a 10-layer tile position (as fft_pass_kernel),
// doubled for bfly2 / ibfly2: slot s of the table holds layer
// lam = clz(1023 - s) - 22, entry s - (1024 - 2^(10 - lam)).  Thread t holds
// slots t, t + 256 (lam 0), t + 512 (lam 1) and t + 768 (lam >= 2), and loads
// all four before storing any, so the block waits for one memory round trip
// instead of one per layer.  CIRCLE: layer0 is 0, whose twiddles come from
// line layer 1 (circle_tw); otherwise layer0 >= 1.
template <bool CIRCLE>
__device__ __forceinline__ void stage_tws10(const FftPass& p, uint64_t hi, uint32_t* tws) {
  const uint32_t* tail = p.tree + p.tree_len;  // tree layer L starts 2^(N - L) words before the end
  const uint32_t N = p.log_domain, L0 = CIRCLE ? 0u : p.layer0, t = threadIdx.x;
  uint32_t val[4];
  const uint64_t h0 = (hi << 9) + t;
  if (CIRCLE) {
    const uint32_t* lt0 = tail - (1ull << (N - 1));
    val[0] = circle_tw(lt0, h0);
    val[1] = circle_tw(lt0, h0 + 256);
  } else {
    const uint32_t* l0 = tail - (1ull << (N - L0)) + h0;
    val[0] = __ldg(l0);
    val[1] = __ldg(l0 + 256);
  }
  val[2] = __ldg(tail - (1ull << (N - L0 - 1)) + (hi << 8) + t);
  const uint32_t u = 255u - t;  // 1023 - slot
  val[3] = 0;
  if (u != 0) {
    const uint32_t lam = __clz(u) - 22;
    const uint64_t h = (hi << (9 - lam)) + (768u + t - (1024u - (1024u >> lam)));
    val[3] = __ldg(tail - (1ull << (N - L0 - lam)) + h);
  }
  tws[t] = val[0] << 1;
  tws[t + 256] = val[1] << 1;
  tws[t + 512] = val[2] << 1;
  if (u != 0) tws[t + 768] = val[3] << 1;
}

// Staged column tile of the contiguous pass: word e of the 1024 at
// (e >> 5) * kTileStride + (e & 31).  Lines of 36 words keep every 16-byte
// chunk aligned for cp.async, and both register layouts read conflict-free:
// lane-major (lane l takes words 32l..32l+31 as 8 x 16 bytes; 8 lanes of a
// quarter-warp cover banks 4l + 4q .. +3, all distinct) and row-major (lane l
// takes word 32j + l: 32 consecutive words).
constexpr uint32_t kTileStride = 36;
constexpr uint32_t kTileWords = 32 * kTileStride;

__device__ __forceinline__ void cp_async16(uint32_t* dst, const uint32_t* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}

// Copies the 1024 words at src (16-byte aligned) into a staged tile; one
// commit group per tile.
__device__ __forceinline__ void tile_prefetch(const uint32_t* __restrict__ src, uint32_t* buf, uint32_t lane) {
#pragma unroll
  for (int i = 0; i < 8; i++) {
    const uint32_t k = lane + 32u * i;  // 16-byte chunk
    cp_async16(buf + (k >> 3) * kTileStride + (k & 7) * 4, src + 4 * k);
  }
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
__device__ __forceinline__ void tile_wait() {
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
  __syncwarp();
}
// Bulk store of one staged-tile line (32 words, written by this thread) to
// 128 bytes of global memory; the fence makes the thread's shared-memory
// writes visible to the bulk copy.
__device__ __forceinline__ void line_bulk_store(uint32_t* gdst, const uint32_t* line) {
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], 128;\n" ::"l"(gdst), "r"(smem_addr(line))
               : "memory");
  asm volatile("cp.async.bulk.commit_group;\n" ::: "memory");
}
// This thread's bulk stores have read their shared-memory source / are done.
__device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory"); }
// Tile position hi of a natural-order column of 2^log_n words (log_n >= 10)
// staged in bit-reversed order, which fuses ColumnOps::bit_reverse_column
// (prover/backend/simd/bit_reverse.rs:21-33) into the first pass: word e of
// the tile is src[rev10(e) * 2^(log_n-10) + rev(hi)].  Lane l copies words
// 32 i + l with 4-byte cp.async; each 32-byte sector holds one word of 8
// tile positions, which read it through L2.  One commit group per tile.
__device__ __forceinline__ void tile_gather_natural(const uint32_t* __restrict__ src, uint32_t log_n, uint64_t hi,
                                                    uint32_t* buf, uint32_t lane) {
  const uint32_t sh = log_n - 10;
  const uint64_t rh = sh ? __brevll(hi) >> (64 - sh) : 0;
#pragma unroll 8
  for (int i = 0; i < 32; i++) {
    const uint32_t e = 32u * i + lane;
    const uint64_t g = ((uint64_t)(__brev(e) >> 22) << sh) | rh;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(smem_addr(buf + i * kTileStride + lane)),
                 "l"(src + g)
                 : "memory");
  }
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
__device__ __forceinline__ void tile_to_lane_major(const uint32_t* buf, uint32_t lane, uint32_t (&v)[32]) {
#pragma unroll
  for (int q = 0; q < 8; q++) {
    const uint4 w = *reinterpret_cast<const uint4*>(buf + lane * kTileStride + 4 * q);
    v[4 * q] = w.x;
    v[4 * q + 1] = w.y;
    v[4 * q + 2] = w.z;
    v[4 * q + 3] = w.w;
  }
}
__device__ __forceinline__ void lane_major_to_tile(uint32_t* buf, uint32_t lane, const uint32_t (&v)[32]) {
#pragma unroll
  for (int q = 0; q < 8; q++)
    *reinterpret_cast<uint4*>(buf + lane * kTileStride + 4 * q) =
        make_uint4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
}

// Contiguous pass (layer0 = 0, C = 0): warp w transforms 1024 consecutive
// words of column g * kWarpCols + w for p.cpb column groups g of one tile
// position, whose twiddles the block stages once.  No block barrier after
// the staging.  Needs 16-byte aligned columns and no source masking.
//   Inverse: each warp streams its tiles through its own staged tile with
// cp.async (the next tile's copy is issued as soon as the transpose has
// freed the buffer, so it lands during the second half of the butterflies
// and the stores), runs layers 0..4 lane-major, 5..9 row-major and stores
// row-major (128 contiguous bytes per instruction).  With p.natural (source
// distinct from destination) the tiles are gathered from a natural-order
// source instead.
//   Forward: each warp loads its tile row-major straight from global memory
// (128 contiguous bytes per instruction), runs layers 9..5, turns the tile
// lane-major through its staged tile, runs layers 4..0 and writes the lane's
// 32 consecutive words back into its own line of the staged tile, from
// where one 128-byte bulk copy per lane stores it.
//   T < 10 (6..9): a pass of T layers.  The 1024 words are 2^(10-T) tiles of
// the pass side by side; layer lam < T pairs the same words and takes the
// same twiddle (word >> (lam + 1) of the layer) as in the 10-layer pass, so
// the kernel runs only the row-major layers 5..T-1.
template <bool INV, int T>
__global__ void __launch_bounds__(256, 4) fft_warp_contig_kernel(FftPass p, FftCols cols) {
  extern __shared__ __align__(16) uint32_t smem[];
  uint32_t* tws = smem;
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint32_t* buf = smem + 1024 + warp * kTileWords;
  const uint64_t hi = (uint64_t)p.tile0 + blockIdx.x;
  const uint64_t base = hi << 10;
  const uint32_t g0 = blockIdx.y * p.cpb;
  uint32_t c = g0 * kWarpCols + warp;
  const bool natural = p.natural != 0;
  if (INV && c < p.n_cols) {
    if (natural)
      tile_gather_natural(cols.src[c], p.log_domain, hi, buf, lane);
    else
      tile_prefetch(cols.src[c] + base, buf, lane);
  }
  stage_tws10<true>(p, hi, tws);
  __syncthreads();
  const uint32_t scale = p.scale;
  for (uint32_t g = 0; g < p.cpb; g++, c += kWarpCols) {
    if (c >= p.n_cols) break;  // no block barrier follows
    uint32_t* __restrict__ dst = cols.dst[c];
    uint32_t v[32];
    if (INV) {
      const uint32_t cn = c + kWarpCols;
      const bool more = g + 1 < p.cpb && cn < p.n_cols;
      tile_wait();
      tile_to_lane_major(buf, lane, v);
      warp_phase_lo<true>(v, tws, lane);
      lane_major_to_tile(buf, lane, v);
      __syncwarp();
#pragma unroll
      for (int j = 0; j < 32; j++) v[j] = buf[j * kTileStride + lane];
      __syncwarp();
      if (more) {
        if (natural)
          tile_gather_natural(cols.src[cn], p.log_domain, hi, buf, lane);
        else
          tile_prefetch(cols.src[cn] + base, buf, lane);
      }
      warp_phase_hi_short<true, T>(v, tws);
#pragma unroll
      for (int j = 0; j < 32; j++) dst[base + j * 32 + lane] = scale != 1u ? m31_mul(v[j], scale) : v[j];
    } else {
      const uint32_t* __restrict__ sp = cols.src[c] + base + lane;
#pragma unroll
      for (int j = 0; j < 32; j++) v[j] = __ldg(sp + 32 * j);
      warp_phase_hi_short<false, T>(v, tws);
      bulk_wait_read();  // the previous tile's bulk stores have read this warp's lines
      __syncwarp();
#pragma unroll
      for (int j = 0; j < 32; j++) buf[j * kTileStride + lane] = v[j];
      __syncwarp();
      tile_to_lane_major(buf, lane, v);
      warp_phase_lo<false>(v, tws, lane);
      if (scale != 1u) {
#pragma unroll
        for (int j = 0; j < 32; j++) v[j] = m31_mul(v[j], scale);
      }
      lane_major_to_tile(buf, lane, v);  // the lane's own line, read just above
      line_bulk_store(dst + base + 32 * lane, buf + lane * kTileStride);
    }
  }
  if (!INV) bulk_wait_all();
}

// Strided pass (C = 3, layer0 >= 3): a block transforms the 8 adjacent
// columns of one tile position, 1024 rows x 8 words (each row one 32-byte
// sector).  Thread (warp w, lane l) works on tile column c = l & 7 with
// m = 4 w + (l >> 3):
//   lane-major: rows 32 m + j (j = 0..31), layers 0..4 of the tile;
//   row-major:  rows 32 j + m, layers 5..9.
// In either layout the 8 lanes of a quarter-warp read or write one whole row
// (a full sector) per instruction, so global memory is read and written
// straight from registers; the one change of layout between the two halves
// goes through shared memory.  Word (r, c) of the exchange tile sits at
// (r + (r >> 5)) * 8 + c: both layouts then touch 32 distinct banks per
// instruction.
constexpr uint32_t kXchWords = (1024 + 32) * 8;
__device__ __forceinline__ uint32_t xch_pos(uint32_t r, uint32_t c) { return (r + (r >> 5)) * 8 + c; }

// A power-of-two source mask that covers every row and column bit of the
// tile (the duplicated coefficients of a blowup evaluation) only changes the
// tile base.
__host__ __device__ __forceinline__ bool strided_mask_on_span(uint64_t mask, uint64_t len, uint32_t span_log) {
  return (mask == ~0ull && len == ~0ull) ||
         (mask != ~0ull && ((mask + 1) & mask) == 0 && mask + 1 >= (1ull << span_log) && len > mask);
}
__host__ __device__ __forceinline__ bool strided_mask_on_base(uint64_t mask, uint64_t len, uint32_t L0) {
  return strided_mask_on_span(mask, len, L0 + 10);
}

// L0T != 0 fixes layer0 at compile time (the row stride 2^L0T words): the
// 32 loads and stores of a thread then address one base register with
// immediate offsets (up to 31 x 2^(L0T+5) words: within the 24-bit signed
// offset of global accesses for L0T <= 11, half of them for L0T = 12).  Those instances take only
// sources whose mask acts on the tile base (checked by the launcher);
// L0T = 0 takes any layer0 and mask.
template <bool INV, int L0T>
__global__ void __launch_bounds__(256, 4) fft_warp_strided_kernel(FftPass p, FftCols cols) {
  extern __shared__ __align__(16) uint32_t smem[];
  uint32_t* tws = smem;
  uint32_t* xch = smem + 1024;
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t c = lane & 7, m = (threadIdx.x >> 5) * 4 + (lane >> 3);
  const uint32_t L0 = L0T ? (uint32_t)L0T : p.layer0;
  const uint64_t t = (uint64_t)p.tile0 + blockIdx.x;
  const uint32_t lo_bits = L0 - 3;
  const uint64_t lo = t & ((1ull << lo_bits) - 1);
  const uint64_t hi = t >> lo_bits;
  const uint64_t base = (hi << (L0 + 10)) | (lo << 3);
  const uint32_t* __restrict__ src = cols.src[blockIdx.y];
  // Rows held in the layout the pass starts from: lane-major for the
  // inverse transform, row-major for the forward one.
  const uint32_t r0 = INV ? 32 * m : m, rs = INV ? 1 : 32;
  uint32_t v[32];
  if (L0T != 0 || strided_mask_on_base(p.src_mask, p.src_len, L0)) {
    const uint32_t* __restrict__ sp = src + (base & p.src_mask) + c + ((uint64_t)r0 << L0);
#pragma unroll
    for (int j = 0; j < 32; j++) v[j] = __ldg(sp + ((uint64_t)(rs * j) << L0));
  } else {
#pragma unroll
    for (int j = 0; j < 32; j++) {
      const uint64_t gi = (base + ((uint64_t)(r0 + rs * j) << L0) + c) & p.src_mask;
      v[j] = gi < p.src_len ? __ldg(src + gi) : 0u;
    }
  }
  stage_tws10<false>(p, hi, tws);
  __syncthreads();
  if (INV) {
    warp_phase_lo<true>(v, tws, m);
#pragma unroll
    for (int j = 0; j < 32; j++) xch[xch_pos(32 * m + j, c)] = v[j];
    __syncthreads();
#pragma unroll
    for (int j = 0; j < 32; j++) v[j] = xch[xch_pos(32 * j + m, c)];
    warp_phase_hi<true>(v, tws);
  } else {
    warp_phase_hi<false>(v, tws);
#pragma unroll
    for (int j = 0; j < 32; j++) xch[xch_pos(32 * j + m, c)] = v[j];
    __syncthreads();
#pragma unroll
    for (int j = 0; j < 32; j++) v[j] = xch[xch_pos(32 * m + j, c)];
    warp_phase_lo<false>(v, tws, m);
  }
  // Stores in the layout the pass ends in: row-major for the inverse
  // transform, lane-major for the forward one.
  const uint32_t scale = p.scale;
  uint32_t* __restrict__ dp = cols.dst[blockIdx.y] + base + c + ((uint64_t)(INV ? m : 32 * m) << L0);
#pragma unroll
  for (int j = 0; j < 32; j++)
    dp[(uint64_t)((INV ? 32 : 1) * j) << L0] = scale != 1u ? m31_mul(v[j], scale) : v[j];
}

// Strided passes of T = 6..9 layers (layer0 = L0, L0 + T >= 13) on the
// thread layout of fft_warp_strided_kernel.  A block again covers 8 adjacent
// columns x 1024 tile rows, but tile row r = r_hi 2^T + r_lo is row r_lo of
// the pass (stride 2^L0 words) in the 8-column group r_hi above the first
// (offset 8 r_hi words): 2^(10-T) tiles of the pass side by side.  Layers
// 0..4 run lane-major and layers 5..T-1 row-major, as in the 10-layer pass.
// A layer's twiddles depend on r_lo and the tile position, not on r_hi, so
// the block stages each layer's table replicated over r_hi and the lookups
// index r >> (lam + 1) unchanged.  Tile position: global words
// (hi << (L0 + T)) | (lo << (13 - T)), lo < 2^(L0 + T - 13).  Sources whose
// mask acts on the tile base only (checked by the launcher).
template <int T>
__device__ __forceinline__ uint64_t short_row_off(uint32_t r, uint32_t L0) {
  return ((uint64_t)(r & ((1u << T) - 1)) << L0) + ((uint64_t)(r >> T) << 3);
}
// The tables of layers 0..T-1 in the slots of stage_tws10 (layer lam at
// 1024 - 2^(10 - lam), 2^(9 - lam) entries), entry e holding twiddle
// (hi << (T - 1 - lam)) + (e mod 2^(T - 1 - lam)) of tree layer L0 + lam,
// doubled.  All loads before any store.
template <int T>
__device__ __forceinline__ void stage_tws_short(const FftPass& p, uint32_t L0, uint64_t hi, uint32_t* tws) {
  const uint32_t* tail = p.tree + p.tree_len;
  const uint32_t N = p.log_domain, t = threadIdx.x;
  uint32_t val[4];
#pragma unroll
  for (int k = 0; k < 4; k++) {
    const uint32_t sl = t + 256u * k;
    const uint32_t lam = sl < 1023u ? __clz(1023u - sl) - 22 : 10u;
    val[k] = 0;
    if (lam < (uint32_t)T) {
      const uint32_t e = sl - (1024u - (1024u >> lam));
      const uint64_t idx = (hi << (T - 1 - lam)) + (e & ((1u << (T - 1 - lam)) - 1));
      val[k] = __ldg(tail - (1ull << (N - L0 - lam)) + idx);
    }
  }
#pragma unroll
  for (int k = 0; k < 4; k++) {
    const uint32_t sl = t + 256u * k;
    if (sl < 1023u && __clz(1023u - sl) - 22 < (uint32_t)T) tws[sl] = val[k] << 1;
  }
}
template <bool INV, int T, int L0T>
__global__ void __launch_bounds__(256, 4) fft_warp_strided_short_kernel(FftPass p, FftCols cols) {
  extern __shared__ __align__(16) uint32_t smem[];
  uint32_t* tws = smem;
  uint32_t* xch = smem + 1024;
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t c = lane & 7, m = (threadIdx.x >> 5) * 4 + (lane >> 3);
  const uint32_t L0 = L0T ? (uint32_t)L0T : p.layer0;
  const uint64_t t = blockIdx.x;
  const uint32_t lo_bits = L0 + T - 13;
  const uint64_t lo = t & ((1ull << lo_bits) - 1);
  const uint64_t hi = t >> lo_bits;
  const uint64_t base = (hi << (L0 + T)) | (lo << (13 - T));
  // Rows held in the layout the pass starts from: lane-major (32 m + j) for
  // the inverse transform, row-major (32 j + m) for the forward one.  With
  // T >= 5, row 32 m + j lies at short_row_off(32 m) + (j << L0), and row
  // 32 j + m at (m << L0) + short_row_off(32 j).
  uint32_t v[32];
  {
    const uint32_t* __restrict__ sp = cols.src[blockIdx.y] + (base & p.src_mask) + c;
    if (INV) {
      sp += short_row_off<T>(32 * m, L0);
#pragma unroll
      for (int j = 0; j < 32; j++) v[j] = __ldg(sp + ((uint64_t)j << L0));
    } else {
      sp += (uint64_t)m << L0;
#pragma unroll
      for (int j = 0; j < 32; j++) v[j] = __ldg(sp + short_row_off<T>(32 * j, L0));
    }
  }
  stage_tws_short<T>(p, L0, hi, tws);
  __syncthreads();
  if (INV) {
    warp_phase_lo<true>(v, tws, m);
#pragma unroll
    for (int j = 0; j < 32; j++) xch[xch_pos(32 * m + j, c)] = v[j];
    __syncthreads();
#pragma unroll
    for (int j = 0; j < 32; j++) v[j] = xch[xch_pos(32 * j + m, c)];
    warp_phase_hi_short<true, T>(v, tws);
  } else {
    warp_phase_hi_short<false, T>(v, tws);
#pragma unroll
    for (int j = 0; j < 32; j++) xch[xch_pos(32 * j + m, c)] = v[j];
    __syncthreads();
#pragma unroll
    for (int j = 0; j < 32; j++) v[j] = xch[xch_pos(32 * m + j, c)];
    warp_phase_lo<false>(v, tws, m);
  }
  // Stores in the layout the pass ends in: row-major for the inverse
  // transform, lane-major for the forward one.
  const uint32_t scale = p.scale;
  uint32_t* __restrict__ dp = cols.dst[blockIdx.y] + base + c;
  if (INV) {
    dp += (uint64_t)m << L0;
#pragma unroll
    for (int j = 0; j < 32; j++) dp[short_row_off<T>(32 * j, L0)] = scale != 1u ? m31_mul(v[j], scale) : v[j];
  } else {
    dp += short_row_off<T>(32 * m, L0);
#pragma unroll
    for (int j = 0; j < 32; j++) dp[(uint64_t)j << L0] = scale != 1u ? m31_mul(v[j], scale) : v[j];
  }
}

// The last pass of an interpolation fused with the first pass of the
// evaluation on the 2^b times larger domain that follows it (interpolate,
// then evaluate_into with the coefficients duplicated onto the 2^b
// subdomains, prover/backend/simd/circle.rs:138-166,413-440).  Both are
// 10-layer strided passes over the same tiles: layers L0..L0+9 of the 2^(L0+10)
// interpolation (one tile position hi = 0) and of the 2^(L0+10+b) evaluation
// (tile positions hi < 2^b, all reading the same coefficient tile).  A block
// loads its tile of the interpolation's intermediate (lane-major), finishes
// the inverse layers, stores the coefficients in place (row-major) and then,
// for each hi, runs the forward layers from them and stores that tile of the
// evaluation (lane-major).  hi = 0 starts from the coefficients in registers;
// the later ones re-read the thread's own stores through L2.  Thread layout,
// exchange tile and twiddle tables are those of fft_warp_strided_kernel; the
// forward tables of all 2^b positions are staged with the inverse one.
// Launched at b = 1 (interpolate_evaluate).
struct FftColsIE {
  uint32_t* coef[kFftMaxCols];  // interpolation intermediate in, coefficients out
  uint32_t* eval[kFftMaxCols];  // evaluation (2^b times longer) out
};
template <int L0T>
__global__ void __launch_bounds__(256, 4) fft_warp_inv_fwd_kernel(FftPass pi, FftPass pf, FftColsIE cols,
                                                                 uint32_t n_hi) {
  extern __shared__ __align__(16) uint32_t smem[];
  uint32_t* twi = smem;
  uint32_t* xch = smem + 1024;
  uint32_t* twf = xch + kXchWords;  // n_hi tables of 1024
  constexpr uint32_t L0 = L0T;
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t c = lane & 7, m = (threadIdx.x >> 5) * 4 + (lane >> 3);
  const uint64_t base = ((uint64_t)blockIdx.x << 3) + c;
  uint32_t* __restrict__ coef = cols.coef[blockIdx.y] + base;
  uint32_t* __restrict__ ev = cols.eval[blockIdx.y] + base;
  uint32_t v[32];
  {
    const uint32_t* __restrict__ sp = coef + ((uint64_t)(32 * m) << L0);
#pragma unroll
    for (int j = 0; j < 32; j++) v[j] = __ldg(sp + ((uint64_t)j << L0));
  }
  stage_tws10<false>(pi, 0, twi);
  for (uint32_t h = 0; h < n_hi; h++) stage_tws10<false>(pf, h, twf + 1024 * h);
  __syncthreads();
  warp_phase_lo<true>(v, twi, m);
#pragma unroll
  for (int j = 0; j < 32; j++) xch[xch_pos(32 * m + j, c)] = v[j];
  __syncthreads();
#pragma unroll
  for (int j = 0; j < 32; j++) v[j] = xch[xch_pos(32 * j + m, c)];
  warp_phase_hi<true>(v, twi);
  uint32_t* __restrict__ cp = coef + ((uint64_t)m << L0);
  const uint32_t scale = pi.scale;
#pragma unroll
  for (int j = 0; j < 32; j++) {
    v[j] = m31_mul(v[j], scale);
    cp[(uint64_t)(32 * j) << L0] = v[j];
  }
  for (uint32_t h = 0; h < n_hi; h++) {
    if (h > 0) {
#pragma unroll
      for (int j = 0; j < 32; j++) v[j] = __ldcg(cp + ((uint64_t)(32 * j) << L0));
    }
    const uint32_t* tw = twf + 1024 * h;
    __syncthreads();  // every thread has read its words of the previous exchange
    warp_phase_hi<false>(v, tw);
#pragma unroll
    for (int j = 0; j < 32; j++) xch[xch_pos(32 * j + m, c)] = v[j];
    __syncthreads();
#pragma unroll
    for (int j = 0; j < 32; j++) v[j] = xch[xch_pos(32 * m + j, c)];
    warp_phase_lo<false>(v, tw, m);
    uint32_t* __restrict__ dp = ev + ((uint64_t)h << (L0 + 10)) + ((uint64_t)(32 * m) << L0);
#pragma unroll
    for (int j = 0; j < 32; j++) dp[(uint64_t)j << L0] = v[j];
  }
}

// ---- contiguous passes of 11 and 12 layers (T = 10 + K) ----
// A group of 2^K warps owns one 2^T-row column tile, 32 values per thread,
// in three layouts (q: the warp's 1024-row quarter of the tile, l: lane):
//   lane-major (layers 0..4):    rows 1024 q + 32 l + j           (v[j]);
//   row-major  (layers 5..9):    rows 1024 q + 32 j + l           (v[j]);
//   top        (layers 10..T-1): rows 1024 k + 32 (q I + i) + l   (v[k I + i]),
//                                k < 2^K, i < I = 32 >> K.
// Each addresses the group's staged tile (row r at (r >> 5) * kTileStride +
// (r & 31)) without bank conflicts.  Lane-major <-> row-major stays inside a
// warp (its own quarter, as in the 10-layer pass); row-major <-> top crosses
// the group's warps through a named barrier of the group.  The inverse pass
// streams its quarter in with cp.async and stores the top layout (128
// contiguous bytes per instruction); the forward pass loads the top layout
// straight from global memory and stores each lane's line with a bulk copy.

// Layers 5..9 of a 2^T-row tile on v[j] = row 1024 q + 32 j + l:
// row >> (lam + 1) = (q << (9 - lam)) + (j >> (lam - 4)).
template <bool INV, int T>
__device__ __forceinline__ void group_phase_hi(uint32_t (&v)[32], const uint32_t* __restrict__ tws, uint32_t q) {
#pragma unroll
  for (int kk = 0; kk < 5; kk++) {
    const int k = INV ? kk : 4 - kk;  // bit of j, layer 5 + k
    const uint32_t* tl = tws + ((1u << T) - (1u << (T - 5 - k))) + (q << (4 - k));
    uint32_t t[16];
#pragma unroll
    for (int m = 0; m < (1 << (4 - k)); m++) t[m] = tl[m];
#pragma unroll
    for (int j = 0; j < 32; j++) {
      if (j & (1 << k)) continue;
      if (INV)
        ibfly2(v[j], v[j | (1 << k)], t[j >> (k + 1)]);
      else
        bfly2(v[j], v[j | (1 << k)], t[j >> (k + 1)]);
    }
  }
}
// Layers 0..4 on v[j] = row 32 b + j of a 2^T-row tile.
template <bool INV, int T>
__device__ __forceinline__ void group_phase_lo(uint32_t (&v)[32], const uint32_t* __restrict__ tws, uint32_t b) {
#pragma unroll
  for (int kk = 0; kk < 5; kk++) {
    const int lam = INV ? kk : 4 - kk;
    const uint32_t* tl = tws + ((1u << T) - (1u << (T - lam))) + (b << (4 - lam));
    uint32_t t[16];
#pragma unroll
    for (int m = 0; m < (1 << (4 - lam)); m++) t[m] = tl[m];
#pragma unroll
    for (int j = 0; j < 32; j++) {
      if (j & (1 << lam)) continue;
      if (INV)
        ibfly2(v[j], v[j | (1 << lam)], t[j >> (lam + 1)]);
      else
        bfly2(v[j], v[j | (1 << lam)], t[j >> (lam + 1)]);
    }
  }
}
// Layers 10..T-1 on the top layout: layer 10 + kk pairs k and k | 2^kk, with
// row >> (11 + kk) = k >> (kk + 1).
template <bool INV, int K>
__device__ __forceinline__ void group_phase_top(uint32_t (&v)[32], const uint32_t* __restrict__ tws) {
  constexpr int T = 10 + K, I = 32 >> K;
#pragma unroll
  for (int k0 = 0; k0 < K; k0++) {
    const int kk = INV ? k0 : K - 1 - k0;
    const uint32_t* tl = tws + ((1u << T) - (1u << (T - 10 - kk)));
#pragma unroll
    for (int k = 0; k < (1 << K); k++) {
      if (k & (1 << kk)) continue;
      const uint32_t t = tl[k >> (kk + 1)];
#pragma unroll
      for (int i = 0; i < I; i++) {
        if (INV)
          ibfly2(v[k * I + i], v[(k | (1 << kk)) * I + i], t);
        else
          bfly2(v[k * I + i], v[(k | (1 << kk)) * I + i], t);
      }
    }
  }
}
// The 2^T - 1 twiddles of a contiguous T-layer tile position (layer0 = 0),
// doubled, in the slot order of stage_tws10: layer lam at 2^T - 2^(T - lam),
// 2^(T-1-lam) entries; layer 0 (the circle layer) from line layer 1.
template <int T>
__device__ __forceinline__ void stage_tws_contig(const FftPass& p, uint64_t hi, uint32_t* tws) {
  const uint32_t* tail = p.tree + p.tree_len;
  const uint32_t N = p.log_domain, t = threadIdx.x;
  {
    constexpr uint32_t R = (1u << (T - 1)) / 256;
    const uint32_t* lt0 = tail - (1ull << (N - 1));
    uint32_t val[R];
#pragma unroll
    for (uint32_t r = 0; r < R; r++) val[r] = circle_tw(lt0, (hi << (T - 1)) + t + 256 * r);
#pragma unroll
    for (uint32_t r = 0; r < R; r++) tws[t + 256 * r] = val[r] << 1;
  }
#pragma unroll
  for (int lam = 1; lam < T; lam++) {
    const uint32_t cnt = 1u << (T - 1 - lam), off = (1u << T) - (1u << (T - lam));
    const uint32_t* l = tail - (1ull << (N - lam)) + (hi << (T - 1 - lam));
#pragma unroll
    for (uint32_t e = 0; e < cnt; e += 256)
      if (e + t < cnt) tws[off + e + t] = __ldg(l + e + t) << 1;
  }
}
// Named barrier 1 + grp of the n_threads threads of group grp (< 4; barrier 0
// is the block's).  Immediate ids, so that a block holds 5 barriers.
__device__ __forceinline__ void group_barrier(uint32_t grp, uint32_t n_threads) {
  switch (grp) {
    case 0: asm volatile("bar.sync 1, %0;\n" ::"r"(n_threads) : "memory"); break;
    case 1: asm volatile("bar.sync 2, %0;\n" ::"r"(n_threads) : "memory"); break;
    case 2: asm volatile("bar.sync 3, %0;\n" ::"r"(n_threads) : "memory"); break;
    default: asm volatile("bar.sync 4, %0;\n" ::"r"(n_threads) : "memory"); break;
  }
}

template <bool INV, int K>
__global__ void __launch_bounds__(256, 4) fft_group_contig_kernel(FftPass p, FftCols cols) {
  constexpr int T = 10 + K;
  constexpr uint32_t W = 1u << K, G = 8u / W, I = 32u >> K;
  constexpr uint32_t kLines = 1u << (T - 5);
  extern __shared__ __align__(16) uint32_t smem[];
  uint32_t* tws = smem;
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t grp = warp / W, q = warp % W;
  uint32_t* buf = smem + (1u << T) + grp * kLines * kTileStride;
  uint32_t* qb = buf + 32 * q * kTileStride;  // the warp's quarter: 32 lines
  const uint64_t hi = (uint64_t)p.tile0 + blockIdx.x;
  const uint64_t base = hi << T;
  // group grp transforms columns (blockIdx.y * cpb + g) * G + grp, g < cpb,
  // of this tile position with the twiddles staged once
  uint32_t c = blockIdx.y * p.cpb * G + grp;
  uint32_t v[32];
  auto load_top = [&](uint32_t col) {
    const uint32_t* __restrict__ sp = cols.src[col] + base + 32 * (q * I) + lane;
#pragma unroll
    for (uint32_t k = 0; k < W; k++)
#pragma unroll
      for (uint32_t i = 0; i < I; i++) v[k * I + i] = __ldg(sp + 1024 * k + 32 * i);
  };
  if (INV && c < p.n_cols) tile_prefetch(cols.src[c] + base + 1024 * q, qb, lane);
  stage_tws_contig<T>(p, hi, tws);
  __syncthreads();
  const uint32_t n_bar = 32 * W;
  const uint32_t scale = p.scale;
  // c is uniform over a group: whole groups leave, the barriers below are per group
  for (uint32_t g = 0; g < p.cpb && c < p.n_cols; g++, c += G) {
    const uint32_t cn = c + G;
    const bool more = g + 1 < p.cpb && cn < p.n_cols;
    if (INV) {
      tile_wait();
      tile_to_lane_major(qb, lane, v);
      group_phase_lo<true, T>(v, tws, 32 * q + lane);
      lane_major_to_tile(qb, lane, v);
      __syncwarp();
#pragma unroll
      for (int j = 0; j < 32; j++) v[j] = qb[j * kTileStride + lane];
      group_phase_hi<true, T>(v, tws, q);
#pragma unroll
      for (int j = 0; j < 32; j++) qb[j * kTileStride + lane] = v[j];
      group_barrier(grp, n_bar);
#pragma unroll
      for (uint32_t k = 0; k < W; k++)
#pragma unroll
        for (uint32_t i = 0; i < I; i++) v[k * I + i] = buf[(32 * k + q * I + i) * kTileStride + lane];
      if (more) {
        group_barrier(grp, n_bar);  // every warp has read its top rows out of the quarters
        tile_prefetch(cols.src[cn] + base + 1024 * q, qb, lane);
      }
      group_phase_top<true, K>(v, tws);
      uint32_t* __restrict__ dp = cols.dst[c] + base + 32 * (q * I) + lane;
#pragma unroll
      for (uint32_t k = 0; k < W; k++)
#pragma unroll
        for (uint32_t i = 0; i < I; i++) {
          const uint32_t x = v[k * I + i];
          dp[1024 * k + 32 * i] = scale != 1u ? m31_mul(x, scale) : x;
        }
    } else {
      load_top(c);
      group_phase_top<false, K>(v, tws);
      if (g > 0) {
        bulk_wait_read();  // this warp's bulk stores of the previous column have read its lines
        group_barrier(grp, n_bar);
      }
#pragma unroll
      for (uint32_t k = 0; k < W; k++)
#pragma unroll
        for (uint32_t i = 0; i < I; i++) buf[(32 * k + q * I + i) * kTileStride + lane] = v[k * I + i];
      group_barrier(grp, n_bar);
#pragma unroll
      for (int j = 0; j < 32; j++) v[j] = qb[j * kTileStride + lane];
      group_phase_hi<false, T>(v, tws, q);
#pragma unroll
      for (int j = 0; j < 32; j++) qb[j * kTileStride + lane] = v[j];
      __syncwarp();
      tile_to_lane_major(qb, lane, v);
      group_phase_lo<false, T>(v, tws, 32 * q + lane);
      if (scale != 1u) {
#pragma unroll
        for (int j = 0; j < 32; j++) v[j] = m31_mul(v[j], scale);
      }
      lane_major_to_tile(qb, lane, v);  // the lane's own line, read just above
      line_bulk_store(cols.dst[c] + base + 1024 * q + 32 * lane, qb + lane * kTileStride);
    }
  }
  if (!INV) bulk_wait_all();
}

template <bool INV, int K>
static int launch_group_contig(const FftPass& q, const FftCols& cols, uint64_t tiles, size_t nc, cudaStream_t s,
                               char* err, size_t err_len) {
  constexpr int T = 10 + K;
  constexpr uint32_t G = 8u >> K;
  constexpr size_t smem = ((1u << T) + G * (1u << (T - 5)) * kTileStride) * sizeof(uint32_t);
  static std::atomic<uint32_t> attr{0};
  STWO_CUDA_TRY(ensure_smem_limit(fft_group_contig_kernel<INV, K>, (int)smem, attr));
  // up to 16 columns per group: fewer twiddle stagings while the grid still
  // has six waves of blocks
  const uint32_t groups = (uint32_t)((nc + G - 1) / G);
  FftPass qq = q;
  qq.cpb = std::max<uint32_t>(1, std::min<uint32_t>(16, (uint32_t)((tiles * groups) / (148 * 4 * 6))));
  dim3 grid((unsigned)tiles, (unsigned)((groups + qq.cpb - 1) / qq.cpb));
  fft_group_contig_kernel<INV, K><<<grid, 256, smem, s>>>(qq, cols);
  STWO_CHECK_LAUNCH();
  return STWO_B200_OK;
}

// A contiguous pass of T = 6..10 layers over `chunks` 1024-word chunks.
template <bool INV, int T>
static int launch_warp_contig(const FftPass& q, const FftCols& cols, uint64_t chunks, size_t nc, cudaStream_t s,
                              char* err, size_t err_len) {
  constexpr size_t smem = (1024 + kWarpCols * kTileWords) * sizeof(uint32_t);
  static std::atomic<uint32_t> attr{0};
  STWO_CUDA_TRY(ensure_smem_limit(fft_warp_contig_kernel<INV, T>, (int)smem, attr));
  // up to 16 column groups per block: fewer twiddle stagings while the grid
  // still has six waves of blocks
  const uint32_t groups = (uint32_t)((nc + kWarpCols - 1) / kWarpCols);
  FftPass qq = q;
  qq.cpb = std::max<uint32_t>(1, std::min<uint32_t>(16, (uint32_t)((chunks * groups) / (148 * 4 * 6))));
  dim3 grid((unsigned)chunks, (unsigned)((groups + qq.cpb - 1) / qq.cpb));
  fft_warp_contig_kernel<INV, T><<<grid, 32 * kWarpCols, smem, s>>>(qq, cols);
  STWO_CHECK_LAUNCH();
  return STWO_B200_OK;
}

template <bool INV>
static int launch_warp_pass(const FftPass& q, const FftCols& cols, uint64_t tiles, size_t nc, cudaStream_t s,
                            char* err, size_t err_len) {
  if (q.C == 0) {
    switch (q.T) {
      case 6: return launch_warp_contig<INV, 6>(q, cols, tiles >> 4, nc, s, err, err_len);
      case 7: return launch_warp_contig<INV, 7>(q, cols, tiles >> 3, nc, s, err, err_len);
      case 8: return launch_warp_contig<INV, 8>(q, cols, tiles >> 2, nc, s, err, err_len);
      case 9: return launch_warp_contig<INV, 9>(q, cols, tiles >> 1, nc, s, err, err_len);
      default: return launch_warp_contig<INV, 10>(q, cols, tiles, nc, s, err, err_len);
    }
  } else {
    constexpr size_t smem = (1024 + kXchWords) * sizeof(uint32_t);
    static std::atomic<uint32_t> attr10{0}, attr11{0}, attr{0};
    static std::atomic<uint32_t> attr12{0};
    const bool fixed = q.layer0 >= 10 && q.layer0 <= 12 && strided_mask_on_base(q.src_mask, q.src_len, q.layer0);
    dim3 grid((unsigned)tiles, (unsigned)nc);
    if (fixed && q.layer0 == 10) {
      STWO_CUDA_TRY(ensure_smem_limit(fft_warp_strided_kernel<INV, 10>, (int)smem, attr10));
      fft_warp_strided_kernel<INV, 10><<<grid, 256, smem, s>>>(q, cols);
    } else if (fixed && q.layer0 == 11) {
      STWO_CUDA_TRY(ensure_smem_limit(fft_warp_strided_kernel<INV, 11>, (int)smem, attr11));
      fft_warp_strided_kernel<INV, 11><<<grid, 256, smem, s>>>(q, cols);
    } else if (fixed) {
      STWO_CUDA_TRY(ensure_smem_limit(fft_warp_strided_kernel<INV, 12>, (int)smem, attr12));
      fft_warp_strided_kernel<INV, 12><<<grid, 256, smem, s>>>(q, cols);
    } else {
      STWO_CUDA_TRY(ensure_smem_limit(fft_warp_strided_kernel<INV, 0>, (int)smem, attr));
      fft_warp_strided_kernel<INV, 0><<<grid, 256, smem, s>>>(q, cols);
    }
  }
  STWO_CHECK_LAUNCH();
  return STWO_B200_OK;
}

template <bool INV, int T>
static int launch_strided_short_t(const FftPass& q, const FftCols& cols, uint64_t blocks, size_t nc, cudaStream_t s,
                                  char* err, size_t err_len) {
  constexpr size_t smem = (1024 + kXchWords) * sizeof(uint32_t);
  static std::atomic<uint32_t> attr10{0}, attr11{0}, attr{0};
  dim3 grid((unsigned)blocks, (unsigned)nc);
  if (q.layer0 == 10) {
    STWO_CUDA_TRY(ensure_smem_limit(fft_warp_strided_short_kernel<INV, T, 10>, (int)smem, attr10));
    fft_warp_strided_short_kernel<INV, T, 10><<<grid, 256, smem, s>>>(q, cols);
  } else if (q.layer0 == 11) {
    STWO_CUDA_TRY(ensure_smem_limit(fft_warp_strided_short_kernel<INV, T, 11>, (int)smem, attr11));
    fft_warp_strided_short_kernel<INV, T, 11><<<grid, 256, smem, s>>>(q, cols);
  } else {
    STWO_CUDA_TRY(ensure_smem_limit(fft_warp_strided_short_kernel<INV, T, 0>, (int)smem, attr));
    fft_warp_strided_short_kernel<INV, T, 0><<<grid, 256, smem, s>>>(q, cols);
  }
  STWO_CHECK_LAUNCH();
  return STWO_B200_OK;
}

// A whole strided pass of 6..9 layers: 2^(10 - T) of its tiles per block.
template <bool INV>
static int launch_strided_short(const FftPass& q, const FftCols& cols, uint64_t tiles, size_t nc, cudaStream_t s,
                                char* err, size_t err_len) {
  const uint64_t blocks = tiles >> (10 - q.T);
  switch (q.T) {
    case 6: return launch_strided_short_t<INV, 6>(q, cols, blocks, nc, s, err, err_len);
    case 7: return launch_strided_short_t<INV, 7>(q, cols, blocks, nc, s, err, err_len);
    case 8: return launch_strided_short_t<INV, 8>(q, cols, blocks, nc, s, err, err_len);
    default: return launch_strided_short_t<INV, 9>(q, cols, blocks, nc, s, err, err_len);
  }
}

template <bool INV, int T, int C, int CPB>
static int launch_tile(const FftPass& q, const FftCols& cols, dim3 grid, cudaStream_t s, char* err, size_t err_len) {
  constexpr int NT = fft_threads(T, C, CPB);
  constexpr size_t E = (size_t)1 << (T + C);
  constexpr size_t smem = ((size_t)CPB * tile_stride_words(E) + ((size_t)1 << T)) * sizeof(uint32_t);
  static_assert(smem <= 200 * 1024, "FFT tile exceeds shared memory");
  static std::atomic<uint32_t> attr{0};
  STWO_CUDA_TRY(ensure_smem_limit(fft_pass_kernel<INV, T, C, CPB, NT>, (int)smem, attr));
  fft_pass_kernel<INV, T, C, CPB, NT><<<grid, NT, smem, s>>>(q, cols);
  STWO_CHECK_LAUNCH();
  return STWO_B200_OK;
}

template <bool INV, int C, int CPB>
static int dispatch_tile(const FftPass& q, const FftCols& cols, dim3 grid, cudaStream_t s, char* err,
                         size_t err_len) {
  switch (q.T) {
#define STWO_FFT_T(TT) \
  case TT: return launch_tile<INV, TT, C, CPB>(q, cols, grid, s, err, err_len);
    STWO_FFT_T(1) STWO_FFT_T(2) STWO_FFT_T(3) STWO_FFT_T(4) STWO_FFT_T(5) STWO_FFT_T(6)
    STWO_FFT_T(7) STWO_FFT_T(8) STWO_FFT_T(9) STWO_FFT_T(10) STWO_FFT_T(11) STWO_FFT_T(12)
#undef STWO_FFT_T
    default: break;
  }
  return set_err(err, err_len, STWO_B200_EARG, "unsupported FFT pass size T=%u", q.T);
}

// One pass over every tile position, or over tile positions
// [tile0, tile0 + tile_cnt) when tile_cnt != 0.
template <bool INV>
static int launch_pass(const FftPass& p, const std::vector<const uint32_t*>& srcs, const std::vector<uint32_t*>& dsts,
                       uint64_t total_log, cudaStream_t s, char* err, size_t err_len, uint64_t tile0 = 0,
                       uint64_t tile_cnt = 0) {
  const uint64_t all_tiles = 1ull << (total_log - p.T - p.C);
  STWO_ARG_CHECK(tile0 + tile_cnt <= all_tiles && tile0 <= 0xffffffffull, "tile range out of the pass");
  uint64_t tiles = tile_cnt ? tile_cnt : all_tiles;
  size_t E = (size_t)1 << (p.T + p.C);
  STWO_ARG_CHECK(p.C == 0 || p.C == 3, "unsupported FFT tile width");
  // Contiguous passes (small tiles, twiddles as large as the data) share one
  // staged twiddle table between 4 columns of the same tile position.
  const uint32_t cpb = (p.C == 0 && E <= 4096 && srcs.size() >= 4) ? 4u : 1u;
  STWO_ARG_CHECK(tiles <= 0x7fffffffull, "too many tiles");
  for (size_t c0 = 0; c0 < srcs.size(); c0 += kFftMaxCols) {
    FftCols cols;
    size_t nc = std::min<size_t>(kFftMaxCols, srcs.size() - c0);
    bool aligned = true;
    for (size_t i = 0; i < nc; i++) {
      cols.src[i] = srcs[c0 + i];
      cols.dst[i] = dsts[c0 + i];
      aligned = aligned && (reinterpret_cast<uintptr_t>(cols.src[i]) % 16 == 0) &&
                (reinterpret_cast<uintptr_t>(cols.dst[i]) % 16 == 0);
    }
    FftPass q = p;
    q.tile0 = (uint32_t)tile0;
    q.vec_io = aligned && (p.C >= 2 || p.layer0 == 0) && E >= 4 && (p.src_mask & 3) == 3 &&
               (p.src_len == ~0ull || p.src_len % 4 == 0);
    q.cpb = cpb;
    q.n_cols = (uint32_t)nc;
    dim3 grid((unsigned)tiles, (unsigned)((nc + cpb - 1) / cpb));
    int rc;
    // 6..9 layers: whole passes over domains of at least 1024 words (a block
    // covers 2^(10 - T) tiles)
    const bool warp_contig = p.C == 0 && p.layer0 == 0 && aligned && p.src_mask == ~0ull && p.src_len == ~0ull &&
                             (p.T == 10 || (p.T >= 6 && p.T < 10 && total_log >= 10 && p.log_domain >= 10 &&
                                            tile_cnt == 0 && tile0 == 0));
    const bool warp_strided = p.T == 10 && p.C == 3 && p.layer0 >= 3;
    // whole passes only: its blocks cover 2^(10 - T) tiles each
    const bool warp_short = p.C == 3 && p.T >= 6 && p.T <= 9 && p.layer0 + p.T >= 13 && tile_cnt == 0 &&
                            tile0 == 0 && strided_mask_on_span(p.src_mask, p.src_len, p.layer0 + p.T);
    const bool group_contig = (p.T == 11 || p.T == 12) && p.C == 0 && p.layer0 == 0 && aligned && !p.natural &&
                              p.src_mask == ~0ull && p.src_len == ~0ull;
    STWO_ARG_CHECK(!p.natural || (INV && p.C == 0 && p.layer0 == 0 && p.src_mask == ~0ull && p.src_len == ~0ull),
                   "natural-order source needs an unmasked first inverse pass");
    if (warp_contig || warp_strided)
      rc = launch_warp_pass<INV>(q, cols, tiles, nc, s, err, err_len);
    else if (warp_short)
      rc = launch_strided_short<INV>(q, cols, tiles, nc, s, err, err_len);
    else if (group_contig)
      rc = p.T == 11 ? launch_group_contig<INV, 1>(q, cols, tiles, nc, s, err, err_len)
                     : launch_group_contig<INV, 2>(q, cols, tiles, nc, s, err, err_len);
    else if (p.C == 3)
      rc = dispatch_tile<INV, 3, 1>(q, cols, grid, s, err, err_len);
    else if (cpb == 4)
      rc = dispatch_tile<INV, 0, 4>(q, cols, grid, s, err, err_len);
    else
      rc = dispatch_tile<INV, 0, 1>(q, cols, grid, s, err, err_len);
    if (rc) return rc;
  }
  return STWO_B200_OK;
}

}  // namespace stwo_b200

using namespace stwo_b200;

// Bit reversal of columns of one log size, kFftMaxCols per launch: into dst
// (out of place) or in place where dst == src.
static int bit_reverse_group(const uint32_t* const* src, uint32_t* const* dst, uint32_t n_cols, uint32_t lg,
                             cudaStream_t s, char* err, size_t err_len) {
  for (uint32_t a = 0; a < n_cols; a += kFftMaxCols) {
    const uint32_t nc = std::min<uint32_t>(kFftMaxCols, n_cols - a);
    FftCols t;
    for (uint32_t k = 0; k < nc; k++) {
      STWO_ARG_CHECK(src[a + k] && dst[a + k], "null column %u", a + k);
      t.src[k] = src[a + k];
      t.dst[k] = dst[a + k];
    }
    if (lg > 0) {
      const uint64_t n = 1ull << lg;
      const unsigned bx = (unsigned)std::min<uint64_t>((n + 255) / 256, std::max<uint64_t>(1, 148 * 32 / nc));
      bit_reverse_cols_kernel<<<dim3(bx, nc), 256, 0, s>>>(t, lg);
      STWO_CHECK_LAUNCH();
    } else {
      for (uint32_t k = 0; k < nc; k++)
        if (t.src[k] != t.dst[k]) STWO_CUDA_TRY(cudaMemcpyAsync(t.dst[k], t.src[k], 4, cudaMemcpyDeviceToDevice, s));
    }
  }
  return STWO_B200_OK;
}

// natural: the sources are in natural order (CircleEvaluation<_, _,
// NaturalOrder>::bit_reverse, core/poly/circle/evaluation.rs:61-64, before
// the interpolation).  Where every source of a size group is distinct from
// its destination, the bit reversal happens in the loads of the first pass
// (warp or tile form); otherwise (in place, or log size <= 2) one batched
// bit-reversal launch into the destinations precedes the transform.
static int interpolate_impl(const uint32_t* const* d_src, uint32_t* const* d_cols, const uint32_t* log_sizes,
                            const uint64_t* half_initial_indices, uint32_t n_cols, const uint32_t* d_itwiddles,
                            uint32_t tree_log_size, cudaStream_t s, char* err, size_t err_len,
                            bool natural = false) {
  STWO_ARG_CHECK(n_cols == 0 || (d_src && d_cols && log_sizes), "null column arrays");
  // Group columns by log size: one launch per (size, pass).
  std::vector<uint32_t> order(n_cols);
  for (uint32_t i = 0; i < n_cols; i++) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return log_sizes[a] < log_sizes[b]; });
  SmallCols small;
  uint32_t n_small = 0;
  for (size_t a = 0; a < order.size();) {
    uint32_t n = log_sizes[order[a]];
    size_t b = a;
    while (b < order.size() && log_sizes[order[b]] == n) b++;
    STWO_ARG_CHECK(n <= 30, "column log size %u too large", n);
    if (n == 0) {
      a = b;
      continue;
    }
    if (n <= 2) {
      if (natural) {
        std::vector<const uint32_t*> gs;
        std::vector<uint32_t*> gd;
        for (size_t i = a; i < b; i++) {
          gs.push_back(d_src[order[i]]);
          gd.push_back(d_cols[order[i]]);
        }
        int rc = bit_reverse_group(gs.data(), gd.data(), (uint32_t)gs.size(), n, s, err, err_len);
        if (rc) return rc;
      }
      for (size_t i = a; i < b; i++) {
        uint32_t c = order[i];
        uint64_t hi = half_initial_indices ? half_initial_indices[c] : (1ull << (31 - (n + 1)));
        if (n_small == kFftMaxCols) {
          small_fft_kernel<<<1, kFftMaxCols, 0, s>>>(small, n_small, 1);
          STWO_CHECK_LAUNCH();
          n_small = 0;
        }
        small.src[n_small] = natural ? d_cols[c] : d_src[c];
        small.dst[n_small] = d_cols[c];
        index_point(hi, small.x[n_small], small.y[n_small]);
        small.log_src[n_small] = n;
        small.log_dst[n_small] = n;
        n_small++;
      }
      a = b;
      continue;
    }
    STWO_ARG_CHECK(d_itwiddles && n - 1 <= tree_log_size, "twiddle tree (log %u) too small for log size %u",
                   tree_log_size, n);
    std::vector<const uint32_t*> srcs;
    std::vector<uint32_t*> dsts;
    for (size_t i = a; i < b; i++) {
      srcs.push_back(d_src[order[i]]);
      dsts.push_back(d_cols[order[i]]);
    }
    std::vector<const uint32_t*> inplace(dsts.begin(), dsts.end());
    auto plan = plan_passes(n);
    bool fuse = natural;  // the first pass (C = 0, layer 0) gathers, when it does not overwrite its source
    for (size_t i = 0; fuse && i < srcs.size(); i++) fuse = srcs[i] != dsts[i];
    if (natural && !fuse) {
      int rc = bit_reverse_group(srcs.data(), dsts.data(), (uint32_t)srcs.size(), n, s, err, err_len);
      if (rc) return rc;
      srcs = inplace;
    }
    for (size_t pi = 0; pi < plan.size(); pi++) {
      FftPass p;
      p.tree = d_itwiddles;
      p.tree_len = 1ull << tree_log_size;
      p.src_mask = ~0ull;
      p.src_len = ~0ull;
      p.log_domain = n;
      p.layer0 = plan[pi].layer0;
      p.T = plan[pi].T;
      p.C = plan[pi].C;
      p.scale = (pi + 1 == plan.size()) ? host_pow2_inv(n) : 1u;
      p.natural = (pi == 0 && fuse) ? 1u : 0u;
      int rc = launch_pass<true>(p, pi == 0 ? srcs : inplace, dsts, n, s, err, err_len);
      if (rc) return rc;
    }
    a = b;
  }
  if (n_small) {
    small_fft_kernel<<<1, kFftMaxCols, 0, s>>>(small, n_small, 1);
    STWO_CHECK_LAUNCH();
  }
  return ok(err, err_len);
}

extern "C" int stwo_b200_interpolate_columns(uint32_t* const* d_cols, const uint32_t* log_sizes,
                                             const uint64_t* half_initial_indices, uint32_t n_cols,
                                             const uint32_t* d_itwiddles, uint32_t tree_log_size, void* stream,
                                             char* err, size_t err_len) {
  int rc = interpolate_impl(d_cols, d_cols, log_sizes, half_initial_indices, n_cols, d_itwiddles, tree_log_size,
                            as_stream(stream), err, err_len);
  return rc ? rc : ok(err, err_len);
}

extern "C" int stwo_b200_interpolate_columns_into(const uint32_t* const* d_evals, uint32_t* const* d_coeffs,
                                                  const uint32_t* log_sizes, const uint64_t* half_initial_indices,
                                                  uint32_t n_cols, const uint32_t* d_itwiddles,
                                                  uint32_t tree_log_size, void* stream, char* err, size_t err_len) {
  int rc = interpolate_impl(d_evals, d_coeffs, log_sizes, half_initial_indices, n_cols, d_itwiddles, tree_log_size,
                            as_stream(stream), err, err_len);
  return rc ? rc : ok(err, err_len);
}

extern "C" int stwo_b200_interpolate_columns_natural(const uint32_t* const* d_natural, uint32_t* const* d_coeffs,
                                                     const uint32_t* log_sizes, const uint64_t* half_initial_indices,
                                                     uint32_t n_cols, const uint32_t* d_itwiddles,
                                                     uint32_t tree_log_size, void* stream, char* err, size_t err_len) {
  int rc = interpolate_impl(d_natural, d_coeffs, log_sizes, half_initial_indices, n_cols, d_itwiddles, tree_log_size,
                            as_stream(stream), err, err_len, true);
  return rc ? rc : ok(err, err_len);
}

namespace stwo_b200 {

std::vector<uint32_t> fft_split(uint32_t log_n) { return split_for(log_n); }

// Pass `pi` of the interpolation (the inverse transform) of same-size columns
// of 2^log_n bit-reversed evaluations, in place, under the pass split
// `split` (fft_split, fetched once by the caller so that both halves of a
// split transform use the same plan).  For pi = 0 only the rows
// [row_begin, row_end) are transformed: whole tiles of the first pass, whose
// 2^split[0] rows are consecutive; the later passes take every row.
int interpolate_pass(uint32_t* const* cols, uint32_t n_cols, uint32_t log_n, const std::vector<uint32_t>& split,
                     uint32_t pi, uint64_t row_begin, uint64_t row_end, const uint32_t* d_itwiddles,
                     uint32_t tree_log_size, cudaStream_t s, char* err, size_t err_len, const uint32_t* const* src) {
  STWO_ARG_CHECK(log_n >= 3 && log_n <= 30 && pi < split.size(), "interpolate pass out of range");
  STWO_ARG_CHECK(d_itwiddles && log_n - 1 <= tree_log_size, "twiddle tree (log %u) too small for log size %u",
                 tree_log_size, log_n);
  uint32_t l0 = 0;
  for (uint32_t k = 0; k < pi; k++) l0 += split[k];
  FftPass p;
  p.tree = d_itwiddles;
  p.tree_len = 1ull << tree_log_size;
  p.src_mask = ~0ull;
  p.src_len = ~0ull;
  p.log_domain = log_n;
  p.layer0 = l0;
  p.T = split[pi];
  p.C = l0 == 0 ? 0u : 3u;
  p.scale = (pi + 1 == split.size()) ? host_pow2_inv(log_n) : 1u;
  std::vector<const uint32_t*> srcs(cols, cols + n_cols);
  std::vector<uint32_t*> dsts(cols, cols + n_cols);
  if (pi == 0 && src) srcs.assign(src, src + n_cols);
  if (pi == 0) {
    const uint64_t tile_rows = 1ull << p.T;
    STWO_ARG_CHECK(row_begin % tile_rows == 0 && row_end % tile_rows == 0 && row_begin < row_end &&
                       row_end <= (1ull << log_n),
                   "rows [%llu, %llu) are not whole tiles of the first pass", (unsigned long long)row_begin,
                   (unsigned long long)row_end);
    return launch_pass<true>(p, srcs, dsts, log_n, s, err, err_len, row_begin / tile_rows,
                             (row_end - row_begin) / tile_rows);
  }
  return launch_pass<true>(p, srcs, dsts, log_n, s, err, err_len);
}

int interpolate_evaluate(uint32_t* const* coeffs, uint32_t* const* evals, uint32_t n_cols, uint32_t log_n,
                         uint32_t log_blowup, const std::vector<uint32_t>& split, uint32_t first_pass,
                         const uint32_t* d_itwiddles, const uint32_t* d_twiddles, uint32_t tree_log_size,
                         cudaStream_t s, char* err, size_t err_len, const uint32_t* const* src0) {
  const uint32_t np = (uint32_t)split.size();
  const uint32_t N = log_n + log_blowup;
  STWO_ARG_CHECK(log_n >= 3 && N <= 30 && first_pass < np && split == split_for(log_n),
                 "interpolate_evaluate: log size %u, blowup %u, pass %u", log_n, log_blowup, first_pass);
  STWO_ARG_CHECK(d_twiddles && N - 1 <= tree_log_size, "twiddle tree (log %u) too small for log size %u",
                 tree_log_size, N);
  const uint32_t L0 = log_n - split.back();
  // Blowup 1 only: at blowup 2 the fused kernel (four forward tables, three
  // halves re-read through L2) measured 3-4% slower than the two passes.
  const bool fused = np >= 2 && split.back() == 10 && L0 >= 10 && L0 <= 12 && log_blowup == 1;
  const uint32_t* const* src = first_pass == 0 ? src0 : nullptr;
  if (!fused) {
    for (uint32_t pi = first_pass; pi < np; pi++) {
      int rc = interpolate_pass(coeffs, n_cols, log_n, split, pi, 0, 1ull << log_n, d_itwiddles, tree_log_size, s,
                                err, err_len, src);
      if (rc) return rc;
    }
    std::vector<uint32_t> logs(n_cols, log_n);
    return stwo_b200_evaluate_polynomials(const_cast<const uint32_t* const*>(coeffs), logs.data(), n_cols,
                                          log_blowup, evals, d_twiddles, tree_log_size, s, err, err_len);
  }
  for (uint32_t pi = first_pass; pi + 1 < np; pi++) {
    int rc = interpolate_pass(coeffs, n_cols, log_n, split, pi, 0, 1ull << log_n, d_itwiddles, tree_log_size, s, err,
                              err_len, src);
    if (rc) return rc;
  }
  FftPass pi;
  pi.tree = d_itwiddles;
  pi.tree_len = 1ull << tree_log_size;
  pi.src_mask = ~0ull;
  pi.src_len = ~0ull;
  pi.log_domain = log_n;
  pi.layer0 = L0;
  pi.T = 10;
  pi.C = 3;
  pi.scale = host_pow2_inv(log_n);
  FftPass pf = pi;
  pf.tree = d_twiddles;
  pf.log_domain = N;
  pf.scale = 1u;
  const uint32_t n_hi = 1u << log_blowup;
  const size_t smem = (1024 + kXchWords + 1024 * n_hi) * sizeof(uint32_t);
  static std::atomic<uint32_t> attr10{0}, attr11{0}, attr12{0};
  STWO_CUDA_TRY(L0 == 10   ? ensure_smem_limit(fft_warp_inv_fwd_kernel<10>, (int)smem, attr10)
                : L0 == 11 ? ensure_smem_limit(fft_warp_inv_fwd_kernel<11>, (int)smem, attr11)
                           : ensure_smem_limit(fft_warp_inv_fwd_kernel<12>, (int)smem, attr12));
  for (uint32_t c0 = 0; c0 < n_cols; c0 += kFftMaxCols) {
    const uint32_t nc = std::min<uint32_t>(kFftMaxCols, n_cols - c0);
    FftColsIE cols;
    for (uint32_t i = 0; i < nc; i++) {
      STWO_ARG_CHECK(coeffs[c0 + i] && evals[c0 + i], "null column %u", c0 + i);
      cols.coef[i] = coeffs[c0 + i];
      cols.eval[i] = evals[c0 + i];
    }
    const dim3 grid(1u << (L0 - 3), nc);
    if (L0 == 10)
      fft_warp_inv_fwd_kernel<10><<<grid, 256, smem, s>>>(pi, pf, cols, n_hi);
    else if (L0 == 11)
      fft_warp_inv_fwd_kernel<11><<<grid, 256, smem, s>>>(pi, pf, cols, n_hi);
    else
      fft_warp_inv_fwd_kernel<12><<<grid, 256, smem, s>>>(pi, pf, cols, n_hi);
    STWO_CHECK_LAUNCH();
  }
  // The remaining evaluation passes, in place, top layers first (as
  // stwo_b200_evaluate_polynomials).
  const std::vector<PassPlan> plan = plan_passes(log_n);
  std::vector<const uint32_t*> srcs(evals, evals + n_cols);
  std::vector<uint32_t*> dsts(evals, evals + n_cols);
  for (size_t k = plan.size() - 1; k-- > 0;) {
    FftPass p;
    p.tree = d_twiddles;
    p.tree_len = 1ull << tree_log_size;
    p.log_domain = N;
    p.layer0 = plan[k].layer0;
    p.T = plan[k].T;
    p.C = plan[k].C;
    p.scale = 1u;
    p.src_mask = ~0ull;
    p.src_len = ~0ull;
    int rc = launch_pass<false>(p, srcs, dsts, N, s, err, err_len);
    if (rc) return rc;
  }
  return STWO_B200_OK;
}

}  // namespace stwo_b200

extern "C" int stwo_b200_evaluate_polynomials(const uint32_t* const* d_coeffs, const uint32_t* log_sizes,
                                              uint32_t n_cols, uint32_t log_blowup, uint32_t* const* d_evals,
                                              const uint32_t* d_twiddles, uint32_t tree_log_size, void* stream,
                                              char* err, size_t err_len) {
  cudaStream_t s = as_stream(stream);
  STWO_ARG_CHECK(n_cols == 0 || (d_coeffs && log_sizes && d_evals), "null column arrays");
  std::vector<uint32_t> order(n_cols);
  for (uint32_t i = 0; i < n_cols; i++) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return log_sizes[a] < log_sizes[b]; });
  SmallCols small;
  uint32_t n_small = 0;
  for (size_t a = 0; a < order.size();) {
    uint32_t n = log_sizes[order[a]];
    size_t b = a;
    while (b < order.size() && log_sizes[order[b]] == n) b++;
    uint32_t N = n + log_blowup;
    STWO_ARG_CHECK(N <= 30, "evaluation log size %u too large", N);
    STWO_ARG_CHECK(N >= 1, "evaluation domain log size must be >= 1");
    if (N <= 2) {
      for (size_t i = a; i < b; i++) {
        uint32_t c = order[i];
        if (n_small == kFftMaxCols) {
          small_fft_kernel<<<1, kFftMaxCols, 0, s>>>(small, n_small, 0);
          STWO_CHECK_LAUNCH();
          n_small = 0;
        }
        small.src[n_small] = d_coeffs[c];
        small.dst[n_small] = d_evals[c];
        index_point(1ull << (31 - (N + 1)), small.x[n_small], small.y[n_small]);
        small.log_src[n_small] = n;
        small.log_dst[n_small] = N;
        n_small++;
      }
      a = b;
      continue;
    }
    STWO_ARG_CHECK(d_twiddles && N - 1 <= tree_log_size, "twiddle tree (log %u) too small for log size %u",
                   tree_log_size, N);
    std::vector<const uint32_t*> srcs;
    std::vector<uint32_t*> dsts;
    for (size_t i = a; i < b; i++) {
      srcs.push_back(d_coeffs[order[i]]);
      dsts.push_back(d_evals[order[i]]);
    }
    // simd/circle.rs:403-411: below log 5 the CPU path zero-extends the
    // coefficients and runs every layer of the big domain; otherwise each of
    // the 2^blowup subdomains transforms a copy of the coefficients with the
    // layers below n only (simd/circle.rs:413-440).
    const bool cpu_path = n < 5;
    const uint32_t layers = cpu_path ? N : n;
    auto plan = plan_passes(layers);
    for (size_t k = plan.size(); k-- > 0;) {
      FftPass p;
      p.tree = d_twiddles;
      p.tree_len = 1ull << tree_log_size;
      p.log_domain = N;
      p.layer0 = plan[k].layer0;
      p.T = plan[k].T;
      p.C = plan[k].C;
      p.scale = 1u;
      const bool first = (k + 1 == plan.size());
      if (first) {
        p.src_mask = cpu_path ? ((1ull << N) - 1) : ((1ull << n) - 1);
        p.src_len = 1ull << n;
        int rc = launch_pass<false>(p, srcs, dsts, N, s, err, err_len);
        if (rc) return rc;
      } else {
        p.src_mask = ~0ull;
        p.src_len = ~0ull;
        std::vector<const uint32_t*> inplace(dsts.begin(), dsts.end());
        int rc = launch_pass<false>(p, inplace, dsts, N, s, err, err_len);
        if (rc) return rc;
      }
    }
    a = b;
  }
  if (n_small) {
    small_fft_kernel<<<1, kFftMaxCols, 0, s>>>(small, n_small, 0);
    STWO_CHECK_LAUNCH();
  }
  return ok(err, err_len);
}

// interpolate_columns + evaluate_polynomials of one column size, as the
// commitment of a trace runs them (prover/pcs/mod.rs:707-781); the
// interpolation's last pass and the evaluation's first share a kernel where
// interpolate_evaluate allows it.
extern "C" int stwo_b200_interpolate_evaluate_columns(const uint32_t* const* d_src, uint32_t* const* d_coeffs,
                                                      uint32_t* const* d_evals, uint32_t n_cols, uint32_t log_size,
                                                      uint32_t log_blowup, const uint32_t* d_itwiddles,
                                                      const uint32_t* d_twiddles, uint32_t tree_log_size,
                                                      void* stream, char* err, size_t err_len) {
  cudaStream_t s = as_stream(stream);
  STWO_ARG_CHECK(n_cols == 0 || (d_coeffs && d_evals), "null column arrays");
  STWO_ARG_CHECK(log_size <= 30 && log_size + log_blowup <= 30, "log size %u + blowup %u too large", log_size,
                 log_blowup);
  if (n_cols == 0) return ok(err, err_len);
  std::vector<uint32_t> logs(n_cols, log_size);
  int rc;
  if (log_size < 3) {
    rc = d_src ? interpolate_impl(d_src, d_coeffs, logs.data(), nullptr, n_cols, d_itwiddles, tree_log_size, s, err,
                                  err_len)
               : interpolate_impl(d_coeffs, d_coeffs, logs.data(), nullptr, n_cols, d_itwiddles, tree_log_size, s,
                                  err, err_len);
    if (rc == 0)
      rc = stwo_b200_evaluate_polynomials(const_cast<const uint32_t* const*>(d_coeffs), logs.data(), n_cols,
                                          log_blowup, d_evals, d_twiddles, tree_log_size, stream, err, err_len);
  } else {
    STWO_ARG_CHECK(d_itwiddles && log_size - 1 <= tree_log_size, "twiddle tree (log %u) too small for log size %u",
                   tree_log_size, log_size);
    rc = interpolate_evaluate(d_coeffs, d_evals, n_cols, log_size, log_blowup, split_for(log_size), 0, d_itwiddles,
                              d_twiddles, tree_log_size, s, err, err_len, d_src);
  }
  return rc ? rc : ok(err, err_len);
}

extern "C" int stwo_b200_fft_set_plan(uint32_t log_size, const uint32_t* pass_layers, uint32_t n_passes, char* err,
                                      size_t err_len) {
  STWO_ARG_CHECK(log_size >= 1 && log_size <= 30, "log size %u out of range", log_size);
  if (n_passes == 0) {
    std::lock_guard<std::mutex> g(g_plan_mu);
    g_plan_override[log_size].clear();
    return ok(err, err_len);
  }
  STWO_ARG_CHECK(pass_layers != nullptr, "null plan");
  STWO_ARG_CHECK(plan_is_valid(log_size, pass_layers, n_passes),
                 "invalid plan for log size %u: 1-4 passes of 1-12 layers summing to the size, first >= 3 if split",
                 log_size);
  std::lock_guard<std::mutex> g(g_plan_mu);
  g_plan_override[log_size].assign(pass_layers, pass_layers + n_passes);
  return ok(err, err_len);
}

extern "C" int stwo_b200_fft_get_plan(uint32_t log_size, uint32_t* pass_layers, uint32_t cap, uint32_t* n_passes,
                                      char* err, size_t err_len) {
  STWO_ARG_CHECK(log_size >= 1 && log_size <= 30, "log size %u out of range", log_size);
  STWO_ARG_CHECK(n_passes != nullptr, "null n_passes");
  const std::vector<uint32_t> t = split_for(log_size);
  *n_passes = (uint32_t)t.size();
  STWO_ARG_CHECK(pass_layers == nullptr || cap >= t.size(), "plan has %zu passes, capacity %u", t.size(), cap);
  if (pass_layers)
    for (size_t i = 0; i < t.size(); i++) pass_layers[i] = t[i];
  return ok(err, err_len);
}

extern "C" int stwo_b200_bit_reverse_columns(const uint32_t* const* d_src, uint32_t* const* d_dst,
                                             const uint32_t* log_sizes, uint32_t n_cols, void* stream, char* err,
                                             size_t err_len) {
  STWO_ARG_CHECK(n_cols == 0 || (d_src && d_dst && log_sizes), "null argument");
  // one launch per run of equal sizes (at most kFftMaxCols columns each)
  for (uint32_t a = 0; a < n_cols;) {
    const uint32_t lg = log_sizes[a];
    STWO_ARG_CHECK(lg <= 31, "log size %u too large", lg);
    uint32_t b = a;
    while (b < n_cols && log_sizes[b] == lg) b++;
    int rc = bit_reverse_group(d_src + a, d_dst + a, b - a, lg, as_stream(stream), err, err_len);
    if (rc) return rc;
    a = b;
  }
  return ok(err, err_len);
}

extern "C" int stwo_b200_butterfly_probe(uint32_t blocks, uint32_t iters, uint32_t* d_out, void* stream, char* err,
                                         size_t err_len) {
  STWO_ARG_CHECK(d_out && blocks >= 1 && blocks <= (1u << 20), "bad probe arguments");
  butterfly_probe_kernel<<<blocks, 256, 0, as_stream(stream)>>>(iters, d_out);
  STWO_CHECK_LAUNCH();
  return ok(err, err_len);
}

extern "C" int stwo_b200_bit_reverse_column(uint32_t* d_col, uint32_t log_size, void* stream, char* err,
                                            size_t err_len) {
  STWO_ARG_CHECK(log_size <= 31, "log size %u too large", log_size);
  if (log_size == 0) return ok(err, err_len);
  uint64_t n = 1ull << log_size;
  uint64_t blocks = std::min<uint64_t>((n + 255) / 256, 148 * 32);
  bit_reverse_kernel<<<(unsigned)blocks, 256, 0, as_stream(stream)>>>(d_col, log_size);
  STWO_CHECK_LAUNCH();
  return ok(err, err_len);
}
