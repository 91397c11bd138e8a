// Blake2s Merkle trees for sm_100a: lifted leaves, node layers and the
// mixed-degree commit_on_layer.
//
// Lifted leaf i (crates/stwo/src/prover/backend/cpu/merkle_lifted.rs:44-78)
// is Blake2s-256 of the byte stream LE32(col_c[lift(i, L - log_c)]) over the
// columns sorted by length, lift(i, r) = ((i >> (r+1)) << 1) + (i & 1).  One
// thread per leaf absorbs 16 columns per compression; for every column a warp
// reads 32 consecutive (or pairwise repeated) words, so loads are coalesced
// without a shared-memory transpose.  Node layers hash 64-byte child pairs with
// one final compression (core/vcs_lifted/blake2_merkle.rs:18-25); a block
// builds up to 8 layers of a subtree in shared memory per launch.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "blake2s.cuh"
#include "common.cuh"
#include "field.cuh"

namespace stwo_b200 {

constexpr int kLeafMaxCols = 1024;
constexpr uint8_t kMixedShift = 0xFF;
struct LeafCols {
  const uint32_t* col[kLeafMaxCols];
  uint8_t shift[kLeafMaxCols];  // L - log_size
  // shift shared by the columns [16g, min(16g + 16, n)) of one compression,
  // or kMixedShift when they differ
  uint8_t group_shift[kLeafMaxCols / 16];
};

__device__ __forceinline__ void store_hash(uint8_t* out, uint64_t i, const uint32_t h[8], bool m31) {
  uint4* o = reinterpret_cast<uint4*>(out + i * 32);
  uint32_t w[8];
#pragma unroll
  for (int k = 0; k < 8; k++) w[k] = m31 ? m31_reduce_u32(h[k]) : h[k];
  o[0] = make_uint4(w[0], w[1], w[2], w[3]);
  o[1] = make_uint4(w[4], w[5], w[6], w[7]);
}

__device__ __forceinline__ uint32_t lift_index(uint32_t i, uint32_t r) {
  return r == 0 ? i : (((i >> (r + 1)) << 1) + (i & 1));
}

// One stage of the lifted leaves.  The leaf hash absorbs the sorted columns
// 16 per compression, and the chaining value after a compression depends
// only on columns of log size <= that compression's largest, so it is a
// function of lift(i, L - that log size): it is computed once per index of
// that size and lifted (lift(lift(i, a), b) = lift(i, a + b)), as SimdBackend
// does (backend/simd/blake2s_lifted.rs:42-160).  A stage runs the
// compressions of the columns in `t` (all of log size <= S, t.shift[c] =
// S - log_c) for the 2^S indices of size S.  It starts from the initial state
// (prev == nullptr) or from the chaining values of size 2^(S - prev_r) in
// `prev` (8 planes of 2^(S - prev_r) words), read at lift(i, prev_r); it
// leaves its chaining values in `next` (8 planes of 2^S words; may be `prev`
// when prev_r == 0, each thread reading its own entries first) or, in the
// last stage, the finalized leaf hashes in `out`.
__global__ void __launch_bounds__(256) lifted_leaves_kernel(LeafCols t, uint32_t n_cols, uint32_t S, int m31,
                                                           uint32_t bytes_before, uint32_t total_bytes,
                                                           const uint32_t* prev, uint32_t prev_r, uint32_t* next,
                                                           int is_last, uint8_t* out) {
  const uint32_t n = 1u << S;  // S <= 30
  const uint32_t n_prev = n >> prev_r;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    uint32_t h[8];
    if (prev == nullptr) {
      blake2s_init(h);
    } else {
      const uint32_t j = lift_index(i, prev_r);
#pragma unroll
      for (int k = 0; k < 8; k++) h[k] = prev[(uint64_t)k * n_prev + j];
    }
    uint32_t m[16];
    uint32_t done = bytes_before;
    if (n_cols == 0 && is_last) {
#pragma unroll
      for (int k = 0; k < 16; k++) m[k] = 0;
      blake2s_compress(h, m, done, true);
    }
    for (uint32_t c0 = 0; c0 < n_cols; c0 += 16) {
      const uint32_t gs = t.group_shift[c0 >> 4];
      if (gs != kMixedShift) {
        // one lifted row index for the whole group (full or the last, partial
        // one): no per-column index work
        const uint32_t li = lift_index(i, gs);
        if (c0 + 16 <= n_cols) {
#pragma unroll
          for (int k = 0; k < 16; k++) m[k] = __ldg(t.col[c0 + k] + li);
        } else {
#pragma unroll
          for (int k = 0; k < 16; k++) m[k] = c0 + k < n_cols ? __ldg(t.col[c0 + k] + li) : 0u;
        }
      } else {
#pragma unroll
        for (int k = 0; k < 16; k++) {
          uint32_t c = c0 + k;
          m[k] = c < n_cols ? __ldg(t.col[c] + lift_index(i, t.shift[c])) : 0u;
        }
      }
      uint32_t nb = min(16u, n_cols - c0) * 4;
      done += nb;
      blake2s_compress(h, m, done, is_last && done == total_bytes);
    }
    if (is_last) {
      store_hash(out, i, h, m31 != 0);
    } else {
#pragma unroll
      for (int k = 0; k < 8; k++) next[(uint64_t)k * n + i] = h[k];
    }
  }
}

// Hashes `levels` consecutive node layers.  Block b hashes `width` parents
// of `in` (2^in_log hashes) at the first level, keeps them in shared memory
// and continues up its subtree; every produced layer lv goes to outs[lv].
struct NodeOuts {
  uint8_t* out[8];
};

// LAT selects the shortest-dependency Blake2s form, for launches of a few
// blocks where one compression's latency (not throughput) sets the time.
template <bool LAT>
__global__ void __launch_bounds__(256) node_layers_kernel(const uint8_t* in, uint32_t in_log, uint32_t levels, int m31,
                                                         NodeOuts outs) {
  __shared__ uint32_t buf[2][256 * 8];
  // level 0: parents of `in`
  uint64_t parents0 = 1ull << (in_log - 1);
  uint32_t width = parents0 < 256 ? (uint32_t)parents0 : 256u;  // parents of this block at level 0
  uint64_t first_parent = (uint64_t)blockIdx.x * width;
  uint32_t tid = threadIdx.x;
  int cur = 0;
  if (tid < width) {
    uint64_t p = first_parent + tid;
    const uint4* src = reinterpret_cast<const uint4*>(in + p * 64);
    uint32_t m[16];
    uint4 a = src[0], b = src[1], c = src[2], d = src[3];
    m[0] = a.x; m[1] = a.y; m[2] = a.z; m[3] = a.w;
    m[4] = b.x; m[5] = b.y; m[6] = b.z; m[7] = b.w;
    m[8] = c.x; m[9] = c.y; m[10] = c.z; m[11] = c.w;
    m[12] = d.x; m[13] = d.y; m[14] = d.z; m[15] = d.w;
    uint32_t h[8];
    blake2s_init(h);
    if (LAT)
      blake2s_compress_lat(h, m, 64, true);
    else
      blake2s_compress(h, m, 64, true);
    if (m31) {
#pragma unroll
      for (int k = 0; k < 8; k++) h[k] = m31_reduce_u32(h[k]);
    }
    store_hash(outs.out[0], p, h, false);
#pragma unroll
    for (int k = 0; k < 8; k++) buf[cur][tid * 8 + k] = h[k];
  }
  __syncthreads();
  for (uint32_t lv = 1; lv < levels; lv++) {
    width >>= 1;
    if (width == 0) break;
    uint64_t first = first_parent >> lv;
    if (tid < width) {
      uint32_t m[16];
#pragma unroll
      for (int k = 0; k < 16; k++) m[k] = buf[cur][tid * 16 + k];
      uint32_t h[8];
      blake2s_init(h);
      if (LAT)
      blake2s_compress_lat(h, m, 64, true);
    else
      blake2s_compress(h, m, 64, true);
      if (m31) {
#pragma unroll
        for (int k = 0; k < 8; k++) h[k] = m31_reduce_u32(h[k]);
      }
      store_hash(outs.out[lv], first + tid, h, false);
#pragma unroll
      for (int k = 0; k < 8; k++) buf[cur ^ 1][tid * 8 + k] = h[k];
    }
    cur ^= 1;
    __syncthreads();
  }
}

// Parent hash of the 64-byte child pair in m (throughput form), reduced to
// M31 words when the tree stores M31 hashes.
__device__ __forceinline__ void hash_children(const uint32_t m[16], bool m31, uint32_t h[8]) {
  blake2s_init(h);
  blake2s_compress(h, m, 64, true);
  if (m31) {
#pragma unroll
    for (int k = 0; k < 8; k++) h[k] = m31_reduce_u32(h[k]);
  }
}

__device__ __forceinline__ void load_children(const uint4* src, uint32_t m[16]) {
  const uint4 a = __ldg(src), b = __ldg(src + 1), c = __ldg(src + 2), d = __ldg(src + 3);
  m[0] = a.x; m[1] = a.y; m[2] = a.z; m[3] = a.w;
  m[4] = b.x; m[5] = b.y; m[6] = b.z; m[7] = b.w;
  m[8] = c.x; m[9] = c.y; m[10] = c.z; m[11] = c.w;
  m[12] = d.x; m[13] = d.y; m[14] = d.z; m[15] = d.w;
}

// Three node layers per thread, for layers wide enough to fill the GPU:
// thread t reads child hashes 8t..8t+7 of `in` and writes parents 4t..4t+3
// (out0), 2t, 2t+1 (out1) and t (out2).  Every thread does 7 compressions
// with no barrier and no idle lanes; the block-cooperative kernel above idles
// half its threads at each level it climbs.
__global__ void __launch_bounds__(256) node_subtree3_kernel(const uint8_t* in, uint64_t n, int m31, uint8_t* out0,
                                                           uint8_t* out1, uint8_t* out2) {
  // Rolled loops keep three copies of the compression in the code instead of
  // seven, so the instruction cache holds the kernel's working set.
  for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < n; t += (uint64_t)gridDim.x * blockDim.x) {
    const uint4* src = reinterpret_cast<const uint4*>(in + t * 256);
    uint32_t m[16], h[8], g0[8];
#pragma unroll 1
    for (int half = 0; half < 2; half++) {
      uint32_t a[8];
#pragma unroll 1
      for (int e = 0; e < 2; e++) {
        load_children(src + 8 * half + 4 * e, m);
        hash_children(m, m31 != 0, h);
        store_hash(out0, 4 * t + 2 * half + e, h, false);
#pragma unroll
        for (int k = 0; k < 8; k++) a[k] = e == 0 ? h[k] : a[k];
      }
#pragma unroll
      for (int k = 0; k < 8; k++) {
        m[k] = a[k];
        m[k + 8] = h[k];
      }
      hash_children(m, m31 != 0, h);
      store_hash(out1, 2 * t + half, h, false);
#pragma unroll
      for (int k = 0; k < 8; k++) g0[k] = half == 0 ? h[k] : g0[k];
    }
#pragma unroll
    for (int k = 0; k < 8; k++) {
      m[k] = g0[k];
      m[k + 8] = h[k];
    }
    hash_children(m, m31 != 0, h);
    store_hash(out2, t, h, false);
  }
}

// Mixed-degree node: Blake2s(prev[2i] || prev[2i+1] || LE32 cols[c][i] ...).
__global__ void __launch_bounds__(256) commit_on_layer_kernel(uint32_t log_size, const uint8_t* prev, LeafCols t,
                                                             uint32_t n_cols, int m31, uint8_t* out) {
  uint64_t n = 1ull << log_size;
  const uint32_t total = (prev ? 64u : 0u) + 4u * n_cols;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t h[8];
    blake2s_init(h);
    uint32_t m[16];
    uint32_t done = 0;
    uint32_t c0 = 0;
    if (prev) {
      const uint4* src = reinterpret_cast<const uint4*>(prev + i * 64);
      uint4 a = src[0], b = src[1], c = src[2], d = src[3];
      m[0] = a.x; m[1] = a.y; m[2] = a.z; m[3] = a.w;
      m[4] = b.x; m[5] = b.y; m[6] = b.z; m[7] = b.w;
      m[8] = c.x; m[9] = c.y; m[10] = c.z; m[11] = c.w;
      m[12] = d.x; m[13] = d.y; m[14] = d.z; m[15] = d.w;
      done = 64;
      blake2s_compress(h, m, done, done == total);
    }
    if (total == 0) {
#pragma unroll
      for (int k = 0; k < 16; k++) m[k] = 0;
      blake2s_compress(h, m, 0, true);
    }
    for (; c0 < n_cols; c0 += 16) {
#pragma unroll
      for (int k = 0; k < 16; k++) {
        uint32_t c = c0 + k;
        m[k] = c < n_cols ? __ldg(t.col[c] + i) : 0u;
      }
      done += min(16u, n_cols - c0) * 4;
      blake2s_compress(h, m, done, done == total);
    }
    store_hash(out, i, h, m31 != 0);
  }
}

// Blake2s throughput probe: every thread chains `iters` compressions on
// register-resident data (no memory traffic), giving the integer-pipe ceiling
// for exactly the op mix the leaf and node kernels execute.
__global__ void __launch_bounds__(256) blake2s_probe_kernel(uint32_t iters, uint32_t* out) {
  uint32_t h[8];
  blake2s_init(h);
  uint32_t m[16];
#pragma unroll
  for (int k = 0; k < 16; k++) m[k] = threadIdx.x * 16 + k + blockIdx.x;
  for (uint32_t it = 0; it < iters; it++) {
    blake2s_compress(h, m, 64 * (it + 1), false);
    m[it & 15] ^= h[0];
  }
  uint32_t x = 0;
#pragma unroll
  for (int k = 0; k < 8; k++) x ^= h[k];
  if (x == 0x12345678u) out[0] = x;  // keeps the chain live
}

static unsigned grid_for(uint64_t n, unsigned threads) {
  uint64_t b = (n + threads - 1) / threads;
  return (unsigned)std::min<uint64_t>(std::max<uint64_t>(b, 1), 148ull * 64);
}

// Leaves of the lifted tree in stages.  Compression group g (columns
// [16g, 16g + 16) of the sorted list) runs at the size of its largest column,
// the last group at L (it writes the leaves); consecutive groups of one size
// form a stage, one launch per up to kLeafMaxCols columns.  The chaining
// values between stages of size S < L go to layer_ws[S] when the caller
// passes the tree's layer buffers (2^S hashes of 32 bytes each, rebuilt by
// the node layers afterwards), else to a temporary buffer that packs size S
// at byte offset 32 * 2^S.
int build_leaves_impl(const uint32_t* const* d_cols, const uint32_t* log_sizes, uint32_t n_cols, uint32_t L,
                      int m31, uint8_t* d_leaves, uint8_t* const* layer_ws, cudaStream_t s, char* err,
                      size_t err_len) {
  STWO_ARG_CHECK(d_leaves != nullptr, "null leaves");
  if (n_cols == 0) {
    LeafCols t{};
    lifted_leaves_kernel<<<1, 32, 0, s>>>(t, 0, 0, m31, 0, 0, nullptr, 0, nullptr, 1, d_leaves);
    STWO_CHECK_LAUNCH();
    return STWO_B200_OK;
  }
  STWO_ARG_CHECK(L <= 30, "lifting log size %u too large", L);
  for (uint32_t c = 0; c < n_cols; c++) {
    STWO_ARG_CHECK(log_sizes[c] >= 1, "A column must be of length >= 2.");
    STWO_ARG_CHECK(log_sizes[c] <= L, "column log size %u exceeds lifting log size %u", log_sizes[c], L);
    STWO_ARG_CHECK(c == 0 || log_sizes[c - 1] <= log_sizes[c], "columns must be sorted by length");
  }
  const uint32_t n_groups = (n_cols + 15) / 16;
  auto group_size = [&](uint32_t g) {
    return g + 1 == n_groups ? L : log_sizes[std::min<uint32_t>(16 * g + 15, n_cols - 1)];
  };
  struct Launch {
    uint32_t g0, g1, S;
  };
  std::vector<Launch> launches;
  for (uint32_t g = 0; g < n_groups;) {
    uint32_t e = g + 1;
    while (e < n_groups && e - g < kLeafMaxCols / 16 && group_size(e) == group_size(g)) e++;
    launches.push_back({g, e, group_size(g)});
    g = e;
  }
  // temporary state: sizes below L packed (when the caller gave no layer
  // buffers), and one buffer of size L for a last stage of > kLeafMaxCols
  // columns
  bool need_small = false, need_top = false;
  for (size_t k = 0; k + 1 < launches.size(); k++) {
    if (launches[k].S < L)
      need_small |= layer_ws == nullptr;
    else
      need_top = true;
  }
  const uint64_t top_bytes = 32ull << L;
  uint8_t* ws = nullptr;
  const uint64_t ws_bytes = (need_small ? top_bytes : 0) + (need_top ? top_bytes : 0);
  if (ws_bytes) STWO_CUDA_TRY(cudaMallocAsync(&ws, ws_bytes, s));
  auto state_of = [&](uint32_t S) -> uint32_t* {
    if (S == L) return reinterpret_cast<uint32_t*>(ws + (need_small ? top_bytes : 0));
    if (layer_ws) return reinterpret_cast<uint32_t*>(layer_ws[S]);
    return reinterpret_cast<uint32_t*>(ws + (32ull << S));
  };
  const uint32_t total_bytes = 4u * n_cols;
  const uint32_t* prev = nullptr;
  uint32_t prev_S = 0;
  for (size_t k = 0; k < launches.size(); k++) {
    const Launch& ln = launches[k];
    const bool last = k + 1 == launches.size();
    const uint32_t c0 = 16 * ln.g0, c1 = std::min<uint32_t>(16 * ln.g1, n_cols);
    const uint32_t nc = c1 - c0;
    LeafCols t;
    for (uint32_t c = 0; c < nc; c++) {
      t.col[c] = d_cols[c0 + c];
      t.shift[c] = (uint8_t)(ln.S - log_sizes[c0 + c]);
    }
    for (uint32_t g = 0; g < kLeafMaxCols / 16; g++) {
      const uint32_t k0 = 16 * g;
      bool uniform = k0 < nc;
      for (uint32_t c = k0 + 1; uniform && c < std::min<uint32_t>(k0 + 16, nc); c++) uniform = t.shift[c] == t.shift[k0];
      t.group_shift[g] = uniform ? t.shift[k0] : kMixedShift;
    }
    uint32_t* next = last ? nullptr : state_of(ln.S);
    lifted_leaves_kernel<<<grid_for(1ull << ln.S, 256), 256, 0, s>>>(t, nc, ln.S, m31, 4u * c0, total_bytes, prev,
                                                                     ln.S - prev_S, next, last, d_leaves);
    STWO_CHECK_LAUNCH();
    prev = next;
    prev_S = ln.S;
  }
  if (ws) STWO_CUDA_TRY(cudaFreeAsync(ws, s));
  return STWO_B200_OK;
}

constexpr uint32_t kSubtree3MinLog = 19;

// Builds layers [in_log - 1 .. stop_log] from layer `in` (2^in_log hashes);
// outs_by_log[k] is the destination of layer log k.
int build_node_layers_impl(const uint8_t* in, uint32_t in_log, uint32_t stop_log, int m31,
                           uint8_t* const* outs_by_log, cudaStream_t s, char* err, size_t err_len) {
  uint32_t cur_log = in_log;
  const uint8_t* cur = in;
  while (cur_log > stop_log) {
    // Wide layers: three levels per thread while the third level still has
    // 2^16 parents (256 blocks of 256 threads).
    if (cur_log - stop_log >= 3 && cur_log >= kSubtree3MinLog) {
      const uint64_t n = 1ull << (cur_log - 3);
      node_subtree3_kernel<<<grid_for(n, 256), 256, 0, s>>>(cur, n, m31, outs_by_log[cur_log - 1],
                                                            outs_by_log[cur_log - 2], outs_by_log[cur_log - 3]);
      STWO_CHECK_LAUNCH();
      cur = outs_by_log[cur_log - 3];
      cur_log -= 3;
      continue;
    }
    uint32_t levels = std::min<uint32_t>(8, cur_log - stop_log);
    uint64_t parents0 = 1ull << (cur_log - 1);
    uint32_t width = (uint32_t)std::min<uint64_t>(256, parents0);
    // a block produces width >> (lv) parents at level lv; keep it >= 1
    while (levels > 1 && (width >> (levels - 1)) == 0) levels--;
    NodeOuts o;
    for (uint32_t lv = 0; lv < levels; lv++) o.out[lv] = outs_by_log[cur_log - 1 - lv];
    unsigned blocks = (unsigned)(parents0 / width);
    if (blocks <= 148)
      node_layers_kernel<true><<<blocks, 256, 0, s>>>(cur, cur_log, levels, m31, o);
    else
      node_layers_kernel<false><<<blocks, 256, 0, s>>>(cur, cur_log, levels, m31, o);
    STWO_CHECK_LAUNCH();
    cur = outs_by_log[cur_log - levels];
    cur_log -= levels;
  }
  return STWO_B200_OK;
}

}  // namespace stwo_b200

using namespace stwo_b200;

extern "C" int stwo_b200_merkle_build_leaves(const uint32_t* const* d_cols, const uint32_t* log_sizes,
                                             uint32_t n_cols, uint32_t lifting_log_size, int m31_output,
                                             uint8_t* d_leaves, void* stream, char* err, size_t err_len) {
  int rc = build_leaves_impl(d_cols, log_sizes, n_cols, lifting_log_size, m31_output, d_leaves, nullptr,
                             as_stream(stream), err, err_len);
  return rc ? rc : ok(err, err_len);
}

extern "C" int stwo_b200_merkle_build_next_layer(const uint8_t* d_prev, uint32_t prev_log_size, int m31_output,
                                                 uint8_t* d_out, void* stream, char* err, size_t err_len) {
  STWO_ARG_CHECK(prev_log_size >= 1 && prev_log_size <= 31, "bad layer log size %u", prev_log_size);
  std::vector<uint8_t*> outs(prev_log_size, nullptr);
  outs[prev_log_size - 1] = d_out;
  int rc = build_node_layers_impl(d_prev, prev_log_size, prev_log_size - 1, m31_output, outs.data(),
                                  as_stream(stream), err, err_len);
  return rc ? rc : ok(err, err_len);
}

extern "C" int stwo_b200_merkle_build_layers(const uint32_t* const* d_cols, const uint32_t* log_sizes,
                                             uint32_t n_cols, uint32_t lifting_log_size, int m31_output,
                                             uint8_t* const* d_layers, void* stream, char* err, size_t err_len) {
  cudaStream_t s = as_stream(stream);
  STWO_ARG_CHECK(d_layers != nullptr, "null layers");
  if (n_cols == 0) {
    STWO_ARG_CHECK(lifting_log_size == 0, "empty commitment needs lifting_log_size 0");
    int rc = build_leaves_impl(nullptr, nullptr, 0, 0, m31_output, d_layers[0], nullptr, s, err, err_len);
    return rc ? rc : ok(err, err_len);
  }
  // prover/vcs_lifted/ops.rs:37 stable sort by length.
  std::vector<uint32_t> order(n_cols);
  for (uint32_t i = 0; i < n_cols; i++) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return log_sizes[a] < log_sizes[b]; });
  std::vector<const uint32_t*> cols(n_cols);
  std::vector<uint32_t> logs(n_cols);
  for (uint32_t i = 0; i < n_cols; i++) {
    cols[i] = d_cols[order[i]];
    logs[i] = log_sizes[order[i]];
  }
  const uint32_t L = lifting_log_size;
  int rc = build_leaves_impl(cols.data(), logs.data(), n_cols, L, m31_output, d_layers[L], d_layers, s, err, err_len);
  if (rc) return rc;
  rc = build_node_layers_impl(d_layers[L], L, 0, m31_output, d_layers, s, err, err_len);
  return rc ? rc : ok(err, err_len);
}

extern "C" int stwo_b200_merkle_build_nodes(uint8_t* const* d_layers, uint32_t lifting_log_size, int m31_output,
                                            void* stream, char* err, size_t err_len) {
  STWO_ARG_CHECK(d_layers != nullptr, "null layers");
  STWO_ARG_CHECK(lifting_log_size <= 31, "bad lifting log size");
  int rc = build_node_layers_impl(d_layers[lifting_log_size], lifting_log_size, 0, m31_output, d_layers,
                                  as_stream(stream), err, err_len);
  return rc ? rc : ok(err, err_len);
}

extern "C" int stwo_b200_merkle_build_leaves_layers(const uint32_t* const* d_cols, const uint32_t* log_sizes,
                                                    uint32_t n_cols, uint32_t lifting_log_size, int m31_output,
                                                    uint8_t* const* d_layers, void* stream, char* err,
                                                    size_t err_len) {
  STWO_ARG_CHECK(d_layers != nullptr, "null layers");
  STWO_ARG_CHECK(lifting_log_size <= 30, "lifting log size %u too large", lifting_log_size);
  int rc = build_leaves_impl(d_cols, log_sizes, n_cols, lifting_log_size, m31_output, d_layers[lifting_log_size],
                             d_layers, as_stream(stream), err, err_len);
  return rc ? rc : ok(err, err_len);
}

extern "C" int stwo_b200_blake2s_probe(uint32_t blocks, uint32_t iters, uint32_t* d_out, void* stream, char* err,
                                       size_t err_len) {
  STWO_ARG_CHECK(blocks >= 1 && d_out, "bad probe arguments");
  blake2s_probe_kernel<<<blocks, 256, 0, as_stream(stream)>>>(iters, d_out);
  STWO_CHECK_LAUNCH();
  return ok(err, err_len);
}

extern "C" int stwo_b200_commit_on_layer(uint32_t log_size, const uint8_t* d_prev, const uint32_t* const* d_cols,
                                         uint32_t n_cols, int m31_output, uint8_t* d_out, void* stream, char* err,
                                         size_t err_len) {
  STWO_ARG_CHECK(log_size <= 30, "log size %u too large", log_size);
  STWO_ARG_CHECK(n_cols <= kLeafMaxCols, "at most %d columns per layer", kLeafMaxCols);
  LeafCols t;
  for (uint32_t c = 0; c < n_cols; c++) {
    t.col[c] = d_cols[c];
    t.shift[c] = 0;
  }
  uint64_t n = 1ull << log_size;
  commit_on_layer_kernel<<<grid_for(n, 256), 256, 0, as_stream(stream)>>>(log_size, d_prev, t, n_cols, m31_output,
                                                                           d_out);
  STWO_CHECK_LAUNCH();
  return ok(err, err_len);
}
