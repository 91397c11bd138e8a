// Trace commitment of a whole column set (the CommitmentTreeProver path of
// crates/stwo/src/prover/pcs/mod.rs:707-781: interpolate_columns, then
// evaluate_polynomials on the blowup domain, then the lifted Blake2s Merkle
// tree of crates/stwo/src/prover/vcs_lifted/prover.rs:33-42), in three forms:
//
//  - per-column: every column its own FFT launches (SimdBackend's per-column
//    structure, ops.rs:29-40, run on the GPU);
//  - batched: one launch per (column size, pass), all columns of a size at
//    once;
//  - batched + graph: the batched launches captured once per buffer set as a
//    CUDA graph and replayed.
//
// The FFT pass plan of every size is a global table (fft.cu); the autotuner
// here times candidate splits per (log_size, n_columns) group on the caller's
// buffers and keeps the fastest, optionally cached in a text file.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <functional>
#include <map>
#include <string>
#include <vector>

#include "common.cuh"
#include "stwo_b200.h"

namespace stwo_b200 {

struct Committer {
  std::vector<uint32_t> logs;
  uint32_t blowup = 0, L = 0, tree_log = 0, flags = 0;
  int m31 = 0;
  const uint32_t* tw = nullptr;
  const uint32_t* itw = nullptr;
  cudaStream_t s = nullptr;
  cudaEvent_t ev_in = nullptr, ev_out = nullptr;
  std::vector<const void*> key;  // buffers the cached graph was captured with
  cudaGraphExec_t exec = nullptr;
  uint64_t graph_launches = 0;

  // host-streamed commits: the H2D copies run on `cs`, one size group at a
  // time, and each group's transforms wait only for that group's copies
  cudaStream_t cs = nullptr;
  std::vector<cudaEvent_t> ev_group;

  ~Committer() {
    if (s) cudaStreamSynchronize(s);
    if (cs) cudaStreamSynchronize(cs);
    if (exec) cudaGraphExecDestroy(exec);
    if (ev_in) cudaEventDestroy(ev_in);
    if (ev_out) cudaEventDestroy(ev_out);
    for (cudaEvent_t e : ev_group) cudaEventDestroy(e);
    if (cs) cudaStreamDestroy(cs);
    if (s) cudaStreamDestroy(s);
  }

  // commit() with the columns still in host memory: copies them into d_evals
  // size group by size group, largest first, on a copy stream, so the
  // transforms of the groups already on the device overlap the copies of the
  // rest; the tree follows once every group is transformed.  Host columns in
  // pinned memory make the copies asynchronous.
  int commit_from_host(const uint32_t* const* h_evals, uint32_t* const* d_evals, uint32_t* const* coeffs,
                       uint32_t* const* ldes, uint8_t* const* layers, cudaStream_t user, char* err, size_t err_len) {
    std::map<uint32_t, std::vector<uint32_t>, std::greater<uint32_t>> groups;
    for (uint32_t i = 0; i < logs.size(); i++) groups[logs[i]].push_back(i);
    if (!cs) STWO_CUDA_TRY(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    while (ev_group.size() < groups.size()) {
      cudaEvent_t e;
      STWO_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
      ev_group.push_back(e);
    }
    STWO_CUDA_TRY(cudaEventRecord(ev_in, user));
    STWO_CUDA_TRY(cudaStreamWaitEvent(s, ev_in, 0));
    STWO_CUDA_TRY(cudaStreamWaitEvent(cs, ev_in, 0));
    int rc = 0;
    size_t g = 0;
    for (const auto& kv : groups) {
      for (uint32_t i : kv.second)
        STWO_CUDA_TRY(cudaMemcpyAsync(d_evals[i], h_evals[i], sizeof(uint32_t) << logs[i], cudaMemcpyHostToDevice, cs));
      STWO_CUDA_TRY(cudaEventRecord(ev_group[g], cs));
      STWO_CUDA_TRY(cudaStreamWaitEvent(s, ev_group[g], 0));
      g++;
      if (flags & STWO_B200_COMMIT_PER_COLUMN) {
        for (uint32_t i : kv.second)
          if ((rc = transform(d_evals, coeffs, ldes, {i}, err, err_len))) return rc;
      } else if ((rc = transform(d_evals, coeffs, ldes, kv.second, err, err_len))) {
        return rc;
      }
    }
    const uint32_t n = (uint32_t)logs.size();
    std::vector<uint32_t> lde_logs(n);
    for (uint32_t i = 0; i < n; i++) lde_logs[i] = logs[i] + blowup;
    rc = stwo_b200_merkle_build_layers(const_cast<const uint32_t* const*>(ldes), lde_logs.data(), n, L, m31, layers, s,
                                       err, err_len);
    cudaEventRecord(ev_out, s);
    cudaStreamWaitEvent(user, ev_out, 0);
    return rc;
  }

  // interpolate + evaluate of the columns `cols`: one
  // stwo_b200_interpolate_evaluate_columns call per log size (the
  // interpolation's last pass and the evaluation's first share a kernel where
  // the pass plan allows); the columns below log 3 in one batched pair of
  // calls.
  int transform(const uint32_t* const* evals, uint32_t* const* coeffs, uint32_t* const* ldes,
                const std::vector<uint32_t>& cols, char* err, size_t err_len) {
    std::map<uint32_t, std::vector<uint32_t>> by_size;
    std::vector<const uint32_t*> se;
    std::vector<uint32_t*> sc, sd;
    std::vector<uint32_t> slg;
    for (uint32_t i : cols) {
      if (logs[i] >= 3) {
        by_size[logs[i]].push_back(i);
      } else {
        se.push_back(evals[i]);
        sc.push_back(coeffs[i]);
        sd.push_back(ldes[i]);
        slg.push_back(logs[i]);
      }
    }
    int rc;
    if (!se.empty()) {
      const uint32_t n = (uint32_t)se.size();
      if ((rc = stwo_b200_interpolate_columns_into(se.data(), sc.data(), slg.data(), nullptr, n, itw, tree_log, s, err,
                                                   err_len)))
        return rc;
      if ((rc = stwo_b200_evaluate_polynomials(sc.data(), slg.data(), n, blowup, sd.data(), tw, tree_log, s, err,
                                               err_len)))
        return rc;
    }
    for (const auto& kv : by_size) {
      std::vector<const uint32_t*> e;
      std::vector<uint32_t*> c, d;
      for (uint32_t i : kv.second) {
        e.push_back(evals[i]);
        c.push_back(coeffs[i]);
        d.push_back(ldes[i]);
      }
      if ((rc = stwo_b200_interpolate_evaluate_columns(e.data(), c.data(), d.data(), (uint32_t)e.size(), kv.first,
                                                       blowup, itw, tw, tree_log, s, err, err_len)))
        return rc;
    }
    return STWO_B200_OK;
  }

  int enqueue(const uint32_t* const* evals, uint32_t* const* coeffs, uint32_t* const* ldes, uint8_t* const* layers,
              char* err, size_t err_len) {
    const uint32_t n = (uint32_t)logs.size();
    int rc;
    if (flags & STWO_B200_COMMIT_PER_COLUMN) {
      for (uint32_t i = 0; i < n; i++)
        if ((rc = transform(evals, coeffs, ldes, {i}, err, err_len))) return rc;
    } else {
      std::vector<uint32_t> all(n);
      for (uint32_t i = 0; i < n; i++) all[i] = i;
      if ((rc = transform(evals, coeffs, ldes, all, err, err_len))) return rc;
    }
    std::vector<uint32_t> lde_logs(n);
    for (uint32_t i = 0; i < n; i++) lde_logs[i] = logs[i] + blowup;
    return stwo_b200_merkle_build_layers(const_cast<const uint32_t* const*>(ldes), lde_logs.data(), n, L, m31, layers,
                                         s, err, err_len);
  }

  int commit(const uint32_t* const* evals, uint32_t* const* coeffs, uint32_t* const* ldes, uint8_t* const* layers,
             cudaStream_t user, char* err, size_t err_len) {
    STWO_CUDA_TRY(cudaEventRecord(ev_in, user));
    STWO_CUDA_TRY(cudaStreamWaitEvent(s, ev_in, 0));
    int rc = 0;
    if (flags & STWO_B200_COMMIT_GRAPH) {
      const uint32_t n = (uint32_t)logs.size();
      std::vector<const void*> k;
      for (uint32_t i = 0; i < n; i++) {
        k.push_back(evals[i]);
        k.push_back(coeffs[i]);
        k.push_back(ldes[i]);
      }
      for (uint32_t i = 0; i <= L; i++) k.push_back(layers[i]);
      if (!exec || k != key) {
        if (exec) {
          cudaGraphExecDestroy(exec);
          exec = nullptr;
        }
        const uint64_t before = g_kernel_launches.load();
        STWO_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        rc = enqueue(evals, coeffs, ldes, layers, err, err_len);
        cudaGraph_t g = nullptr;
        const cudaError_t ce = cudaStreamEndCapture(s, &g);
        const uint64_t launched = g_kernel_launches.load() - before;
        g_kernel_launches.fetch_sub(launched);  // nothing ran during capture
        if (rc) {
          if (g) cudaGraphDestroy(g);
          return rc;
        }
        if (ce != cudaSuccess)
          return set_err(err, err_len, STWO_B200_ECUDA, "commit graph capture: %s", cudaGetErrorString(ce));
        const cudaError_t ie = cudaGraphInstantiate(&exec, g, 0);
        cudaGraphDestroy(g);
        if (ie != cudaSuccess) {
          exec = nullptr;
          return set_err(err, err_len, STWO_B200_ECUDA, "commit graph instantiate: %s", cudaGetErrorString(ie));
        }
        key = k;
        graph_launches = launched;
      }
      STWO_CUDA_TRY(cudaGraphLaunch(exec, s));
      g_kernel_launches.fetch_add(graph_launches);
    } else {
      rc = enqueue(evals, coeffs, ldes, layers, err, err_len);
    }
    cudaEventRecord(ev_out, s);
    cudaStreamWaitEvent(user, ev_out, 0);
    return rc;
  }

  void drop_graph() {
    if (exec) cudaGraphExecDestroy(exec);
    exec = nullptr;
    key.clear();
  }
};

// Candidate pass splits of an n-layer transform: one pass up to 12 layers,
// every two-pass split, and three-pass splits near thirds.
static std::vector<std::vector<uint32_t>> candidate_splits(uint32_t n) {
  std::vector<std::vector<uint32_t>> c;
  if (n <= 12) c.push_back({n});
  for (uint32_t a = 3; a <= 12 && a < n; a++)
    if (n - a >= 1 && n - a <= 12) c.push_back({a, n - a});
  if (n >= 15)
    for (uint32_t a = std::max(3u, n / 3 - 1); a <= std::min(12u, n / 3 + 1); a++)
      for (uint32_t b = std::max(1u, (n - a) / 2 - 1); b <= std::min(12u, (n - a) / 2 + 1); b++)
        if (n - a - b >= 1 && n - a - b <= 12) c.push_back({a, b, n - a - b});
  return c;
}

static std::string split_str(const std::vector<uint32_t>& t) {
  std::string s;
  for (size_t i = 0; i < t.size(); i++) s += (i ? "," : "") + std::to_string(t[i]);
  return s;
}

}  // namespace stwo_b200

using namespace stwo_b200;

struct stwo_b200_committer {
  Committer c;
};

extern "C" int stwo_b200_committer_create(const uint32_t* log_sizes, uint32_t n_cols, uint32_t log_blowup,
                                          int m31_output, const uint32_t* d_twiddles, const uint32_t* d_itwiddles,
                                          uint32_t tree_log_size, uint32_t flags, stwo_b200_committer** out,
                                          char* err, size_t err_len) {
  STWO_ARG_CHECK(out != nullptr, "null out");
  STWO_ARG_CHECK(n_cols >= 1 && log_sizes != nullptr, "a commitment needs at least one column");
  STWO_ARG_CHECK(log_blowup >= 1 && log_blowup <= 8, "log_blowup %u out of range", log_blowup);
  STWO_ARG_CHECK(d_twiddles && d_itwiddles, "null twiddle tree");
  STWO_ARG_CHECK((flags & ~(uint32_t)(STWO_B200_COMMIT_PER_COLUMN | STWO_B200_COMMIT_GRAPH)) == 0, "unknown flags");
  uint32_t mx = 0;
  for (uint32_t i = 0; i < n_cols; i++) {
    STWO_ARG_CHECK(log_sizes[i] >= 1 && log_sizes[i] + log_blowup <= 30, "column log size %u out of range",
                   log_sizes[i]);
    mx = std::max(mx, log_sizes[i]);
  }
  STWO_ARG_CHECK(mx + log_blowup - 1 <= tree_log_size, "twiddle tree (log %u) too small", tree_log_size);
  auto* h = new stwo_b200_committer();
  Committer& c = h->c;
  c.logs.assign(log_sizes, log_sizes + n_cols);
  c.blowup = log_blowup;
  c.L = mx + log_blowup;
  c.m31 = m31_output;
  c.tw = d_twiddles;
  c.itw = d_itwiddles;
  c.tree_log = tree_log_size;
  c.flags = flags;
  cudaError_t e = cudaStreamCreateWithFlags(&c.s, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c.ev_in, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c.ev_out, cudaEventDisableTiming);
  if (e != cudaSuccess) {
    delete h;
    return set_err(err, err_len, STWO_B200_ECUDA, "committer: %s", cudaGetErrorString(e));
  }
  *out = h;
  return ok(err, err_len);
}

extern "C" int stwo_b200_committer_destroy(stwo_b200_committer* c, char* err, size_t err_len) {
  delete c;
  return ok(err, err_len);
}

extern "C" int stwo_b200_committer_lifting_log_size(const stwo_b200_committer* c, uint32_t* out, char* err,
                                                    size_t err_len) {
  STWO_ARG_CHECK(c && out, "null argument");
  *out = c->c.L;
  return ok(err, err_len);
}

extern "C" int stwo_b200_committer_commit(stwo_b200_committer* c, const uint32_t* const* d_evals,
                                          uint32_t* const* d_coeffs, uint32_t* const* d_ldes,
                                          uint8_t* const* d_layers, void* stream, char* err, size_t err_len) {
  STWO_ARG_CHECK(c && d_evals && d_coeffs && d_ldes && d_layers, "null argument");
  int rc = c->c.commit(d_evals, d_coeffs, d_ldes, d_layers, as_stream(stream), err, err_len);
  return rc ? rc : ok(err, err_len);
}

extern "C" int stwo_b200_committer_commit_from_host(stwo_b200_committer* c, const uint32_t* const* h_evals,
                                                    uint32_t* const* d_evals, uint32_t* const* d_coeffs,
                                                    uint32_t* const* d_ldes, uint8_t* const* d_layers, void* stream,
                                                    char* err, size_t err_len) {
  STWO_ARG_CHECK(c && h_evals && d_evals && d_coeffs && d_ldes && d_layers, "null argument");
  int rc = c->c.commit_from_host(h_evals, d_evals, d_coeffs, d_ldes, d_layers, as_stream(stream), err, err_len);
  return rc ? rc : ok(err, err_len);
}

extern "C" int stwo_b200_committer_autotune(stwo_b200_committer* h, const uint32_t* const* d_evals,
                                            uint32_t* const* d_coeffs, uint32_t* const* d_ldes,
                                            const char* cache_path, uint32_t reps, char* err, size_t err_len) {
  STWO_ARG_CHECK(h && d_evals && d_coeffs && d_ldes, "null argument");
  Committer& c = h->c;
  // groups: log size -> columns
  std::map<uint32_t, std::vector<uint32_t>> groups;
  for (uint32_t i = 0; i < c.logs.size(); i++) groups[c.logs[i]].push_back(i);
  // cache: "log_size n_columns T1,T2,..." per line
  std::map<std::pair<uint32_t, uint32_t>, std::vector<uint32_t>> cache;
  if (cache_path) {
    if (FILE* f = std::fopen(cache_path, "r")) {
      unsigned n, k;
      char buf[64];
      while (std::fscanf(f, "%u %u %63s", &n, &k, buf) == 3) {
        std::vector<uint32_t> t;
        for (char* p = buf; *p;) {
          t.push_back((uint32_t)std::strtoul(p, &p, 10));
          if (*p == ',') p++;
        }
        cache[{n, k}] = t;
      }
      std::fclose(f);
    }
  }
  bool tuned_any = false;
  reps = std::max<uint32_t>(1, std::min<uint32_t>(reps, 20));
  cudaEvent_t a, b;
  STWO_CUDA_TRY(cudaEventCreate(&a));
  STWO_CUDA_TRY(cudaEventCreate(&b));
  int rc = 0;
  for (auto& kv : groups) {
    const uint32_t n = kv.first, k = (uint32_t)kv.second.size();
    auto hit = cache.find({n, k});
    if (hit != cache.end()) {
      if ((rc = stwo_b200_fft_set_plan(n, hit->second.data(), (uint32_t)hit->second.size(), err, err_len))) break;
      continue;
    }
    std::vector<uint32_t> best;
    float best_ms = 1e30f;
    for (const auto& cand : candidate_splits(n)) {
      if ((rc = stwo_b200_fft_set_plan(n, cand.data(), (uint32_t)cand.size(), err, err_len))) break;
      if ((rc = c.transform(d_evals, d_coeffs, d_ldes, kv.second, err, err_len))) break;  // warm-up
      cudaEventRecord(a, c.s);
      for (uint32_t r = 0; r < reps && !rc; r++)
        rc = c.transform(d_evals, d_coeffs, d_ldes, kv.second, err, err_len);
      cudaEventRecord(b, c.s);
      if (rc) break;
      if (cudaEventSynchronize(b) != cudaSuccess) {
        rc = set_err(err, err_len, STWO_B200_ECUDA, "autotune: %s", cudaGetErrorString(cudaGetLastError()));
        break;
      }
      float ms = 0;
      cudaEventElapsedTime(&ms, a, b);
      if (ms < best_ms) {
        best_ms = ms;
        best = cand;
      }
    }
    if (rc) break;
    if ((rc = stwo_b200_fft_set_plan(n, best.data(), (uint32_t)best.size(), err, err_len))) break;
    cache[{n, k}] = best;
    tuned_any = true;
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  if (rc) return rc;
  c.drop_graph();  // plans changed: recapture on the next commit
  if (cache_path && tuned_any) {
    if (FILE* f = std::fopen(cache_path, "w")) {
      for (auto& kv : cache) std::fprintf(f, "%u %u %s\n", kv.first.first, kv.first.second, split_str(kv.second).c_str());
      std::fclose(f);
    }
  }
  return ok(err, err_len);
}
