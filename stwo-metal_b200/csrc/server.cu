// Prove-request serving on one GPU: continuous batching of Wide-Fibonacci
// proofs (the serving pattern of the commit + FRI path; the reference proves
// one request at a time through prover::prove, crates/stwo/src/prover/mod.rs:
// 32-138, and has no serving loop).
//
// - `slots` worker threads; each admitted request runs on its own prover and
//   stream, so requests that are admitted while others run overlap on the
//   device (their host-side Fiat-Shamir steps and launch gaps fill each other's
//   idle time).
// - Resident provers: device buffers, twiddles and the captured FRI graph of a
//   (log_n_rows, column class, PCS config) shape stay allocated between
//   requests; the column class is the width rounded up to a multiple of 64, so
//   any width up to it reuses the buffers (stwo_b200_prove_wide_fib_cols).
// - Admission by HBM footprint: a request is admitted when a slot is free and
//   its shape has an idle resident prover, or a new one fits the budget after
//   evicting idle residents, least recently used first.  The queue is scanned
//   in arrival order and the first admissible request is taken.
// The proof of a request does not depend on what else runs: every prover owns
// its buffers and stream, and the kernels are deterministic.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <list>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "common.cuh"
#include "stwo_b200.h"

namespace stwo_b200 {

using Clock = std::chrono::steady_clock;

struct ShapeKey {
  uint32_t v[8];
  bool operator==(const ShapeKey& o) const { return std::memcmp(v, o.v, sizeof(v)) == 0; }
};

static ShapeKey shape_of(const stwo_b200_wide_fib_config& c, uint32_t cap) {
  return ShapeKey{{c.log_n_rows, cap, c.log_blowup, c.pow_bits, c.n_queries, c.log_last_layer_degree_bound,
                   c.line_fold_step, (uint32_t)c.m31_channel}};
}

struct Resident {
  ShapeKey key;
  stwo_b200_wide_fib_config cfg;  // n_cols = the column class
  stwo_b200_prover* prover = nullptr;
  cudaStream_t stream = nullptr;
  uint32_t* d_a = nullptr;
  uint32_t* d_b = nullptr;
  size_t bytes = 0;
  bool busy = false, ready = false;
  uint64_t last_used = 0;
};

struct Request {
  uint64_t ticket = 0;
  stwo_b200_wide_fib_config cfg;
  std::vector<uint32_t> a, b;
  size_t need = 0;
  Clock::time_point t_submit, t_admit, t_done;
  std::vector<uint8_t> proof;
  int rc = 0;
  std::string err;
  bool done = false;
};

constexpr size_t kMaxProofBytes = (size_t)16 << 20;  // far above any Wide-Fibonacci proof

static uint32_t column_class(uint32_t n_cols) { return std::min<uint32_t>((n_cols + 63) / 64 * 64, 1016); }

struct Server {
  size_t budget = 0, used = 0;
  uint32_t slots = 1;
  int device = 0;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Request*> queue;
  std::map<uint64_t, Request*> reqs;
  std::list<Resident*> residents;
  uint64_t next_ticket = 1, tick = 0;
  bool stopping = false;
  uint64_t n_done = 0, n_created = 0, n_reused = 0, n_evicted = 0;
  uint32_t running = 0, max_running = 0;
  std::vector<std::thread> workers;

  static void destroy_resident(Resident* r) {
    if (r->prover) stwo_b200_prover_destroy(r->prover, nullptr, 0);
    if (r->d_a) cudaFree(r->d_a);
    if (r->d_b) cudaFree(r->d_b);
    if (r->stream) cudaStreamDestroy(r->stream);
    delete r;
  }

  // Under mu.  An idle resident of r's shape, or a reservation for a new one
  // (after evicting idle residents into *evict); nullptr when r must wait.
  Resident* acquire(Request* r, std::vector<Resident*>* evict) {
    const uint32_t cap = column_class(r->cfg.n_cols);
    const ShapeKey key = shape_of(r->cfg, cap);
    for (Resident* x : residents)
      if (!x->busy && x->ready && x->key == key) {
        x->busy = true;
        n_reused++;
        return x;
      }
    if (used + r->need > budget) {
      std::vector<Resident*> idle;
      size_t freeable = 0;
      for (Resident* x : residents)
        if (!x->busy && x->ready) {
          idle.push_back(x);
          freeable += x->bytes;
        }
      if (used - freeable + r->need > budget) return nullptr;
      std::sort(idle.begin(), idle.end(), [](Resident* p, Resident* q) { return p->last_used < q->last_used; });
      for (Resident* x : idle) {
        if (used + r->need <= budget) break;
        residents.remove(x);
        used -= x->bytes;
        evict->push_back(x);
        n_evicted++;
      }
    }
    Resident* x = new Resident();
    x->key = key;
    x->cfg = r->cfg;
    x->cfg.n_cols = cap;
    x->bytes = r->need;
    x->busy = true;
    used += r->need;
    residents.push_back(x);
    n_created++;
    return x;
  }

  void worker() {
    cudaSetDevice(device);
    char err[512];
    for (;;) {
      Request* r = nullptr;
      Resident* res = nullptr;
      std::vector<Resident*> evict;
      {
        std::unique_lock<std::mutex> lk(mu);
        cv_work.wait(lk, [&] {
          for (auto it = queue.begin(); it != queue.end(); ++it)
            if ((res = acquire(*it, &evict))) {
              r = *it;
              queue.erase(it);
              return true;
            }
          return stopping && queue.empty();
        });
        if (!r) return;
        r->t_admit = Clock::now();
        max_running = std::max(max_running, ++running);
      }
      for (Resident* e : evict) destroy_resident(e);
      int rc = 0;
      err[0] = 0;
      if (!res->ready) {
        cudaError_t ce = cudaStreamCreateWithFlags(&res->stream, cudaStreamNonBlocking);
        if (ce == cudaSuccess) ce = cudaMalloc(&res->d_a, 4ull << res->cfg.log_n_rows);
        if (ce == cudaSuccess) ce = cudaMalloc(&res->d_b, 4ull << res->cfg.log_n_rows);
        if (ce != cudaSuccess)
          rc = set_err(err, sizeof(err), STWO_B200_ENOMEM, "resident buffers: %s", cudaGetErrorString(ce));
        if (!rc) rc = stwo_b200_prover_create(&res->cfg, &res->prover, res->stream, err, sizeof(err));
      }
      const size_t nb = 4ull << r->cfg.log_n_rows;
      if (!rc) rc = stwo_b200_memcpy_h2d(res->d_a, r->a.data(), nb, res->stream, err, sizeof(err));
      if (!rc) rc = stwo_b200_memcpy_h2d(res->d_b, r->b.data(), nb, res->stream, err, sizeof(err));
      size_t len = 0;
      if (!rc) {
        r->proof.resize(kMaxProofBytes);
        rc = stwo_b200_prove_wide_fib_cols(res->prover, r->cfg.n_cols, res->d_a, res->d_b, r->proof.data(),
                                           r->proof.size(), &len, err, sizeof(err));
        r->proof.resize(rc ? 0 : len);
      }
      std::lock_guard<std::mutex> lk(mu);
      r->rc = rc;
      if (rc) r->err = err;
      r->t_done = Clock::now();
      r->done = true;
      running--;
      n_done++;
      if (rc && !res->ready) {  // a resident that never came up: release its reservation
        residents.remove(res);
        used -= res->bytes;
        destroy_resident(res);
      } else {
        res->ready = true;
        res->busy = false;
        res->last_used = ++tick;
      }
      cv_done.notify_all();
      cv_work.notify_all();
    }
  }
};

}  // namespace stwo_b200

using namespace stwo_b200;

struct stwo_b200_server {
  Server s;
};

extern "C" int stwo_b200_server_create(size_t hbm_budget_bytes, uint32_t slots, stwo_b200_server** out, char* err,
                                       size_t err_len) {
  STWO_ARG_CHECK(out, "null out");
  STWO_ARG_CHECK(slots >= 1 && slots <= 16, "slots %u out of range [1, 16]", slots);
  STWO_ARG_CHECK(hbm_budget_bytes > 0, "zero HBM budget");
  auto* h = new stwo_b200_server();
  h->s.budget = hbm_budget_bytes;
  h->s.slots = slots;
  cudaGetDevice(&h->s.device);
  for (uint32_t i = 0; i < slots; i++) h->s.workers.emplace_back([h] { h->s.worker(); });
  *out = h;
  return ok(err, err_len);
}

extern "C" int stwo_b200_server_destroy(stwo_b200_server* h, char* err, size_t err_len) {
  if (!h) return ok(err, err_len);
  {
    std::lock_guard<std::mutex> lk(h->s.mu);
    h->s.stopping = true;
  }
  h->s.cv_work.notify_all();
  for (auto& t : h->s.workers) t.join();
  for (Resident* r : h->s.residents) Server::destroy_resident(r);
  for (auto& kv : h->s.reqs) delete kv.second;
  delete h;
  return ok(err, err_len);
}

extern "C" int stwo_b200_server_submit(stwo_b200_server* h, const stwo_b200_wide_fib_config* cfg, const uint32_t* a,
                                       const uint32_t* b, uint64_t* ticket, char* err, size_t err_len) {
  STWO_ARG_CHECK(h && cfg && a && b && ticket, "null argument");
  STWO_ARG_CHECK(cfg->n_cols >= 3 && cfg->n_cols <= 1016, "n_cols %u out of range [3, 1016]", cfg->n_cols);
  stwo_b200_wide_fib_config klass = *cfg;
  klass.n_cols = column_class(cfg->n_cols);
  size_t fp = 0;
  int rc = stwo_b200_prover_footprint(&klass, &fp, err, err_len);
  if (rc) return rc;
  const size_t need = fp + (8ull << cfg->log_n_rows);  // + the two input columns
  STWO_ARG_CHECK(need <= h->s.budget, "request needs %zu bytes, more than the HBM budget %zu", need, h->s.budget);
  auto* r = new Request();
  r->cfg = *cfg;
  const size_t n = (size_t)1 << cfg->log_n_rows;
  r->a.assign(a, a + n);
  r->b.assign(b, b + n);
  r->need = need;
  r->t_submit = Clock::now();
  {
    std::lock_guard<std::mutex> lk(h->s.mu);
    STWO_ARG_CHECK(!h->s.stopping, "server is stopping");
    r->ticket = h->s.next_ticket++;
    h->s.reqs[r->ticket] = r;
    h->s.queue.push_back(r);
    *ticket = r->ticket;
  }
  h->s.cv_work.notify_all();
  return ok(err, err_len);
}

extern "C" int stwo_b200_server_wait(stwo_b200_server* h, uint64_t ticket, uint8_t* proof_out, size_t proof_cap,
                                     size_t* proof_len, double* times_ms, char* err, size_t err_len) {
  STWO_ARG_CHECK(h && proof_len, "null argument");
  Request* r = nullptr;
  {
    std::unique_lock<std::mutex> lk(h->s.mu);
    auto it = h->s.reqs.find(ticket);
    STWO_ARG_CHECK(it != h->s.reqs.end(), "unknown ticket %llu", (unsigned long long)ticket);
    r = it->second;
    h->s.cv_done.wait(lk, [&] { return r->done; });
    h->s.reqs.erase(ticket);
  }
  std::unique_ptr<Request> own(r);
  if (times_ms) {
    using ms = std::chrono::duration<double, std::milli>;
    times_ms[0] = ms(r->t_admit - r->t_submit).count();  // queued
    times_ms[1] = ms(r->t_done - r->t_admit).count();    // on a prover
    times_ms[2] = ms(r->t_done - r->t_submit).count();   // latency
  }
  if (r->rc) return set_err(err, err_len, r->rc, "%s", r->err.c_str());
  *proof_len = r->proof.size();
  if (proof_out) {
    STWO_ARG_CHECK(proof_cap >= r->proof.size(), "proof buffer too small (%zu < %zu)", proof_cap, r->proof.size());
    std::memcpy(proof_out, r->proof.data(), r->proof.size());
  }
  return ok(err, err_len);
}

extern "C" int stwo_b200_server_get_stats(stwo_b200_server* h, stwo_b200_server_stats* out, char* err, size_t err_len) {
  STWO_ARG_CHECK(h && out, "null argument");
  std::lock_guard<std::mutex> lk(h->s.mu);
  out->completed = h->s.n_done;
  out->provers_created = h->s.n_created;
  out->provers_reused = h->s.n_reused;
  out->provers_evicted = h->s.n_evicted;
  out->resident_bytes = h->s.used;
  out->residents = (uint32_t)h->s.residents.size();
  out->max_running = h->s.max_running;
  out->queued = (uint32_t)h->s.queue.size();
  return ok(err, err_len);
}
