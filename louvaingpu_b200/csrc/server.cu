// Request server over the batched runner (continuous batching).
//
// n_slots worker threads each own one lvg_ctx (its own CUDA stream and a
// device arena of hbm_budget / n_slots bytes, reserved on first use and kept).
// A slot that is free takes the queued requests in arrival order -- as many as
// its arena holds by lvg_batch_footprint, within the entry and graph caps --
// and runs them as one batched dendrogram run; the slots run at the same time
// on their own streams, so new requests start while earlier batches are still
// on the device.  A request that arrives alone runs through lvg_run.  The
// reference has no serving path: it runs one graph per process
// (LouvainCPP.cpp:209).
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/lvg.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Req {
  int64_t id, tag;
  const int32_t* src;
  const int32_t* dst;
  const float* w;
  int64_t E;
  int32_t V;
  int32_t* part_out;
  int64_t t_submit;
};

}  // namespace

struct lvg_server {
  lvg_config cfg{};
  int32_t n_slots = 0;
  int64_t slot_bytes = 0;
  int64_t max_entries = 0;
  int32_t max_graphs = 0;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Req> pending;
  std::deque<lvg_serve_result> done;
  int64_t submitted = 0, completed = 0, batches = 0, next_id = 0;
  int32_t live_slots = 0, used_slots = 0, started = 0;
  bool stopping = false;
  std::string err;
  std::vector<std::thread> workers;
  Clock::time_point t0;

  int64_t now() const {
    return std::chrono::duration_cast<std::chrono::nanoseconds>(Clock::now() - t0).count();
  }
};

namespace {

int64_t footprint(int64_t V, int64_t E, int32_t G) {
  int64_t b = 0;
  lvg_batch_footprint(V, E, G, &b);
  return b;
}

void post(lvg_server* S, const std::vector<lvg_serve_result>& rs) {
  std::lock_guard<std::mutex> lk(S->mu);
  for (const auto& r : rs) S->done.push_back(r);
  S->completed += (int64_t)rs.size();
  S->cv_done.notify_all();
}

lvg_serve_result result_of(const Req& r, int64_t t_start) {
  lvg_serve_result x;
  std::memset(&x, 0, sizeof x);
  x.id = r.id;
  x.tag = r.tag;
  x.t_submit_ns = r.t_submit;
  x.t_start_ns = t_start;
  return x;
}

// One request alone: the plain path.
void run_one(lvg_server* S, lvg_ctx* ctx, const Req& r, int64_t t_start) {
  lvg_serve_result x = result_of(r, t_start);
  x.batch_graphs = 1;
  lvg_status st = lvg_load_edges_device(ctx, r.src, r.dst, r.w, r.E, r.V);
  if (st == LVG_OK) {
    lvg_result res;
    st = lvg_run(ctx, &res);
    if (st == LVG_OK || st == LVG_ERR_NOT_CONVERGED) {
      x.n_levels = res.n_levels;
      x.n_comms = res.n_comms;
      x.q_final = res.q_final;
      if (r.part_out && r.V > 0) {
        lvg_status ps = lvg_get_partition(ctx, 0x7fffffff, r.part_out);   // last level
        if (ps != LVG_OK) st = ps;
      }
    }
  }
  x.status = st;
  x.t_done_ns = S->now();
  post(S, {x});
}

// A group as one batched run; on an arena overflow the group is split in two.
void run_group(lvg_server* S, lvg_ctx* ctx, const std::vector<Req>& grp, int64_t t_start) {
  const int32_t G = (int32_t)grp.size();
  if (G == 1) {
    run_one(S, ctx, grp[0], t_start);
    return;
  }
  std::vector<const int32_t*> src(G), dst(G);
  std::vector<const float*> w(G);
  std::vector<int64_t> ne(G);
  std::vector<int32_t> nv(G), lev(G), com(G), stat(G);
  std::vector<double> q(G);
  int64_t V = 0;
  for (int32_t g = 0; g < G; ++g) {
    src[g] = grp[g].src;
    dst[g] = grp[g].dst;
    w[g] = grp[g].w;
    ne[g] = grp[g].E;
    nv[g] = grp[g].V;
    V += grp[g].V;
  }
  std::vector<int32_t> part((size_t)std::max<int64_t>(V, 1));
  lvg_status st = lvg_batch_run_graphs(ctx, G, src.data(), dst.data(), w.data(), ne.data(), nv.data(), part.data(),
                                       q.data(), lev.data(), com.data(), stat.data());
  if (st == LVG_ERR_OOM) {
    std::vector<Req> a(grp.begin(), grp.begin() + G / 2), b(grp.begin() + G / 2, grp.end());
    run_group(S, ctx, a, t_start);
    run_group(S, ctx, b, t_start);
    return;
  }
  const int64_t t_done = S->now();
  std::vector<lvg_serve_result> rs;
  rs.reserve(G);
  int64_t off = 0;
  for (int32_t g = 0; g < G; ++g) {
    lvg_serve_result x = result_of(grp[g], t_start);
    x.batch_graphs = G;
    x.status = st == LVG_OK ? stat[g] : st;
    if (st == LVG_OK) {
      x.n_levels = lev[g];
      x.n_comms = com[g];
      x.q_final = q[g];
      if (grp[g].part_out && grp[g].V > 0)
        std::memcpy(grp[g].part_out, part.data() + off, sizeof(int32_t) * grp[g].V);
    }
    off += grp[g].V;
    x.t_done_ns = t_done;
    rs.push_back(x);
  }
  post(S, rs);
}

void fail_pending(lvg_server* S, std::unique_lock<std::mutex>& lk, lvg_status why) {
  while (!S->pending.empty()) {
    lvg_serve_result x = result_of(S->pending.front(), S->now());
    x.status = why;
    x.t_done_ns = x.t_start_ns;
    S->done.push_back(x);
    S->pending.pop_front();
    S->completed += 1;
  }
  S->cv_done.notify_all();
  (void)lk;
}

void worker(lvg_server* S) {
  lvg_config cfg = S->cfg;
  cfg.arena_bytes = S->slot_bytes;
  cfg.l2_persist = 0;      // the persisting-L2 window is per device, not per slot
  lvg_ctx* ctx = nullptr;
  lvg_status cs = lvg_create(&cfg, &ctx);
  if (cs == LVG_OK) cs = lvg_reserve(ctx, S->slot_bytes);   // the slot's share of the budget, once
  std::unique_lock<std::mutex> lk(S->mu);
  S->started += 1;
  S->cv_done.notify_all();
  if (cs != LVG_OK) {
    S->err = "a serving slot could not create its context or reserve its memory";
    if (ctx) {
      lk.unlock();
      lvg_destroy(ctx);
      lk.lock();
    }
    if (--S->live_slots == 0) fail_pending(S, lk, cs);
    return;
  }
  S->used_slots += 1;
  for (;;) {
    S->cv_work.wait(lk, [&] { return S->stopping || !S->pending.empty(); });
    if (S->pending.empty()) {
      if (S->stopping) break;
      continue;
    }
    std::vector<Req> grp;
    int64_t E = 0, V = 0;
    while (!S->pending.empty() && (int32_t)grp.size() < S->max_graphs) {
      const Req& r = S->pending.front();
      if (!grp.empty() && (E + r.E > S->max_entries ||
                           footprint(V + r.V, E + r.E, (int32_t)grp.size() + 1) > S->slot_bytes))
        break;
      grp.push_back(r);
      S->pending.pop_front();
      E += r.E;
      V += r.V;
    }
    S->batches += 1;
    const int64_t t_start = S->now();
    lk.unlock();
    run_group(S, ctx, grp, t_start);
    lk.lock();
    S->cv_work.notify_all();
  }
  lk.unlock();
  lvg_destroy(ctx);
}

}  // namespace

extern "C" {

lvg_status lvg_server_create(const lvg_config* cfg, int32_t n_slots, int64_t hbm_budget_bytes,
                             int64_t max_batch_entries, int32_t max_batch_graphs, lvg_server** out) {
  if (!out) return LVG_ERR_INVALID_ARG;
  *out = nullptr;
  if (n_slots < 1 || hbm_budget_bytes <= 0 || max_batch_entries < 1 || max_batch_graphs < 1)
    return LVG_ERR_INVALID_ARG;
  auto* S = new (std::nothrow) lvg_server();
  if (!S) return LVG_ERR_OOM;
  if (cfg) S->cfg = *cfg;
  else lvg_config_default(&S->cfg);
  S->n_slots = n_slots;
  S->slot_bytes = hbm_budget_bytes / n_slots;
  S->max_entries = max_batch_entries;
  S->max_graphs = max_batch_graphs;
  S->t0 = Clock::now();
  S->live_slots = n_slots;
  try {
    for (int32_t k = 0; k < n_slots; ++k) S->workers.emplace_back(worker, S);
  } catch (...) {
    {
      std::lock_guard<std::mutex> lk(S->mu);
      S->stopping = true;
      S->live_slots = (int32_t)S->workers.size();
    }
    S->cv_work.notify_all();
    for (auto& t : S->workers) t.join();
    delete S;
    return LVG_ERR_OOM;
  }
  {
    // every slot has its memory (or has failed) before the first request
    std::unique_lock<std::mutex> lk(S->mu);
    S->cv_done.wait(lk, [&] { return S->started >= n_slots; });
  }
  *out = S;
  return LVG_OK;
}

lvg_status lvg_server_submit(lvg_server* S, const int32_t* d_src, const int32_t* d_dst, const float* d_w,
                             int64_t n_entries, int32_t n_vertices, int32_t* part_out, int64_t tag,
                             int64_t* id_out) {
  if (!S || n_entries < 0 || n_vertices < 0 || (n_entries > 0 && (!d_src || !d_dst || !d_w)))
    return LVG_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(S->mu);
  if (S->stopping) {
    S->err = "server is stopping";
    return LVG_ERR_STATE;
  }
  if (S->live_slots == 0) {
    S->err = "no serving slot is alive";
    return LVG_ERR_STATE;
  }
  if (footprint(n_vertices, n_entries, 1) > S->slot_bytes) {
    S->err = "the graph needs more device memory than one slot holds";
    return LVG_ERR_CAPACITY;
  }
  Req r{S->next_id++, tag, d_src, d_dst, d_w, n_entries, n_vertices, part_out, S->now()};
  S->pending.push_back(r);
  S->submitted += 1;
  if (id_out) *id_out = r.id;
  S->cv_work.notify_one();
  return LVG_OK;
}

lvg_status lvg_server_poll(lvg_server* S, lvg_serve_result* out, int32_t max, int32_t* n_out) {
  if (!S || !n_out || max < 0 || (max > 0 && !out)) return LVG_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(S->mu);
  int32_t n = 0;
  while (n < max && !S->done.empty()) {
    out[n++] = S->done.front();
    S->done.pop_front();
  }
  *n_out = n;
  return LVG_OK;
}

lvg_status lvg_server_drain(lvg_server* S, int64_t timeout_ms) {
  if (!S) return LVG_ERR_INVALID_ARG;
  std::unique_lock<std::mutex> lk(S->mu);
  auto all_done = [&] { return S->completed >= S->submitted; };
  if (timeout_ms < 0) {
    S->cv_done.wait(lk, all_done);
    return LVG_OK;
  }
  if (!S->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), all_done)) {
    S->err = "drain timed out";
    return LVG_ERR_STATE;
  }
  return LVG_OK;
}

lvg_status lvg_server_stats(lvg_server* S, int64_t* submitted, int64_t* completed, int64_t* batches,
                            int64_t* reserved_bytes) {
  if (!S) return LVG_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(S->mu);
  if (submitted) *submitted = S->submitted;
  if (completed) *completed = S->completed;
  if (batches) *batches = S->batches;
  if (reserved_bytes) *reserved_bytes = (int64_t)S->used_slots * S->slot_bytes;
  return LVG_OK;
}

// Workers write the message under the lock; the caller gets a copy that stays
// valid until its own thread's next call.
const char* lvg_server_last_error(const lvg_server* S) {
  if (!S) return "null server";
  static thread_local std::string copy;
  std::lock_guard<std::mutex> lk(const_cast<lvg_server*>(S)->mu);
  copy = S->err;
  return copy.c_str();
}

lvg_status lvg_server_destroy(lvg_server* S) {
  if (!S) return LVG_ERR_INVALID_ARG;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->stopping = true;
  }
  S->cv_work.notify_all();
  for (auto& t : S->workers)
    if (t.joinable()) t.join();
  delete S;
  return LVG_OK;
}

}  // extern "C"
