// Context, level driver and the extern "C" entry points of liblvg.
//
// The level loop restates generate_dendogram (LouvainCPP.cpp:209-553):
// level 0 runs CSR build -> Q of the singleton state -> one-level -> renumber ->
// induce; every further level runs CSR build -> one-level -> renumber, stops
// when the level's Q gain is below level_min_gain (LouvainCPP.cpp:466), else
// induces the next level.  Unlike the reference, the level input lists stay on
// the device between levels (no host round trip, LouvainCPP.cpp:390-412,477-499).
#include <algorithm>
#include <atomic>
#include <climits>
#include <cmath>
#include <numeric>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "louvain.cuh"
#include "prims.cuh"

using namespace lvg;

namespace lvg {
static std::atomic<int64_t> g_launches{0};
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
}  // namespace lvg

namespace {

struct LevelRec {
  lvg_level_info info;
  int32_t* d_part = nullptr;    // renumbered partition (arena high end, run lifetime)
  int32_t* d_labels = nullptr;  // community labels before renumbering
};

}  // namespace

struct lvg_ctx {
  lvg_config cfg;
  Tuning tune;
  int device = 0;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  Arena arena;
  std::string err;
  // level-0 graph
  bool loaded = false;
  int32_t V0 = 0;
  int64_t E0 = 0;
  const int32_t* src0 = nullptr;
  const int32_t* dst0 = nullptr;
  const float* w0 = nullptr;
  int32_t* composed = nullptr;   // partition of the level-0 vertices through the last renumbered level
  size_t base_lo = 0;            // arena low mark above the level-0 list and `composed`
  size_t run_hi = 0;             // arena high mark above the per-level partitions
  // current level
  int level = 0;
  LevelGraph g;
  CommState st;
  bool have_state = false;
  bool renumbered = false;
  bool pristine = false;         // level 0 as loaded: no pass, state change or renumbering since
  bool symmetric0 = false;       // the level-0 list was found sorted and symmetric at load
  int32_t* d_part_cur = nullptr;
  int32_t C_cur = 0;
  std::vector<LevelRec> levels;
  std::vector<float> pass_ms;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  cudaEvent_t pev[6] = {};        // phase timing: build, renumber, induce (start, end)
  SideStreams side{};
  bool have_side = false;
  std::vector<cudaEvent_t> mev;   // move-phase events, two per pass
  cudaGraphExec_t g_moves = nullptr;   // captured move kernels of one pass (current level)
  cudaGraphExec_t g_commit = nullptr;  // captured commit + pass control
  size_t persist_max = 0;         // device limits for L2 persistence
  size_t window_max = 0;
  double move_ms = 0.0;
  int64_t move_passes = 0;
  std::vector<float> move_pass_ms;  // move kernels of each pass of the last one-level phase
  PreCsr pre0;                    // level-0 CSR built during a chunked host upload
  PreCsr pre_next;                // CSR of the level just coarsened into, written by the coarsening
  cudaStream_t copy_stream = nullptr;   // host-list upload chunks (lvg_load_edges)
  std::vector<cudaEvent_t> load_ev;     // one per upload chunk
};

namespace {

lvg_status fail(lvg_ctx* c, lvg_status s, const std::string& m) {
  if (c) c->err = m;
  return s;
}

template <typename F>
lvg_status guarded(lvg_ctx* c, F&& f) {
  try {
    f();
    if (c) c->err.clear();
    return LVG_OK;
  } catch (const Error& e) {
    return fail(c, e.status, e.what());
  } catch (const std::bad_alloc&) {
    return fail(c, LVG_ERR_OOM, "host allocation failed");
  } catch (const std::exception& e) {
    return fail(c, LVG_ERR_CUDA, e.what());
  }
}

void require(bool ok, lvg_status s, const char* m) {
  if (!ok) throw Error(s, m);
}

float elapsed(cudaEvent_t a, cudaEvent_t b) {
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, a, b);
  return ms;
}

// Device bytes for a level-0 graph of V vertices and E entries: level-0 list
// copy, composed partition, CSR + per-vertex arrays + community state, and the
// largest phase scratch (the doubled-list sort of the CSR build).
size_t arena_estimate(int64_t V, int64_t E, bool copy_list) {
  size_t b = 0;
  if (copy_list) b += 12 * (size_t)E;
  b += 4 * (size_t)V;                       // composed
  b += 16 * (size_t)E + 80 * (size_t)V;     // CSR (<= 2E entries) + per-vertex + state
  b += 88 * (size_t)E + 24 * (size_t)V;     // build scratch: 2 x 2E x 12 B sort, head/pos, wsum
  b += 16 * (size_t)E;                      // hub tables (degree-bounded) and per-level partitions
  b += 36 * (size_t)V + (size_t)E / 4;      // first-pass chunk lists, partials, int32 degrees
  b += (size_t)64 << 20;
  return b;
}

void sync(lvg_ctx* c) { LVG_CUDA(cudaStreamSynchronize(c->stream)); }

// Prepare the current level (c->g holds the level input list): build, state.
void drop_graphs(lvg_ctx* c) {
  if (c->g_moves) cudaGraphExecDestroy(c->g_moves);
  if (c->g_commit) cudaGraphExecDestroy(c->g_commit);
  c->g_moves = c->g_commit = nullptr;
}

// Capture the two halves of a pass once per level; replaying them replaces
// about a dozen launches and the side-stream fork/join per pass.
void ensure_graphs(lvg_ctx* c) {
  if (c->g_moves && c->g_commit) return;
  cudaStream_t s = c->stream;
  cudaGraph_t gr = nullptr;
  LVG_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  launch_moves(c->g, c->st, s, &c->side);
  LVG_CUDA(cudaStreamEndCapture(s, &gr));
  LVG_CUDA(cudaGraphInstantiate(&c->g_moves, gr, 0));
  cudaGraphDestroy(gr);
  LVG_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  launch_commit(c->g, c->st, s);
  LVG_CUDA(cudaStreamEndCapture(s, &gr));
  LVG_CUDA(cudaGraphInstantiate(&c->g_commit, gr, 0));
  cudaGraphDestroy(gr);
}

void prepare_level(lvg_ctx* c) {
  drop_graphs(c);
  LVG_CUDA(cudaEventRecord(c->pev[0], c->stream));
  build_level(c->g, c->tune, c->arena, c->stream);
  c->st.gid = nullptr;     // one graph (a batch that failed part-way may have left its maps)
  c->st.gdone = nullptr;
  alloc_state(c->g, c->st, c->arena);
  init_state(c->g, c->st, 0.0, c->cfg.pass_min_gain, c->cfg.max_passes, c->arena, c->stream);
  LVG_CUDA(cudaEventRecord(c->pev[1], c->stream));   // read once the stream has synchronised
  c->have_state = true;
  c->renumbered = false;
}

void load_common(lvg_ctx* c, const int32_t* d_src, const int32_t* d_dst, const float* d_w, int64_t E,
                 int32_t V) {
  c->V0 = V;
  c->E0 = E;
  c->src0 = d_src;
  c->dst0 = d_dst;
  c->w0 = d_w;
  c->composed = c->arena.lo_n<int32_t>(V);
  iota(c->composed, V, c->stream);
  c->base_lo = c->arena.lo;
  c->run_hi = c->arena.hi;
  c->levels.clear();
  c->level = 0;
  c->g = LevelGraph();
  c->g.V = V;
  c->g.E = E;
  c->g.src = d_src;
  c->g.dst = d_dst;
  c->g.w = d_w;
  c->g.pre = &c->pre0;
  prepare_level(c);
  c->symmetric0 = c->g.sorted_symmetric;
  c->loaded = true;
  c->pristine = true;
}

void reset_to_level0(lvg_ctx* c) {
  // rebuild level 0 from the loaded list (used by lvg_run after partial steps)
  c->arena.lo = c->base_lo;
  c->arena.hi = c->run_hi = c->arena.cap;
  std::vector<int32_t> iota(c->V0);
  for (int32_t i = 0; i < c->V0; ++i) iota[i] = i;
  LVG_CUDA(cudaMemcpyAsync(c->composed, iota.data(), sizeof(int32_t) * c->V0, cudaMemcpyHostToDevice, c->stream));
  sync(c);
  c->levels.clear();
  c->level = 0;
  c->g = LevelGraph();
  c->g.V = c->V0;
  c->g.E = c->E0;
  c->g.src = c->src0;
  c->g.dst = c->dst0;
  c->g.w = c->w0;
  c->g.pre = &c->pre0;
  prepare_level(c);
  c->pristine = true;
}

double read_q(lvg_ctx* c) {
  HiScope hs(c->arena);
  double* d = c->arena.hi_n<double>(1);
  launch_q(c->g, c->st, d, c->stream);
  double q = 0.0;
  LVG_CUDA(cudaMemcpyAsync(&q, d, sizeof q, cudaMemcpyDeviceToHost, c->stream));
  sync(c);
  return q;
}

constexpr int kHardPassCap = 1 << 20;

// Keeps the gathered community arrays (tot, comm, size) in L2 while the move
// passes stream the CSR through it; the streams' previous windows come back
// when the scope ends.
struct L2Window {
  lvg_ctx* c;
  cudaStream_t streams[4];
  cudaStreamAttrValue saved[4];
  int n = 0;
  L2Window(lvg_ctx* ctx, const CommState& st) : c(ctx) {
    if (!c->cfg.l2_persist || c->persist_max == 0 || c->window_max == 0 || st.hot_bytes == 0) return;
    cudaStreamAttrValue v = {};
    size_t bytes = std::min(st.hot_bytes, c->window_max);
    v.accessPolicyWindow.base_ptr = (void*)st.tot;
    v.accessPolicyWindow.num_bytes = bytes;
    v.accessPolicyWindow.hitRatio = (float)std::min(1.0, (double)c->persist_max / (double)bytes);
    v.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
    v.accessPolicyWindow.missProp = cudaAccessPropertyStreaming;
    streams[0] = c->stream;
    for (int k = 0; k < 3; ++k) streams[k + 1] = c->side.side[k];
    for (int k = 0; k < 4; ++k) {
      if (cudaStreamGetAttribute(streams[k], cudaStreamAttributeAccessPolicyWindow, &saved[k]) != cudaSuccess) break;
      if (cudaStreamSetAttribute(streams[k], cudaStreamAttributeAccessPolicyWindow, &v) != cudaSuccess) break;
      n = k + 1;
    }
  }
  ~L2Window() {
    for (int k = 0; k < n; ++k) cudaStreamSetAttribute(streams[k], cudaStreamAttributeAccessPolicyWindow, &saved[k]);
    if (n) cudaCtxResetPersistingL2Cache();
  }
};

// One-level phase (oneLevelCUDA, OneLevelKernel.cu:518-954).
void one_level(lvg_ctx* c, double lower, double* q_out, int32_t* passes_out, int32_t* status_out,
               double* q_start_out) {
  cudaStream_t s = c->stream;
  c->pristine = false;
  init_state(c->g, c->st, lower, c->cfg.pass_min_gain, c->cfg.max_passes, c->arena, s);
  L2Window l2(c, c->st);
  // The first pass runs the singleton kernels and a level usually stops at
  // its second pass, so the hashing pass is captured only when a third pass
  // is launched.
  const bool use_graphs = c->cfg.use_graphs != 0;
  PassCtl h;
  const int chunk = c->cfg.passes_per_sync > 0 ? c->cfg.passes_per_sync : 4;
  c->pass_ms.clear();
  LVG_CUDA(cudaEventRecord(c->ev0, s));
  int launched = 0;
  for (;;) {
    for (int p = 0; p < chunk; ++p) {
      size_t e = 2 * (size_t)launched;
      while (c->mev.size() < e + 2) {
        cudaEvent_t ev;
        LVG_CUDA(cudaEventCreate(&ev));
        c->mev.push_back(ev);
      }
      LVG_CUDA(cudaEventRecord(c->mev[e], s));
      const bool graph = use_graphs && launched >= 2;
      if (graph) ensure_graphs(c);
      if (launched == 0) launch_moves_singleton(c->g, c->st, s, &c->side);   // state is singletons
      else if (graph) LVG_CUDA(cudaGraphLaunch(c->g_moves, s));
      else launch_moves(c->g, c->st, s, &c->side);
      LVG_CUDA(cudaEventRecord(c->mev[e + 1], s));
      if (graph) LVG_CUDA(cudaGraphLaunch(c->g_commit, s));
      else launch_commit(c->g, c->st, s);
      ++launched;
    }
    LVG_CUDA(cudaMemcpyAsync(&h, c->st.ctl, sizeof h, cudaMemcpyDeviceToHost, s));
    sync(c);
    if (h.done) break;
    if (h.err) throw Error(LVG_ERR_CAPACITY, "neighbour-community table probe limit exceeded");
    // every pass must raise Q by pass_min_gain over a bounded range, so a
    // level that runs this long has lost its state: stop with an error
    if (launched >= kHardPassCap) throw Error(LVG_ERR_NOT_CONVERGED, "hard pass cap reached");
  }
  launch_merge(c->g, c->st, s);
  LVG_CUDA(cudaEventRecord(c->ev1, s));
  LVG_CUDA(cudaMemcpyAsync(&h, c->st.ctl, sizeof h, cudaMemcpyDeviceToHost, s));
  sync(c);
  if (h.err) throw Error(LVG_ERR_CAPACITY, "neighbour-community table probe limit exceeded");
  c->pass_ms.push_back(elapsed(c->ev0, c->ev1));
  c->move_ms = 0.0;
  c->move_passes = h.passes;
  c->move_pass_ms.clear();
  for (int p = 0; p < h.passes && 2 * (size_t)p + 1 < c->mev.size(); ++p) {
    const float ms = elapsed(c->mev[2 * p], c->mev[2 * p + 1]);
    c->move_pass_ms.push_back(ms);
    c->move_ms += ms;
  }
  if (q_out) *q_out = h.q_ret;
  if (passes_out) *passes_out = h.passes;
  if (status_out) *status_out = h.status;
  (void)q_start_out;
  (void)launched;
}

// Renumber the current level; the partition and labels live on the arena's
// high end for the rest of the run.
int32_t renumber_level(lvg_ctx* c) {
  const int32_t V = c->g.V;
  c->pristine = false;
  c->arena.hi = c->run_hi;
  int32_t* part = c->arena.hi_n<int32_t>(V);
  int32_t* labels = c->arena.hi_n<int32_t>(V);
  c->run_hi = c->arena.hi;
  LVG_CUDA(cudaMemcpyAsync(labels, c->st.comm, sizeof(int32_t) * std::max(V, 1), cudaMemcpyDeviceToDevice,
                           c->stream));
  LVG_CUDA(cudaEventRecord(c->pev[2], c->stream));
  int32_t C = renumber(c->g, c->st.comm, part, c->arena, c->stream);
  compose(c->composed, part, c->V0, c->stream);    // partitionAtLevel (LouvainCPP.cpp:82-106)
  LVG_CUDA(cudaEventRecord(c->pev[3], c->stream));
  c->d_part_cur = part;
  c->C_cur = C;
  c->renumbered = true;
  LevelRec r;
  std::memset(&r.info, 0, sizeof r.info);
  r.d_part = part;
  r.d_labels = labels;
  r.info.n_vertices = V;
  r.info.n_entries = c->g.E;
  r.info.nnz = c->g.nnz;
  r.info.n_comms = C;
  r.info.ms_build = elapsed(c->pev[0], c->pev[1]);   // complete: renumber synchronised the stream
  c->levels.push_back(r);
  return C;
}

// Coarsen into the next level and build it.
void induce_level(lvg_ctx* c) {
  int32_t *os = nullptr, *od = nullptr;
  float* ow = nullptr;
  c->arena.hi = c->run_hi;
  LVG_CUDA(cudaEventRecord(c->pev[4], c->stream));
  PreCsr hi_csr;
  int64_t n = induce(c->g, c->d_part_cur, c->C_cur, &os, &od, &ow, c->arena, c->stream, &hi_csr, c->tune.coarsen);
  // the next level's list (and its CSR, when the coarsening wrote it) moves
  // down to the start of the level region
  c->arena.lo = c->base_lo;
  int32_t* ns = c->arena.lo_n<int32_t>(n);
  int32_t* nd = c->arena.lo_n<int32_t>(n);
  float* nw = c->arena.lo_n<float>(n);
  auto down = [&](void* dst, const void* src, size_t bytes) {
    if (bytes) LVG_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, c->stream));
  };
  down(ns, os, sizeof(int32_t) * n);
  down(nd, od, sizeof(int32_t) * n);
  down(nw, ow, sizeof(float) * n);
  const int32_t C1 = c->C_cur;
  c->pre_next = PreCsr();
  if (hi_csr.valid) {
    PreCsr& p = c->pre_next;
    p.off = c->arena.lo_n<int64_t>((int64_t)C1 + 1);
    p.col = c->arena.lo_n<int32_t>(hi_csr.nnz);
    p.cw = c->arena.lo_n<float>(hi_csr.nnz);
    p.k = c->arena.lo_n<double>(C1);
    p.loopw = c->arena.lo_n<float>(C1);
    p.has_loop = c->arena.lo_n<uint8_t>(C1);
    down(p.off, hi_csr.off, sizeof(int64_t) * ((size_t)C1 + 1));
    down(p.col, hi_csr.col, sizeof(int32_t) * hi_csr.nnz);
    down(p.cw, hi_csr.cw, sizeof(float) * hi_csr.nnz);
    down(p.k, hi_csr.k, sizeof(double) * C1);
    down(p.loopw, hi_csr.loopw, sizeof(float) * C1);
    down(p.has_loop, hi_csr.has_loop, C1);
    p.m = hi_csr.m;
    p.nnz = hi_csr.nnz;
    p.valid = true;
  }
  LVG_CUDA(cudaEventRecord(c->pev[5], c->stream));
  sync(c);
  if (!c->levels.empty()) {
    c->levels.back().info.ms_renumber = elapsed(c->pev[2], c->pev[3]);
    c->levels.back().info.ms_induce = elapsed(c->pev[4], c->pev[5]);
  }
  c->arena.hi = c->run_hi;
  int32_t C = c->C_cur;
  c->g = LevelGraph();
  c->g.V = C;
  c->g.E = n;
  c->g.src = ns;
  c->g.dst = nd;
  c->g.w = nw;
  c->g.pre = &c->pre_next;
  c->level += 1;
  prepare_level(c);
}

void check_ctx(lvg_ctx* c) {
  require(c != nullptr, LVG_ERR_INVALID_ARG, "null context");
  LVG_CUDA(cudaSetDevice(c->device));
}

}  // namespace

extern "C" {

const char* lvg_status_string(lvg_status s) {
  switch (s) {
    case LVG_OK: return "ok";
    case LVG_ERR_INVALID_ARG: return "invalid argument";
    case LVG_ERR_OOM: return "out of device memory";
    case LVG_ERR_CAPACITY: return "capacity exceeded";
    case LVG_ERR_NOT_CONVERGED: return "not converged";
    case LVG_ERR_CUDA: return "CUDA error";
    case LVG_ERR_STATE: return "call out of order";
  }
  return "unknown status";
}

lvg_status lvg_config_default(lvg_config* cfg) {
  if (!cfg) return LVG_ERR_INVALID_ARG;
  std::memset(cfg, 0, sizeof *cfg);
  cfg->device = 0;
  cfg->pass_min_gain = 1e-7;   // __MIN (OneLevelKernel.cu:425)
  cfg->level_min_gain = 1e-7;  // __MIN (LouvainCPP.cpp:55)
  cfg->max_passes = -1;        // __PASS_MAX (OneLevelKernel.cu:424)
  cfg->max_levels = -1;
  cfg->arena_bytes = 0;
  cfg->tile_max_degree = 512;
  cfg->block_max_degree = 4096;
  cfg->passes_per_sync = 2;   // a level of this method stops at its second pass
  cfg->use_graphs = 1;
  cfg->l2_persist = 1;
  return LVG_OK;
}

lvg_status lvg_create(const lvg_config* cfg, lvg_ctx** out) {
  if (!out) return LVG_ERR_INVALID_ARG;
  *out = nullptr;
  lvg_ctx* c = new (std::nothrow) lvg_ctx();
  if (!c) return LVG_ERR_OOM;
  lvg_status s = guarded(c, [&] {
    if (cfg) c->cfg = *cfg;
    else lvg_config_default(&c->cfg);
    require(c->cfg.tile_max_degree >= 0 && c->cfg.block_max_degree >= 0, LVG_ERR_INVALID_ARG,
            "bucket thresholds must be >= 0");
    c->tune.warp_max = c->cfg.tile_max_degree > 0 ? std::min(c->cfg.tile_max_degree, 512) : 512;
    c->tune.block_max = c->cfg.block_max_degree > 0 ? std::min(c->cfg.block_max_degree, 8192) : 4096;
    if (c->tune.block_max < c->tune.warp_max) c->tune.block_max = c->tune.warp_max;
    require(c->cfg.coarsen_mode >= 0 && c->cfg.coarsen_mode <= 3, LVG_ERR_INVALID_ARG,
            "coarsen_mode must be 0, 1, 2 or 3");
    c->tune.coarsen = c->cfg.coarsen_mode;
    c->device = c->cfg.device;
    int n = 0;
    LVG_CUDA(cudaGetDeviceCount(&n));
    require(c->device >= 0 && c->device < n, LVG_ERR_INVALID_ARG, "no such CUDA device");
    LVG_CUDA(cudaSetDevice(c->device));
    LVG_CUDA(cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking));
    c->stream = c->own_stream;
    LVG_CUDA(cudaEventCreate(&c->ev0));
    LVG_CUDA(cudaEventCreate(&c->ev1));
    for (auto& e : c->pev) LVG_CUDA(cudaEventCreate(&e));
    for (int k = 0; k < 3; ++k) {
      LVG_CUDA(cudaStreamCreateWithFlags(&c->side.side[k], cudaStreamNonBlocking));
      LVG_CUDA(cudaEventCreateWithFlags(&c->side.join[k], cudaEventDisableTiming));
    }
    LVG_CUDA(cudaEventCreateWithFlags(&c->side.fork, cudaEventDisableTiming));
    c->have_side = true;
    cudaDeviceProp prop;
    LVG_CUDA(cudaGetDeviceProperties(&prop, c->device));
    c->persist_max = (size_t)prop.persistingL2CacheMaxSize;
    c->window_max = (size_t)prop.accessPolicyMaxWindowSize;
    if (c->persist_max > 0)   // per-context limit, released with the context
      LVG_CUDA(cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, c->persist_max));
  });
  if (s != LVG_OK) {
    lvg_destroy(c);
    return s;
  }
  *out = c;
  return LVG_OK;
}

lvg_status lvg_destroy(lvg_ctx* c) {
  if (!c) return LVG_OK;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  drop_graphs(c);
  c->arena.release();
  if (c->ev0) cudaEventDestroy(c->ev0);
  if (c->ev1) cudaEventDestroy(c->ev1);
  for (auto& e : c->pev)
    if (e) cudaEventDestroy(e);
  for (cudaEvent_t e : c->mev) cudaEventDestroy(e);
  if (c->have_side) {
    for (int k = 0; k < 3; ++k) {
      cudaStreamDestroy(c->side.side[k]);
      cudaEventDestroy(c->side.join[k]);
    }
    cudaEventDestroy(c->side.fork);
  }
  for (cudaEvent_t e : c->load_ev) cudaEventDestroy(e);
  if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
  if (c->own_stream) cudaStreamDestroy(c->own_stream);
  delete c;
  return LVG_OK;
}

const char* lvg_last_error(const lvg_ctx* c) { return c ? c->err.c_str() : "null context"; }

lvg_status lvg_set_stream(lvg_ctx* c, void* stream) {
  return guarded(c, [&] {
    check_ctx(c);
    c->stream = stream ? (cudaStream_t)stream : c->own_stream;
  });
}

lvg_status lvg_load_edges(lvg_ctx* c, const int32_t* src, const int32_t* dst, const float* w, int64_t E,
                          int32_t V) {
  return guarded(c, [&] {
    check_ctx(c);
    require(V >= 0 && E >= 0, LVG_ERR_INVALID_ARG, "negative size");
    require(E == 0 || (src && dst && w), LVG_ERR_INVALID_ARG, "null edge array");
    c->loaded = false;
    c->pre0 = PreCsr();
    size_t need = c->cfg.arena_bytes > 0 ? (size_t)c->cfg.arena_bytes : arena_estimate(V, E, true);
    c->arena.reserve(need);
    int32_t* s = c->arena.lo_n<int32_t>(E);
    int32_t* d = c->arena.lo_n<int32_t>(E);
    float* ww = c->arena.lo_n<float>(E);
    int64_t chunk = c->cfg.load_chunk_entries > 0 ? c->cfg.load_chunk_entries : ((int64_t)1 << 25);
    chunk = (chunk + 2047) / 2048 * 2048;
    bool ok;
    if (E >= 2 * chunk) {   // copy in chunks, checking and building level 0 as they arrive
      if (!c->copy_stream) LVG_CUDA(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
      ok = stream_load_level0(src, dst, w, s, d, ww, E, V, chunk, c->pre0, c->load_ev, c->arena, c->stream,
                              c->copy_stream);
    } else {
      if (E > 0) {
        LVG_CUDA(cudaMemcpyAsync(s, src, sizeof(int32_t) * E, cudaMemcpyHostToDevice, c->stream));
        LVG_CUDA(cudaMemcpyAsync(d, dst, sizeof(int32_t) * E, cudaMemcpyHostToDevice, c->stream));
        LVG_CUDA(cudaMemcpyAsync(ww, w, sizeof(float) * E, cudaMemcpyHostToDevice, c->stream));
      }
      ok = validate_edges(s, d, ww, E, V, c->arena, c->stream);
    }
    require(ok, LVG_ERR_INVALID_ARG, "edge list has a vertex id out of range or a negative / non-finite weight");
    load_common(c, s, d, ww, E, V);
  });
}

lvg_status lvg_load_edges_device(lvg_ctx* c, const int32_t* src, const int32_t* dst, const float* w, int64_t E,
                                 int32_t V) {
  return guarded(c, [&] {
    check_ctx(c);
    require(V >= 0 && E >= 0, LVG_ERR_INVALID_ARG, "negative size");
    require(E == 0 || (src && dst && w), LVG_ERR_INVALID_ARG, "null edge array");
    c->loaded = false;
    c->pre0 = PreCsr();
    size_t need = c->cfg.arena_bytes > 0 ? (size_t)c->cfg.arena_bytes : arena_estimate(V, E, false);
    c->arena.reserve(need);
    require(validate_edges(src, dst, w, E, V, c->arena, c->stream), LVG_ERR_INVALID_ARG,
            "edge list has a vertex id out of range or a negative / non-finite weight");
    load_common(c, src, dst, w, E, V);
  });
}

lvg_status lvg_modularity(lvg_ctx* c, double* q) {
  return guarded(c, [&] {
    check_ctx(c);
    require(c->loaded && c->have_state, LVG_ERR_STATE, "no graph loaded");
    require(q != nullptr, LVG_ERR_INVALID_ARG, "null output");
    *q = read_q(c);
  });
}

lvg_status lvg_one_level(lvg_ctx* c, double lower, double* q, int32_t* passes) {
  int32_t status = 0;
  lvg_status s = guarded(c, [&] {
    check_ctx(c);
    require(c->loaded && c->have_state, LVG_ERR_STATE, "no graph loaded");
    one_level(c, lower, q, passes, &status, nullptr);
  });
  if (s == LVG_OK && status != 0) return fail(c, (lvg_status)status, "pass cap reached before convergence");
  return s;
}

lvg_status lvg_renumber(lvg_ctx* c, int32_t* comm_out, int32_t* n_comms) {
  return guarded(c, [&] {
    check_ctx(c);
    require(c->loaded && c->have_state, LVG_ERR_STATE, "no graph loaded");
    int32_t C = renumber_level(c);
    if (comm_out && c->g.V > 0)
      LVG_CUDA(cudaMemcpyAsync(comm_out, c->d_part_cur, sizeof(int32_t) * c->g.V, cudaMemcpyDeviceToHost,
                               c->stream));
    sync(c);
    if (n_comms) *n_comms = C;
  });
}

lvg_status lvg_induce(lvg_ctx* c) {
  return guarded(c, [&] {
    check_ctx(c);
    require(c->loaded && c->renumbered, LVG_ERR_STATE, "lvg_induce needs lvg_renumber first");
    induce_level(c);
  });
}

lvg_status lvg_run(lvg_ctx* c, lvg_result* res) {
  int32_t run_status = 0;
  lvg_status s = guarded(c, [&] {
    check_ctx(c);
    require(c->loaded, LVG_ERR_STATE, "no graph loaded");
    if (!c->pristine) reset_to_level0(c);   // a run starts from level 0 as loaded
    if (res) std::memset(res, 0, sizeof *res);
    if (c->E0 == 0) {
      // LouvainCPP.cpp:211-230: an empty edge list yields one identity partition
      renumber_level(c);
      c->levels.back().info.passes = 0;
      if (res) { res->n_levels = 1; res->n_comms = c->V0; res->q_final = 0.0; }
      return;
    }
    double mod = 0.0;
    int64_t pass_entries = 0;
    for (;;) {
      double q0 = read_q(c);                      // modularityCUDA (LouvainCPP.cpp:356)
      double lower = c->level == 0 ? q0 : mod;
      double ql = 0.0;
      int32_t passes = 0, st = 0;
      one_level(c, lower, &ql, &passes, &st, nullptr);
      float ms_passes = c->pass_ms.empty() ? 0.0f : c->pass_ms.back();
      renumber_level(c);
      LevelRec& r = c->levels.back();
      r.info.passes = passes;
      r.info.q_start = q0;
      r.info.q_level = ql;
      r.info.ms_passes = ms_passes;
      pass_entries += c->g.nnz * (int64_t)passes;
      if (st != 0) { run_status = st; break; }
      if (c->level > 0 && (ql - mod) < c->cfg.level_min_gain) break;   // LouvainCPP.cpp:466
      if (c->cfg.max_levels >= 0 && c->level + 1 >= c->cfg.max_levels) { run_status = LVG_ERR_NOT_CONVERGED; break; }
      mod = ql;
      induce_level(c);
    }
    if (res) {
      res->n_levels = (int32_t)c->levels.size();
      res->n_comms = c->C_cur;
      res->pass_entries = pass_entries;
      res->status = run_status;
      res->q_final = modularity_fp64(c->src0, c->dst0, c->w0, c->E0, std::max(c->C_cur, 1), c->composed,
                                     c->arena, c->stream, c->symmetric0);
    }
    sync(c);
    if (!c->levels.empty()) c->levels.back().info.ms_renumber = elapsed(c->pev[2], c->pev[3]);
  });
  if (s == LVG_OK && run_status != 0) return fail(c, (lvg_status)run_status, "cap reached before convergence");
  return s;
}

lvg_status lvg_num_levels(const lvg_ctx* c, int32_t* n) {
  if (!c || !n) return LVG_ERR_INVALID_ARG;
  *n = (int32_t)c->levels.size();
  return LVG_OK;
}

lvg_status lvg_get_level_info(const lvg_ctx* c, int32_t level, lvg_level_info* info) {
  if (!c || !info || level < 0 || level >= (int32_t)c->levels.size()) return LVG_ERR_INVALID_ARG;
  *info = c->levels[level].info;
  return LVG_OK;
}

lvg_status lvg_get_level_partition(const lvg_ctx* cc, int32_t level, int32_t* part) {
  lvg_ctx* c = const_cast<lvg_ctx*>(cc);
  return guarded(c, [&] {
    check_ctx(c);
    require(part && level >= 0 && level < (int32_t)c->levels.size(), LVG_ERR_INVALID_ARG, "bad level");
    const LevelRec& r = c->levels[level];
    if (r.info.n_vertices > 0)
      LVG_CUDA(cudaMemcpyAsync(part, r.d_part, sizeof(int32_t) * r.info.n_vertices, cudaMemcpyDeviceToHost,
                               c->stream));
    sync(c);
  });
}

lvg_status lvg_get_level_labels(const lvg_ctx* cc, int32_t level, int32_t* labels) {
  lvg_ctx* c = const_cast<lvg_ctx*>(cc);
  return guarded(c, [&] {
    check_ctx(c);
    require(labels && level >= 0 && level < (int32_t)c->levels.size(), LVG_ERR_INVALID_ARG, "bad level");
    const LevelRec& r = c->levels[level];
    if (r.info.n_vertices > 0)
      LVG_CUDA(cudaMemcpyAsync(labels, r.d_labels, sizeof(int32_t) * r.info.n_vertices,
                               cudaMemcpyDeviceToHost, c->stream));
    sync(c);
  });
}

lvg_status lvg_get_partition(const lvg_ctx* cc, int32_t level, int32_t* part) {
  lvg_ctx* c = const_cast<lvg_ctx*>(cc);
  return guarded(c, [&] {
    check_ctx(c);
    int32_t L = (int32_t)c->levels.size();
    require(part && L > 0 && level >= 0, LVG_ERR_INVALID_ARG, "bad level");
    if (level >= L - 1) {
      if (c->V0 > 0)
        LVG_CUDA(cudaMemcpyAsync(part, c->composed, sizeof(int32_t) * c->V0, cudaMemcpyDeviceToHost, c->stream));
      sync(c);
      return;
    }
    // compose levels 0..level on the host side from the per-level partitions
    std::vector<int32_t> cur(c->V0), lv;
    LVG_CUDA(cudaMemcpyAsync(cur.data(), c->levels[0].d_part, sizeof(int32_t) * c->V0, cudaMemcpyDeviceToHost,
                             c->stream));
    sync(c);
    for (int32_t l = 1; l <= level; ++l) {
      lv.resize(c->levels[l].info.n_vertices);
      LVG_CUDA(cudaMemcpyAsync(lv.data(), c->levels[l].d_part, sizeof(int32_t) * lv.size(),
                               cudaMemcpyDeviceToHost, c->stream));
      sync(c);
      for (auto& x : cur) x = lv[x];
    }
    std::memcpy(part, cur.data(), sizeof(int32_t) * c->V0);
  });
}

lvg_status lvg_count_partitions(const int32_t* part, int64_t n, int32_t* count) {
  if (!count || (n > 0 && !part) || n < 0) return LVG_ERR_INVALID_ARG;
  int32_t mx = 0;                                // countPartitions (LouvainCPP.cpp:116-127)
  for (int64_t i = 0; i < n; ++i) mx = std::max(mx, part[i]);
  *count = 1 + mx;
  return LVG_OK;
}

lvg_status lvg_modularity_fp64(lvg_ctx* c, const int32_t* part, double* q) {
  return guarded(c, [&] {
    check_ctx(c);
    require(c->loaded, LVG_ERR_STATE, "no graph loaded");
    require(part && q, LVG_ERR_INVALID_ARG, "null argument");
    int32_t C = 0;
    for (int32_t i = 0; i < c->V0; ++i) {
      require(part[i] >= 0 && part[i] < std::max(c->V0, 1), LVG_ERR_INVALID_ARG, "partition id out of range");
      C = std::max(C, part[i] + 1);
    }
    HiScope hs(c->arena);
    int32_t* dp = c->arena.hi_n<int32_t>(c->V0);
    if (c->V0 > 0)
      LVG_CUDA(cudaMemcpyAsync(dp, part, sizeof(int32_t) * c->V0, cudaMemcpyHostToDevice, c->stream));
    *q = modularity_fp64(c->src0, c->dst0, c->w0, c->E0, std::max(C, 1), dp, c->arena, c->stream, c->symmetric0);
  });
}

lvg_status lvg_get_csr(const lvg_ctx* cc, int32_t* n_vertices, int64_t* nnz, double* m, int64_t* off,
                       int32_t* col, float* w, double* k, float* loopw, uint8_t* has_loop) {
  lvg_ctx* c = const_cast<lvg_ctx*>(cc);
  return guarded(c, [&] {
    check_ctx(c);
    require(c->loaded && c->have_state, LVG_ERR_STATE, "no graph loaded");
    const LevelGraph& g = c->g;
    if (n_vertices) *n_vertices = g.V;
    if (nnz) *nnz = g.nnz;
    if (m) *m = g.m;
    cudaStream_t s = c->stream;
    if (off) LVG_CUDA(cudaMemcpyAsync(off, g.off, sizeof(int64_t) * (g.V + 1), cudaMemcpyDeviceToHost, s));
    if (col && g.nnz) LVG_CUDA(cudaMemcpyAsync(col, g.col, sizeof(int32_t) * g.nnz, cudaMemcpyDeviceToHost, s));
    if (w && g.nnz) LVG_CUDA(cudaMemcpyAsync(w, g.cw, sizeof(float) * g.nnz, cudaMemcpyDeviceToHost, s));
    if (k && g.V) LVG_CUDA(cudaMemcpyAsync(k, g.k, sizeof(double) * g.V, cudaMemcpyDeviceToHost, s));
    if (loopw && g.V) LVG_CUDA(cudaMemcpyAsync(loopw, g.loopw, sizeof(float) * g.V, cudaMemcpyDeviceToHost, s));
    if (has_loop && g.V) LVG_CUDA(cudaMemcpyAsync(has_loop, g.has_loop, g.V, cudaMemcpyDeviceToHost, s));
    sync(c);
  });
}

lvg_status lvg_get_level_edges(const lvg_ctx* cc, int64_t* n_entries, int32_t* src, int32_t* dst, float* w) {
  lvg_ctx* c = const_cast<lvg_ctx*>(cc);
  return guarded(c, [&] {
    check_ctx(c);
    require(c->loaded && c->have_state, LVG_ERR_STATE, "no graph loaded");
    const LevelGraph& g = c->g;
    if (n_entries) *n_entries = g.E;
    cudaStream_t s = c->stream;
    if (src && g.E) LVG_CUDA(cudaMemcpyAsync(src, g.src, sizeof(int32_t) * g.E, cudaMemcpyDeviceToHost, s));
    if (dst && g.E) LVG_CUDA(cudaMemcpyAsync(dst, g.dst, sizeof(int32_t) * g.E, cudaMemcpyDeviceToHost, s));
    if (w && g.E) LVG_CUDA(cudaMemcpyAsync(w, g.w, sizeof(float) * g.E, cudaMemcpyDeviceToHost, s));
    sync(c);
  });
}

lvg_status lvg_set_communities(lvg_ctx* c, const int32_t* comm) {
  return guarded(c, [&] {
    check_ctx(c);
    require(c->loaded && c->have_state, LVG_ERR_STATE, "no graph loaded");
    require(comm != nullptr, LVG_ERR_INVALID_ARG, "null communities");
    const int32_t V = c->g.V;
    for (int32_t i = 0; i < V; ++i)
      require(comm[i] >= 0 && comm[i] < V, LVG_ERR_INVALID_ARG, "community id out of range");
    HiScope hs(c->arena);
    int32_t* d = c->arena.hi_n<int32_t>(V);
    if (V > 0) LVG_CUDA(cudaMemcpyAsync(d, comm, sizeof(int32_t) * V, cudaMemcpyHostToDevice, c->stream));
    c->pristine = false;
    set_state_from(c->g, c->st, d, c->stream);
    sync(c);
  });
}

lvg_status lvg_move_decide(lvg_ctx* c, int32_t* next, int32_t* cand) {
  return guarded(c, [&] {
    check_ctx(c);
    require(c->loaded && c->have_state, LVG_ERR_STATE, "no graph loaded");
    const int32_t V = c->g.V;
    cudaStream_t s = c->stream;
    reset_ctl(c->st, 0.0, c->cfg.pass_min_gain, -1, s);
    clear_deltas(c->g, c->st, s);
    launch_moves(c->g, c->st, s, &c->side);
    if (next && V) LVG_CUDA(cudaMemcpyAsync(next, c->st.next, sizeof(int32_t) * V, cudaMemcpyDeviceToHost, s));
    if (cand && V) LVG_CUDA(cudaMemcpyAsync(cand, c->st.cand, sizeof(int32_t) * V, cudaMemcpyDeviceToHost, s));
    PassCtl h;
    LVG_CUDA(cudaMemcpyAsync(&h, c->st.ctl, sizeof h, cudaMemcpyDeviceToHost, s));
    // leave the committed state as it was
    clear_deltas(c->g, c->st, s);
    if (V) LVG_CUDA(cudaMemcpyAsync(c->st.next, c->st.comm, sizeof(int32_t) * V, cudaMemcpyDeviceToDevice, s));
    sync(c);
    require(h.err == 0, LVG_ERR_CAPACITY, "neighbour-community table probe limit exceeded");
  });
}

lvg_status lvg_last_pass_times(const lvg_ctx* c, float* ms, int32_t cap, int32_t* n) {
  if (!c) return LVG_ERR_INVALID_ARG;
  int32_t k = (int32_t)c->pass_ms.size();
  if (ms)
    for (int32_t i = 0; i < k && i < cap; ++i) ms[i] = c->pass_ms[i];
  if (n) *n = k;
  return LVG_OK;
}

lvg_status lvg_move_pass_times(const lvg_ctx* c, float* ms, int32_t cap, int32_t* n) {
  if (!c) return LVG_ERR_INVALID_ARG;
  const int32_t k = (int32_t)c->move_pass_ms.size();
  if (ms)
    for (int32_t i = 0; i < k && i < cap; ++i) ms[i] = c->move_pass_ms[i];
  if (n) *n = k;
  return LVG_OK;
}

lvg_status lvg_move_stats(const lvg_ctx* c, double* ms_total, int64_t* n_passes) {
  if (!c) return LVG_ERR_INVALID_ARG;
  if (ms_total) *ms_total = c->move_ms;
  if (n_passes) *n_passes = c->move_passes;
  return LVG_OK;
}

lvg_status lvg_kernel_launches(int64_t* n) {
  if (!n) return LVG_ERR_INVALID_ARG;
  *n = lvg::g_launches.load();
  return LVG_OK;
}

lvg_status lvg_memory(const lvg_ctx* c, int64_t* capacity, int64_t* peak) {
  if (!c) return LVG_ERR_INVALID_ARG;
  if (capacity) *capacity = (int64_t)c->arena.cap;
  if (peak) *peak = (int64_t)c->arena.peak;
  return LVG_OK;
}

}  // extern "C"

// ============================================================================
// Autotuner of the degree-class thresholds (no counterpart in the reference,
// whose launch shapes are fixed: <<<N,32>>> per vertex, OneLevelKernel.cu:248-386).
namespace {

using ShapeKey = std::tuple<int, int, int, int, int>;   // device, log2 V, log2 nnz, log2 max degree, integral
std::mutex g_tune_mu;
std::map<ShapeKey, std::pair<int32_t, int32_t>> g_tune_cache;

int floor_log2(int64_t x) {
  int l = -1;
  for (; x > 0; x >>= 1) ++l;
  return l;
}

ShapeKey shape_key(lvg_ctx* c) {
  const int64_t dmax = max_degree(c->g, c->arena, c->stream);
  return ShapeKey(c->device, floor_log2(c->g.V), floor_log2(c->g.nnz), floor_log2(dmax), c->g.int_acc ? 1 : 0);
}

void set_tuning(lvg_ctx* c, int32_t tile, int32_t block) {
  c->tune.warp_max = tile;
  c->tune.block_max = block;
  c->cfg.tile_max_degree = tile;
  c->cfg.block_max_degree = block;
}

}  // namespace

extern "C" lvg_status lvg_tune_pick(const lvg_tune_point* p, int32_t n, int32_t pref_tile, int32_t pref_block,
                                    int32_t* best_index) {
  if (!best_index || n < 0 || (n > 0 && !p)) return LVG_ERR_INVALID_ARG;
  int32_t b = -1;
  for (int32_t i = 0; i < n; ++i)
    if (p[i].move_ms >= 0.0f && (b < 0 || p[i].move_ms < p[b].move_ms)) b = i;
  if (b >= 0) {
    for (int32_t i = 0; i < n; ++i) {
      if (p[i].tile_max_degree == pref_tile && p[i].block_max_degree == pref_block && p[i].move_ms >= 0.0f &&
          (double)p[i].move_ms <= 1.02 * (double)p[b].move_ms) {
        b = i;
        break;
      }
    }
  }
  *best_index = b;
  return LVG_OK;
}

extern "C" lvg_status lvg_tune_cache_clear(void) {
  std::lock_guard<std::mutex> lock(g_tune_mu);
  g_tune_cache.clear();
  return LVG_OK;
}

extern "C" lvg_status lvg_get_thresholds(const lvg_ctx* c, int32_t* tile_max_degree, int32_t* block_max_degree) {
  if (!c) return LVG_ERR_INVALID_ARG;
  if (tile_max_degree) *tile_max_degree = c->tune.warp_max;
  if (block_max_degree) *block_max_degree = c->tune.block_max;
  return LVG_OK;
}

extern "C" lvg_status lvg_autotune(lvg_ctx* c, const lvg_tune_space* sp, lvg_tune_point* points, int32_t cap,
                                   int32_t* n_points, lvg_tune_point* best) {
  return guarded(c, [&] {
    check_ctx(c);
    require(c->loaded, LVG_ERR_STATE, "no graph loaded");
    require(cap >= 0 && (cap == 0 || points), LVG_ERR_INVALID_ARG, "bad points buffer");
    static const int32_t kTiles[] = {64, 128, 256, 512};
    static const int32_t kBlocks[] = {1024, 2048, 4096, 8192};
    const int32_t* tl = sp && sp->tile_max_degrees ? sp->tile_max_degrees : kTiles;
    const int32_t nt = sp && sp->tile_max_degrees ? sp->n_tile : 4;
    const int32_t* bl = sp && sp->block_max_degrees ? sp->block_max_degrees : kBlocks;
    const int32_t nb = sp && sp->block_max_degrees ? sp->n_block : 4;
    require(nt > 0 && nb > 0, LVG_ERR_INVALID_ARG, "empty candidate list");
    for (int32_t i = 0; i < nt; ++i)
      require(tl[i] >= 32 && tl[i] <= 512, LVG_ERR_INVALID_ARG, "tile_max_degree candidates must be in [32, 512]");
    for (int32_t i = 0; i < nb; ++i)
      require(bl[i] >= 32 && bl[i] <= 8192, LVG_ERR_INVALID_ARG, "block_max_degree candidates must be in [32, 8192]");
    const int reps = sp && sp->reps > 0 ? sp->reps : 3;
    std::vector<std::pair<int32_t, int32_t>> cands;
    for (int32_t i = 0; i < nt; ++i)
      for (int32_t j = 0; j < nb; ++j)
        if (bl[j] >= tl[i] && std::find(cands.begin(), cands.end(), std::make_pair(tl[i], bl[j])) == cands.end())
          cands.emplace_back(tl[i], bl[j]);
    require(!cands.empty(), LVG_ERR_INVALID_ARG, "no candidate pair has tile_max_degree <= block_max_degree");
    if (n_points) *n_points = 0;
    const int32_t pref_tile = c->tune.warp_max, pref_block = c->tune.block_max;
    if (!c->pristine) reset_to_level0(c);   // tune from level 0 as loaded
    if (c->E0 == 0 || c->g.nnz == 0) {   // no move pass to time (lvg_run runs none either)
      if (best) *best = lvg_tune_point{pref_tile, pref_block, -1.0f, -1.0f};
      return;
    }
    const ShapeKey key = shape_key(c);
    if (sp && sp->use_cache) {
      std::pair<int32_t, int32_t> hit(0, 0);
      {
        std::lock_guard<std::mutex> lock(g_tune_mu);
        auto it = g_tune_cache.find(key);
        if (it != g_tune_cache.end()) hit = it->second;
      }
      if (hit.first > 0) {
        set_tuning(c, hit.first, hit.second);
        reset_to_level0(c);
        if (best) *best = lvg_tune_point{hit.first, hit.second, -1.0f, -1.0f};
        return;
      }
    }
    std::vector<lvg_tune_point> pts;
    std::vector<int32_t> labels, ref_labels;
    double ref_q = 0.0;
    int32_t ref_passes = -1;
    try {
      for (const auto& cand : cands) {
        lvg_tune_point pt{cand.first, cand.second, -1.0f, -1.0f};
        set_tuning(c, cand.first, cand.second);
        try {
          reset_to_level0(c);
        } catch (const Error& e) {
          if (e.status != LVG_ERR_OOM) throw;
          pts.push_back(pt);   // this pair's hub tables do not fit the context's arena
          continue;
        }
        const double q0 = read_q(c);   // synchronises: the build events are complete
        pt.build_ms = elapsed(c->pev[0], c->pev[1]);
        std::vector<float> ms;
        for (int r = 0; r <= reps; ++r) {
          double q = 0.0;
          int32_t passes = 0, status = 0;
          one_level(c, q0, &q, &passes, &status, nullptr);
          if (r == 0) {
            // the thresholds route vertices to kernels; the decisions must not move
            labels.resize((size_t)c->g.V);
            if (c->g.V > 0)
              LVG_CUDA(cudaMemcpyAsync(labels.data(), c->st.comm, sizeof(int32_t) * c->g.V, cudaMemcpyDeviceToHost,
                                       c->stream));
            sync(c);
            if (ref_passes < 0) {
              ref_q = q;
              ref_passes = passes;
              ref_labels = labels;
            } else {
              require(q == ref_q && passes == ref_passes && labels == ref_labels, LVG_ERR_STATE,
                      "autotune: two threshold pairs gave different level-0 results");
            }
            continue;
          }
          float h = 0.0f;
          for (size_t p = 1; p < c->move_pass_ms.size(); ++p) h += c->move_pass_ms[p];
          ms.push_back(h);
        }
        std::sort(ms.begin(), ms.end());
        pt.move_ms = ms[ms.size() / 2];
        pts.push_back(pt);
      }
    } catch (...) {
      // leave the context built with the pair it had before the call
      set_tuning(c, pref_tile, pref_block);
      try {
        reset_to_level0(c);
      } catch (...) {
      }
      throw;
    }
    int32_t bi = -1;
    lvg_tune_pick(pts.data(), (int32_t)pts.size(), pref_tile, pref_block, &bi);
    const int32_t tile = bi >= 0 ? pts[bi].tile_max_degree : pref_tile;
    const int32_t block = bi >= 0 ? pts[bi].block_max_degree : pref_block;
    set_tuning(c, tile, block);
    reset_to_level0(c);
    if (bi >= 0) {
      std::lock_guard<std::mutex> lock(g_tune_mu);
      g_tune_cache[key] = std::make_pair(tile, block);
    }
    const int32_t n = (int32_t)pts.size();
    for (int32_t i = 0; i < std::min(n, cap); ++i) points[i] = pts[i];
    if (n_points) *n_points = n;
    if (best) *best = bi >= 0 ? pts[bi] : lvg_tune_point{tile, block, -1.0f, -1.0f};
  });
}

// ============================================================================
// Batched runs (no counterpart in the reference, which runs one graph per
// process, LouvainCPP.cpp:209): every level of every graph in one set of
// launches over the disjoint union of the graphs still running.
namespace {

struct BatchLevel {
  std::vector<int32_t> act;     // original graph of each level graph
  std::vector<int32_t> vbase;   // [G+1] vertex ranges of the level graphs
};

// Input of a batched run: graph g has vertex_off[g+1]-vertex_off[g] vertices
// and entry_off[g+1]-entry_off[g] entries at src[g], dst[g], w[g] (device
// pointers, or host pointers when `host` is set).
struct BatchInput {
  int32_t G = 0;
  const int64_t* eoff = nullptr;
  const int32_t* voff = nullptr;
  std::vector<const int32_t*> src, dst;
  std::vector<const float*> w;
  bool host = false;
};

void batch_run(lvg_ctx* c, const BatchInput& in, int32_t* part_out, double* q_out, int32_t* levels_out,
               int32_t* comms_out, int32_t* status_out) {
  cudaStream_t s = c->stream;
  const int32_t G0 = in.G;
  const int64_t* eoff = in.eoff;
  const int32_t* voff = in.voff;
  const int64_t E0 = eoff[G0];
  const int32_t V0 = voff[G0];
  for (int32_t g = 0; g < G0; ++g) {
    require(eoff[g + 1] >= eoff[g] && voff[g + 1] >= voff[g], LVG_ERR_INVALID_ARG, "offsets must not decrease");
    require((int64_t)(voff[g + 1] - voff[g]) <= (int64_t)kGroup * kGroup, LVG_ERR_CAPACITY,
            "a batched graph may have at most 2048*2048 vertices");
    require(eoff[g + 1] == eoff[g] || (in.src[g] && in.dst[g] && in.w[g]), LVG_ERR_INVALID_ARG, "null edge array");
  }
  require(E0 < ((int64_t)1 << 31), LVG_ERR_CAPACITY, "a batch may hold at most 2^31-1 entries");
  drop_graphs(c);
  c->pre0 = PreCsr();   // the batch reuses the arena
  c->loaded = false;
  c->have_state = false;
  size_t need = c->cfg.arena_bytes > 0 ? (size_t)c->cfg.arena_bytes
                                       : arena_estimate(V0, E0, true) + 256 * (size_t)G0 + 8 * (size_t)V0;
  c->arena.reserve(need);
  Arena& a = c->arena;
  // level-0 union list with global vertex ids
  int32_t* src0 = a.lo_n<int32_t>(E0);
  int32_t* dst0 = a.lo_n<int32_t>(E0);
  float* w0 = a.lo_n<float>(E0);
  int32_t* gid0 = a.lo_n<int32_t>(V0);
  int32_t* local0 = a.lo_n<int32_t>(V0);
  {
    HiScope hs(a);
    std::vector<const void*> ptrs(3 * (size_t)G0);
    if (in.host) {
      // stage the host lists (graph by graph, in entry order) and point into the copy
      int32_t* ss = a.hi_n<int32_t>(E0);
      int32_t* sd = a.hi_n<int32_t>(E0);
      float* sw = a.hi_n<float>(E0);
      bool packed = G0 > 0 && in.src[0] && in.dst[0] && in.w[0];
      for (int32_t g = 0; packed && g < G0; ++g)
        packed = in.src[g] == in.src[0] + eoff[g] && in.dst[g] == in.dst[0] + eoff[g] && in.w[g] == in.w[0] + eoff[g];
      if (packed && E0 > 0) {   // one copy per array
        LVG_CUDA(cudaMemcpyAsync(ss, in.src[0], sizeof(int32_t) * E0, cudaMemcpyHostToDevice, s));
        LVG_CUDA(cudaMemcpyAsync(sd, in.dst[0], sizeof(int32_t) * E0, cudaMemcpyHostToDevice, s));
        LVG_CUDA(cudaMemcpyAsync(sw, in.w[0], sizeof(float) * E0, cudaMemcpyHostToDevice, s));
      }
      for (int32_t g = 0; g < G0; ++g) {
        const int64_t e0 = eoff[g], n = eoff[g + 1] - eoff[g];
        if (n > 0 && !packed) {
          LVG_CUDA(cudaMemcpyAsync(ss + e0, in.src[g], sizeof(int32_t) * n, cudaMemcpyHostToDevice, s));
          LVG_CUDA(cudaMemcpyAsync(sd + e0, in.dst[g], sizeof(int32_t) * n, cudaMemcpyHostToDevice, s));
          LVG_CUDA(cudaMemcpyAsync(sw + e0, in.w[g], sizeof(float) * n, cudaMemcpyHostToDevice, s));
        }
        ptrs[g] = ss + e0;
        ptrs[G0 + g] = sd + e0;
        ptrs[2 * G0 + g] = sw + e0;
      }
    } else {
      for (int32_t g = 0; g < G0; ++g) {
        ptrs[g] = in.src[g];
        ptrs[G0 + g] = in.dst[g];
        ptrs[2 * G0 + g] = in.w[g];
      }
    }
    const void** dptrs = a.hi_n<const void*>(3 * (int64_t)G0);
    int64_t* deoff = a.hi_n<int64_t>(G0 + 1);
    int32_t* dvoff = a.hi_n<int32_t>(G0 + 1);
    uint32_t* bad = a.hi_n<uint32_t>(1);
    LVG_CUDA(cudaMemcpyAsync(dptrs, ptrs.data(), sizeof(void*) * ptrs.size(), cudaMemcpyHostToDevice, s));
    LVG_CUDA(cudaMemcpyAsync(deoff, eoff, sizeof(int64_t) * (G0 + 1), cudaMemcpyHostToDevice, s));
    LVG_CUDA(cudaMemcpyAsync(dvoff, voff, sizeof(int32_t) * (G0 + 1), cudaMemcpyHostToDevice, s));
    LVG_CUDA(cudaMemsetAsync(bad, 0, sizeof(uint32_t), s));
    batch_globalize((const int32_t* const*)dptrs, (const int32_t* const*)(dptrs + G0),
                    (const float* const*)(dptrs + 2 * G0), E0, deoff, dvoff, G0, src0, dst0, w0, bad, s);
    batch_vgid(dvoff, G0, V0, gid0, s);
    batch_local_ids(gid0, dvoff, V0, local0, s);
    uint32_t h = 0;
    LVG_CUDA(cudaMemcpyAsync(&h, bad, sizeof h, cudaMemcpyDeviceToHost, s));
    sync(c);
    require(h == 0, LVG_ERR_INVALID_ARG, "edge list has a vertex id out of its graph or a negative / non-finite weight");
  }
  const size_t base_lo = a.lo;
  std::vector<double> mod(G0, 0.0);
  std::vector<int32_t> levels(G0, 0), comms(G0, 0), status(G0, 0);
  BatchLevel L;
  L.act.resize(G0);
  std::iota(L.act.begin(), L.act.end(), 0);
  L.vbase.assign(voff, voff + G0 + 1);
  const int32_t *lsrc_d = src0, *ldst_d = dst0;
  const float* lw_d = w0;
  int64_t E = E0;
  c->levels.clear();
  for (int level = 0;; ++level) {
    const int32_t G = (int32_t)L.act.size();
    const int32_t V = L.vbase[G];
    LevelGraph& g = c->g;
    g = LevelGraph();
    g.V = V;
    g.E = E;
    g.src = lsrc_d;
    g.dst = ldst_d;
    g.w = lw_d;
    // per-level graph arrays
    int32_t* vbase_d = a.lo_n<int32_t>(G + 1);
    int32_t* vgid = a.lo_n<int32_t>(V);
    double* gm = a.lo_n<double>(G);
    LVG_CUDA(cudaMemcpyAsync(vbase_d, L.vbase.data(), sizeof(int32_t) * (G + 1), cudaMemcpyHostToDevice, s));
    batch_vgid(vbase_d, G, V, vgid, s);
    batch_m(lsrc_d, lw_d, E, vgid, gm, G, s);
    g.gm = gm;
    g.vgid = vgid;
    build_level(g, c->tune, a, s);
    CommState& st = c->st;
    alloc_state(g, st, a);
    // commit plan: groups of 2048 communities per graph
    std::vector<int32_t> blk_g, blk_c0, gblk0(G + 1);
    for (int32_t j = 0; j < G; ++j) {
      gblk0[j] = (int32_t)blk_g.size();
      for (int32_t c0 = L.vbase[j]; c0 < L.vbase[j + 1]; c0 += kGroup) {
        blk_g.push_back(j);
        blk_c0.push_back(c0);
      }
    }
    gblk0[G] = (int32_t)blk_g.size();
    BatchPlan bp;
    bp.nblk = (int64_t)blk_g.size();
    int32_t* d_blk_g = a.lo_n<int32_t>(bp.nblk);
    int32_t* d_blk_c0 = a.lo_n<int32_t>(bp.nblk);
    int32_t* d_gblk0 = a.lo_n<int32_t>(G + 1);
    double* partials = a.lo_n<double>(bp.nblk);
    LVG_CUDA(cudaMemcpyAsync(d_blk_g, blk_g.data(), sizeof(int32_t) * bp.nblk, cudaMemcpyHostToDevice, s));
    LVG_CUDA(cudaMemcpyAsync(d_blk_c0, blk_c0.data(), sizeof(int32_t) * bp.nblk, cudaMemcpyHostToDevice, s));
    LVG_CUDA(cudaMemcpyAsync(d_gblk0, gblk0.data(), sizeof(int32_t) * (G + 1), cudaMemcpyHostToDevice, s));
    bp.vbase = vbase_d;
    bp.blk_g = d_blk_g;
    bp.blk_c0 = d_blk_c0;
    bp.gblk0 = d_gblk0;
    st.partials = partials;
    // per-graph control
    BatchCtl C;
    C.q_prev = a.lo_n<double>(G);
    C.cur = a.lo_n<double>(G);
    C.lower = a.lo_n<double>(G);
    C.q_ret = a.lo_n<double>(G);
    int32_t* ints = a.lo_n<int32_t>(6 * (int64_t)G + 1);
    C.pass = ints;
    C.stop_now = ints + G;
    C.done = ints + 2 * G;
    C.status = ints + 3 * G;
    C.passes = ints + 4 * G;
    C.ndone = ints + 6 * G;
    C.pass_min = c->cfg.pass_min_gain;
    C.max_passes = c->cfg.max_passes;
    st.gid = vgid;
    st.gdone = C.done;
    batch_init(g, st, s);
    reset_ctl(st, 0.0, c->cfg.pass_min_gain, -1, s);
    batch_commit(0, bp, gm, g.k, st, C, s);
    batch_ctl(1, bp, st, C, G, s);
    std::vector<double> q0(G), hv(G);
    LVG_CUDA(cudaMemcpyAsync(q0.data(), C.q_prev, sizeof(double) * G, cudaMemcpyDeviceToHost, s));
    sync(c);
    for (int32_t j = 0; j < G; ++j) hv[j] = level == 0 ? q0[j] : mod[L.act[j]];   // lower (LouvainCPP.cpp:356,446)
    LVG_CUDA(cudaMemcpyAsync(C.lower, hv.data(), sizeof(double) * G, cudaMemcpyHostToDevice, s));
    std::fill(hv.begin(), hv.end(), -1.0);                                        // curMod = -1
    LVG_CUDA(cudaMemcpyAsync(C.cur, hv.data(), sizeof(double) * G, cudaMemcpyHostToDevice, s));
    // a graph without entries keeps its identity partition after one level
    // (LouvainCPP.cpp:211-230): its pass loop is over before it starts
    std::vector<int32_t> empty(G, 0);
    int32_t n_empty = 0;
    if (level == 0)
      for (int32_t j = 0; j < G; ++j) n_empty += (empty[j] = eoff[j + 1] == eoff[j] ? 1 : 0);
    {
      std::vector<int32_t> iv(6 * (size_t)G + 1, 0);
      for (int32_t j = 0; j < G; ++j) {
        iv[j] = 1;                                                                 // pass 1
        iv[2 * G + j] = empty[j];                                                  // done
      }
      iv[6 * G] = n_empty;                                                         // ndone
      LVG_CUDA(cudaMemcpyAsync(ints, iv.data(), sizeof(int32_t) * iv.size(), cudaMemcpyHostToDevice, s));
    }
    // pass loop of all graphs
    if (n_empty < G) {
      L2Window l2(c, st);
      const int chunk = c->cfg.passes_per_sync > 0 ? c->cfg.passes_per_sync : 4;
      PassCtl h;
      int launched = 0;
      for (;;) {
        for (int p = 0; p < chunk; ++p) {
          if (launched == 0) launch_moves_singleton(g, st, s, &c->side);   // from batch_init's singletons
          else launch_moves(g, st, s, &c->side);
          batch_commit(1, bp, gm, g.k, st, C, s);
          batch_ctl(0, bp, st, C, G, s);
          ++launched;
        }
        LVG_CUDA(cudaMemcpyAsync(&h, st.ctl, sizeof h, cudaMemcpyDeviceToHost, s));
        sync(c);
        if (h.done) break;
        if (h.err) throw Error(LVG_ERR_CAPACITY, "neighbour-community table probe limit exceeded");
        if (launched >= kHardPassCap) throw Error(LVG_ERR_NOT_CONVERGED, "hard pass cap reached");
      }
    }
    launch_merge_deltas(g, st, s);
    batch_commit(2, bp, gm, g.k, st, C, s);
    batch_ctl(2, bp, st, C, G, s);
    std::vector<double> qret(G);
    std::vector<int32_t> passes(G), stat(G);
    LVG_CUDA(cudaMemcpyAsync(qret.data(), C.q_ret, sizeof(double) * G, cudaMemcpyDeviceToHost, s));
    LVG_CUDA(cudaMemcpyAsync(passes.data(), C.passes, sizeof(int32_t) * G, cudaMemcpyDeviceToHost, s));
    LVG_CUDA(cudaMemcpyAsync(stat.data(), C.status, sizeof(int32_t) * G, cudaMemcpyDeviceToHost, s));
    // renumber, compose, decide who goes on
    const size_t run_hi = a.hi;
    int32_t* part = a.hi_n<int32_t>(V);
    uint32_t* pos = a.hi_n<uint32_t>(V + 1);
    int32_t Ctot = renumber_pos(g, st.comm, part, pos, a, s);
    int32_t* cbase_d = a.hi_n<int32_t>(G + 1);
    gather_u32(pos, vbase_d, G + 1, cbase_d, s);
    std::vector<int32_t> cbase(G + 1);
    LVG_CUDA(cudaMemcpyAsync(cbase.data(), cbase_d, sizeof(int32_t) * (G + 1), cudaMemcpyDeviceToHost, s));
    int64_t* ecnt_d = a.hi_n<int64_t>(G);
    batch_count(lsrc_d, E, vgid, ecnt_d, G, s);
    std::vector<int64_t> ecnt(G);
    LVG_CUDA(cudaMemcpyAsync(ecnt.data(), ecnt_d, sizeof(int64_t) * G, cudaMemcpyDeviceToHost, s));
    std::vector<int32_t> lidx(G0, -1);
    for (int32_t j = 0; j < G; ++j) lidx[L.act[j]] = j;
    int32_t* lidx_d = a.hi_n<int32_t>(G0);
    LVG_CUDA(cudaMemcpyAsync(lidx_d, lidx.data(), sizeof(int32_t) * G0, cudaMemcpyHostToDevice, s));
    batch_compose(local0, gid0, V0, lidx_d, vbase_d, cbase_d, part, s);
    sync(c);
    (void)Ctot;
    BatchLevel N;
    std::vector<int32_t> shift(G, INT_MIN);
    int64_t E_keep = 0;
    N.vbase.push_back(0);
    for (int32_t j = 0; j < G; ++j) {
      const int32_t g0 = L.act[j];
      const int32_t Cj = cbase[j + 1] - cbase[j];
      levels[g0] = level + 1;
      comms[g0] = Cj;
      bool stop = stat[j] != LVG_OK || empty[j];
      if (stop) status[g0] = stat[j];
      if (!stop && level > 0 && (qret[j] - mod[g0]) < c->cfg.level_min_gain) stop = true;   // LouvainCPP.cpp:466
      if (!stop && c->cfg.max_levels >= 0 && level + 1 >= c->cfg.max_levels) {
        stop = true;
        status[g0] = LVG_ERR_NOT_CONVERGED;
      }
      mod[g0] = qret[j];
      if (!stop) {
        shift[j] = N.vbase.back() - cbase[j];
        N.act.push_back(g0);
        N.vbase.push_back(N.vbase.back() + Cj);
        E_keep += ecnt[j];
      }
    }
    (void)passes;
    if (N.act.empty()) {
      a.hi = run_hi;
      break;
    }
    int32_t* shift_d = a.hi_n<int32_t>(G);
    LVG_CUDA(cudaMemcpyAsync(shift_d, shift.data(), sizeof(int32_t) * G, cudaMemcpyHostToDevice, s));
    int32_t *os = nullptr, *od = nullptr;
    float* ow = nullptr;
    int64_t n = batch_induce(g, part, vgid, shift_d, N.vbase.back(), E_keep, &os, &od, &ow, a, s);
    a.lo = base_lo;
    int32_t* ns = a.lo_n<int32_t>(n);
    int32_t* nd = a.lo_n<int32_t>(n);
    float* nw = a.lo_n<float>(n);
    if (n > 0) {
      LVG_CUDA(cudaMemcpyAsync(ns, os, sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, s));
      LVG_CUDA(cudaMemcpyAsync(nd, od, sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, s));
      LVG_CUDA(cudaMemcpyAsync(nw, ow, sizeof(float) * n, cudaMemcpyDeviceToDevice, s));
    }
    sync(c);
    a.hi = run_hi;
    lsrc_d = ns;
    ldst_d = nd;
    lw_d = nw;
    E = n;
    L = std::move(N);
  }
  // per-graph FP64 Newman modularity of the final partitions
  {
    std::vector<int32_t> coff(G0 + 1, 0);
    for (int32_t g0 = 0; g0 < G0; ++g0) coff[g0 + 1] = coff[g0] + comms[g0];
    const int32_t Ctot = coff[G0];
    std::vector<int32_t> cg(std::max(Ctot, 1), 0), blk_g, blk_c0, gblk0(G0 + 1);
    for (int32_t g0 = 0; g0 < G0; ++g0) {
      gblk0[g0] = (int32_t)blk_g.size();
      for (int32_t k = coff[g0]; k < coff[g0 + 1]; ++k) cg[k] = g0;
      for (int32_t c0 = coff[g0]; c0 < coff[g0 + 1]; c0 += kGroup) {
        blk_g.push_back(g0);
        blk_c0.push_back(c0);
      }
    }
    gblk0[G0] = (int32_t)blk_g.size();
    HiScope hs(a);
    BatchPlan cp;
    cp.nblk = (int64_t)blk_g.size();
    int32_t* coff_d = a.hi_n<int32_t>(G0 + 1);
    int32_t* cg_d = a.hi_n<int32_t>(std::max(Ctot, 1));
    int32_t* bg_d = a.hi_n<int32_t>(std::max<int64_t>(cp.nblk, 1));
    int32_t* bc_d = a.hi_n<int32_t>(std::max<int64_t>(cp.nblk, 1));
    int32_t* gb_d = a.hi_n<int32_t>(G0 + 1);
    double* q_d = a.hi_n<double>(G0);
    LVG_CUDA(cudaMemcpyAsync(coff_d, coff.data(), sizeof(int32_t) * (G0 + 1), cudaMemcpyHostToDevice, s));
    LVG_CUDA(cudaMemcpyAsync(cg_d, cg.data(), sizeof(int32_t) * cg.size(), cudaMemcpyHostToDevice, s));
    if (cp.nblk > 0) {
      LVG_CUDA(cudaMemcpyAsync(bg_d, blk_g.data(), sizeof(int32_t) * cp.nblk, cudaMemcpyHostToDevice, s));
      LVG_CUDA(cudaMemcpyAsync(bc_d, blk_c0.data(), sizeof(int32_t) * cp.nblk, cudaMemcpyHostToDevice, s));
    }
    LVG_CUDA(cudaMemcpyAsync(gb_d, gblk0.data(), sizeof(int32_t) * (G0 + 1), cudaMemcpyHostToDevice, s));
    cp.vbase = coff_d;
    cp.blk_g = bg_d;
    cp.blk_c0 = bc_d;
    cp.gblk0 = gb_d;
    batch_modularity(src0, dst0, w0, E0, gid0, local0, cp, cg_d, Ctot, G0, q_d, a, s);
    if (q_out) LVG_CUDA(cudaMemcpyAsync(q_out, q_d, sizeof(double) * G0, cudaMemcpyDeviceToHost, s));
    if (part_out && V0 > 0)
      LVG_CUDA(cudaMemcpyAsync(part_out, local0, sizeof(int32_t) * V0, cudaMemcpyDeviceToHost, s));
    sync(c);
  }
  if (levels_out) std::copy(levels.begin(), levels.end(), levels_out);
  if (comms_out) std::copy(comms.begin(), comms.end(), comms_out);
  if (status_out) std::copy(status.begin(), status.end(), status_out);
  c->g = LevelGraph();
  c->st = CommState();
}

}  // namespace

namespace {
BatchInput packed_input(const int32_t* src, const int32_t* dst, const float* w, const int64_t* entry_off,
                        const int32_t* vertex_off, int32_t n_graphs, bool host) {
  require(n_graphs >= 1 && entry_off && vertex_off, LVG_ERR_INVALID_ARG, "need at least one graph and offsets");
  require(entry_off[0] == 0 && vertex_off[0] == 0, LVG_ERR_INVALID_ARG, "offsets must start at 0");
  require(entry_off[n_graphs] == 0 || (src && dst && w), LVG_ERR_INVALID_ARG, "null edge array");
  BatchInput in;
  in.G = n_graphs;
  in.eoff = entry_off;
  in.voff = vertex_off;
  in.host = host;
  in.src.resize(n_graphs);
  in.dst.resize(n_graphs);
  in.w.resize(n_graphs);
  for (int32_t g = 0; g < n_graphs; ++g) {
    const int64_t e0 = entry_off[g];
    in.src[g] = src ? src + e0 : nullptr;
    in.dst[g] = dst ? dst + e0 : nullptr;
    in.w[g] = w ? w + e0 : nullptr;
  }
  return in;
}
}  // namespace

extern "C" lvg_status lvg_batch_run(lvg_ctx* c, const int32_t* src, const int32_t* dst, const float* w,
                                    const int64_t* entry_off, const int32_t* vertex_off, int32_t n_graphs,
                                    int32_t* part_out, double* q_out, int32_t* levels_out, int32_t* comms_out,
                                    int32_t* status_out) {
  return guarded(c, [&] {
    check_ctx(c);
    BatchInput in = packed_input(src, dst, w, entry_off, vertex_off, n_graphs, true);
    batch_run(c, in, part_out, q_out, levels_out, comms_out, status_out);
  });
}

extern "C" lvg_status lvg_batch_run_graphs(lvg_ctx* c, int32_t n_graphs, const int32_t* const* d_src,
                                           const int32_t* const* d_dst, const float* const* d_w,
                                           const int64_t* n_entries, const int32_t* n_vertices, int32_t* part_out,
                                           double* q_out, int32_t* levels_out, int32_t* comms_out,
                                           int32_t* status_out) {
  return guarded(c, [&] {
    check_ctx(c);
    require(n_graphs >= 1 && d_src && d_dst && d_w && n_entries && n_vertices, LVG_ERR_INVALID_ARG,
            "need at least one graph and its arrays");
    std::vector<int64_t> eoff(n_graphs + 1, 0);
    std::vector<int32_t> voff(n_graphs + 1, 0);
    for (int32_t g = 0; g < n_graphs; ++g) {
      require(n_entries[g] >= 0 && n_vertices[g] >= 0, LVG_ERR_INVALID_ARG, "negative size");
      require((int64_t)voff[g] + n_vertices[g] < ((int64_t)1 << 31), LVG_ERR_CAPACITY,
              "a batch may hold at most 2^31-1 vertices");
      eoff[g + 1] = eoff[g] + n_entries[g];
      voff[g + 1] = voff[g] + n_vertices[g];
    }
    BatchInput in;
    in.G = n_graphs;
    in.eoff = eoff.data();
    in.voff = voff.data();
    in.src.assign(d_src, d_src + n_graphs);
    in.dst.assign(d_dst, d_dst + n_graphs);
    in.w.assign(d_w, d_w + n_graphs);
    batch_run(c, in, part_out, q_out, levels_out, comms_out, status_out);
  });
}

extern "C" lvg_status lvg_reserve(lvg_ctx* c, int64_t bytes) {
  return guarded(c, [&] {
    check_ctx(c);
    require(bytes >= 0, LVG_ERR_INVALID_ARG, "negative size");
    require(!c->loaded, LVG_ERR_STATE, "reserve before loading a graph");
    c->arena.reserve((size_t)bytes);
  });
}

extern "C" lvg_status lvg_batch_footprint(int64_t n_vertices, int64_t n_entries, int32_t n_graphs, int64_t* bytes) {
  if (!bytes || n_vertices < 0 || n_entries < 0 || n_graphs < 0) return LVG_ERR_INVALID_ARG;
  *bytes = (int64_t)(arena_estimate(n_vertices, n_entries, true) + 256 * (size_t)n_graphs +
                     8 * (size_t)n_vertices);
  return LVG_OK;
}

extern "C" lvg_status lvg_batch_run_device(lvg_ctx* c, const int32_t* d_src, const int32_t* d_dst,
                                           const float* d_w, const int64_t* entry_off, const int32_t* vertex_off,
                                           int32_t n_graphs, int32_t* part_out, double* q_out, int32_t* levels_out,
                                           int32_t* comms_out, int32_t* status_out) {
  return guarded(c, [&] {
    check_ctx(c);
    BatchInput in = packed_input(d_src, d_dst, d_w, entry_off, vertex_off, n_graphs, false);
    batch_run(c, in, part_out, q_out, levels_out, comms_out, status_out);
  });
}
