// Level data structures and host-side phase functions of the Louvain hot path.
#pragma once
#include <vector>

#include "lvg_internal.cuh"

namespace lvg {

// Control block of the pass loop, resident on the device so that a whole
// level of passes runs without host round trips.  Kernels of a pass that
// start after `done` is set return at once.
struct PassCtl {
  double q_prev;     // Q of the committed state, tested by this pass
  double cur;        // running floor (curMod, OneLevelKernel.cu:528,894-896)
  double lower;      // floor given by the caller
  double pass_min;   // __MIN (OneLevelKernel.cu:425)
  double q_ret;      // Q after the isolated-vertex merge
  int32_t pass;      // 1-based pass in progress
  int32_t max_passes;
  int32_t stop_now;  // 1: gain below threshold this pass, 2: pass cap
  int32_t done;
  int32_t status;    // LVG_OK or LVG_ERR_NOT_CONVERGED
  int32_t passes;    // passes executed
  uint32_t err;      // device-side error bits
  int32_t pad;
};

enum : uint32_t { kErrProbe = 1u };

// Degree classes of the move kernels (see bucket_of).
enum { kB4 = 0, kB8, kB16, kB32, kBTile, kBBlock, kBHub, kNumBuckets };

// Level-0 CSR built while the list streamed in from the host
// (stream_load_level0); valid only if the whole list was in range, strictly
// sorted and symmetric.  Lives below the level region of the arena, so a
// rerun from level 0 uses it again.
struct PreCsr {
  bool valid = false;
  int64_t* off = nullptr;
  int32_t* col = nullptr;
  float* cw = nullptr;
  double* k = nullptr;
  float* loopw = nullptr;
  uint8_t* has_loop = nullptr;
  double m = 0.0;
  int64_t nnz = 0;
};

// One level of the graph on the device.
struct LevelGraph {
  int32_t V = 0;
  int64_t E = 0;                  // level input list
  const int32_t* src = nullptr;
  const int32_t* dst = nullptr;
  const float* w = nullptr;
  int64_t nnz = 0;                // merged doubled list, self loops removed
  int64_t* off = nullptr;         // [V+1]
  int32_t* col = nullptr;         // [nnz]
  float* cw = nullptr;            // [nnz]
  double* k = nullptr;            // degree (InitKernel.cu:154-179), 0 for vertices without entries
  double* kfrac = nullptr;        // k / 2m
  float* loopw = nullptr;         // last self-loop weight (InitKernel.cu:181-194,239-242)
  uint8_t* has_loop = nullptr;
  double m = 0.0;                 // sum of input weights (NeighbourCompute.cu:46)
  bool sorted_symmetric = false;  // CSR built without sorting (list sorted and symmetric)
  const PreCsr* pre = nullptr;    // level 0 only: CSR built during the upload
  const double* gm = nullptr;     // batched runs: m of each graph (device)
  const int32_t* vgid = nullptr;  // batched runs: graph of each vertex (device)
  int32_t* blist = nullptr;       // vertices grouped by degree class, in index order inside a class
  int64_t nbucket[kNumBuckets] = {};
  int64_t bstart[kNumBuckets] = {};
  int32_t max_deg = 0;
  int32_t block_max = 4096;       // largest degree of the block class (the context's threshold)
  // sliced-ELL copies of the degree classes up to 32 (slots of class b from ell_base[b])
  int32_t* ell_col = nullptr;
  float* ell_w = nullptr;
  int64_t ell_base[kNumBuckets] = {};
  struct VInfo* ell_info = nullptr;  // per item of the classes up to 32, from bstart[kB4]; filled by init_state
  // tiles of the small-degree bucket
  int32_t* tile_start = nullptr;  // [ntiles+1] first bucket index of each tile
  int64_t ntiles = 0;
  bool int_acc = false;           // integral weights, degrees < 2^30: exact int32 sums
  int32_t* k32 = nullptr;         // k as int32 when int_acc (the first pass's gathered totals)
  // hubs: 4096-entry chunks of the hub rows, each hub's communities hashed
  // into a power-of-two number of buckets (see hub_part/hub_agg kernels)
  int32_t* chunk_hub = nullptr;   // [nchunk] hub index of the chunk
  int64_t* chunk_beg = nullptr;   // [nchunk] first CSR entry of the chunk
  int64_t* chunk_cbo = nullptr;   // [nchunk] first of the chunk's bucket offsets in cb_off
  int64_t* chunk_stg = nullptr;   // [nchunk] first staging slot of the chunk
  int64_t nchunk = 0;
  int32_t* hub_plog = nullptr;    // [nhub] log2 bucket count
  int32_t* hub_cb0 = nullptr;     // [nhub+1] first chunk of each hub
  int32_t* hub_bb0 = nullptr;     // [nhub+1] first bucket of each hub
  int32_t* bucket_hub = nullptr;  // [nhub_bucket] hub of each bucket
  int64_t nhub_bucket = 0;
  uint16_t* cb_off = nullptr;     // per chunk: bucket offsets inside the chunk
  unsigned long long* stage = nullptr;  // [hub entries] pairs grouped by bucket per chunk
  uint32_t* hub_sawown = nullptr;
  struct HubPartial* hub_part = nullptr;  // [nhub_bucket]
  // singleton first pass: chunks {vertex, piece} of the rows longer than 32,
  // rows of more than one chunk {vertex, first chunk}, per-chunk partials
  int2* sp_chunk = nullptr;
  int64_t sp_nchunk = 0;
  int2* sp_multi = nullptr;
  int64_t sp_nmulti = 0;
  struct HubPartial* sp_part = nullptr;
};

// Pass deltas of one community in one 32-byte sector, so that a move's three
// updates of a community (total, internal weight, size) touch one sector.
// `out` / `iw_out` carry the own side of a move out of a singleton community
// (the first pass of a level): written without atomics by the community's
// only vertex, applied by the commit.
struct __align__(32) Delta {
  double tot;
  double in;
  int32_t size;
  int32_t out;
  double iw_out;
};

struct CommState {
  int32_t* comm = nullptr;
  int32_t* next = nullptr;
  double* tot = nullptr;
  double* in = nullptr;
  int32_t* size = nullptr;
  Delta* delta = nullptr;
  int32_t* cand = nullptr;
  double* partials = nullptr;     // level-1 group partials of Q
  double* partials2 = nullptr;
  PassCtl* ctl = nullptr;
  int64_t ngroups = 0;
  size_t hot_bytes = 0;           // tot | comm | size, contiguous from tot
  const int32_t* gid = nullptr;   // batched runs: graph of each vertex
  int32_t* gdone = nullptr;       // batched runs: per-graph stop flags
  unsigned long long* queue = nullptr;   // work counters of the persistent move kernels (batched runs)
};
constexpr int kQueueSlots = 8;    // hub buckets, tiles, up to six block-class degree bands

struct Tuning {
  int32_t warp_max = 512;         // largest degree packed into tiles
  int32_t block_max = 4096;       // largest degree with a block-private table
  int32_t coarsen = 0;            // coarsening method (kCoarsen*)
};

// Coarsening methods of a level (lvg_config.coarsen_mode).
enum : int32_t { kCoarsenAuto = 0, kCoarsenChunks = 1, kCoarsenTransposed = 2, kCoarsenSort = 3 };

// Validate an input list on the device: ids in range, weights finite >= 0.
bool validate_edges(const int32_t* src, const int32_t* dst, const float* w, int64_t E, int32_t V,
                    Arena& a, cudaStream_t s);

// Build the level CSR, degrees, loops and buckets (NeighbourCompute.cu:42-117,
// InitKernel.cu:245-339).  Level arrays go to the arena's low end.
void build_level(LevelGraph& g, const Tuning& t, Arena& a, cudaStream_t s);
// Copies a host list into (src, dst, w) in chunks of `chunk` entries on
// `copy` while kernels on `s` check each arrived chunk (ids in range, finite
// non-negative weights, strict order, symmetry fingerprints) and build the
// sorted-symmetric CSR into `pre`, allocated at the arena's low end (and
// released again, pre.valid false, when the list is not in that form).
// Returns false if an entry failed the range or weight check.
bool stream_load_level0(const int32_t* hsrc, const int32_t* hdst, const float* hw, int32_t* src, int32_t* dst,
                        float* w, int64_t E, int32_t V, int64_t chunk, PreCsr& pre, std::vector<cudaEvent_t>& evs,
                        Arena& a, cudaStream_t s, cudaStream_t copy);

// Allocate community state for g (low end) and set the singleton state
// (InitKernel.cu:196-216, OneLevelKernel.cu:80-91); ctl->q_prev = Q(S0).
void alloc_state(const LevelGraph& g, CommState& st, Arena& a);
void init_state(const LevelGraph& g, CommState& st, double lower, double pass_min, int32_t max_passes,
                Arena& a, cudaStream_t s);

// Side streams on which the smaller degree classes of a pass run.
struct SideStreams {
  cudaStream_t side[3];
  cudaEvent_t fork;
  cudaEvent_t join[3];
};

// Launch one pass: move kernels + conditional commit + control.
void launch_pass(const LevelGraph& g, CommState& st, cudaStream_t s, const SideStreams* ss);
// The ΔQ test, conditional commit and pass control of one pass.
void launch_commit(const LevelGraph& g, CommState& st, cudaStream_t s);
// Launch only the move kernels (decisions, accumulations into d*).
void launch_moves(const LevelGraph& g, CommState& st, cudaStream_t s, const SideStreams* ss);
// The move kernels of a pass from the singleton state (the first pass of a
// level, right after init_state / batch_init): same decisions, no tables.
void launch_moves_singleton(const LevelGraph& g, CommState& st, cudaStream_t s, const SideStreams* ss);
// After the loop is done: isolated-vertex merge, final commit, ctl->q_ret.
void launch_merge(const LevelGraph& g, CommState& st, cudaStream_t s);
// Q of the committed state into *dst (device).
void launch_q(const LevelGraph& g, CommState& st, double* dst, cudaStream_t s);
// Overwrite the committed state from comm (device) and recompute totals.
void set_state_from(const LevelGraph& g, CommState& st, const int32_t* d_comm, cudaStream_t s);
void clear_deltas(const LevelGraph& g, CommState& st, cudaStream_t s);
void reset_ctl(CommState& st, double lower, double pass_min, int32_t max_passes, cudaStream_t s);

// Renumber (RenumberKernel.cu:63-221): part[i] = rank of comm[i] by smallest
// member index; returns the community count (synchronises).
int32_t renumber(const LevelGraph& g, const int32_t* comm, int32_t* part, Arena& a, cudaStream_t s);

// Coarsen (InducedGraphKernel.cu:50-113): writes the next level input list to
// high-end scratch and returns its size; out_* point into that scratch.
// Coarsening of a strictly sorted, symmetric level list without a device-wide
// sort of all its entries (induce.cu).  Writes the same list as the
// sort-based path into osrc/odst/ow (capacity E) and its length into *count;
// returns false, having done nothing, when the list is not in that form or
// the arena lacks room.  With `next` (arrays of capacity E entries / C rows
// given), also writes the coarse list's CSR as build_csr_fast would build it
// and marks it valid.
bool induce_sorted(const LevelGraph& g, const int32_t* part, int32_t C, int32_t* osrc, int32_t* odst, float* ow,
                   int64_t* count, PreCsr* next, Arena& a, cudaStream_t s);
// The same list (and CSR) by transposition (induce.cu): the keys listed in
// segment order of the second community, then one stable sort by the first.
// Same preconditions and return value as induce_sorted.
bool induce_transposed(const LevelGraph& g, const int32_t* part, int32_t C, int32_t* osrc, int32_t* odst,
                       float* ow, int64_t* count, PreCsr* next, Arena& a, cudaStream_t s);
// Coarse list of the level under `part` (C communities), left at the arena's
// high end.  With `next`: when the sort-free path runs, also the next level's
// CSR (high end, next->valid set); otherwise next->valid stays false.
int64_t induce(const LevelGraph& g, const int32_t* part, int32_t C, int32_t** out_src, int32_t** out_dst,
               float** out_w, Arena& a, cudaStream_t s, PreCsr* next = nullptr, int32_t mode = kCoarsenAuto);

// FP64 Newman modularity of part[] (values < C) over an input list (device).
// symmetric: the list is known to hold (v, u, w) for every (u, v, w) (its
// community strengths are then summed from the source side alone).
double modularity_fp64(const int32_t* src, const int32_t* dst, const float* w, int64_t E, int32_t C,
                       const int32_t* part, Arena& a, cudaStream_t s, bool symmetric = false);

// The same modularity with caller-provided scratch: Kc, Ain, t of C doubles,
// partials of ceil(C/2048) doubles; twoW_q[0] = 2W, twoW_q[1] = Q (device).
// Community ids outside [0, C) are left out of the sums and set *bad (device
// flag, nullable).
void modularity_fp64_scratch(const int32_t* src, const int32_t* dst, const float* w, int64_t E, int32_t C,
                             const int32_t* part, double* Kc, double* Ain, double* t, double* partials,
                             double* twoW_q, uint32_t* bad, cudaStream_t s);

// ---------------------------------------------------------------- batched runs
// Per-graph pass control of a batched run (device arrays of the level's graphs).
struct BatchCtl {
  double* q_prev;
  double* cur;
  double* lower;
  double* q_ret;
  int32_t* pass;
  int32_t* stop_now;
  int32_t* done;
  int32_t* status;
  int32_t* passes;
  int32_t* ndone;
  double pass_min;
  int32_t max_passes;
};

// Commit blocks of a batched level: block b sums communities
// blk_c0[b]..+2048 of graph blk_g[b]; graph j owns blocks gblk0[j]..gblk0[j+1].
struct BatchPlan {
  const int32_t* vbase = nullptr;   // [G+1]
  const int32_t* blk_g = nullptr;
  const int32_t* blk_c0 = nullptr;
  const int32_t* gblk0 = nullptr;   // [G+1]
  int64_t nblk = 0;
};

// Union list of the graphs' own lists (device pointer arrays of G entries);
// *bad |= 1 on an id outside its graph or a negative / non-finite weight.
void batch_globalize(const int32_t* const* psrc, const int32_t* const* pdst, const float* const* pw, int64_t E,
                     const int64_t* eoff, const int32_t* voff, int32_t G, int32_t* gsrc, int32_t* gdst, float* gw,
                     uint32_t* bad, cudaStream_t s);
void batch_vgid(const int32_t* vbase, int32_t G, int32_t V, int32_t* vgid, cudaStream_t s);
// local[i] = i - voff[gid[i]]
void batch_local_ids(const int32_t* gid, const int32_t* voff, int32_t V, int32_t* local, cudaStream_t s);
void batch_m(const int32_t* src, const float* w, int64_t E, const int32_t* vgid, double* gm, int32_t G,
             cudaStream_t s);
void batch_init(const LevelGraph& g, CommState& st, cudaStream_t s);
// mode: 0 init (Q only), 1 pass (per-graph ΔQ test + commit), 2 force commit
// g_k: degrees of the level's vertices (the own side of first-pass moves).
void batch_commit(int mode, const BatchPlan& bp, const double* gm, const double* g_k, CommState& st,
                  const BatchCtl& C, cudaStream_t s);
// mode: 0 end of pass, 1 Q of the state into q_prev, 2 into q_ret
void batch_ctl(int mode, const BatchPlan& bp, const CommState& st, const BatchCtl& C, int32_t G, cudaStream_t s);
void launch_merge_deltas(const LevelGraph& g, CommState& st, cudaStream_t s);
// renumber() that also leaves the head-flag scan in pos[0..V] (pos[v] = new
// ids of the communities whose smallest member is below v).
int32_t renumber_pos(const LevelGraph& g, const int32_t* comm, int32_t* part, uint32_t* pos, Arena& a,
                     cudaStream_t s);
// Coarsen the graphs still running: part[v] + shift[graph] (INT_MIN: dropped).
int64_t batch_induce(const LevelGraph& g, const int32_t* part, const int32_t* vgid, const int32_t* shift,
                     int32_t C_next, int64_t E_keep, int32_t** out_src, int32_t** out_dst, float** out_w, Arena& a,
                     cudaStream_t s);
// out[j] = pos[idx[j]]
void gather_u32(const uint32_t* pos, const int32_t* idx, int32_t n, int32_t* out, cudaStream_t s);
// entries of the list per graph
void batch_count(const int32_t* src, int64_t E, const int32_t* vgid, int64_t* cnt, int32_t G, cudaStream_t s);
void batch_compose(int32_t* local0, const int32_t* gid0, int64_t n, const int32_t* lidx, const int32_t* vbase,
                   const int32_t* cbase, const int32_t* part, cudaStream_t s);
// FP64 Newman modularity of every graph: community ids coff[g] + local0[v]
// with coff = cp.vbase, cp the 2048-groups of each graph's communities,
// cg[c] = graph of community c; q[g] on the device, summed on the fixed tree.
void batch_modularity(const int32_t* src, const int32_t* dst, const float* w, int64_t E, const int32_t* gid0,
                      const int32_t* local0, const BatchPlan& cp, const int32_t* cg, int32_t Ctot, int32_t G,
                      double* q, Arena& a, cudaStream_t s);

// Largest row of the level CSR (synchronises).
int64_t max_degree(const LevelGraph& g, Arena& a, cudaStream_t s);

// x[i] = i for i < n.
void iota(int32_t* x, int64_t n, cudaStream_t s);
// part_out[i] = part_level[composed[i]] for i < n.
void compose(int32_t* composed, const int32_t* part_level, int64_t n, cudaStream_t s);

}  // namespace lvg
