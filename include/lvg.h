/*
 * lvg.h -- C ABI of liblvg, the B200 (sm_100a) Louvain hot path.
 *
 * Each entry point replaces one function of the reference's GPU phase API,
 * the six `extern` functions its level driver links against
 * (LouvainCUDA/LouvainCPP.cpp:129-134), or a driver-side step of
 * generate_dendogram (LouvainCPP.cpp:209-553).  The reference file:line each
 * one replaces is given beside it.
 *
 * Conventions
 *  - Vertices are dense indices 0..n_vertices-1 (the reference's CUDPP
 *    id->index hash, InitKernel.cu:276-306, becomes the caller's dense ids).
 *  - An edge list is SoA (src, dst, w) of n_entries entries, exactly what the
 *    reference copies to the device (LouvainCPP.cpp:283-287).  Both directions
 *    of an undirected edge are listed by the caller; the library appends the
 *    reversed copy of every entry as the reference does (NeighbourCompute.cu:66-68).
 *  - Weights are finite and >= 0.
 *  - Every function returns lvg_status; nothing throws across the ABI.  On
 *    error lvg_last_error(ctx) describes the failure.
 *  - A context owns one CUDA stream (or the one given by lvg_set_stream), its
 *    device arena and all device state.  Contexts are independent; one
 *    context must not be used by two host threads at once.
 *  - Host pointers are only read during the call (inputs) or written before
 *    it returns (outputs).  Device pointers passed to lvg_load_edges_device
 *    must stay valid until the next load or lvg_destroy.
 */
#ifndef LVG_H
#define LVG_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  LVG_OK = 0,
  LVG_ERR_INVALID_ARG = 1, /* bad pointer, size, id out of range, negative/non-finite weight */
  LVG_ERR_OOM = 2,         /* device arena or cudaMalloc exhausted */
  LVG_ERR_CAPACITY = 3,    /* a size limit of this build was exceeded */
  LVG_ERR_NOT_CONVERGED = 4, /* pass or level cap reached before the gain threshold */
  LVG_ERR_CUDA = 5,        /* CUDA runtime error */
  LVG_ERR_STATE = 6        /* call out of order (e.g. one_level before load) */
} lvg_status;

typedef struct lvg_ctx lvg_ctx;

typedef struct {
  int32_t device;          /* CUDA device ordinal (reference: cudaSetDevice(0), LouvainCPP.cpp:774) */
  double pass_min_gain;    /* stop a level when Q gains less (reference __MIN = 1e-7, OneLevelKernel.cu:425) */
  double level_min_gain;   /* stop the run when a level gains less (LouvainCPP.cpp:55,466) */
  int32_t max_passes;      /* <0: unbounded like __PASS_MAX=-1 (OneLevelKernel.cu:424) */
  int32_t max_levels;      /* <0: unbounded */
  int64_t arena_bytes;     /* 0: sized from the level-0 graph at load */
  int32_t tile_max_degree; /* vertices up to this degree are packed into shared-memory tiles (<= 512) */
  int32_t block_max_degree;/* up to this degree a block-per-vertex shared table; above, global tables */
  int32_t passes_per_sync; /* passes launched between host checks of convergence (0: default) */
  int32_t use_graphs;      /* replay each pass from CUDA graphs captured once per level (1: on) */
  int32_t l2_persist;      /* keep the gathered community arrays in an L2 persisting window (1: on) */
  int64_t load_chunk_entries; /* lvg_load_edges: the host list is copied in chunks of this many entries
                              * while the level-0 CSR is built from the chunks already on the device
                              * (0: 2^25; rounded up to a multiple of 2048; lists of fewer than two
                              * chunks are copied whole, then built) */
  int32_t coarsen_mode;    /* coarsening of a sorted symmetric level list (InducedGraphKernel.cu:50-113):
                            * 0 automatic, 1 segment chunks, 2 by transposition, 3 sort of all keys;
                            * every mode writes the same coarse list */
} lvg_config;

/* Per-level record of a run (the reference keeps one Partition per level,
 * LouvainCPP.cpp:384,464). */
typedef struct {
  int32_t n_vertices;      /* vertices of the level graph */
  int64_t n_entries;       /* entries of the level input list */
  int64_t nnz;             /* merged CSR entries (doubled list, loops removed) */
  int32_t n_comms;         /* communities after the level (next level's vertices) */
  int32_t passes;          /* move passes, including the last (breaking) one */
  double q_start;          /* Q of the singleton state of the level */
  double q_level;          /* Q returned by the one-level phase (oneLevelCUDA's return value) */
  double ms_build, ms_passes, ms_renumber, ms_induce; /* device time of each phase */
} lvg_level_info;

typedef struct {
  int32_t n_levels;
  int32_t n_comms;         /* communities of the final partition */
  double q_final;          /* FP64 Newman modularity of the final partition on the level-0 graph */
  int64_t pass_entries;    /* sum over levels of nnz * passes (edges processed by move passes) */
  int32_t status;          /* LVG_OK or LVG_ERR_NOT_CONVERGED */
} lvg_result;

/* Defaults: pass/level gain 1e-7 (the reference's), unbounded caps. */
lvg_status lvg_config_default(lvg_config* cfg);

lvg_status lvg_create(const lvg_config* cfg, lvg_ctx** out);
lvg_status lvg_destroy(lvg_ctx* ctx);
const char* lvg_last_error(const lvg_ctx* ctx);
const char* lvg_status_string(lvg_status s);
/* Run all work of this context on `stream` (a cudaStream_t); NULL restores the
 * context's own stream. */
lvg_status lvg_set_stream(lvg_ctx* ctx, void* stream);

/* Load the level-0 edge list from HOST memory and build the level CSR, degrees
 * and self-loop weights.  Replaces the driver's H2D copies
 * (LouvainCPP.cpp:283-287) followed by CalculateNeighbour (NeighbourCompute.cu:42)
 * and initCUDA (InitKernel.cu:245). */
lvg_status lvg_load_edges(lvg_ctx* ctx, const int32_t* src, const int32_t* dst, const float* w,
                          int64_t n_entries, int32_t n_vertices);
/* As lvg_load_edges, with the edge list already in device memory. */
lvg_status lvg_load_edges_device(lvg_ctx* ctx, const int32_t* d_src, const int32_t* d_dst,
                                 const float* d_w, int64_t n_entries, int32_t n_vertices);

/* Q of the current level's committed community state.
 * Replaces modularityCUDA (OneLevelKernel.cu:965-980). */
lvg_status lvg_modularity(lvg_ctx* ctx, double* q);

/* Run the move passes of the current level until the Q gain falls below
 * pass_min_gain, then the isolated-vertex merge.  `lower` is the floor of the
 * running Q (the `lower` argument of the reference).  Replaces oneLevelCUDA
 * (OneLevelKernel.cu:518-954). */
lvg_status lvg_one_level(lvg_ctx* ctx, double lower, double* q, int32_t* passes);

/* Number the current level's communities 0..C-1 in order of their smallest
 * member vertex.  comm_out (host, nullable) receives n_vertices entries.
 * Replaces renumberCUDA (RenumberKernel.cu:63-221). */
lvg_status lvg_renumber(lvg_ctx* ctx, int32_t* comm_out, int32_t* n_comms);

/* Coarsen: the level input list mapped through the renumbered partition,
 * weight 0 -> 1, equal (cu,cv) keys summed, becomes the next level's input
 * list; its CSR is built.  Replaces inducedGraphCUDA (InducedGraphKernel.cu:50-113)
 * and the CalculateNeighbour/initCUDA calls of the next level. */
lvg_status lvg_induce(lvg_ctx* ctx);

/* Whole dendrogram from the loaded graph.  Replaces generate_dendogram
 * (LouvainCPP.cpp:209-553). */
lvg_status lvg_run(lvg_ctx* ctx, lvg_result* res);

/* Results of the last lvg_run / step sequence. */
lvg_status lvg_num_levels(const lvg_ctx* ctx, int32_t* n_levels);
lvg_status lvg_get_level_info(const lvg_ctx* ctx, int32_t level, lvg_level_info* info);
/* Renumbered partition of the level's vertices (the Partition pushed per level,
 * RenumberKernel.cu:202-203), as a dense array of that level's size. */
lvg_status lvg_get_level_partition(const lvg_ctx* ctx, int32_t level, int32_t* part);
/* Community ids of the level before renumbering (vertex-index labels). */
lvg_status lvg_get_level_labels(const lvg_ctx* ctx, int32_t level, int32_t* labels);
/* Partition of the level-0 vertices composed through levels 0..level.
 * Replaces partitionAtLevel (LouvainCPP.cpp:82-106). */
lvg_status lvg_get_partition(const lvg_ctx* ctx, int32_t level, int32_t* part);
/* 1 + max community id of a composed partition.  Replaces countPartitions
 * (LouvainCPP.cpp:116-127). */
lvg_status lvg_count_partitions(const int32_t* part, int64_t n, int32_t* count);

/* FP64 Newman modularity of a partition (host array over the level-0
 * vertices) on the loaded level-0 graph, computed on the device. */
lvg_status lvg_modularity_fp64(lvg_ctx* ctx, const int32_t* part, double* q);

/* Copy the current level's CSR and per-vertex values to host buffers (any may
 * be NULL): off[V+1], col[nnz], w[nnz], degree k[V], loop weight[V], has_loop[V]. */
lvg_status lvg_get_csr(const lvg_ctx* ctx, int32_t* n_vertices, int64_t* nnz, double* m,
                       int64_t* off, int32_t* col, float* w, double* k, float* loopw,
                       uint8_t* has_loop);

/* Copy the current level's input list to host buffers (any may be NULL):
 * src/dst/w of n_entries entries.  After lvg_induce this is the coarse list
 * inducedGraphCUDA writes (InducedGraphKernel.cu:84-113): one entry per
 * distinct (community of src, community of dst) key in ascending key order,
 * weight = sum over the level's entries of (w == 0 ? 1 : w). */
lvg_status lvg_get_level_edges(const lvg_ctx* ctx, int64_t* n_entries, int32_t* src, int32_t* dst, float* w);

/* Set the committed community state of the current level from host arrays
 * (communities as vertex indices) and recompute its totals; used to drive
 * single passes from a known state. */
lvg_status lvg_set_communities(lvg_ctx* ctx, const int32_t* comm);
/* One synchronous decision pass from the committed state, without commit:
 * next[V] chosen community, cand[V] isolated-merge candidate (-1 none).
 * The state is left unchanged.  Restates one launch of the move kernels
 * (SetNewCommunityWarpShuffle + oneLevelKernel, OneLevelKernel.cu:248-422). */
lvg_status lvg_move_decide(lvg_ctx* ctx, int32_t* next, int32_t* cand);

/* Device-time (ms) of the move passes of the last lvg_one_level, and the
 * per-pass breakdown when `ms` is non-NULL (cap entries). */
lvg_status lvg_last_pass_times(const lvg_ctx* ctx, float* ms, int32_t cap, int32_t* n_passes);

/* Device time of the move kernels of each pass of the last one-level phase
 * (CUDA events around the move launches; the first pass runs the singleton
 * kernels).  Fills up to cap values; *n = number of passes. */
lvg_status lvg_move_pass_times(const lvg_ctx* ctx, float* ms, int32_t cap, int32_t* n);

/* Device time of the move kernels (all degree buckets of a pass, the hot
 * path's dominant work) summed over the passes of the last lvg_one_level /
 * lvg_run, and the number of passes it covers. */
lvg_status lvg_move_stats(const lvg_ctx* ctx, double* ms_total, int64_t* n_passes);

/* Number of CUDA kernels this library has launched in this process. */
lvg_status lvg_kernel_launches(int64_t* n);

/* Batched form: run the whole dendrogram of n_graphs independent graphs at
 * once.  Graph g owns entries entry_off[g]..entry_off[g+1] of the HOST arrays
 * src/dst/w, whose vertex ids are local to the graph (0..n_g-1), and
 * n_g = vertex_off[g+1] - vertex_off[g] vertices.  Every graph gets exactly
 * the result of its own lvg_run (same passes, levels, partitions): the graphs
 * share launches, while m, the pass control, Q and the level break stay per
 * graph.  Outputs (host, each nullable): part_out[vertex_off[n_graphs]] final
 * community of every vertex (local to its graph), q_out[g] FP64 Newman
 * modularity, levels_out[g], comms_out[g], status_out[g] (LVG_OK or
 * LVG_ERR_NOT_CONVERGED).  A graph may have at most 2048*2048 vertices; the
 * batch at most 2^31-1 entries.  The reference runs one graph per process
 * (LouvainCPP.cpp:209); it has no batched form. */
lvg_status lvg_batch_run(lvg_ctx* ctx, const int32_t* src, const int32_t* dst, const float* w,
                         const int64_t* entry_off, const int32_t* vertex_off, int32_t n_graphs,
                         int32_t* part_out, double* q_out, int32_t* levels_out, int32_t* comms_out,
                         int32_t* status_out);

/* lvg_batch_run with the packed list already in device memory (d_src, d_dst,
 * d_w: device pointers, read during the call; d_w is used in place).  The
 * offsets and the outputs stay on the host. */
lvg_status lvg_batch_run_device(lvg_ctx* ctx, const int32_t* d_src, const int32_t* d_dst, const float* d_w,
                                const int64_t* entry_off, const int32_t* vertex_off, int32_t n_graphs,
                                int32_t* part_out, double* q_out, int32_t* levels_out, int32_t* comms_out,
                                int32_t* status_out);

/* lvg_batch_run over graphs held in separate device buffers: graph g has
 * n_entries[g] entries at d_src[g], d_dst[g], d_w[g] (device pointers, ids
 * local to the graph) and n_vertices[g] vertices.  The pointer and size arrays
 * are host arrays; outputs as in lvg_batch_run (part_out packed graph after
 * graph). */
lvg_status lvg_batch_run_graphs(lvg_ctx* ctx, int32_t n_graphs, const int32_t* const* d_src,
                                const int32_t* const* d_dst, const float* const* d_w, const int64_t* n_entries,
                                const int32_t* n_vertices, int32_t* part_out, double* q_out, int32_t* levels_out,
                                int32_t* comms_out, int32_t* status_out);

/* Reserve the context's device arena now (at least `bytes`), so that later
 * calls that fit in it allocate nothing.  Only before a graph is loaded. */
lvg_status lvg_reserve(lvg_ctx* ctx, int64_t bytes);

/* Device bytes a batched run of n_graphs graphs with these totals reserves
 * (the arena lvg_batch_run sizes itself to when lvg_config.arena_bytes is 0). */
lvg_status lvg_batch_footprint(int64_t n_vertices, int64_t n_entries, int32_t n_graphs, int64_t* bytes);

/* ------------------------------------------------------------- serving ----
 * A request server over device-resident graphs (continuous batching).
 * n_slots worker contexts, each on its own host thread and CUDA stream, split
 * an HBM budget evenly (each slot's arena is reserved once).  A free slot
 * takes the queued requests in arrival order as one batched run, as many as
 * fit its arena (lvg_batch_footprint), at most max_batch_entries entries and
 * max_batch_graphs graphs; slots run concurrently, so requests that arrive
 * while others are on the GPU start as soon as a slot frees up.  Each
 * request's result is exactly what lvg_run gives for its graph alone. */
typedef struct lvg_server lvg_server;

typedef struct {
  int64_t id;           /* lvg_server_submit's id */
  int64_t tag;          /* the caller's tag */
  int32_t status;       /* LVG_OK, LVG_ERR_NOT_CONVERGED, or the batch's error */
  int32_t n_levels;
  int32_t n_comms;
  int32_t batch_graphs; /* graphs in the batched run that served it */
  double q_final;       /* FP64 Newman modularity of the final partition */
  int64_t t_submit_ns;  /* steady-clock times since lvg_server_create */
  int64_t t_start_ns;
  int64_t t_done_ns;
} lvg_serve_result;

lvg_status lvg_server_create(const lvg_config* cfg, int32_t n_slots, int64_t hbm_budget_bytes,
                             int64_t max_batch_entries, int32_t max_batch_graphs, lvg_server** out);
/* Queue one graph.  d_src/d_dst/d_w: device arrays complete on the device
 * before the call and kept alive until the result is polled; part_out: host
 * array of n_vertices ints written before the result is posted (nullable). */
lvg_status lvg_server_submit(lvg_server* srv, const int32_t* d_src, const int32_t* d_dst, const float* d_w,
                             int64_t n_entries, int32_t n_vertices, int32_t* part_out, int64_t tag,
                             int64_t* id_out);
/* Move up to max finished results into out; *n_out = how many. */
lvg_status lvg_server_poll(lvg_server* srv, lvg_serve_result* out, int32_t max, int32_t* n_out);
/* Wait until every submitted request has finished (timeout_ms < 0: no limit);
 * LVG_ERR_STATE on timeout. */
lvg_status lvg_server_drain(lvg_server* srv, int64_t timeout_ms);
/* Counters: submitted, completed, batched runs, device bytes reserved. */
lvg_status lvg_server_stats(lvg_server* srv, int64_t* submitted, int64_t* completed, int64_t* batches,
                            int64_t* reserved_bytes);
/* Last error message of the server (a copy, valid until this thread's next call). */
const char* lvg_server_last_error(const lvg_server* srv);
/* Stops the workers after the queue is empty and frees every slot. */
lvg_status lvg_server_destroy(lvg_server* srv);

/* Largest community count lvg_modularity_fp64_noalloc accepts. */
#define LVG_NOALLOC_MAX_COMMS (1 << 18)
/* Size of its fixed device array: 3 * 2^18 + 2^18/2048 + 3 = 786,563 doubles
 * (Kc, Ain and the per-community terms, the tree partials, 2W, Q and a flag). */
#define LVG_NOALLOC_SCRATCH_BYTES 6292504

/* FP64 Newman modularity of a partition, like lvg_modularity_fp64, for
 * callers that cannot allocate device memory when they need the value: a
 * serving process whose caching allocator already holds all free HBM in its
 * own pool (a cudaMalloc would fail, or force that pool to give memory back),
 * and latency-bound loops running beside work on other streams, which cannot
 * take the device-wide synchronisation of cudaMalloc/cudaFree.
 * No counterpart in the reference.
 * Inputs are device pointers: the edge list (n_entries entries, ids that index
 * d_part) and the community of each vertex, values in [0, n_comms).  An id
 * outside that range is left out of the sums and the call returns
 * LVG_ERR_INVALID_ARG.  The result goes to the host double *q.  The call
 * allocates nothing: its scratch is a fixed device array of
 * LVG_NOALLOC_SCRATCH_BYTES bytes that every GPU which loads the library holds
 * until the process exits.  n_comms above LVG_NOALLOC_MAX_COMMS returns
 * LVG_ERR_CAPACITY.  The first call on a device looks up the array's device
 * address (cudaGetSymbolAddress), so make it before any stream capture.  All
 * calls share the array and each call clears what it sums into: calls that
 * overlap on the GPU (other streams, other host threads) race and must be
 * serialised by the caller.  The call synchronises `stream` (a cudaStream_t,
 * NULL for the legacy default stream) before it returns the value. */
lvg_status lvg_modularity_fp64_noalloc(const int32_t* d_src, const int32_t* d_dst, const float* d_w,
                                       int64_t n_entries, const int32_t* d_part, int32_t n_comms,
                                       void* stream, double* q);

/* Test hook of the failure paths (no counterpart in the reference, whose
 * sorts are Thrust's and wait on nothing).  The radix sort of the CSR build
 * and the coarsening finds each tile's offsets by decoupled look-back: a tile
 * waits for the counts its predecessors publish, for at most spin_limit polls
 * (default 1 << 22), then sets an error flag and goes on, and the sort returns
 * LVG_ERR_CUDA ("radix sort look-back did not complete") instead of hanging.
 * hold_tile >= 0 makes that tile of every later sort never publish, so the
 * waits of the tiles after it run out; hold_tile = -1 and the default limit
 * restore normal operation.  Process-wide; for tests only. */
lvg_status lvg_debug_radix_hold(int32_t spin_limit, int64_t hold_tile);

/* Bytes of device memory the context holds (arena capacity) and its peak use. */
lvg_status lvg_memory(const lvg_ctx* ctx, int64_t* capacity, int64_t* peak);

/* ------------------------------------------------------------ autotuner ----
 * The move kernels split a pass's vertices into degree classes: rows up to 32
 * entries (thread/lane kernels), up to tile_max_degree (shared-memory tiles),
 * up to block_max_degree (one block and one shared table per vertex) and
 * above (global hub tables).  Which split is fastest depends on the graph's
 * degree distribution and on the GPU.  The reference has fixed launch shapes
 * (<<<N,32>>> per vertex, OneLevelKernel.cu:248-386, and serial chunks for
 * hubs) and no tuner; these entry points have no counterpart in it.
 *
 * The thresholds change which kernel handles a vertex, never a decision: every
 * kernel computes the same FP64 gains with the same tie-break, so any pair
 * gives the same passes, partitions and Q (the tuner checks this on the graph
 * it measures and fails with LVG_ERR_STATE if a candidate disagrees; on any
 * failure the context is left rebuilt at level 0 with the pair it had). */
typedef struct {
  int32_t tile_max_degree;
  int32_t block_max_degree;
  float move_ms;    /* median device time of the move kernels of the hashing
                       passes (every pass after the first) of one level-0
                       one-level phase; < 0: candidate did not fit the arena */
  float build_ms;   /* device time of the level-0 build with these thresholds */
} lvg_tune_point;

typedef struct {
  const int32_t* tile_max_degrees;   /* candidates, each in [32, 512] (NULL: 64, 128, 256, 512) */
  int32_t n_tile;
  const int32_t* block_max_degrees;  /* candidates, each in [32, 8192] (NULL: 1024, 2048, 4096, 8192) */
  int32_t n_block;
  int32_t reps;                      /* timed one-level phases per candidate (<= 0: 3), after one untimed */
  int32_t use_cache;                 /* 1: reuse the pair tuned earlier in this process for a graph of the
                                        same shape class on the same device, without measuring */
} lvg_tune_space;

/* Measure every (tile, block) pair with tile <= block on the loaded level-0
 * graph and keep the fastest: rebuild level 0 with the pair, run one untimed
 * and `reps` timed level-0 one-level phases, and take the median move time of
 * the hashing passes.  Pairs within 2 % of the fastest defer to the context's
 * configured pair when it is among them (lvg_tune_pick).  The chosen pair is
 * then used by every level built afterwards (this graph's later levels,
 * lvg_run, batched runs of this context) and the context is left at level 0,
 * rebuilt, as after a load.  Shape class = (device, floor(log2 V),
 * floor(log2 nnz), floor(log2 max degree), integral weights); the process-wide
 * cache keeps the pair of each class.  points (nullable, cap entries) receives
 * every measured pair in order, *n_points their number (0 on a cache hit);
 * best (nullable) the chosen one.  Costs one level-0 build and reps+1
 * one-level phases per pair. */
lvg_status lvg_autotune(lvg_ctx* ctx, const lvg_tune_space* space, lvg_tune_point* points, int32_t cap,
                        int32_t* n_points, lvg_tune_point* best);

/* The degree thresholds the context builds levels with. */
lvg_status lvg_get_thresholds(const lvg_ctx* ctx, int32_t* tile_max_degree, int32_t* block_max_degree);

/* The tuner's choice among measured points (host only, no device call): the
 * smallest move_ms >= 0; a point equal to (pref_tile, pref_block) wins when
 * within 2 % of it; among equal times the earlier point.  *best_index = -1
 * when no point has move_ms >= 0. */
lvg_status lvg_tune_pick(const lvg_tune_point* points, int32_t n, int32_t pref_tile, int32_t pref_block,
                         int32_t* best_index);

/* Forget every cached pair. */
lvg_status lvg_tune_cache_clear(void);

#ifdef __cplusplus
}
#endif
#endif
