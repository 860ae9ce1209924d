// Louvain hot path kernels for sm_100a.
//
// Layout in HBM (one level):
//   level input list  src/dst int32[E], w float[E]       (the reference's edge list)
//   CSR               off int64[V+1], col int32[nnz], cw float[nnz]
//                     (doubled list, equal (u,v) merged, self loops removed)
//   per vertex        k/kfrac double, loopw float, has_loop u8
//   community state   comm/next int32, tot/in double, size int32, deltas
//                     deltas (tot, in, size: one 32-byte sector per community), cand int32
//
// Every FP64 expression that feeds a decision is written with explicit
// round-to-nearest intrinsics so it rounds exactly as the CPU oracle does.
#include <algorithm>
#include <climits>
#include <mutex>
#include <vector>

#include "louvain.cuh"
#include "prims.cuh"

namespace lvg {

struct HubPartial {
  double g, w;
  int32_t c, n;
};

// Static per-vertex facts of a level, copied in degree-class item order so
// that a class kernel streams them instead of gathering them by vertex id.
struct VInfo {
  double kfrac;
  double k;
  float loopw;
  int32_t vid_loop;   // vertex id << 1 | has_loop
};

namespace {

__device__ __forceinline__ void delta_clear(Delta& d) {
  d.tot = 0.0; d.in = 0.0; d.size = 0; d.out = 0; d.iw_out = 0.0;
}

// Commit of one community's pass deltas (communitySetKernel,
// OneLevelKernel.cu:93-107): tot/in/size move by the deltas, and a vertex
// that left its singleton community takes its degree and weight out of it.
__device__ __forceinline__ void delta_commit(Delta& d, double kc, double& tot, double& in, int32_t& size) {
  double t = tot, x = in;
  if (d.out) { t = __dsub_rn(t, kc); x = __dsub_rn(x, d.iw_out); }
  tot = __dadd_rn(t, d.tot);
  in = __dadd_rn(x, d.in);
  size += d.size - d.out;
  delta_clear(d);
}

constexpr int kThreads = 256;
constexpr int kHubChunk = 4096;
constexpr int kNone = INT_MAX;

// ------------------------------------------------------------------ validate
__global__ void validate_kernel(const int32_t* src, const int32_t* dst, const float* w, int64_t E,
                                int32_t V, uint32_t* bad) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < E; e += (int64_t)gridDim.x * blockDim.x) {
    int32_t a = src[e], b = dst[e];
    float x = w[e];
    if (a < 0 || a >= V || b < 0 || b >= V || !(x >= 0.0f) || isinf(x)) atomicOr(bad, 1u);
  }
}

// ------------------------------------------------------------------ CSR build
// Doubled list D = input ++ reversed(input) (NeighbourCompute.cu:66-68) as
// 64-bit keys (src << B | dst) with the weight as payload.
__global__ void make_keys_kernel(const int32_t* src, const int32_t* dst, const float* w, int64_t E, int B,
                                 uint64_t* keys, float* vals) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < E; e += (int64_t)gridDim.x * blockDim.x) {
    uint64_t a = (uint32_t)src[e], b = (uint32_t)dst[e];
    float x = w[e];
    keys[e] = (a << B) | b;
    vals[e] = x;
    keys[E + e] = (b << B) | a;
    vals[E + e] = x;
  }
}

// Segmented inclusive warp sum over contiguous runs of equal `seg`.
template <typename K>
__device__ __forceinline__ double seg_warp_sum(double v, K seg) {
  const unsigned full = 0xffffffffu;
  int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    double u = __shfl_up_sync(full, v, o);
    K t = __shfl_up_sync(full, seg, o);
    if (lane >= o && t == seg) v = __dadd_rn(v, u);
  }
  return v;
}

template <typename K>
__device__ __forceinline__ bool seg_warp_last(K seg, bool valid) {
  const unsigned full = 0xffffffffu;
  int lane = threadIdx.x & 31;
  K nx = __shfl_down_sync(full, seg, 1);
  bool nvalid = __shfl_down_sync(full, valid, 1);
  return valid && (lane == 31 || !nvalid || nx != seg);
}

// Per sorted entry: CSR heads, row counts, degree (InitKernel.cu:154-179:
// weight 0 counts 1, a self loop counts twice), last self-loop weight
// (InitKernel.cu:181-194).  Grid covers n exactly in whole warps.
__global__ void csr_scan_kernel(const uint64_t* keys, const float* vals, int64_t n, int B, uint32_t* head,
                                int64_t* rowcnt, double* k, float* loopw, uint8_t* has_loop) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  bool valid = i < n;
  uint64_t mask = (B >= 64) ? ~0ull : ((1ull << B) - 1);
  uint64_t key = valid ? keys[i] : 0ull;
  int64_t row = valid ? (int64_t)(key >> B) : -1;
  uint64_t c = key & mask;
  bool loop = valid && (uint64_t)row == c;
  float x = valid ? vals[i] : 0.0f;
  bool first = valid && (i == 0 || keys[i - 1] != key);
  bool last = valid && (i == n - 1 || keys[i + 1] != key);
  bool h = first && !loop;
  if (valid) head[i] = h ? 1u : 0u;
  if (h) atomicAdd((unsigned long long*)&rowcnt[row], 1ull);
  if (loop && last) { loopw[row] = x; has_loop[row] = 1; }
  float dv = x == 0.0f ? 1.0f : x;
  if (loop) dv *= 2.0f;
  double s = seg_warp_sum<int64_t>(valid ? (double)dv : 0.0, row);
  if (seg_warp_last<int64_t>(row, valid)) atomicAdd(&k[row], s);
}

// CSR column and merged weight of every (u,v), u != v.
__global__ void csr_emit_kernel(const uint64_t* keys, const float* vals, int64_t n, int B, const uint32_t* pos,
                                const uint32_t* head, int32_t* col, double* wsum) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  bool valid = i < n;
  uint64_t mask = (B >= 64) ? ~0ull : ((1ull << B) - 1);
  uint64_t key = valid ? keys[i] : 0ull;
  uint64_t row = key >> B, c = key & mask;
  bool loop = row == c;
  int64_t r = (valid && !loop) ? (int64_t)pos[i] + (int64_t)head[i] - 1 : -1;
  if (valid && head[i]) col[r] = (int32_t)c;
  double s = seg_warp_sum<int64_t>(valid && !loop ? (double)vals[i] : 0.0, r);
  if (seg_warp_last<int64_t>(r, valid) && r >= 0) atomicAdd(&wsum[r], s);
}

// Sort-free build: a level list that is strictly sorted by (src, dst) and
// symmetric with bitwise-equal weights doubles into each entry twice, so the
// merged CSR row of u is its list row without the self loop, weights 2w.
// Entries per row; runs of equal rows inside a warp add once.  Grid covers E
// in whole warps.
__global__ void row_count_kernel(const int32_t* src, int64_t E, int64_t* rowcnt) {
  int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  bool valid = e < E;
  int64_t u = valid ? src[e] : -1;
  double n = seg_warp_sum<int64_t>(valid ? 1.0 : 0.0, u);
  if (seg_warp_last<int64_t>(u, valid)) atomicAdd((unsigned long long*)&rowcnt[u], (unsigned long long)n);
}

enum : uint32_t { kNotSorted = 1u, kNotSymmetric = 2u, kBadEntry = 4u };

// Sortedness (exact) and symmetry of the list in one coalesced pass.  The
// symmetry test compares order-free fingerprints: the sums mod 2^64 of two
// independent 64-bit hashes of (src, dst, weight bits) over the non-loop
// entries against the same sums of (dst, src, weight bits).  A strictly sorted
// list has no repeated entry, so the sums agree when the list equals its
// transpose; a list that is not symmetric passes only on a 128-bit collision.
__device__ __forceinline__ uint64_t edge_hash(uint32_t u, uint32_t v, uint32_t wb, uint64_t key) {
  return mix64(mix64((((uint64_t)u << 32) | v) ^ key) + (uint64_t)wb * 0x9E3779B97F4A7C15ull + key);
}

__global__ void list_check_kernel(const int32_t* src, const int32_t* dst, const float* w, int64_t E,
                                  uint32_t* flags, unsigned long long* sums) {
  const uint64_t K1 = 0x243F6A8885A308D3ull, K2 = 0x13198A2E03707344ull;
  uint64_t d1 = 0, d2 = 0;
  bool unsorted = false;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < E; e += (int64_t)gridDim.x * blockDim.x) {
    const int32_t u = src[e], v = dst[e];
    if (e + 1 < E) {
      const int32_t u2 = src[e + 1], v2 = dst[e + 1];
      if (!(u2 > u || (u2 == u && v2 > v))) unsorted = true;
    }
    if (u != v) {
      const uint32_t wb = __float_as_uint(w[e]);
      d1 += edge_hash((uint32_t)u, (uint32_t)v, wb, K1) - edge_hash((uint32_t)v, (uint32_t)u, wb, K1);
      d2 += edge_hash((uint32_t)u, (uint32_t)v, wb, K2) - edge_hash((uint32_t)v, (uint32_t)u, wb, K2);
    }
  }
  const unsigned full = 0xffffffffu;
#pragma unroll
  for (int o = 16; o >= 1; o >>= 1) {
    d1 += __shfl_down_sync(full, d1, o);
    d2 += __shfl_down_sync(full, d2, o);
  }
  const bool any_unsorted = __any_sync(full, unsorted);
  if ((threadIdx.x & 31) == 0) {
    if (d1) atomicAdd(&sums[0], (unsigned long long)d1);
    if (d2) atomicAdd(&sums[1], (unsigned long long)d2);
    if (any_unsorted) atomicOr(flags, kNotSorted);
  }
}

__global__ void nonloop_flag_kernel(const int32_t* src, const int32_t* dst, int64_t E, uint32_t* flag) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < E; e += (int64_t)gridDim.x * blockDim.x)
    flag[e] = src[e] != dst[e] ? 1u : 0u;
}

__global__ void csr_fast_emit_kernel(const int32_t* src, const int32_t* dst, const float* w, int64_t E,
                                     const uint32_t* pos, int32_t* col, float* cw, double* k, float* loopw,
                                     uint8_t* has_loop) {
  int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  bool valid = e < E;
  int64_t u = valid ? src[e] : -1;
  int32_t v = valid ? dst[e] : -1;
  float x = valid ? w[e] : 0.0f;
  bool loop = valid && u == v;
  if (valid && !loop) {
    uint32_t p = pos[e];
    col[p] = v;
    cw[p] = __double2float_rn(__dadd_rn((double)x, (double)x));
  }
  if (loop) { loopw[u] = x; has_loop[u] = 1; }
  float f = x == 0.0f ? 1.0f : x;             // InitKernel.cu:165-170, both copies of the entry
  if (loop) f *= 2.0f;
  double dv = valid ? __dadd_rn((double)f, (double)f) : 0.0;
  double sum = seg_warp_sum<int64_t>(dv, u);
  if (seg_warp_last<int64_t>(u, valid)) atomicAdd(&k[u], sum);
}

// ---------------------------------------------------------- streamed level-0 build
// The checks and CSR build of a list that arrives from the host chunk by
// chunk, each chunk processed while later ones are still being copied.  The
// CSR is the one build_csr_fast makes; it is kept only if the whole list
// turns out strictly sorted and symmetric.

__device__ __forceinline__ bool entry_ok(int32_t u, int32_t v, float x, int32_t V) {
  return u >= 0 && u < V && v >= 0 && v < V && x >= 0.0f && !isinf(x);   // as validate_kernel
}

// One chunk [b, e_end): range/weight check, strict order against the previous
// entry, the symmetry fingerprints of list_check_kernel, per-row counts of
// non-loop entries (into cnt) and the chunk's non-loop flags (pos[b..e_end),
// scanned next).  Grid covers the chunk in whole warps.
__global__ void pre_chunk_kernel(const int32_t* src, const int32_t* dst, const float* w, int64_t b, int64_t e_end,
                                 int32_t V, uint32_t* flags, unsigned long long* sums, unsigned long long* cnt,
                                 uint32_t* pos) {
  const uint64_t K1 = 0x243F6A8885A308D3ull, K2 = 0x13198A2E03707344ull;   // as list_check_kernel
  const unsigned full = 0xffffffffu;
  const int64_t e = b + blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const bool in = e < e_end;
  const int32_t u = in ? src[e] : 0, v = in ? dst[e] : 0;
  const float x = in ? w[e] : 0.0f;
  const bool ok = in && entry_ok(u, v, x, V);
  bool unsorted = false;
  if (in && e > 0) {
    const int32_t u0 = src[e - 1], v0 = dst[e - 1];
    unsorted = !(u > u0 || (u == u0 && v > v0));
  }
  uint64_t d1 = 0, d2 = 0;
  if (ok && u != v) {
    const uint32_t wb = __float_as_uint(x);
    d1 = edge_hash((uint32_t)u, (uint32_t)v, wb, K1) - edge_hash((uint32_t)v, (uint32_t)u, wb, K1);
    d2 = edge_hash((uint32_t)u, (uint32_t)v, wb, K2) - edge_hash((uint32_t)v, (uint32_t)u, wb, K2);
  }
  if (in) pos[e] = (ok && u != v) ? 1u : 0u;
  const int64_t key = ok ? (int64_t)u : -1;
  const double n = seg_warp_sum<int64_t>((ok && u != v) ? 1.0 : 0.0, key);
  if (seg_warp_last<int64_t>(key, ok) && n > 0.0) atomicAdd(&cnt[u], (unsigned long long)n);
#pragma unroll
  for (int o = 16; o >= 1; o >>= 1) {
    d1 += __shfl_down_sync(full, d1, o);
    d2 += __shfl_down_sync(full, d2, o);
  }
  const bool any_bad = __any_sync(full, in && !ok), any_unsorted = __any_sync(full, unsorted);
  if ((threadIdx.x & 31) == 0) {
    if (d1) atomicAdd(&sums[0], (unsigned long long)d1);
    if (d2) atomicAdd(&sums[1], (unsigned long long)d2);
    if (any_unsorted) atomicOr(flags, kNotSorted);
    if (any_bad) atomicOr(flags, kBadEntry);
  }
}

// carry[i + 1] = carry[i] + (non-loop entries of chunk i)
__global__ void pre_carry_kernel(uint32_t* carry, int64_t i, const uint32_t* chunk_total) {
  carry[i + 1] = carry[i] + *chunk_total;
}

// The chunk's CSR entries, degrees and self loops, as csr_fast_emit_kernel
// does for the whole list (positions: chunk scan + carry).  Entries that
// failed the checks are skipped.  Grid covers the chunk in whole warps.
__global__ void pre_emit_kernel(const int32_t* src, const int32_t* dst, const float* w, int64_t b, int64_t e_end,
                                int32_t V, const uint32_t* pos, const uint32_t* carry, int32_t* col, float* cw,
                                double* k, float* loopw, uint8_t* has_loop) {
  const int64_t e = b + blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const bool in = e < e_end;
  const int32_t u = in ? src[e] : 0, v = in ? dst[e] : 0;
  const float x = in ? w[e] : 0.0f;
  const bool ok = in && entry_ok(u, v, x, V);
  const bool loop = ok && u == v;
  if (ok && !loop) {
    const uint32_t p = pos[e] + *carry;
    col[p] = v;
    cw[p] = __double2float_rn(__dadd_rn((double)x, (double)x));
  }
  if (loop) { loopw[u] = x; has_loop[u] = 1; }
  float f = x == 0.0f ? 1.0f : x;             // InitKernel.cu:165-170, both copies of the entry
  if (loop) f *= 2.0f;
  const double dv = ok ? __dadd_rn((double)f, (double)f) : 0.0;
  const int64_t key = ok ? (int64_t)u : -1;
  const double sum = seg_warp_sum<int64_t>(dv, key);
  if (seg_warp_last<int64_t>(key, ok)) atomicAdd(&k[u], sum);
}

// Group partials of the fixed-tree sum of the weights (as tree_sum_f32's
// first round; group b of the chunk starting at x).
__global__ void __launch_bounds__(kRedThreads) pre_group_kernel(const float* x, int64_t n, double* out) {
  __shared__ double ws[8];
  const int64_t b = blockIdx.x;
  int64_t len = n - b * kGroup;
  if (len > kGroup) len = kGroup;
  const double r = group_sum_block<float>(x + b * kGroup, len, ws);
  if (threadIdx.x == 0) out[b] = r;
}

__global__ void row_off_kernel(const int64_t* rowstart, const uint32_t* pos, int32_t V, int64_t* off) {
  for (int64_t u = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; u <= V; u += (int64_t)gridDim.x * blockDim.x)
    off[u] = pos[rowstart[u]];
}

__global__ void to_float_kernel(const double* x, float* y, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    y[i] = __double2float_rn(x[i]);
}

// ------------------------------------------------------------------ buckets
// Degree classes: 1-4, 5-8, 9-16, 17-32 lanes per vertex (group kernels),
// 33..tile_max (tiles), ..block_max (block per vertex), above (hubs).
__device__ __forceinline__ int bucket_of(int32_t i, const int64_t* off, const double* k, int32_t tmax,
                                         int32_t bmax) {
  if (!(k[i] > 0.0)) return kNumBuckets;  // no entry in the doubled list: never moves
  int64_t d = off[i + 1] - off[i];
  if (d <= 4) return kB4;
  if (d <= 8) return kB8;
  if (d <= 16) return kB16;
  if (d <= 32) return kB32;
  if (d <= tmax) return kBTile;
  return d <= bmax ? kBBlock : kBHub;
}

__global__ void __launch_bounds__(kThreads) bucket_count_kernel(int32_t V, const int64_t* off, const double* k,
                                                                int32_t tmax, int32_t bmax, uint32_t* cnt,
                                                                int64_t nblk) {
  uint32_t c[kNumBuckets] = {};
  int64_t base = (int64_t)blockIdx.x * 2048 + (int64_t)threadIdx.x * 8;
  for (int j = 0; j < 8; ++j) {
    int64_t i = base + j;
    if (i < V) {
      int b = bucket_of((int32_t)i, off, k, tmax, bmax);
      if (b < kNumBuckets) c[b]++;
    }
  }
  for (int b = 0; b < kNumBuckets; ++b) {
    uint32_t tot;
    block_exclusive_scan256<uint32_t>(c[b], &tot);
    if (threadIdx.x == 0) cnt[b * nblk + blockIdx.x] = tot;
  }
}

__global__ void __launch_bounds__(kThreads) bucket_scatter_kernel(int32_t V, const int64_t* off, const double* k,
                                                                  int32_t tmax, int32_t bmax,
                                                                  const uint32_t* offs, int64_t nblk,
                                                                  int32_t* list) {
  int64_t base = (int64_t)blockIdx.x * 2048 + (int64_t)threadIdx.x * 8;
  int8_t bid[8];
  uint32_t c[kNumBuckets] = {};
  for (int j = 0; j < 8; ++j) {
    int64_t i = base + j;
    bid[j] = i < V ? (int8_t)bucket_of((int32_t)i, off, k, tmax, bmax) : (int8_t)kNumBuckets;
    if (bid[j] < kNumBuckets) c[bid[j]]++;
  }
  uint32_t pre[kNumBuckets];
  for (int b = 0; b < kNumBuckets; ++b) {
    uint32_t tot;
    pre[b] = block_exclusive_scan256<uint32_t>(c[b], &tot) + offs[b * nblk + blockIdx.x];
  }
  for (int j = 0; j < 8; ++j) {
    int b = bid[j];
    if (b < kNumBuckets) list[pre[b]++] = (int32_t)(base + j);
  }
}

__global__ void hub_info_kernel(const int32_t* hubs, int64_t nhub, const int64_t* off, int64_t* beg_end) {
  int64_t h = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (h < nhub) {
    int32_t i = hubs[h];
    beg_end[2 * h] = off[i];
    beg_end[2 * h + 1] = off[i + 1];
  }
}

// ------------------------------------------------------------------ state
__global__ void init_state_kernel(int32_t V, const double* k, const float* loopw, double m, double* kfrac,
                                  int32_t* comm, int32_t* next, double* tot, double* in, int32_t* size,
                                  Delta* delta, int32_t* cand) {
  double twom = __dmul_rn(2.0, m);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < V; i += (int64_t)gridDim.x * blockDim.x) {
    comm[i] = (int32_t)i;                 // InitKernel.cu:213-215
    next[i] = (int32_t)i;
    tot[i] = k[i];                        // InitKernel.cu:236
    in[i] = (double)loopw[i];             // InitKernel.cu:242
    size[i] = 1;                          // OneLevelKernel.cu:87
    delta_clear(delta[i]);
    cand[i] = -1;
    kfrac[i] = m > 0.0 ? __ddiv_rn(k[i], twom) : 0.0;  // OneLevelKernel.cu:307
  }
}

struct MoveArgs {
  const int32_t* list;
  int64_t n;
  const int64_t* off;
  const int32_t* col;
  const float* cw;
  const int32_t* comm;
  const double* tot;
  const int32_t* size;
  const double* kfrac;
  const double* k;
  const float* loopw;
  const uint8_t* has_loop;
  int32_t* next;
  int32_t* cand;
  Delta* delta;
  PassCtl* ctl;
  const int32_t* k32;    // degrees as int32 (integral weights), else nullptr: the singleton tot
  const int32_t* gid;    // batched runs: graph of each vertex (nullptr for one graph)
  const int32_t* gdone;  // batched runs: 1 once a graph's level loop has stopped
  unsigned long long* queue;   // batched runs: work counter of this launch (nullptr: grid-stride)
};

// Work items of the block-per-item kernels (block, tile and hub-bucket
// classes).  Without a queue (one graph) a block takes items blockIdx.x,
// blockIdx.x + gridDim.x, ...  With one (batched runs, whose graphs and rows
// are of very uneven sizes) the blocks are persistent and pull kQueueGrab
// consecutive items at a time from a device counter, so that a block that
// finishes early takes more.  Every thread of the block calls these; the
// decisions are the same whichever block takes an item.
constexpr int kQueueGrab = 8;
struct WorkQueue {
  int64_t base, end;
};
__device__ __forceinline__ int64_t work_take(unsigned long long* q, WorkQueue& w) {
  __syncthreads();
  if (threadIdx.x == 0) {
    w.base = (int64_t)atomicAdd(q, (unsigned long long)kQueueGrab);
    w.end = w.base + kQueueGrab;
  }
  __syncthreads();
  return w.base;
}
__device__ __forceinline__ int64_t work_begin(unsigned long long* q, WorkQueue& w) {
  return q ? work_take(q, w) : (int64_t)blockIdx.x;
}
__device__ __forceinline__ int64_t work_advance(unsigned long long* q, int64_t item, WorkQueue& w) {
  if (!q) return item + gridDim.x;
  return item + 1 < w.end ? item + 1 : work_take(q, w);
}

// Candidate order: higher gain first, then lower community id
// (OneLevelKernel.cu:330,358).  Only strictly positive gains are candidates.
__device__ __forceinline__ bool better(double g2, int32_t c2, double g1, int32_t c1) {
  return g2 > g1 || (g2 == g1 && c2 < c1);
}


__device__ __forceinline__ void warp_best(double& bg, int32_t& bc, double& bw) {
  const unsigned full = 0xffffffffu;
#pragma unroll
  for (int o = 16; o >= 1; o >>= 1) {
    double g = __shfl_xor_sync(full, bg, o);
    int32_t c = __shfl_xor_sync(full, bc, o);
    double w = __shfl_xor_sync(full, bw, o);
    if (better(g, c, bg, bc)) { bg = g; bc = c; bw = w; }
  }
}

// remove/insert (OneLevelKernel.cu:52-78) of a vertex of degree ki moving
// with weight iw from community own to best.  SINGLETON: own holds only this
// vertex, so its side is two plain stores the commit applies.
template <bool SINGLETON>
__device__ __forceinline__ void move_deltas(Delta* d, int32_t own, int32_t best, double ki, double iw) {
  if (SINGLETON) {
    d[own].out = 1;
    d[own].iw_out = iw;
  } else {
    atomicAdd(&d[own].tot, -ki);
    atomicAdd(&d[own].in, -iw);
    atomicAdd(&d[own].size, -1);
  }
  atomicAdd(&d[best].tot, ki);
  atomicAdd(&d[best].in, iw);
  atomicAdd(&d[best].size, 1);
}

// The decision for one vertex from its best candidate: singleton-pair rule
// (OneLevelKernel.cu:407-410), remove/insert into the delta buffers
// (OneLevelKernel.cu:52-78, 412-421) and the isolated-merge candidate
// (OneLevelKernel.cu:142-169).
// SINGLETON: the state is the level's initial one (every community a single
// vertex), so both sizes are 1 without reading them.
template <bool SINGLETON = false>
__device__ __forceinline__ void apply_decision_kl(const MoveArgs& P, int32_t i, int32_t own, int32_t bc, double bw,
                                                  int32_t nseg, double ki, float loopw) {
  if (P.gdone && P.gdone[P.gid[i]]) return;   // that graph's pass loop has stopped
  int32_t raw = bc == kNone ? own : bc;
  int32_t so = SINGLETON ? 1 : P.size[own], sb = SINGLETON ? 1 : P.size[raw];
  int32_t best = raw;
  if (so == 1 && sb == 1 && raw > own) best = own;
  P.next[i] = best;
  P.cand[i] = (so == 1 && nseg == 1 && raw != own && own < raw) ? raw : -1;
  if (best != own) move_deltas<SINGLETON>(P.delta, own, best, ki, __dadd_rn(bw, (double)loopw));
}

template <bool SINGLETON = false>
__device__ __forceinline__ void apply_decision(const MoveArgs& P, int32_t i, int32_t own, int32_t bc, double bw,
                                               int32_t nseg) {
  if (P.gdone && P.gdone[P.gid[i]]) return;   // that graph's pass loop has stopped
  int32_t raw = bc == kNone ? own : bc;
  int32_t so = SINGLETON ? 1 : P.size[own], sb = SINGLETON ? 1 : P.size[raw];
  int32_t best = raw;
  if (so == 1 && sb == 1 && raw > own) best = own;
  P.next[i] = best;
  P.cand[i] = (so == 1 && nseg == 1 && raw != own && own < raw) ? raw : -1;
  if (best != own) move_deltas<SINGLETON>(P.delta, own, best, P.k[i], __dadd_rn(bw, (double)P.loopw[i]));
}

// Packed (community << 32 | integer sum) slots are all ones when empty; the
// add of an integral weight cannot carry into the key (sums stay below 2^30).
constexpr unsigned long long kPackedEmpty = ~0ull;

__device__ __forceinline__ uint32_t hash_c(int32_t c, int logT) {
  return (uint32_t)(((uint64_t)(uint32_t)c * 0x9E3779B97F4A7C15ull) >> (64 - logT));
}

__device__ __forceinline__ int ceil_log2(int64_t x) {  // x >= 1
  return x <= 1 ? 0 : 64 - __clzll((unsigned long long)(x - 1));
}

// Open-addressing insert of (c, w) into a table of 2^logT slots.
template <typename Acc>
__device__ __forceinline__ bool table_insert(int32_t* keys, Acc* vals, int logT, int32_t c, Acc w) {
  uint32_t T = 1u << logT;
  uint32_t h = hash_c(c, logT);
  for (uint32_t p = 0; p < T; ++p) {
    int32_t prev = atomicCAS(&keys[h], -1, c);
    if (prev == -1 || prev == c) { atomicAdd(&vals[h], w); return true; }
    h = (h + 1) & (T - 1);
  }
  return false;
}

// Entries [e0 + u*stride) of a row, u < 4: columns and weights first, then
// the four community gathers, so that each thread keeps several loads in
// flight; kNone marks entries past `end`.
constexpr int kUnroll = 4;
__device__ __forceinline__ void gather4(const MoveArgs& P, int64_t e0, int64_t stride, int64_t end,
                                        int32_t (&c)[kUnroll], float (&w)[kUnroll]) {
  int32_t col[kUnroll];
#pragma unroll
  for (int u = 0; u < kUnroll; ++u) {
    const int64_t e = e0 + u * stride;
    col[u] = e < end ? __ldcs(P.col + e) : -1;
    w[u] = e < end ? __ldcs(P.cw + e) : 0.0f;
  }
#pragma unroll
  for (int u = 0; u < kUnroll; ++u) c[u] = col[u] >= 0 ? P.comm[col[u]] : kNone;
}

// Block per vertex for the block class (tile_max < degree <= block_max),
// launched once per degree band (dlo, dhi] with a shared table of
// 2^maxLog >= 2 dhi slots: the narrow bands of low degrees take small tables
// and NT = 128 threads, so that many blocks fit on an SM; int32 sums when
// the weights are integral (exact, half the table bytes).
template <typename Acc, int NT>
__global__ void __launch_bounds__(NT) move_block_kernel(MoveArgs P, int maxLog, int64_t dlo, int64_t dhi) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ double rg[NT / 32], rw[NT / 32];
  __shared__ int32_t rc[NT / 32], rn[NT / 32], rs[NT / 32];
  if (P.ctl->done) return;
  const int Tmax = 1 << maxLog;
  Acc* vals = reinterpret_cast<Acc*>(smem);
  int32_t* keys = reinterpret_cast<int32_t*>(vals + Tmax);
  int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int s = threadIdx.x; s < Tmax; s += NT) { keys[s] = -1; vals[s] = Acc(0); }
  __syncthreads();
  bool overflow = false;
  __shared__ WorkQueue wq;
  for (int64_t item = work_begin(P.queue, wq); item < P.n; item = work_advance(P.queue, item, wq)) {
    int32_t i = P.list[item];
    int64_t beg = P.off[i], end = P.off[i + 1];
    if (end - beg <= dlo || end - beg > dhi) continue;   // another band takes this degree
    int32_t own = P.comm[i];
    int logT = min(maxLog, max(5, ceil_log2(2 * (end - beg))));
    int T = 1 << logT;
    bool sawown = false;
    for (int64_t e0 = beg + threadIdx.x; e0 < end; e0 += kUnroll * NT) {
      int32_t c[kUnroll];
      float wv[kUnroll];
      gather4(P, e0, NT, end, c, wv);
#pragma unroll
      for (int u = 0; u < kUnroll; ++u) {
        if (c[u] != kNone) {
          sawown |= (c[u] == own);
          if (!table_insert<Acc>(keys, vals, logT, c[u], (Acc)wv[u])) overflow = true;
        }
      }
    }
    __syncthreads();
    double kf = P.kfrac[i];
    double bg = 0.0, bw = 0.0;
    int32_t bc = kNone;
    int nocc = 0;
    for (int s0 = threadIdx.x; s0 < T; s0 += kUnroll * NT) {
      int32_t c[kUnroll];
      double W[kUnroll], t[kUnroll];
#pragma unroll
      for (int u = 0; u < kUnroll; ++u) {
        const int s = s0 + u * NT;
        c[u] = s < T ? keys[s] : -1;
        W[u] = c[u] >= 0 ? (double)vals[s] : 0.0;
        if (c[u] >= 0) { keys[s] = -1; vals[s] = Acc(0); }
      }
#pragma unroll
      for (int u = 0; u < kUnroll; ++u) t[u] = (c[u] >= 0 && W[u] != 0.0) ? P.tot[c[u]] : 0.0;
#pragma unroll
      for (int u = 0; u < kUnroll; ++u) {
        if (c[u] >= 0) {
          ++nocc;
          if (W[u] != 0.0) {                                            // OneLevelKernel.cu:303
            const double g = __dsub_rn(W[u], __dmul_rn(t[u], kf));      // OneLevelKernel.cu:307-313
            if (g > 0.0 && better(g, c[u], bg, bc)) { bg = g; bc = c[u]; bw = W[u]; }
          }
        }
      }
    }
    warp_best(bg, bc, bw);
    nocc = __reduce_add_sync(0xffffffffu, (unsigned)nocc);
    int so = __any_sync(0xffffffffu, sawown) ? 1 : 0;
    if (lane == 0) { rg[w] = bg; rc[w] = bc; rw[w] = bw; rn[w] = nocc; rs[w] = so; }
    __syncthreads();
    if (threadIdx.x == 0) {
      double g = rg[0], ww = rw[0];
      int32_t c = rc[0];
      int n = rn[0], sw = rs[0];
      for (int k2 = 1; k2 < NT / 32; ++k2) {
        if (better(rg[k2], rc[k2], g, c)) { g = rg[k2]; c = rc[k2]; ww = rw[k2]; }
        n += rn[k2];
        sw |= rs[k2];
      }
      int32_t nseg = n + ((P.has_loop[i] && !sw) ? 1 : 0);
      apply_decision(P, i, own, c, ww, nseg);
    }
    __syncthreads();
  }
  if (__syncthreads_or(overflow) && threadIdx.x == 0) atomicOr(&P.ctl->err, kErrProbe);
}

// ----------------------------------------------------------------- ELL kernels
// Degree <= 32: vertices of class D (4, 8, 16, 32) keep their entries in a
// sliced-ELL copy of the CSR built once per level: vertex j of the class owns
// slots [j*D, j*D+D), padding holds column -1.
struct EllArgs {
  const int32_t* col;   // [n * G] neighbour of each slot, -1 for padding
  const float* w;       // [n * G]
  const int32_t* list;  // [n] vertex of each item
  const VInfo* info;    // [n] static facts of each item's vertex, in item order
  int64_t n;
};

// One thread per vertex.  The thread loads its ELL row with
// 16-byte loads, gathers the neighbour communities, sorts the (community,
// weight) pairs in registers with a bitonic network and walks them once in
// ascending order: equal communities are adjacent, so each run gives one
// candidate's summed weight, and keeping only strictly larger gains leaves
// the lowest community among equal gains (OneLevelKernel.cu:330,358).
template <int D>
__device__ __forceinline__ void cas_pair(int32_t (&c)[D], float (&w)[D], int a, int b) {
  int32_t ca = c[a], cb = c[b];
  bool sw = ca > cb;
  float wa = w[a], wb = w[b];
  c[a] = sw ? cb : ca; c[b] = sw ? ca : cb;
  w[a] = sw ? wb : wa; w[b] = sw ? wa : wb;
}

template <int D>
__device__ __forceinline__ void bitonic_sort(int32_t (&c)[D], float (&w)[D]) {
#pragma unroll
  for (int k = 2; k <= D; k <<= 1) {
#pragma unroll
    for (int j = k >> 1; j > 0; j >>= 1) {
#pragma unroll
      for (int x = 0; x < D; ++x) {
        int y = x ^ j;
        if (y > x) {
          if ((x & k) == 0) cas_pair<D>(c, w, x, y);
          else cas_pair<D>(c, w, y, x);
        }
      }
    }
  }
}

template <int D>
__global__ void __launch_bounds__(kThreads) move_thread_kernel(MoveArgs P, EllArgs L) {
  if (P.ctl->done) return;
  for (int64_t j = blockIdx.x * (int64_t)kThreads + threadIdx.x; j < L.n; j += (int64_t)gridDim.x * kThreads) {
    int32_t c[D];
    float w[D];
    const int4* cp = reinterpret_cast<const int4*>(L.col + j * D);
    const float4* wp = reinterpret_cast<const float4*>(L.w + j * D);
#pragma unroll
    for (int q = 0; q < D / 4; ++q) {
      int4 a = __ldcs(cp + q);          // streamed once per pass: evict first
      float4 b = __ldcs(wp + q);
      c[4 * q] = a.x; c[4 * q + 1] = a.y; c[4 * q + 2] = a.z; c[4 * q + 3] = a.w;
      w[4 * q] = b.x; w[4 * q + 1] = b.y; w[4 * q + 2] = b.z; w[4 * q + 3] = b.w;
    }
    const VInfo vi = L.info[j];
    const int32_t i = vi.vid_loop >> 1;
#pragma unroll
    for (int q = 0; q < D; ++q) c[q] = c[q] >= 0 ? P.comm[c[q]] : kNone;
    const int32_t own = P.comm[i];
    const double kf = vi.kfrac;
    bitonic_sort<D>(c, w);
    double bg = 0.0, bw = 0.0, run = 0.0;
    int32_t bc = kNone;
    int nseg = 0;
    bool sawown = false;
#pragma unroll
    for (int q = 0; q < D; ++q) {
      const bool ok = c[q] != kNone;
      const bool head = ok && (q == 0 || c[q] != c[q - 1]);
      const bool tail = ok && (q == D - 1 || c[q + 1] != c[q]);
      run = head ? (double)w[q] : __dadd_rn(run, (double)w[q]);
      nseg += head ? 1 : 0;
      sawown |= ok && c[q] == own;
      if (tail && run != 0.0) {                                  // OneLevelKernel.cu:303
        double g = __dsub_rn(run, __dmul_rn(P.tot[c[q]], kf));   // OneLevelKernel.cu:307-313
        if (g > 0.0 && g > bg) { bg = g; bc = c[q]; bw = run; }
      }
    }
    nseg += ((vi.vid_loop & 1) && !sawown) ? 1 : 0;
    apply_decision_kl(P, i, own, bc, bw, nseg, vi.k, vi.loopw);
  }
}

// ------------------------------------------------------- singleton first pass
// The first pass of every level starts from singletons (comm[i] = i,
// tot[i] = k[i], size[i] = 1: InitKernel.cu:213-236, OneLevelKernel.cu:87).
// Then every neighbour is its own candidate community with W = w(i,j) (the
// CSR has one entry per neighbour), own is never a neighbour, and the number
// of distinct neighbour communities is the degree (+1 for a self loop).  The
// best candidate is a plain argmax over the row -- higher gain, then lower
// community -- which splits into independent pieces: no tables, no
// community gather.  Decisions are the general kernels' bit for bit.
template <int D>
__global__ void __launch_bounds__(kThreads) sp_thread_kernel(MoveArgs P, EllArgs L) {
  // D lanes per vertex: lane s of a segment takes ELL slot s (coalesced row
  // loads, one gather per lane, all in flight together), then a segment argmax.
  if (P.ctl->done) return;
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31, sl = lane % D;
  const int64_t per_warp = 32 / D;
  const int64_t nwarps = (int64_t)gridDim.x * (kThreads / 32);
  const int64_t ngroups = (L.n + per_warp - 1) / per_warp;
  for (int64_t grp = blockIdx.x * (int64_t)(kThreads / 32) + (threadIdx.x >> 5); grp < ngroups; grp += nwarps) {
    const int64_t j = grp * per_warp + lane / D;             // item of this lane's segment
    const bool ok = j < L.n;
    const int32_t c = ok ? __ldcs(L.col + j * D + sl) : -1;
    const float wv = ok ? __ldcs(L.w + j * D + sl) : 0.0f;
    const double kf = ok ? L.info[j].kfrac : 0.0;
    const double t = c < 0 ? 0.0 : (P.k32 ? (double)P.k32[c] : P.tot[c]);   // singleton tot = k
    double bg = 0.0, bw = 0.0;
    int32_t bc = kNone;
    const double W = (double)wv;
    if (c >= 0 && W != 0.0) {                                       // OneLevelKernel.cu:303
      const double g = __dsub_rn(W, __dmul_rn(t, kf));              // OneLevelKernel.cu:307-313
      if (g > 0.0) { bg = g; bc = c; bw = W; }
    }
#pragma unroll
    for (int o = D / 2; o >= 1; o >>= 1) {                          // argmax inside the segment
      const double g2 = __shfl_xor_sync(full, bg, o);
      const int32_t c2 = __shfl_xor_sync(full, bc, o);
      const double w2 = __shfl_xor_sync(full, bw, o);
      if (better(g2, c2, bg, bc)) { bg = g2; bc = c2; bw = w2; }
    }
    const unsigned valid = __ballot_sync(full, c >= 0);
    if (ok && sl == 0) {
      const unsigned seg = (D == 32) ? valid : ((valid >> (lane & ~(D - 1))) & ((1u << D) - 1u));
      const VInfo vi = L.info[j];
      const int32_t i = vi.vid_loop >> 1;
      apply_decision_kl<true>(P, i, i, bc, bw, __popc(seg) + (vi.vid_loop & 1), vi.k, vi.loopw);
    }
  }
}

// Rows longer than 32: warp-sized chunks of kSpChunk entries.  A row of one
// chunk is decided by its warp; longer rows leave a partial per chunk for
// sp_combine_kernel.
constexpr int kSpChunk = 512;
constexpr int kSpUnroll = 4;     // entries per lane in flight

__global__ void __launch_bounds__(kThreads) sp_chunk_kernel(MoveArgs P, const int2* chunks, int64_t nch,
                                                            HubPartial* part) {
  if (P.ctl->done) return;
  const int lane = threadIdx.x & 31;
  const int64_t nwarps = (int64_t)gridDim.x * (kThreads / 32);
  for (int64_t q = blockIdx.x * (int64_t)(kThreads / 32) + (threadIdx.x >> 5); q < nch; q += nwarps) {
    const int2 ch = chunks[q];
    const int32_t i = ch.x;
    const int64_t row = P.off[i], deg = P.off[i + 1] - row;
    const int64_t beg = row + (int64_t)ch.y * kSpChunk;
    const int64_t end = min(beg + (int64_t)kSpChunk, row + deg);
    const double kf = P.kfrac[i];
    double bg = 0.0, bw = 0.0;
    int32_t bc = kNone;
    for (int64_t e0 = beg; e0 < end; e0 += kSpUnroll * 32) {
      int32_t c[kSpUnroll];
      float w[kSpUnroll];
      double t[kSpUnroll];
#pragma unroll
      for (int u = 0; u < kSpUnroll; ++u) {
        const int64_t e = e0 + u * 32 + lane;
        c[u] = e < end ? __ldcs(P.col + e) : kNone;
        w[u] = e < end ? __ldcs(P.cw + e) : 0.0f;
      }
#pragma unroll
      for (int u = 0; u < kSpUnroll; ++u)
        t[u] = c[u] == kNone ? 0.0 : (P.k32 ? (double)P.k32[c[u]] : P.tot[c[u]]);   // singleton tot = k
#pragma unroll
      for (int u = 0; u < kSpUnroll; ++u) {
        const double W = (double)w[u];
        if (c[u] != kNone && W != 0.0) {
          const double g = __dsub_rn(W, __dmul_rn(t[u], kf));
          if (g > 0.0 && better(g, c[u], bg, bc)) { bg = g; bc = c[u]; bw = W; }
        }
      }
    }
    warp_best(bg, bc, bw);
    if (lane == 0) {
      if (deg <= kSpChunk) apply_decision<true>(P, i, i, bc, bw, (int32_t)deg + (P.has_loop[i] ? 1 : 0));
      else part[q] = HubPartial{bg, bw, bc, 0};
    }
  }
}

__global__ void sp_combine_kernel(MoveArgs P, const int2* multi, int64_t nmulti, const HubPartial* part) {
  if (P.ctl->done) return;
  for (int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; x < nmulti; x += (int64_t)gridDim.x * blockDim.x) {
    const int32_t i = multi[x].x, first = multi[x].y;
    const int64_t deg = P.off[i + 1] - P.off[i];
    const int32_t n = (int32_t)((deg + kSpChunk - 1) / kSpChunk);
    double g = 0.0, w = 0.0;
    int32_t c = kNone;
    for (int32_t k = 0; k < n; ++k) {
      const HubPartial h = part[first + k];
      if (better(h.g, h.c, g, c)) { g = h.g; c = h.c; w = h.w; }
    }
    apply_decision<true>(P, i, i, c, w, (int32_t)deg + (P.has_loop[i] ? 1 : 0));
  }
}

// Chunk lists of the rows longer than 32 (the classes from kBTile on).
__global__ void sp_count_kernel(const int32_t* list, int64_t n, const int64_t* off, uint32_t* cnt, uint32_t* multi) {
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x) {
    const int32_t i = list[j];
    const int64_t nc = (off[i + 1] - off[i] + kSpChunk - 1) / kSpChunk;
    cnt[j] = (uint32_t)nc;
    multi[j] = nc > 1 ? 1u : 0u;
  }
}

__global__ void sp_fill_kernel(const int32_t* list, int64_t n, const int64_t* off, const uint32_t* first,
                               const uint32_t* mpos, int2* chunks, int2* multi) {
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x) {
    const int32_t i = list[j];
    const uint32_t f = first[j], nc = first[j + 1] - f;
    for (uint32_t k = 0; k < nc; ++k) chunks[f + k] = make_int2(i, (int)k);
    if (mpos[j + 1] != mpos[j]) multi[mpos[j]] = make_int2(i, (int)f);
  }
}

// k/2m; in a batched run m is the vertex's own graph's (gm[vgid[i]]).
__global__ void k32_kernel(int32_t V, const double* k, int32_t* k32) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < V; i += (int64_t)gridDim.x * blockDim.x)
    k32[i] = (int32_t)k[i];   // integral and below 2^30 when called
}

__global__ void kfrac_kernel(int32_t V, const double* k, double m, const double* gm, const int32_t* vgid,
                             double* kfrac) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < V; i += (int64_t)gridDim.x * blockDim.x) {
    double mi = gm ? gm[vgid[i]] : m;
    kfrac[i] = mi > 0.0 ? __ddiv_rn(k[i], __dmul_rn(2.0, mi)) : 0.0;   // OneLevelKernel.cu:307
  }
}

__global__ void vinfo_fill_kernel(const int32_t* list, int64_t n, const double* kfrac, const double* k,
                                  const float* loopw, const uint8_t* has_loop, VInfo* info) {
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x) {
    int32_t i = list[j];
    VInfo v;
    v.kfrac = kfrac[i];
    v.k = k[i];
    v.loopw = loopw[i];
    v.vid_loop = (i << 1) | (has_loop[i] ? 1 : 0);
    info[j] = v;
  }
}

// Sliced-ELL copy of the degree-class rows: slot (class b, item j, lane s).
__global__ void ell_fill_kernel(const int32_t* list, const int64_t* off, const int32_t* col, const float* cw,
                                int64_t n, int G, int32_t* ecol, float* ew) {
  for (int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; x < n * G; x += (int64_t)gridDim.x * blockDim.x) {
    int64_t j = x / G;
    int sl = (int)(x - j * G);
    int32_t i = list[j];
    int64_t b = off[i];
    int64_t d = off[i + 1] - b;
    ecol[x] = sl < d ? col[b + sl] : -1;
    ew[x] = sl < d ? cw[b + sl] : 0.0f;
  }
}

// ---------------------------------------------------------------- tile kernel
// Degrees 33..kTileMaxDeg are packed, in index order, into tiles of about
// kTileCost cost units (degree + 4 per vertex).  One block hashes every
// (vertex, neighbour community) pair of its tile into a shared-memory table
// -- all entry loads of the tile independent of each other -- and keeps the
// claimed slots in a list, then resolves each vertex's best community: the
// largest gain bits (positive doubles order like their bit patterns), then the
// smallest community among equal gains.
constexpr int kTileMaxDeg = 512;
constexpr int kTileUnroll = 4;   // tile entries per thread in flight
constexpr int kTileCost = 1536;
constexpr int kTileVtx = 48;          // >= kTileCost / (33 + 4) + 1
constexpr int kTileSlotsLog = 12;     // 4096 slots for <= kTileCost + kTileMaxDeg + 4 entries
constexpr int kTileSlots = 1 << kTileSlotsLog;
constexpr unsigned long long kEmptyKey = ~0ull;
static_assert(kTileVtx >= kTileCost / 37 + 1, "tile vertex arrays too small");
static_assert(kTileCost + kTileMaxDeg + 4 <= (1 << 11) + 8, "tile table load above one half");
static_assert(kTileCost + kTileMaxDeg + 4 <= 256 * 9, "tile row ids: 9 entries per thread");
static_assert(kTileVtx < 256, "tile row ids are bytes");

template <typename Acc>
struct TileSmem {
  unsigned long long key[kTileSlots];
  Acc val[kTileSlots];
  uint16_t claimed[kTileSlots];
  int64_t beg[kTileVtx];
  double kf[kTileVtx];
  double bestw[kTileVtx];
  unsigned long long bestg[kTileVtx];
  int32_t vid[kTileVtx];
  int32_t own[kTileVtx];
  int32_t rowbeg[kTileVtx + 1];
  int32_t bestc[kTileVtx];
  int32_t nseg[kTileVtx];
  int32_t flags[kTileVtx];   // bit0 saw own community, bit1 has self loop
  int32_t nclaimed;
  uint8_t rowid[kThreads * 9];   // tile vertex of every tile entry
};

template <typename Acc>
__device__ __forceinline__ void tile_insert(TileSmem<Acc>& S, unsigned long long k, Acc w, bool& overflow) {
  uint32_t h = (uint32_t)((k * 0x9E3779B97F4A7C15ull) >> (64 - kTileSlotsLog));
  for (int p = 0; p < kTileSlots; ++p) {
    unsigned long long prev = atomicCAS(&S.key[h], kEmptyKey, k);
    if (prev == kEmptyKey) S.claimed[atomicAdd(&S.nclaimed, 1)] = (uint16_t)h;
    if (prev == kEmptyKey || prev == k) { atomicAdd(&S.val[h], w); return; }
    h = (h + 1) & (kTileSlots - 1);
  }
  overflow = true;
}

__device__ __forceinline__ int tile_find(const int32_t* rowbeg, int nv, int q) {
  int lo = 0, hi = nv - 1;
  while (lo < hi) {            // last j with rowbeg[j] <= q
    int mid = (lo + hi + 1) >> 1;
    if (rowbeg[mid] <= q) lo = mid; else hi = mid - 1;
  }
  return lo;
}

template <typename Acc>
__global__ void __launch_bounds__(kThreads) move_tile_kernel(MoveArgs P, const int32_t* tile_start, int64_t ntiles) {
  extern __shared__ __align__(16) unsigned char smem[];
  TileSmem<Acc>& S = *reinterpret_cast<TileSmem<Acc>*>(smem);
  if (P.ctl->done) return;
  for (int sl = threadIdx.x; sl < kTileSlots; sl += kThreads) { S.key[sl] = kEmptyKey; S.val[sl] = Acc(0); }
  if (threadIdx.x == 0) S.nclaimed = 0;
  bool overflow = false;
  for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int vb = tile_start[t];
    const int nv = tile_start[t + 1] - vb;
    int deg = 0;
    if (threadIdx.x < nv) {
      int32_t i = P.list[vb + threadIdx.x];
      int64_t b = P.off[i];
      deg = (int)(P.off[i + 1] - b);
      S.vid[threadIdx.x] = i;
      S.beg[threadIdx.x] = b;
      S.own[threadIdx.x] = P.comm[i];
      S.kf[threadIdx.x] = P.kfrac[i];
      S.flags[threadIdx.x] = P.has_loop[i] ? 2 : 0;
      S.bestg[threadIdx.x] = 0ull;
      S.bestc[threadIdx.x] = kNone;
      S.nseg[threadIdx.x] = 0;
    }
    int ne;
    int pre = block_exclusive_scan256<int>(deg, &ne);
    if (threadIdx.x < nv) S.rowbeg[threadIdx.x] = pre;
    if (threadIdx.x == 0) S.rowbeg[nv] = ne;
    __syncthreads();
    {   // row ids: one search per run of 9 entries, then a forward walk
      const int q0 = threadIdx.x * 9;
      if (q0 < ne) {
        int j = tile_find(S.rowbeg, nv, q0);
        const int q1 = min(q0 + 9, ne);
        for (int q = q0; q < q1; ++q) {
          while (S.rowbeg[j + 1] <= q) ++j;
          S.rowid[q] = (uint8_t)j;
        }
      }
    }
    __syncthreads();
    for (int q0 = threadIdx.x; q0 < ne; q0 += kTileUnroll * kThreads) {
      int jj[kTileUnroll];
      int32_t cc[kTileUnroll];
      float ww[kTileUnroll];
#pragma unroll
      for (int u = 0; u < kTileUnroll; ++u) {
        int q = q0 + u * kThreads;
        jj[u] = -1;
        if (q < ne) {
          int j = S.rowid[q];
          int64_t e = S.beg[j] + (q - S.rowbeg[j]);
          jj[u] = j;
          cc[u] = __ldcs(P.col + e);
          ww[u] = __ldcs(P.cw + e);
        }
      }
#pragma unroll
      for (int u = 0; u < kTileUnroll; ++u)
        if (jj[u] >= 0) cc[u] = P.comm[cc[u]];
#pragma unroll
      for (int u = 0; u < kTileUnroll; ++u) {
        if (jj[u] >= 0) {
          int j = jj[u];
          if (cc[u] == S.own[j]) atomicOr(&S.flags[j], 1);
          unsigned long long k = ((unsigned long long)(uint32_t)j << 32) | (uint32_t)cc[u];
          tile_insert(S, k, (Acc)ww[u], overflow);
        }
      }
    }
    __syncthreads();
    const int nc = S.nclaimed;
    for (int x = threadIdx.x; x < nc; x += kThreads) {       // count, best gain bits
      int sl = S.claimed[x];
      unsigned long long k = S.key[sl];
      int j = (int)(k >> 32);
      int32_t c = (int32_t)(uint32_t)k;
      atomicAdd(&S.nseg[j], 1);
      double W = (double)S.val[sl];
      if (W != 0.0) {
        double g = __dsub_rn(W, __dmul_rn(P.tot[c], S.kf[j]));
        if (g > 0.0) atomicMax(&S.bestg[j], (unsigned long long)__double_as_longlong(g));
      }
    }
    __syncthreads();
    for (int x = threadIdx.x; x < nc; x += kThreads) {       // smallest community among the best gains
      int sl = S.claimed[x];
      unsigned long long k = S.key[sl];
      int j = (int)(k >> 32);
      int32_t c = (int32_t)(uint32_t)k;
      double W = (double)S.val[sl];
      if (W != 0.0 && S.bestg[j] != 0ull) {
        double g = __dsub_rn(W, __dmul_rn(P.tot[c], S.kf[j]));
        if ((unsigned long long)__double_as_longlong(g) == S.bestg[j]) atomicMin(&S.bestc[j], c);
      }
    }
    __syncthreads();
    for (int x = threadIdx.x; x < nc; x += kThreads) {       // weight to the winner; clear the table
      int sl = S.claimed[x];
      unsigned long long k = S.key[sl];
      int j = (int)(k >> 32);
      int32_t c = (int32_t)(uint32_t)k;
      if (c == S.bestc[j]) S.bestw[j] = (double)S.val[sl];
      S.key[sl] = kEmptyKey;
      S.val[sl] = Acc(0);
    }
    __syncthreads();
    if (threadIdx.x < nv) {
      int j = threadIdx.x;
      int f = S.flags[j];
      int32_t nseg = S.nseg[j] + (((f & 2) && !(f & 1)) ? 1 : 0);
      int32_t bc = S.bestc[j];
      apply_decision(P, S.vid[j], S.own[j], bc, bc == kNone ? 0.0 : S.bestw[j], nseg);
    }
    if (threadIdx.x == 0) S.nclaimed = 0;
    __syncthreads();
  }
  if (__syncthreads_or(overflow) && threadIdx.x == 0) atomicOr(&P.ctl->err, kErrProbe);
}

struct TilePackedSmem {
  unsigned long long slot[kTileSlots];
  uint16_t claimed[kTileSlots];
  int64_t beg[kTileVtx];
  double kf[kTileVtx];
  double bestw[kTileVtx];
  unsigned long long bestg[kTileVtx];
  int32_t vid[kTileVtx];
  int32_t own[kTileVtx];
  int32_t rowbeg[kTileVtx + 1];
  int32_t bestc[kTileVtx];
  int32_t nseg[kTileVtx];
  int32_t flags[kTileVtx];
  int32_t nclaimed;
  uint8_t rowid[kThreads * 9];
};
constexpr int kTilePackedMaxComm = 1 << 26;

__device__ __forceinline__ void tile_packed_insert(TilePackedSmem& S, uint32_t key, uint32_t w, bool& overflow) {
  uint32_t h = (uint32_t)(((unsigned long long)key * 0x9E3779B97F4A7C15ull) >> (64 - kTileSlotsLog));
  for (int p = 0; p < kTileSlots; ++p) {
    const unsigned long long cur = *reinterpret_cast<volatile unsigned long long*>(&S.slot[h]);
    if ((uint32_t)(cur >> 32) == key) { atomicAdd(&S.slot[h], (unsigned long long)w); return; }
    if (cur == kPackedEmpty) {
      const unsigned long long prev = atomicCAS(&S.slot[h], kPackedEmpty, ((unsigned long long)key << 32) | w);
      if (prev == kPackedEmpty) { S.claimed[atomicAdd(&S.nclaimed, 1)] = (uint16_t)h; return; }
      if ((uint32_t)(prev >> 32) == key) { atomicAdd(&S.slot[h], (unsigned long long)w); return; }
    }
    h = (h + 1) & (kTileSlots - 1);
  }
  overflow = true;
}

// The tile kernel with packed slots ((j << 26 | c) << 32 | integer sum, all
// ones when empty; j < 48, so no key is all ones): one shared atomic per
// entry and a smaller table.  Integral weights, community ids below 2^26.
__global__ void __launch_bounds__(kThreads) move_tile_packed_kernel(MoveArgs P, const int32_t* tile_start,
                                                                    int64_t ntiles) {
  extern __shared__ __align__(16) unsigned char smem[];
  TilePackedSmem& S = *reinterpret_cast<TilePackedSmem*>(smem);
  if (P.ctl->done) return;
  for (int sl = threadIdx.x; sl < kTileSlots; sl += kThreads) S.slot[sl] = kPackedEmpty;
  if (threadIdx.x == 0) S.nclaimed = 0;
  bool overflow = false;
  __shared__ WorkQueue wq;
  for (int64_t t = work_begin(P.queue, wq); t < ntiles; t = work_advance(P.queue, t, wq)) {
    const int vb = tile_start[t];
    const int nv = tile_start[t + 1] - vb;
    int deg = 0;
    if (threadIdx.x < nv) {
      int32_t i = P.list[vb + threadIdx.x];
      int64_t b = P.off[i];
      deg = (int)(P.off[i + 1] - b);
      S.vid[threadIdx.x] = i;
      S.beg[threadIdx.x] = b;
      S.own[threadIdx.x] = P.comm[i];
      S.kf[threadIdx.x] = P.kfrac[i];
      S.flags[threadIdx.x] = P.has_loop[i] ? 2 : 0;
      S.bestg[threadIdx.x] = 0ull;
      S.bestc[threadIdx.x] = kNone;
      S.nseg[threadIdx.x] = 0;
    }
    int ne;
    int pre = block_exclusive_scan256<int>(deg, &ne);
    if (threadIdx.x < nv) S.rowbeg[threadIdx.x] = pre;
    if (threadIdx.x == 0) S.rowbeg[nv] = ne;
    __syncthreads();
    {   // row ids: one search per run of 9 entries, then a forward walk
      const int q0 = threadIdx.x * 9;
      if (q0 < ne) {
        int j = tile_find(S.rowbeg, nv, q0);
        const int q1 = min(q0 + 9, ne);
        for (int q = q0; q < q1; ++q) {
          while (S.rowbeg[j + 1] <= q) ++j;
          S.rowid[q] = (uint8_t)j;
        }
      }
    }
    __syncthreads();
    for (int q0 = threadIdx.x; q0 < ne; q0 += kTileUnroll * kThreads) {
      int jj[kTileUnroll];
      int32_t cc[kTileUnroll];
      float ww[kTileUnroll];
#pragma unroll
      for (int u = 0; u < kTileUnroll; ++u) {
        int q = q0 + u * kThreads;
        jj[u] = -1;
        if (q < ne) {
          int j = S.rowid[q];
          int64_t e = S.beg[j] + (q - S.rowbeg[j]);
          jj[u] = j;
          cc[u] = __ldcs(P.col + e);
          ww[u] = __ldcs(P.cw + e);
        }
      }
#pragma unroll
      for (int u = 0; u < kTileUnroll; ++u)
        if (jj[u] >= 0) cc[u] = P.comm[cc[u]];
#pragma unroll
      for (int u = 0; u < kTileUnroll; ++u) {
        if (jj[u] >= 0) {
          int j = jj[u];
          if (cc[u] == S.own[j]) atomicOr(&S.flags[j], 1);
          tile_packed_insert(S, ((uint32_t)j << 26) | (uint32_t)cc[u], (uint32_t)ww[u], overflow);
        }
      }
    }
    __syncthreads();
    const int nc = S.nclaimed;
    for (int x = threadIdx.x; x < nc; x += kThreads) {       // count, best gain bits
      int sl = S.claimed[x];
      const unsigned long long sv = S.slot[sl];
      const uint32_t key = (uint32_t)(sv >> 32);
      int j = (int)(key >> 26);
      int32_t c = (int32_t)(key & ((1u << 26) - 1u));
      atomicAdd(&S.nseg[j], 1);
      double W = (double)(uint32_t)sv;
      if (W != 0.0) {
        double g = __dsub_rn(W, __dmul_rn(P.tot[c], S.kf[j]));
        if (g > 0.0) atomicMax(&S.bestg[j], (unsigned long long)__double_as_longlong(g));
      }
    }
    __syncthreads();
    for (int x = threadIdx.x; x < nc; x += kThreads) {       // smallest community among the best gains
      int sl = S.claimed[x];
      const unsigned long long sv = S.slot[sl];
      const uint32_t key = (uint32_t)(sv >> 32);
      int j = (int)(key >> 26);
      int32_t c = (int32_t)(key & ((1u << 26) - 1u));
      double W = (double)(uint32_t)sv;
      if (W != 0.0 && S.bestg[j] != 0ull) {
        double g = __dsub_rn(W, __dmul_rn(P.tot[c], S.kf[j]));
        if ((unsigned long long)__double_as_longlong(g) == S.bestg[j]) atomicMin(&S.bestc[j], c);
      }
    }
    __syncthreads();
    for (int x = threadIdx.x; x < nc; x += kThreads) {       // weight to the winner; clear the table
      int sl = S.claimed[x];
      const unsigned long long sv = S.slot[sl];
      const uint32_t key = (uint32_t)(sv >> 32);
      int j = (int)(key >> 26);
      int32_t c = (int32_t)(key & ((1u << 26) - 1u));
      if (c == S.bestc[j]) S.bestw[j] = (double)(uint32_t)sv;
      S.slot[sl] = kPackedEmpty;
    }
    __syncthreads();
    if (threadIdx.x < nv) {
      int j = threadIdx.x;
      int f = S.flags[j];
      int32_t nseg = S.nseg[j] + (((f & 2) && !(f & 1)) ? 1 : 0);
      int32_t bc = S.bestc[j];
      apply_decision(P, S.vid[j], S.own[j], bc, bc == kNone ? 0.0 : S.bestw[j], nseg);
    }
    if (threadIdx.x == 0) S.nclaimed = 0;
    __syncthreads();
  }
  if (__syncthreads_or(overflow) && threadIdx.x == 0) atomicOr(&P.ctl->err, kErrProbe);
}

// Tile boundaries: vertex j of the tile bucket belongs to tile
// floor(cumcost_j / kTileCost), cost = degree + 4, so a tile holds at most
// kTileCost / 37 + 1 vertices and kTileCost + kTileMaxDeg + 4 entries.
__global__ void tile_cost_kernel(const int32_t* list, int64_t n, const int64_t* off, int64_t* cost) {
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x) {
    int32_t i = list[j];
    cost[j] = off[i + 1] - off[i] + 4;
  }
}

__global__ void tile_start_kernel(const int64_t* cum, int64_t n, int32_t* tile_start) {
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x) {
    int64_t t = cum[j] / kTileCost;
    if (j == 0 || cum[j - 1] / kTileCost != t) tile_start[t] = (int32_t)j;
    if (j == n - 1) tile_start[t + 1] = (int32_t)n;
  }
}

// Integral weights with small degrees allow an exact int32 accumulator.
__global__ void int_weights_kernel(const float* cw, int64_t nnz, const double* k, int32_t V, uint32_t* notint) {
  int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nnz; e += stride) {
    float x = cw[e];
    if (x != truncf(x)) atomicOr(notint, 1u);
  }
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < V; i += stride)
    if (!(k[i] < 1073741824.0)) atomicOr(notint, 1u);
}

// Hubs: rows longer than block_max.  A pass aggregates a hub's neighbour
// communities in three launches, with no global-memory atomics on the sums:
//  (1) hub_part_kernel -- one block per 4096-entry chunk of a hub row gathers
//      the neighbours' communities and writes the chunk's (community, weight)
//      pairs grouped by bucket (top bits of a hash of the community; a hub of
//      degree d has about d/1024 buckets, a power of two) to a staging area,
//      with the chunk's bucket offsets;
//  (2) hub_agg_kernel -- one block per (hub, bucket) reads that bucket's
//      pairs from every chunk of the hub, sums equal communities in a
//      shared-memory table and keeps the bucket's best candidate and its
//      count of distinct communities;
//  (3) hub_decide_kernel -- one thread per hub combines its buckets in order
//      and decides.
// A bucket holds a disjoint set of communities, so its best candidate and
// count are those of the row restricted to that set, and combining buckets
// with `better` gives the row's argmax and tie-break.
constexpr int kHubPartThreads = 512;              // chunk blocks: 16 warps of 8 entries per lane
constexpr int kHubItems = kHubChunk / kHubPartThreads;
constexpr int kHubBucketTarget = 1024;            // mean entries of a bucket
constexpr int kHubMaxBucketsLog = 12;
constexpr int kAggLog = 11;                       // shared table of 2048 slots
constexpr int kAggSlots = 1 << kAggLog;
constexpr int kAggFull = kAggSlots / 2;           // more claims: the bucket is split into sub-passes
constexpr int kAggMaxSplitLog = 16;               // beyond 2^16 sub-passes: report, give up
static_assert(kHubChunk % kHubPartThreads == 0 && kHubChunk <= 65535, "chunk offsets are 16-bit");

__device__ __forceinline__ uint32_t hub_bucket(int32_t c, int plog) {
  return plog == 0 ? 0u : (uint32_t)(((uint64_t)(uint32_t)c * 0x9E3779B97F4A7C15ull) >> (64 - plog));
}
// sub-pass of a community inside its bucket (an independent hash)
__device__ __forceinline__ uint32_t hub_sub(int32_t c, int slog) {
  return slog == 0 ? 0u : (uint32_t)(((uint64_t)(uint32_t)c * 0xD6E8FEB86659FD93ull) >> (64 - slog));
}
// table slot (a third hash: the communities of one bucket share the top bits of the first)
__device__ __forceinline__ uint32_t agg_slot(int32_t c) {
  return (uint32_t)(((uint64_t)(uint32_t)c * 0xC2B2AE3D27D4EB4Full) >> (64 - kAggLog));
}

struct HubArgs {
  const int32_t* hubs;        // [nhub] hub vertices
  const int32_t* chunk_hub;   // [nchunk] hub of each chunk (a hub's chunks are consecutive)
  const int64_t* chunk_beg;   // [nchunk] first CSR entry of the chunk
  const int64_t* chunk_cbo;   // [nchunk] first of the chunk's bucket offsets in cb_off
  const int64_t* chunk_stg;   // [nchunk] first staging slot of the chunk (hub entries in CSR order)
  const int32_t* hub_plog;    // [nhub] log2 of the hub's bucket count
  const int32_t* hub_cb0;     // [nhub + 1] first chunk of each hub
  const int32_t* hub_bb0;     // [nhub + 1] first bucket of each hub
  const int32_t* bucket_hub;  // [nbucket] hub of each bucket
  uint16_t* cb_off;           // per chunk: 2^plog + 1 bucket offsets inside the chunk
  unsigned long long* stage;  // [hub entries] community << 32 | weight bits, grouped by bucket per chunk
  uint32_t* sawown;           // [nhub] a neighbour is in the hub's own community
  HubPartial* part;           // [nbucket] best candidate and distinct count of each bucket
  int64_t nbucket;
};

__global__ void __launch_bounds__(kHubPartThreads) hub_part_kernel(MoveArgs P, HubArgs H) {
  __shared__ uint32_t cnt[1 << kHubMaxBucketsLog];
  if (P.ctl->done) return;
  const int64_t ch = blockIdx.x;
  const int32_t h = H.chunk_hub[ch];
  const int32_t i = H.hubs[h];
  const int32_t own = P.comm[i];
  const int64_t beg = H.chunk_beg[ch];
  const int64_t end = min(beg + (int64_t)kHubChunk, P.off[i + 1]);
  const int plog = H.hub_plog[h];
  const int nb = 1 << plog;
  for (int x = threadIdx.x; x < nb; x += kHubPartThreads) cnt[x] = 0;
  __syncthreads();
  int32_t c[kHubItems];
  float w[kHubItems];
#pragma unroll
  for (int u = 0; u < kHubItems; ++u) {
    const int64_t e = beg + u * kHubPartThreads + threadIdx.x;
    c[u] = e < end ? __ldcs(P.col + e) : -1;
    w[u] = e < end ? __ldcs(P.cw + e) : 0.0f;
  }
#pragma unroll
  for (int u = 0; u < kHubItems; ++u) c[u] = c[u] >= 0 ? P.comm[c[u]] : -1;   // all gathers in flight
  bool sawown = false;
  uint32_t bk[kHubItems], rk[kHubItems];
#pragma unroll
  for (int u = 0; u < kHubItems; ++u) {
    bk[u] = 0u;
    rk[u] = 0u;
    if (c[u] >= 0) {
      sawown |= c[u] == own;
      bk[u] = hub_bucket(c[u], plog);
      rk[u] = atomicAdd(&cnt[bk[u]], 1u);
    }
  }
  __syncthreads();
  // bucket starts: each thread scans a run of consecutive buckets
  const int per = (nb + kHubPartThreads - 1) / kHubPartThreads;
  const int x0 = min((int)threadIdx.x * per, nb), x1 = min(x0 + per, nb);
  uint32_t local = 0;
  for (int x = x0; x < x1; ++x) local += cnt[x];
  uint32_t total;
  uint32_t run = block_exclusive_scan512<uint32_t>(local, &total);
  uint16_t* off = H.cb_off + H.chunk_cbo[ch];
  for (int x = x0; x < x1; ++x) {
    const uint32_t v = cnt[x];
    cnt[x] = run;
    off[x] = (uint16_t)run;
    run += v;
  }
  if (threadIdx.x == 0) off[nb] = (uint16_t)total;
  __syncthreads();
  unsigned long long* st = H.stage + H.chunk_stg[ch];
#pragma unroll
  for (int u = 0; u < kHubItems; ++u)
    if (c[u] >= 0) st[cnt[bk[u]] + rk[u]] = ((unsigned long long)(uint32_t)c[u] << 32) | __float_as_uint(w[u]);
  if (__syncthreads_or(sawown) && threadIdx.x == 0) atomicOr(&H.sawown[h], 1u);
}

// Shared-memory tables of hub_agg_kernel.  Packed (integral weights):
// community << 32 | integer sum, all ones when empty, one atomic per entry.
template <bool PACKED>
struct AggTable {
  unsigned long long slot[kAggSlots];
  __device__ __forceinline__ void clear(int s) { slot[s] = kPackedEmpty; }
  __device__ __forceinline__ void get(int s, int32_t& c, double& W) const {
    c = (int32_t)(uint32_t)(slot[s] >> 32);
    W = (double)(uint32_t)slot[s];
  }
  // 1: added to an existing community, 2: claimed a slot, 0: table full
  __device__ __forceinline__ int insert(int32_t c, float w, uint32_t& where) {
    const uint32_t wi = (uint32_t)w;
    uint32_t h = agg_slot(c);
    for (int p = 0; p < kAggSlots; ++p) {
      const unsigned long long cur = *reinterpret_cast<volatile unsigned long long*>(&slot[h]);
      if ((uint32_t)(cur >> 32) == (uint32_t)c) { atomicAdd(&slot[h], (unsigned long long)wi); return 1; }
      if (cur == kPackedEmpty) {
        const unsigned long long prev = atomicCAS(&slot[h], kPackedEmpty, ((unsigned long long)(uint32_t)c << 32) | wi);
        if (prev == kPackedEmpty) { where = h; return 2; }
        if ((uint32_t)(prev >> 32) == (uint32_t)c) { atomicAdd(&slot[h], (unsigned long long)wi); return 1; }
      }
      h = (h + 1) & (kAggSlots - 1);
    }
    return 0;
  }
};

template <>
struct AggTable<false> {
  int32_t key[kAggSlots];
  double val[kAggSlots];
  __device__ __forceinline__ void clear(int s) { key[s] = -1; val[s] = 0.0; }
  __device__ __forceinline__ void get(int s, int32_t& c, double& W) const { c = key[s]; W = val[s]; }
  __device__ __forceinline__ int insert(int32_t c, float w, uint32_t& where) {
    uint32_t h = agg_slot(c);
    for (int p = 0; p < kAggSlots; ++p) {
      const int32_t prev = atomicCAS(&key[h], -1, c);
      if (prev == -1 || prev == c) {
        atomicAdd(&val[h], (double)w);
        if (prev == -1) { where = h; return 2; }
        return 1;
      }
      h = (h + 1) & (kAggSlots - 1);
    }
    return 0;
  }
};

struct int2x64 {
  int64_t base;
  int32_t len;
};

struct AggCtl {
  int64_t segbase[kThreads];   // staging slot of each segment's first pair
  uint16_t claimed[kAggSlots];
  int32_t segpre[kThreads + 1];
  double rg[kThreads / 32], rw[kThreads / 32];
  int32_t rc[kThreads / 32], rn[kThreads / 32];
  int32_t nclaimed;
  int32_t full;
};

template <bool PACKED>
constexpr size_t agg_smem_bytes() {
  return sizeof(AggTable<PACKED>) + sizeof(AggCtl);
}

struct AggBest {
  double g, w;
  int32_t c, n;
};

// One staged pair into the table, when its community belongs to sub-pass
// `sub` of 2^slog; a claimed slot is listed, and a table past half full
// marks the sub-pass as split.
template <bool PACKED>
__device__ __forceinline__ void agg_insert(AggTable<PACKED>& T, AggCtl& S, unsigned long long x, int slog,
                                           uint32_t sub) {
  const int32_t c = (int32_t)(uint32_t)(x >> 32);
  if (slog > 0 && hub_sub(c, slog) != sub) return;
  uint32_t where = 0;
  const int r = T.insert(c, __uint_as_float((uint32_t)x), where);
  if (r == 2) {
    const int n = atomicAdd(&S.nclaimed, 1);
    S.claimed[n] = (uint16_t)where;
    if (n + 1 > kAggFull) S.full = 1;
  } else if (r == 0) {
    S.full = 1;
  }
}

// Sums the staged pairs of K segments (segment k starts at staging slot
// seg(k).x and holds seg(k).y pairs) per community in the shared table T,
// and leaves the best candidate (gain w - tot_c * kf, higher gain then lower
// community; OneLevelKernel.cu:303,307-313,330,358) and the count of distinct
// communities in thread 0.  The table is left empty.  When the pairs claim
// more than half the table, the communities are split by a second hash into
// 2, 4, ... sub-passes, each re-reading the pairs, until every sub-pass fits;
// still too full at 2^16 sub-passes, the pass's error flag is set (reported
// as a capacity error, never a wrong sum).  All threads of the block call it.
template <bool PACKED, typename SegFn>
__device__ AggBest agg_segments(const MoveArgs& P, AggTable<PACKED>& T, AggCtl& S, const unsigned long long* stage,
                                int32_t K, SegFn seg, double kf) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  double bg = 0.0, bw = 0.0;
  int32_t bc = kNone;
  int nocc = 0;
  for (int slog = 0;; ++slog) {
    bg = 0.0; bw = 0.0; bc = kNone; nocc = 0;
    bool split = false;
    for (uint32_t sub = 0; sub < (1u << slog) && !split; ++sub) {
      if (K == 1) {   // one segment (a block-class row): no scan, no search
        const int2x64 sg = seg(0);
        for (int32_t q = threadIdx.x; q < sg.len; q += kThreads) {
          if (*reinterpret_cast<volatile int32_t*>(&S.full)) break;
          const unsigned long long x = stage[sg.base + q];
          agg_insert(T, S, x, slog, sub);
        }
        __syncthreads();
      }
      for (int32_t k0 = 0; K > 1 && k0 < K; k0 += kThreads) {
        const int32_t k = k0 + (int32_t)threadIdx.x;
        int64_t base = 0;
        int32_t len = 0;
        if (k < K) {
          const int2x64 sg = seg(k);
          base = sg.base;
          len = sg.len;
        }
        int32_t tot;
        const int32_t pre = block_exclusive_scan256<int32_t>(len, &tot);
        S.segpre[threadIdx.x] = pre;
        S.segbase[threadIdx.x] = base;
        __syncthreads();
        const int nseg = min(kThreads, K - k0);
        for (int32_t q = threadIdx.x; q < tot; q += kThreads) {
          if (*reinterpret_cast<volatile int32_t*>(&S.full)) break;   // this sub-pass is discarded anyway
          int jlo = 0, jhi = nseg - 1;                 // last segment starting at or before q
          while (jlo < jhi) {
            const int mid = (jlo + jhi + 1) >> 1;
            if (S.segpre[mid] <= q) jlo = mid; else jhi = mid - 1;
          }
          const unsigned long long x = stage[S.segbase[jlo] + (q - S.segpre[jlo])];
          agg_insert(T, S, x, slog, sub);
        }
        __syncthreads();
      }
      const bool full = S.full != 0;
      const int nc = S.nclaimed;
      for (int x = threadIdx.x; x < nc; x += kThreads) {
        const int sl = S.claimed[x];
        if (!full) {
          int32_t c;
          double W;
          T.get(sl, c, W);
          ++nocc;
          if (W != 0.0) {                                            // OneLevelKernel.cu:303
            const double g = __dsub_rn(W, __dmul_rn(P.tot[c], kf));  // OneLevelKernel.cu:307-313
            if (g > 0.0 && better(g, c, bg, bc)) { bg = g; bc = c; bw = W; }
          }
        }
        T.clear(sl);
      }
      __syncthreads();
      if (threadIdx.x == 0) { S.nclaimed = 0; S.full = 0; }
      __syncthreads();
      split = full;
    }
    if (!split) break;
    if (slog == kAggMaxSplitLog) {
      if (threadIdx.x == 0) atomicOr(&P.ctl->err, kErrProbe);
      break;
    }
  }
  warp_best(bg, bc, bw);
  nocc = __reduce_add_sync(0xffffffffu, (unsigned)nocc);
  if (lane == 0) { S.rg[wid] = bg; S.rc[wid] = bc; S.rw[wid] = bw; S.rn[wid] = nocc; }
  __syncthreads();
  AggBest r{S.rg[0], S.rw[0], S.rc[0], S.rn[0]};
  if (threadIdx.x == 0) {
    for (int k2 = 1; k2 < kThreads / 32; ++k2) {
      if (better(S.rg[k2], S.rc[k2], r.g, r.c)) { r.g = S.rg[k2]; r.c = S.rc[k2]; r.w = S.rw[k2]; }
      r.n += S.rn[k2];
    }
  }
  __syncthreads();
  return r;   // valid in thread 0
}

template <bool PACKED>
__device__ __forceinline__ void agg_init(AggTable<PACKED>& T, AggCtl& S) {
  for (int x = threadIdx.x; x < kAggSlots; x += kThreads) T.clear(x);
  if (threadIdx.x == 0) { S.nclaimed = 0; S.full = 0; }
  __syncthreads();
}

// One block per (hub, bucket), blocks persistent over the buckets: the
// bucket's segments are its slice of every chunk of the hub.
template <bool PACKED>
__global__ void __launch_bounds__(kThreads) hub_agg_kernel(MoveArgs P, HubArgs H) {
  extern __shared__ __align__(16) unsigned char smem[];
  AggTable<PACKED>& T = *reinterpret_cast<AggTable<PACKED>*>(smem);
  AggCtl& S = *reinterpret_cast<AggCtl*>(smem + sizeof(AggTable<PACKED>));
  if (P.ctl->done) return;
  agg_init(T, S);
  __shared__ WorkQueue wq;
  for (int64_t gb = work_begin(P.queue, wq); gb < H.nbucket; gb = work_advance(P.queue, gb, wq)) {
    const int32_t h = H.bucket_hub[gb];
    const int32_t b = (int32_t)(gb - H.hub_bb0[h]);
    const int32_t c0 = H.hub_cb0[h], K = H.hub_cb0[h + 1] - c0;
    const AggBest r = agg_segments<PACKED>(
        P, T, S, H.stage, K,
        [&](int32_t k) {
          const uint16_t* off = H.cb_off + H.chunk_cbo[c0 + k];
          return int2x64{H.chunk_stg[c0 + k] + off[b], (int32_t)off[b + 1] - (int32_t)off[b]};
        },
        P.kfrac[H.hubs[h]]);
    if (threadIdx.x == 0) H.part[gb] = HubPartial{r.g, r.w, r.c, r.n};
  }
}

__global__ void hub_decide_kernel(MoveArgs P, HubArgs H, int64_t nhub) {
  if (P.ctl->done) return;
  int64_t h = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (h >= nhub) return;
  int32_t i = H.hubs[h];
  int32_t own = P.comm[i];
  double g = 0.0, ww = 0.0;
  int32_t c = kNone;
  int n = 0;
  for (int32_t bk = H.hub_bb0[h]; bk < H.hub_bb0[h + 1]; ++bk) {
    HubPartial q = H.part[bk];
    if (better(q.g, q.c, g, c)) { g = q.g; c = q.c; ww = q.w; }
    n += q.n;
  }
  bool sw = H.sawown[h] != 0;
  H.sawown[h] = 0;
  int32_t nseg = n + ((P.has_loop[i] && !sw) ? 1 : 0);
  apply_decision(P, i, own, c, ww, nseg);
}

// ------------------------------------------------------------------ commit + Q
// term_c = in_c/m - (tot_c/2m)^2 (OneLevelKernel.cu:447-448), zero when m <= 0.
__device__ __forceinline__ double q_term(double in, double tot, double m, double twom) {
  if (!(m > 0.0)) return 0.0;
  double a = __ddiv_rn(in, m);
  double b = __ddiv_rn(tot, twom);
  return __dsub_rn(a, __dmul_rn(b, b));
}

enum { kCommitInit = 0, kCommitPass = 1, kCommitForce = 2 };

// kCommitPass: the ΔQ test of the pass (OneLevelKernel.cu:889-896), then
// communitySetKernel (:93-107) and the Q of the new state; on a stop the
// deltas are dropped (mergeInitKernel, :109-120).  kCommitForce commits
// unconditionally (mergeSetKernel, :122-136).  kCommitInit only sums Q.
template <int MODE>
__global__ void __launch_bounds__(kRedThreads) commit_kernel(int32_t V, double m, int32_t* comm, const int32_t* next,
                                                             double* tot, double* in, int32_t* size, Delta* delta,
                                                             const double* k, double* partials, PassCtl* ctl) {
  __shared__ double ws[8];
  int64_t base = (int64_t)blockIdx.x * kGroup + threadIdx.x;
  if (MODE == kCommitPass) {
    if (ctl->done) return;
    bool stop = __dsub_rn(ctl->q_prev, ctl->cur) < ctl->pass_min;
    bool capped = ctl->max_passes >= 0 && ctl->pass >= ctl->max_passes;
    if (stop || capped) {
      for (int j = 0; j < 8; ++j) {
        int64_t c = base + (int64_t)j * 256;
        if (c < V) delta_clear(delta[c]);
      }
      if (blockIdx.x == 0 && threadIdx.x == 0) ctl->stop_now = stop ? 1 : 2;
      return;
    }
  }
  double twom = __dmul_rn(2.0, m);
  double s = 0.0;
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    int64_t c = base + (int64_t)j * 256;
    if (c < V) {
      double t, x;
      if (MODE != kCommitInit) {
        t = tot[c]; x = in[c];
        int32_t sz = size[c];
        delta_commit(delta[c], k[c], t, x, sz);
        tot[c] = t; in[c] = x; size[c] = sz;
        comm[c] = next[c];
      } else {
        t = tot[c]; x = in[c];
      }
      s = __dadd_rn(s, q_term(x, t, m, twom));
    }
  }
  double r = block_tree256(s, ws);
  if (threadIdx.x == 0) partials[blockIdx.x] = r;
}

// Intermediate tree level when a level has more than 2048 groups.
__global__ void __launch_bounds__(kRedThreads) tree_level_ctl_kernel(const double* x, int64_t n, double* out,
                                                                     const PassCtl* ctl, int respect_ctl) {
  __shared__ double ws[8];
  if (respect_ctl && (ctl->done || ctl->stop_now)) return;
  int64_t b = blockIdx.x;
  int64_t len = n - b * kGroup;
  if (len > kGroup) len = kGroup;
  double r = group_sum_block<double>(x + b * kGroup, len, ws);
  if (threadIdx.x == 0) out[b] = r;
}

// End of a pass: either finish the level loop or move the floor and Q on.
__global__ void __launch_bounds__(kRedThreads) ctl_pass_kernel(const double* partials, int64_t np, PassCtl* ctl) {
  __shared__ double ws[8];
  __shared__ int flag;
  if (threadIdx.x == 0) flag = ctl->done ? 2 : (ctl->stop_now ? 1 : 0);
  __syncthreads();
  int f = flag;
  if (f == 2) return;
  if (f == 1) {
    if (threadIdx.x == 0) {
      ctl->status = ctl->stop_now == 2 ? LVG_ERR_NOT_CONVERGED : LVG_OK;
      ctl->passes = ctl->pass;
      ctl->stop_now = 0;
      ctl->done = 1;
    }
    return;
  }
  double q = group_sum_block<double>(partials, np, ws);
  if (threadIdx.x == 0) {
    double cur = ctl->q_prev;            // curMod = newMod; if (curMod < lower) curMod = lower
    if (cur < ctl->lower) cur = ctl->lower;
    ctl->cur = cur;
    ctl->q_prev = q;
    ctl->pass += 1;
  }
}

__global__ void __launch_bounds__(kRedThreads) ctl_q_kernel(const double* partials, int64_t np, double* dst) {
  __shared__ double ws[8];
  double q = group_sum_block<double>(partials, np, ws);
  if (threadIdx.x == 0) *dst = q;
}

__global__ void ctl_init_kernel(PassCtl* ctl, double lower, double pass_min, int32_t max_passes) {
  ctl->cur = -1.0;                       // curMod = -1 (OneLevelKernel.cu:528)
  ctl->lower = lower;
  ctl->pass_min = pass_min;
  ctl->q_ret = 0.0;
  ctl->pass = 1;
  ctl->max_passes = max_passes;
  ctl->stop_now = 0;
  ctl->done = 0;
  ctl->status = 0;
  ctl->passes = 0;
  ctl->err = 0;
}

// Isolated-vertex merge (OneLevelKernel.cu:138-171) from the candidates of
// the last pass; weight 0, so `in` moves by the loop weight only.
__global__ void merge_kernel(int32_t V, const int32_t* comm, int32_t* next, const int32_t* cand, const double* k,
                             const float* loopw, Delta* delta) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < V; i += (int64_t)gridDim.x * blockDim.x) {
    int32_t c = cand[i];
    if (c >= 0) {
      int32_t own = comm[i];
      next[i] = c;
      double ki = k[i];
      move_deltas<false>(delta, own, c, ki, __dadd_rn(0.0, (double)loopw[i]));
    }
  }
}

__global__ void set_state_kernel(int32_t V, const int32_t* src_comm, const double* k, const float* loopw,
                                 int32_t* comm, int32_t* next, double* tot, double* in, int32_t* size) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < V; i += (int64_t)gridDim.x * blockDim.x) {
    int32_t c = src_comm[i];
    comm[i] = c;
    next[i] = c;
    atomicAdd(&tot[c], k[i]);
    atomicAdd(&in[c], (double)loopw[i]);
    atomicAdd(&size[c], 1);
  }
}

__global__ void clear_deltas_kernel(int32_t V, Delta* delta, int32_t* cand) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < V; i += (int64_t)gridDim.x * blockDim.x) {
    delta_clear(delta[i]);
    if (cand) cand[i] = -1;
  }
}

// ------------------------------------------------------------------ renumber
// Smallest member of every community.  A block takes one contiguous range
// of vertices and keeps the minimum of the communities it meets in a small
// shared table (open addressing, a few probes; a community that finds no
// slot updates the global minimum directly), flushed once: the few very
// large communities would otherwise serialise atomics on their counter.
constexpr int kMinHotLog = 9;
constexpr int kMinHot = 1 << kMinHotLog;
__global__ void __launch_bounds__(kThreads) min_member_kernel(int32_t V, const int32_t* comm, int32_t* minidx) {
  __shared__ int32_t hk[kMinHot], hv[kMinHot];
  for (int x = threadIdx.x; x < kMinHot; x += kThreads) { hk[x] = -1; hv[x] = 0x7fffffff; }
  __syncthreads();
  const int64_t per = ((int64_t)V + gridDim.x - 1) / gridDim.x;
  const int64_t i0 = (int64_t)blockIdx.x * per;
  const int64_t i1 = min((int64_t)V, i0 + per);
  for (int64_t i = i0 + threadIdx.x; i < i1; i += kThreads) {
    const int32_t c = comm[i];
    uint32_t h = hash_c(c, kMinHotLog);
    bool done = false;
    for (int p = 0; p < 8 && !done; ++p) {
      const int32_t prev = atomicCAS(&hk[h], -1, c);
      if (prev == -1 || prev == c) {
        atomicMin(&hv[h], (int32_t)i);
        done = true;
      }
      h = (h + 1) & (kMinHot - 1);
    }
    if (!done) atomicMin(&minidx[c], (int32_t)i);
  }
  __syncthreads();
  for (int x = threadIdx.x; x < kMinHot; x += kThreads)
    if (hk[x] >= 0) atomicMin(&minidx[hk[x]], hv[x]);
}

__global__ void head_flag_kernel(int32_t V, const int32_t* comm, const int32_t* minidx, uint32_t* flag) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < V) flag[i] = minidx[comm[i]] == (int32_t)i ? 1u : 0u;
}

__global__ void renumber_apply_kernel(int32_t V, const int32_t* comm, const uint32_t* flag, const uint32_t* pos,
                                      int32_t* newid_of_comm) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < V; i += (int64_t)gridDim.x * blockDim.x)
    if (flag[i]) newid_of_comm[comm[i]] = (int32_t)pos[i];
}

__global__ void gather_kernel(int32_t V, const int32_t* comm, const int32_t* newid_of_comm, int32_t* part) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < V; i += (int64_t)gridDim.x * blockDim.x)
    part[i] = newid_of_comm[comm[i]];
}

// ------------------------------------------------------------------ induce
__global__ void induce_keys_kernel(const int32_t* src, const int32_t* dst, const float* w, int64_t E,
                                   const int32_t* part, int B, uint64_t* keys, float* vals) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < E; e += (int64_t)gridDim.x * blockDim.x) {
    uint64_t a = (uint32_t)part[src[e]], b = (uint32_t)part[dst[e]];
    keys[e] = (a << B) | b;
    float x = w[e];
    vals[e] = x == 0.0f ? 1.0f : x;       // InducedGraphKernel.cu:38-39
  }
}

__global__ void run_head_kernel(const uint64_t* keys, int64_t n, uint32_t* head) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    head[i] = (i == 0 || keys[i - 1] != keys[i]) ? 1u : 0u;
}

__global__ void run_sum_kernel(const uint64_t* keys, const float* vals, int64_t n, int B, const uint32_t* pos,
                               const uint32_t* head, int32_t* osrc, int32_t* odst, double* wsum) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  bool valid = i < n;
  uint64_t mask = (B >= 64) ? ~0ull : ((1ull << B) - 1);
  uint64_t key = valid ? keys[i] : 0ull;
  int64_t r = valid ? (int64_t)pos[i] + (int64_t)head[i] - 1 : -1;
  if (valid && head[i]) {
    osrc[r] = (int32_t)(key >> B);
    odst[r] = (int32_t)(key & mask);
  }
  double s = seg_warp_sum<int64_t>(valid ? (double)vals[i] : 0.0, r);
  if (seg_warp_last<int64_t>(r, valid)) atomicAdd(&wsum[r], s);
}

// ------------------------------------------------------------------ modularity
// Community strength Kc (both endpoints of every entry) and internal weight
// Ain (2w for entries inside one community).  Few communities: block-private
// shared-memory sums flushed once per block; many: global atomics.
constexpr int kNmSmemMax = 4096;
// Lanes of a warp holding the same key add their values before one atomic:
// large communities (the last levels have few) would otherwise serialise on a
// handful of addresses.  Every lane gets its group's sum; the lowest lane of
// the group adds it.  Lanes with key < 0 take no part.
__device__ __forceinline__ void warp_group_add(double* arr, int32_t key, double x) {
  const unsigned full = 0xffffffffu;
  const unsigned peers = __match_any_sync(full, key);
  double sum = 0.0;
#pragma unroll
  for (int l = 0; l < 32; ++l) {
    const double v = __shfl_sync(full, x, l);
    if ((peers >> l) & 1u) sum += v;
  }
  if (key >= 0 && (threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(&arr[key], sum);
}

// Community ids of an entry's endpoints as accumulation keys: -1 (no part in
// the sums) for a lane past the end, and for an id outside [0, C), which also
// sets *bad when the caller passes a flag (callers that validated the ids on
// the host pass none).
__device__ __forceinline__ void nm_keys(const int32_t* part, const int32_t* src, const int32_t* dst, int64_t e,
                                        bool ok, int32_t C, uint32_t* bad, int32_t& a, int32_t& b) {
  a = ok ? part[src[e]] : -1;
  b = ok ? part[dst[e]] : -1;
  const bool oob = ok && ((uint32_t)a >= (uint32_t)C || (uint32_t)b >= (uint32_t)C);
  if (oob) {
    if (bad) atomicOr(bad, 1u);
    a = (uint32_t)a < (uint32_t)C ? a : -1;
    b = (uint32_t)b < (uint32_t)C ? b : -1;
  }
}

__global__ void __launch_bounds__(kThreads) nm_accum_smem_kernel(const int32_t* src, const int32_t* dst,
                                                                 const float* w, int64_t E, const int32_t* part,
                                                                 int32_t C, double* Kc, double* Ain, uint32_t* bad) {
  extern __shared__ __align__(16) unsigned char smem[];
  double* sK = reinterpret_cast<double*>(smem);
  double* sA = sK + C;
  for (int c = threadIdx.x; c < 2 * C; c += kThreads) sK[c] = 0.0;
  __syncthreads();
  // few communities: lanes with the same community add first (warp-uniform loop)
  for (int64_t e0 = blockIdx.x * (int64_t)blockDim.x; e0 < E; e0 += (int64_t)gridDim.x * blockDim.x) {
    const int64_t e = e0 + threadIdx.x;
    const bool ok = e < E;
    const double x = ok ? (double)w[e] : 0.0;
    int32_t a, b;
    nm_keys(part, src, dst, e, ok, C, bad, a, b);
    warp_group_add(sK, a, x);
    warp_group_add(sK, b, x);
    warp_group_add(sA, (a >= 0 && a == b) ? a : -1, 2.0 * x);
  }
  __syncthreads();
  for (int c = threadIdx.x; c < C; c += kThreads) {
    if (sK[c] != 0.0) atomicAdd(&Kc[c], sK[c]);
    if (sA[c] != 0.0) atomicAdd(&Ain[c], sA[c]);
  }
}

// Kc, Ain of modularity_fp64 for many communities: grid-stride over whole
// warps, warp-aggregated atomics.
__global__ void nm_accum_agg_kernel(const int32_t* src, const int32_t* dst, const float* w, int64_t E,
                                    const int32_t* part, int32_t C, double* Kc, double* Ain, uint32_t* bad) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t e0 = blockIdx.x * (int64_t)blockDim.x; e0 < E; e0 += stride) {
    const int64_t e = e0 + threadIdx.x;
    const bool ok = e < E;
    const double x = ok ? (double)w[e] : 0.0;
    int32_t a, b;
    nm_keys(part, src, dst, e, ok, C, bad, a, b);
    warp_group_add(Kc, a, x);
    warp_group_add(Kc, b, x);
    warp_group_add(Ain, (a >= 0 && a == b) ? a : -1, 2.0 * x);
  }
}

__global__ void nm_term_kernel(const double* Kc, const double* Ain, int32_t C, const double* twoW, double* t) {
  double tw = *twoW;
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < C; c += (int64_t)gridDim.x * blockDim.x) {
    double f = __ddiv_rn(Kc[c], tw);
    t[c] = tw > 0.0 ? __dsub_rn(__ddiv_rn(Ain[c], tw), __dmul_rn(f, f)) : 0.0;
  }
}

__global__ void iota_kernel(int32_t* x, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    x[i] = (int32_t)i;
}

__global__ void compose_kernel(int32_t* composed, const int32_t* part_level, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    composed[i] = part_level[composed[i]];
}

int sm_count() {
  static const int sms = [] {   // thread-safe one-time initialisation
    int dev = 0, n = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    return n > 0 ? n : 148;
  }();
  return sms;
}

unsigned sm_grid(int64_t n, int threads) {
  int sms = sm_count();
  int64_t g = (n + threads - 1) / threads;
  int64_t cap = (int64_t)sms * 16;
  if (g > cap) g = cap;
  return (unsigned)(g > 0 ? g : 1);
}

MoveArgs move_args(const LevelGraph& g, CommState& st) {
  MoveArgs P;
  P.list = nullptr; P.n = 0;
  P.off = g.off; P.col = g.col; P.cw = g.cw;
  P.comm = st.comm; P.tot = st.tot; P.size = st.size;
  P.kfrac = g.kfrac; P.k = g.k; P.loopw = g.loopw; P.has_loop = g.has_loop;
  P.next = st.next; P.cand = st.cand;
  P.delta = st.delta;
  P.ctl = st.ctl;
  P.k32 = g.k32;
  P.gid = st.gid;
  P.gdone = st.gdone;
  P.queue = nullptr;
  return P;
}

}  // namespace

// ============================================================================ host

bool validate_edges(const int32_t* src, const int32_t* dst, const float* w, int64_t E, int32_t V, Arena& a,
                    cudaStream_t s) {
  if (E == 0) return true;
  HiScope hs(a);
  uint32_t* bad = a.hi_n<uint32_t>(1);
  LVG_CUDA(cudaMemsetAsync(bad, 0, sizeof(uint32_t), s));
  validate_kernel<<<sm_grid(E, kThreads), kThreads, 0, s>>>(src, dst, w, E, V, bad);
  LVG_LAUNCH();
  uint32_t h = 0;
  LVG_CUDA(cudaMemcpyAsync(&h, bad, sizeof h, cudaMemcpyDeviceToHost, s));
  LVG_CUDA(cudaStreamSynchronize(s));
  return h == 0;
}

bool stream_load_level0(const int32_t* hsrc, const int32_t* hdst, const float* hw, int32_t* src, int32_t* dst,
                        float* w, int64_t E, int32_t V, int64_t chunk, PreCsr& pre, std::vector<cudaEvent_t>& evs,
                        Arena& a, cudaStream_t s, cudaStream_t copy) {
  pre = PreCsr();
  chunk = std::max<int64_t>(kGroup, (chunk + kGroup - 1) / kGroup * kGroup);
  const int64_t nchunks = (E + chunk - 1) / chunk;
  const size_t mark = a.lo;
  pre.off = a.lo_n<int64_t>((int64_t)V + 1);
  pre.col = a.lo_n<int32_t>(E);
  pre.cw = a.lo_n<float>(E);
  pre.k = a.lo_n<double>(V);
  pre.loopw = a.lo_n<float>(V);
  pre.has_loop = a.lo_n<uint8_t>(V);
  bool valid = false, bad = false;
  {
    HiScope hs(a);
    uint32_t* pos = a.hi_n<uint32_t>(E + 1);
    const int64_t ngroups = (E + kGroup - 1) / kGroup;
    double* gpart = a.hi_n<double>(ngroups);
    double* d_m = a.hi_n<double>(1);
    unsigned long long* chk = a.hi_n<unsigned long long>(3);   // flags, two fingerprint sums
    uint32_t* carry = a.hi_n<uint32_t>(nchunks + 1);
    LVG_CUDA(cudaMemsetAsync(pre.off, 0, sizeof(int64_t) * ((size_t)V + 1), s));
    LVG_CUDA(cudaMemsetAsync(pre.k, 0, sizeof(double) * std::max<int32_t>(V, 1), s));
    LVG_CUDA(cudaMemsetAsync(pre.loopw, 0, sizeof(float) * std::max<int32_t>(V, 1), s));
    LVG_CUDA(cudaMemsetAsync(pre.has_loop, 0, std::max<int32_t>(V, 1), s));
    LVG_CUDA(cudaMemsetAsync(chk, 0, 3 * sizeof(unsigned long long), s));
    LVG_CUDA(cudaMemsetAsync(carry, 0, sizeof(uint32_t), s));
    while ((int64_t)evs.size() < nchunks + 1) {
      cudaEvent_t ev;
      LVG_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
      evs.push_back(ev);
    }
    // the copies start once earlier work of the stream (which may still use
    // this memory) is done; chunk i's kernels start once its copies are
    LVG_CUDA(cudaEventRecord(evs[nchunks], s));
    LVG_CUDA(cudaStreamWaitEvent(copy, evs[nchunks], 0));
    // chunk i's copies are issued before chunk i-1's kernels, so that the
    // kernels overlap the next copy even when a copy from pageable memory
    // holds the host thread until it is staged
    auto issue_copy = [&](int64_t i) {
      const int64_t b = i * chunk, n = std::min(chunk, E - b);
      LVG_CUDA(cudaMemcpyAsync(src + b, hsrc + b, sizeof(int32_t) * n, cudaMemcpyHostToDevice, copy));
      LVG_CUDA(cudaMemcpyAsync(dst + b, hdst + b, sizeof(int32_t) * n, cudaMemcpyHostToDevice, copy));
      LVG_CUDA(cudaMemcpyAsync(w + b, hw + b, sizeof(float) * n, cudaMemcpyHostToDevice, copy));
      LVG_CUDA(cudaEventRecord(evs[i], copy));
    };
    issue_copy(0);
    for (int64_t i = 0; i < nchunks; ++i) {
      const int64_t b = i * chunk, n = std::min(chunk, E - b);
      if (i + 1 < nchunks) issue_copy(i + 1);
      LVG_CUDA(cudaStreamWaitEvent(s, evs[i], 0));
      pre_chunk_kernel<<<grid_for(n, kThreads), kThreads, 0, s>>>(src, dst, w, b, b + n, V, (uint32_t*)chk, chk + 1,
                                                                   (unsigned long long*)pre.off, pos);
      LVG_LAUNCH();
      scan_u32(pos + b, pos + b, n, a, s);
      pre_carry_kernel<<<1, 1, 0, s>>>(carry, i, pos + b + n);
      LVG_LAUNCH();
      pre_emit_kernel<<<grid_for(n, kThreads), kThreads, 0, s>>>(src, dst, w, b, b + n, V, pos, carry + i, pre.col,
                                                                  pre.cw, pre.k, pre.loopw, pre.has_loop);
      LVG_LAUNCH();
      pre_group_kernel<<<(unsigned)((n + kGroup - 1) / kGroup), kRedThreads, 0, s>>>(w + b, n, gpart + b / kGroup);
      LVG_LAUNCH();
    }
    tree_finish(gpart, ngroups, d_m, a, s);
    unsigned long long h[3] = {0, 0, 0};
    LVG_CUDA(cudaMemcpyAsync(h, chk, sizeof h, cudaMemcpyDeviceToHost, s));
    LVG_CUDA(cudaMemcpyAsync(&pre.m, d_m, sizeof(double), cudaMemcpyDeviceToHost, s));
    LVG_CUDA(cudaStreamSynchronize(s));
    bad = (h[0] & kBadEntry) != 0;
    valid = !bad && h[0] == 0 && h[1] == 0 && h[2] == 0;
    if (valid) {
      scan_i64(pre.off, pre.off, V, a, s);   // non-loop entries before each row
      LVG_CUDA(cudaMemcpyAsync(&pre.nnz, pre.off + V, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
      LVG_CUDA(cudaStreamSynchronize(s));
    }
  }
  if (!valid) {
    a.lo = mark;   // the list is not in that form: the level build makes the CSR
    pre = PreCsr();
  }
  pre.valid = valid;
  return !bad;
}

// Sort-free CSR build; returns false (and builds nothing) unless the level
// list is strictly sorted and symmetric.
static void set_move_attributes();

static bool build_csr_fast(LevelGraph& g, Arena& a, cudaStream_t s) {
  const int32_t V = g.V;
  const int64_t E = g.E;
  if (E >= ((int64_t)1 << 32) - 1) return false;
  HiScope hs(a);
  int64_t* rowstart = a.hi_n<int64_t>(V + 1);
  unsigned long long* chk = a.hi_n<unsigned long long>(3);   // flags, two fingerprint sums
  LVG_CUDA(cudaMemsetAsync(chk, 0, 3 * sizeof(unsigned long long), s));
  list_check_kernel<<<sm_grid(E, kThreads), kThreads, 0, s>>>(g.src, g.dst, g.w, E, (uint32_t*)chk, chk + 1);
  LVG_LAUNCH();
  unsigned long long h[3] = {0, 0, 0};
  LVG_CUDA(cudaMemcpyAsync(h, chk, sizeof h, cudaMemcpyDeviceToHost, s));
  LVG_CUDA(cudaStreamSynchronize(s));
  if (h[0] != 0 || h[1] != 0 || h[2] != 0) return false;
  LVG_CUDA(cudaMemsetAsync(rowstart, 0, sizeof(int64_t) * (V + 1), s));
  row_count_kernel<<<grid_for(E, kThreads), kThreads, 0, s>>>(g.src, E, rowstart);
  LVG_LAUNCH();
  scan_i64(rowstart, rowstart, V, a, s);
  uint32_t* pos = a.hi_n<uint32_t>(E + 1);
  nonloop_flag_kernel<<<sm_grid(E, kThreads), kThreads, 0, s>>>(g.src, g.dst, E, pos);
  LVG_LAUNCH();
  scan_u32(pos, pos, E, a, s);
  uint32_t nnz = 0;
  LVG_CUDA(cudaMemcpyAsync(&nnz, pos + E, sizeof nnz, cudaMemcpyDeviceToHost, s));
  LVG_CUDA(cudaStreamSynchronize(s));
  g.nnz = nnz;
  g.col = a.lo_n<int32_t>(nnz);
  g.cw = a.lo_n<float>(nnz);
  csr_fast_emit_kernel<<<grid_for(E, kThreads), kThreads, 0, s>>>(g.src, g.dst, g.w, E, pos, g.col, g.cw, g.k,
                                                                    g.loopw, g.has_loop);
  LVG_LAUNCH();
  row_off_kernel<<<sm_grid(V + 1, kThreads), kThreads, 0, s>>>(rowstart, pos, V, g.off);
  LVG_LAUNCH();
  return true;
}

void build_level(LevelGraph& g, const Tuning& t, Arena& a, cudaStream_t s) {
  const int32_t V = g.V;
  const int64_t E = g.E;
  const int64_t n = 2 * E;
  if (n >= ((int64_t)1 << 32)) throw Error(LVG_ERR_CAPACITY, "doubled edge list exceeds 2^32-1 entries");
  // per-vertex arrays (low end, level lifetime)
  const bool pre = g.pre && g.pre->valid;
  g.kfrac = a.lo_n<double>(V);
  double* d_m = a.lo_n<double>(1);
  if (pre) {   // level 0 built while it streamed in (stream_load_level0)
    g.off = g.pre->off;
    g.col = g.pre->col;
    g.cw = g.pre->cw;
    g.k = g.pre->k;
    g.loopw = g.pre->loopw;
    g.has_loop = g.pre->has_loop;
    g.nnz = g.pre->nnz;
    LVG_CUDA(cudaMemcpyAsync(d_m, &g.pre->m, sizeof(double), cudaMemcpyHostToDevice, s));
    g.sorted_symmetric = true;
  } else {
    g.off = a.lo_n<int64_t>(V + 1);
    g.k = a.lo_n<double>(V);
    g.loopw = a.lo_n<float>(V);
    g.has_loop = a.lo_n<uint8_t>(V);
    LVG_CUDA(cudaMemsetAsync(g.k, 0, sizeof(double) * std::max<int32_t>(V, 1), s));
    LVG_CUDA(cudaMemsetAsync(g.loopw, 0, sizeof(float) * std::max<int32_t>(V, 1), s));
    LVG_CUDA(cudaMemsetAsync(g.has_loop, 0, std::max<int32_t>(V, 1), s));
    tree_sum_f32(g.w, E, d_m, a, s);                                  // NeighbourCompute.cu:46
    g.sorted_symmetric = E > 0 && build_csr_fast(g, a, s);
  }
  if (!g.sorted_symmetric) {
    HiScope hs(a);
    const int B = std::max(1, bits_for(V));
    uint64_t* k0 = a.hi_n<uint64_t>(n);
    float* v0 = a.hi_n<float>(n);
    uint64_t* k1 = a.hi_n<uint64_t>(n);
    float* v1 = a.hi_n<float>(n);
    uint32_t* head = a.hi_n<uint32_t>(n + 1);
    uint32_t* pos = a.hi_n<uint32_t>(n + 1);
    int64_t* rowcnt = a.hi_n<int64_t>(V + 1);
    LVG_CUDA(cudaMemsetAsync(rowcnt, 0, sizeof(int64_t) * (V + 1), s));
    if (E > 0) {
      make_keys_kernel<<<sm_grid(E, kThreads), kThreads, 0, s>>>(g.src, g.dst, g.w, E, B, k0, v0);
      LVG_LAUNCH();
    }
    int which = radix_sort_pairs(k0, v0, k1, v1, n, 2 * B, a, s);   // NeighbourCompute.cu:82
    uint64_t* keys = which ? k1 : k0;
    float* vals = which ? v1 : v0;
    if (n > 0) {
      csr_scan_kernel<<<grid_for(n, kThreads), kThreads, 0, s>>>(keys, vals, n, B, head, rowcnt, g.k, g.loopw,
                                                                  g.has_loop);
      LVG_LAUNCH();
    }
    scan_u32(head, pos, n, a, s);
    scan_i64(rowcnt, g.off, V, a, s);
    int64_t nnz = 0;
    LVG_CUDA(cudaMemcpyAsync(&nnz, g.off + V, sizeof nnz, cudaMemcpyDeviceToHost, s));
    LVG_CUDA(cudaStreamSynchronize(s));
    g.nnz = nnz;
    // exact CSR on the low end
    g.col = a.lo_n<int32_t>(nnz);
    g.cw = a.lo_n<float>(nnz);
    double* wsum = a.hi_n<double>(nnz);
    LVG_CUDA(cudaMemsetAsync(wsum, 0, sizeof(double) * std::max<int64_t>(nnz, 1), s));
    if (n > 0) {
      csr_emit_kernel<<<grid_for(n, kThreads), kThreads, 0, s>>>(keys, vals, n, B, pos, head, g.col, wsum);
      LVG_LAUNCH();
    }
    if (nnz > 0) {
      to_float_kernel<<<sm_grid(nnz, kThreads), kThreads, 0, s>>>(wsum, g.cw, nnz);
      LVG_LAUNCH();
    }
  }
  LVG_CUDA(cudaMemcpyAsync(&g.m, d_m, sizeof(double), cudaMemcpyDeviceToHost, s));
  LVG_CUDA(cudaStreamSynchronize(s));
  // degree buckets (stable by vertex index)
  g.blist = a.lo_n<int32_t>(V);
  {
    HiScope hs(a);
    int64_t nblk = (V + 2047) / 2048;
    if (nblk == 0) nblk = 1;
    uint32_t* cnt = a.hi_n<uint32_t>(kNumBuckets * nblk + 1);
    bucket_count_kernel<<<(unsigned)nblk, kThreads, 0, s>>>(V, g.off, g.k, t.warp_max, t.block_max, cnt, nblk);
    LVG_LAUNCH();
    std::vector<uint32_t> host_cnt(kNumBuckets * nblk);
    LVG_CUDA(cudaMemcpyAsync(host_cnt.data(), cnt, sizeof(uint32_t) * kNumBuckets * nblk, cudaMemcpyDeviceToHost,
                             s));
    scan_u32(cnt, cnt, kNumBuckets * nblk, a, s);
    bucket_scatter_kernel<<<(unsigned)nblk, kThreads, 0, s>>>(V, g.off, g.k, t.warp_max, t.block_max, cnt, nblk,
                                                              g.blist);
    LVG_LAUNCH();
    LVG_CUDA(cudaStreamSynchronize(s));
    int64_t acc = 0;
    for (int b = 0; b < kNumBuckets; ++b) {
      int64_t c = 0;
      for (int64_t j = 0; j < nblk; ++j) c += host_cnt[b * nblk + j];
      g.nbucket[b] = c;
      g.bstart[b] = acc;
      acc += c;
    }
  }
  // sliced-ELL copies of the degree classes up to 32
  {
    static const int kG[4] = {4, 8, 16, 32};
    int64_t slots = 0;
    for (int b = kB4; b <= kB32; ++b) {
      g.ell_base[b] = slots;
      slots += g.nbucket[b] * kG[b - kB4];
    }
    g.ell_col = a.lo_n<int32_t>(slots);
    g.ell_w = a.lo_n<float>(slots);
    for (int b = kB4; b <= kB32; ++b) {
      int64_t nb = g.nbucket[b];
      if (nb == 0) continue;
      int G = kG[b - kB4];
      ell_fill_kernel<<<sm_grid(nb * G, kThreads), kThreads, 0, s>>>(g.blist + g.bstart[b], g.off, g.col, g.cw, nb,
                                                                      G, g.ell_col + g.ell_base[b],
                                                                      g.ell_w + g.ell_base[b]);
      LVG_LAUNCH();
    }
  }
  // k/2m and the class-ordered vertex facts of the thread kernels
  if (V > 0) {
    kfrac_kernel<<<sm_grid(V, kThreads), kThreads, 0, s>>>(V, g.k, g.m, g.gm, g.vgid, g.kfrac);
    LVG_LAUNCH();
  }
  {
    int64_t nitems = g.bstart[kB32] + g.nbucket[kB32] - g.bstart[kB4];
    g.ell_info = a.lo_n<VInfo>(nitems);
    if (nitems > 0) {
      vinfo_fill_kernel<<<sm_grid(nitems, kThreads), kThreads, 0, s>>>(g.blist + g.bstart[kB4], nitems, g.kfrac, g.k,
                                                                       g.loopw, g.has_loop, g.ell_info);
      LVG_LAUNCH();
    }
  }
  // tiles of the small-degree bucket
  g.ntiles = 0;
  const int64_t n0 = g.nbucket[kBTile];
  const int32_t* tlist = g.blist + g.bstart[kBTile];
  g.tile_start = a.lo_n<int32_t>(n0 + 2);
  if (n0 > 0) {
    HiScope hs(a);
    int64_t* cum = a.hi_n<int64_t>(n0 + 1);
    tile_cost_kernel<<<sm_grid(n0, kThreads), kThreads, 0, s>>>(tlist, n0, g.off, cum);
    LVG_LAUNCH();
    scan_i64(cum, cum, n0, a, s);
    tile_start_kernel<<<sm_grid(n0, kThreads), kThreads, 0, s>>>(cum, n0, g.tile_start);
    LVG_LAUNCH();
    int64_t last = 0;
    LVG_CUDA(cudaMemcpyAsync(&last, cum + n0 - 1, sizeof last, cudaMemcpyDeviceToHost, s));
    LVG_CUDA(cudaStreamSynchronize(s));
    g.ntiles = last / kTileCost + 1;
  }
  {
    HiScope hs(a);
    uint32_t* notint = a.hi_n<uint32_t>(1);
    LVG_CUDA(cudaMemsetAsync(notint, 0, sizeof(uint32_t), s));
    int_weights_kernel<<<sm_grid(std::max<int64_t>(g.nnz, V), kThreads), kThreads, 0, s>>>(g.cw, g.nnz, g.k, V,
                                                                                          notint);
    LVG_LAUNCH();
    uint32_t h = 0;
    LVG_CUDA(cudaMemcpyAsync(&h, notint, sizeof h, cudaMemcpyDeviceToHost, s));
    LVG_CUDA(cudaStreamSynchronize(s));
    g.int_acc = h == 0;
  }
  // the first pass gathers a neighbour's singleton total k as int32 when exact
  g.k32 = nullptr;
  if (g.int_acc && V > 0) {
    g.k32 = a.lo_n<int32_t>(V);
    k32_kernel<<<sm_grid(V, kThreads), kThreads, 0, s>>>(V, g.k, g.k32);
    LVG_LAUNCH();
  }
  // hubs: chunks of kHubChunk entries and ~kHubBucketTarget entries per bucket
  g.nchunk = 0;
  g.nhub_bucket = 0;
  const int64_t nhub = g.nbucket[kBHub];
  if (nhub > 0) {
    const int32_t* hubs = g.blist + g.bstart[kBHub];
    std::vector<int64_t> be(2 * nhub);
    {
      HiScope hs(a);
      int64_t* d_be = a.hi_n<int64_t>(2 * nhub);
      hub_info_kernel<<<grid_for(nhub, kThreads), kThreads, 0, s>>>(hubs, nhub, g.off, d_be);
      LVG_LAUNCH();
      LVG_CUDA(cudaMemcpyAsync(be.data(), d_be, sizeof(int64_t) * 2 * nhub, cudaMemcpyDeviceToHost, s));
      LVG_CUDA(cudaStreamSynchronize(s));
    }
    std::vector<int32_t> plog(nhub), cb0(nhub + 1), bb0(nhub + 1), chub, bhub;
    std::vector<int64_t> cbeg, cbo, cstg;
    int64_t noff = 0, nstg = 0;
    for (int64_t h = 0; h < nhub; ++h) {
      const int64_t d = be[2 * h + 1] - be[2 * h];
      int l = 0;
      while (l < kHubMaxBucketsLog && ((int64_t)kHubBucketTarget << l) < d) ++l;
      plog[h] = l;
      cb0[h] = (int32_t)chub.size();
      bb0[h] = (int32_t)bhub.size();
      for (int64_t b = be[2 * h]; b < be[2 * h + 1]; b += kHubChunk) {
        chub.push_back((int32_t)h);
        cbeg.push_back(b);
        cbo.push_back(noff);
        cstg.push_back(nstg + (b - be[2 * h]));
        noff += ((int64_t)1 << l) + 1;
      }
      nstg += d;
      bhub.insert(bhub.end(), (size_t)1 << l, (int32_t)h);
    }
    cb0[nhub] = (int32_t)chub.size();
    bb0[nhub] = (int32_t)bhub.size();
    g.nchunk = (int64_t)chub.size();
    g.nhub_bucket = (int64_t)bhub.size();
    g.chunk_hub = a.lo_n<int32_t>(g.nchunk);
    g.chunk_beg = a.lo_n<int64_t>(g.nchunk);
    g.chunk_cbo = a.lo_n<int64_t>(g.nchunk);
    g.chunk_stg = a.lo_n<int64_t>(g.nchunk);
    g.hub_plog = a.lo_n<int32_t>(nhub);
    g.hub_cb0 = a.lo_n<int32_t>(nhub + 1);
    g.hub_bb0 = a.lo_n<int32_t>(nhub + 1);
    g.bucket_hub = a.lo_n<int32_t>(g.nhub_bucket);
    g.cb_off = a.lo_n<uint16_t>(noff);
    g.stage = a.lo_n<unsigned long long>(nstg);
    g.hub_sawown = a.lo_n<uint32_t>(nhub);
    g.hub_part = a.lo_n<HubPartial>(g.nhub_bucket);
    LVG_CUDA(cudaMemcpyAsync(g.chunk_hub, chub.data(), sizeof(int32_t) * g.nchunk, cudaMemcpyHostToDevice, s));
    LVG_CUDA(cudaMemcpyAsync(g.chunk_beg, cbeg.data(), sizeof(int64_t) * g.nchunk, cudaMemcpyHostToDevice, s));
    LVG_CUDA(cudaMemcpyAsync(g.chunk_cbo, cbo.data(), sizeof(int64_t) * g.nchunk, cudaMemcpyHostToDevice, s));
    LVG_CUDA(cudaMemcpyAsync(g.chunk_stg, cstg.data(), sizeof(int64_t) * g.nchunk, cudaMemcpyHostToDevice, s));
    LVG_CUDA(cudaMemcpyAsync(g.hub_plog, plog.data(), sizeof(int32_t) * nhub, cudaMemcpyHostToDevice, s));
    LVG_CUDA(cudaMemcpyAsync(g.hub_cb0, cb0.data(), sizeof(int32_t) * (nhub + 1), cudaMemcpyHostToDevice, s));
    LVG_CUDA(cudaMemcpyAsync(g.hub_bb0, bb0.data(), sizeof(int32_t) * (nhub + 1), cudaMemcpyHostToDevice, s));
    LVG_CUDA(cudaMemcpyAsync(g.bucket_hub, bhub.data(), sizeof(int32_t) * g.nhub_bucket, cudaMemcpyHostToDevice,
                             s));
    LVG_CUDA(cudaMemsetAsync(g.hub_sawown, 0, sizeof(uint32_t) * nhub, s));
    LVG_CUDA(cudaStreamSynchronize(s));  // host vectors go out of scope
  }
  // singleton first pass: warp chunks of the rows longer than 32
  g.sp_nchunk = 0;
  g.sp_nmulti = 0;
  {
    const int64_t nl = g.nbucket[kBTile] + g.nbucket[kBBlock] + g.nbucket[kBHub];
    const int32_t* llist = g.blist + g.bstart[kBTile];
    if (nl > 0) {
      HiScope hs(a);
      uint32_t* cnt = a.hi_n<uint32_t>(nl + 1);
      uint32_t* mul = a.hi_n<uint32_t>(nl + 1);
      sp_count_kernel<<<sm_grid(nl, kThreads), kThreads, 0, s>>>(llist, nl, g.off, cnt, mul);
      LVG_LAUNCH();
      scan_u32(cnt, cnt, nl, a, s);
      scan_u32(mul, mul, nl, a, s);
      uint32_t tot[2] = {0, 0};
      LVG_CUDA(cudaMemcpyAsync(&tot[0], cnt + nl, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
      LVG_CUDA(cudaMemcpyAsync(&tot[1], mul + nl, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
      LVG_CUDA(cudaStreamSynchronize(s));
      g.sp_nchunk = tot[0];
      g.sp_nmulti = tot[1];
      g.sp_chunk = a.lo_n<int2>(g.sp_nchunk);
      g.sp_multi = a.lo_n<int2>(g.sp_nmulti);
      g.sp_part = a.lo_n<HubPartial>(g.sp_nmulti > 0 ? g.sp_nchunk : 0);
      sp_fill_kernel<<<sm_grid(nl, kThreads), kThreads, 0, s>>>(llist, nl, g.off, cnt, mul, g.sp_chunk, g.sp_multi);
      LVG_LAUNCH();
    }
  }
  g.block_max = t.block_max;
  set_move_attributes();
}

void alloc_state(const LevelGraph& g, CommState& st, Arena& a) {
  const int32_t V = g.V;
  // comm, tot and size are gathered per entry / per candidate: keep them
  // adjacent so that one L2 persistence window covers them
  st.tot = a.lo_n<double>(V);
  st.comm = a.lo_n<int32_t>(V);
  st.size = a.lo_n<int32_t>(V);
  st.hot_bytes = (size_t)((char*)(st.size + std::max<int32_t>(V, 1)) - (char*)st.tot);
  st.next = a.lo_n<int32_t>(V);
  st.in = a.lo_n<double>(V);
  st.delta = a.lo_n<Delta>(V);
  st.cand = a.lo_n<int32_t>(V);
  st.ngroups = (V + kGroup - 1) / kGroup;
  if (st.ngroups == 0) st.ngroups = 1;
  st.partials = a.lo_n<double>(st.ngroups);
  st.partials2 = a.lo_n<double>((st.ngroups + kGroup - 1) / kGroup);
  st.ctl = a.lo_n<PassCtl>(1);
  st.queue = a.lo_n<unsigned long long>(kQueueSlots);
}

// Q of the committed state through the fixed tree into *dst.
static void q_tail(const CommState& st, double* dst, cudaStream_t s, bool respect_ctl) {
  const double* p = st.partials;
  int64_t np = st.ngroups;
  if (np > kGroup) {
    int64_t nb = (np + kGroup - 1) / kGroup;
    tree_level_ctl_kernel<<<(unsigned)nb, kRedThreads, 0, s>>>(p, np, st.partials2, st.ctl, respect_ctl ? 1 : 0);
    LVG_LAUNCH();
    p = st.partials2;
    np = nb;
  }
  if (respect_ctl) {
    ctl_pass_kernel<<<1, kRedThreads, 0, s>>>(p, np, st.ctl);
  } else {
    ctl_q_kernel<<<1, kRedThreads, 0, s>>>(p, np, dst);
  }
  LVG_LAUNCH();
}

void init_state(const LevelGraph& g, CommState& st, double lower, double pass_min, int32_t max_passes, Arena& a,
                cudaStream_t s) {
  (void)a;
  const int32_t V = g.V;
  if (V > 0) {
    init_state_kernel<<<sm_grid(V, kThreads), kThreads, 0, s>>>(V, g.k, g.loopw, g.m, g.kfrac, st.comm, st.next,
                                                                st.tot, st.in, st.size, st.delta, st.cand);
    LVG_LAUNCH();
  }
  ctl_init_kernel<<<1, 1, 0, s>>>(st.ctl, lower, pass_min, max_passes);
  LVG_LAUNCH();
  launch_q(g, st, &st.ctl->q_prev, s);
}

void launch_q(const LevelGraph& g, CommState& st, double* dst, cudaStream_t s) {
  commit_kernel<kCommitInit><<<(unsigned)st.ngroups, kRedThreads, 0, s>>>(
      g.V, g.m, st.comm, st.next, st.tot, st.in, st.size, st.delta, g.k, st.partials, st.ctl);
  LVG_LAUNCH();
  q_tail(st, dst, s, false);
}

// Dynamic shared memory limits of the move kernels, set before any capture.
// Dynamic shared memory limits of the move kernels, set once per device
// before any capture.
static void set_move_attributes() {
  constexpr int kDevs = 64;
  static std::mutex mu;
  static bool done[kDevs] = {};
  int dev = 0;
  LVG_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(mu);   // contexts on several host threads
  if (dev >= 0 && dev < kDevs && done[dev]) return;
  LVG_CUDA(cudaFuncSetAttribute(move_tile_kernel<int>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)sizeof(TileSmem<int>)));
  LVG_CUDA(cudaFuncSetAttribute(move_tile_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)sizeof(TileSmem<double>)));
  LVG_CUDA(cudaFuncSetAttribute(move_tile_packed_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)sizeof(TilePackedSmem)));
  LVG_CUDA(cudaFuncSetAttribute(hub_agg_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)agg_smem_bytes<true>()));
  LVG_CUDA(cudaFuncSetAttribute(hub_agg_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)agg_smem_bytes<false>()));
  // block bands: up to 2 * 8192 slots of int32 key + f64 sum (block_max <= 8192)
  const int big = (int)((size_t)16384 * (sizeof(double) + sizeof(int32_t)));
  LVG_CUDA(cudaFuncSetAttribute(move_block_kernel<int, 128>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  LVG_CUDA(cudaFuncSetAttribute(move_block_kernel<int, 256>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  LVG_CUDA(cudaFuncSetAttribute(move_block_kernel<double, 128>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  LVG_CUDA(cudaFuncSetAttribute(move_block_kernel<double, 256>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  if (dev >= 0 && dev < kDevs) done[dev] = true;
}

template <typename Acc>
static void launch_tiles(const LevelGraph& g, MoveArgs P, cudaStream_t s) {
  size_t smem = sizeof(TileSmem<Acc>);
  int per_sm = (int)((227u * 1024u) / (smem + 1024));
  if (per_sm < 1) per_sm = 1;
  int64_t grid = std::min<int64_t>(g.ntiles, (int64_t)sm_count() * per_sm);
  move_tile_kernel<Acc><<<(unsigned)std::max<int64_t>(grid, 1), kThreads, smem, s>>>(P, g.tile_start, g.ntiles);
  LVG_LAUNCH();
}

template <int D>
static void launch_thread(const LevelGraph& g, MoveArgs P, int bucket, cudaStream_t s) {
  EllArgs L;
  L.n = g.nbucket[bucket];
  if (L.n == 0) return;
  L.col = g.ell_col + g.ell_base[bucket];
  L.w = g.ell_w + g.ell_base[bucket];
  L.list = g.blist + g.bstart[bucket];
  L.info = g.ell_info + (g.bstart[bucket] - g.bstart[kB4]);
  int64_t blocks = std::min<int64_t>((L.n + kThreads - 1) / kThreads, (int64_t)sm_count() * 8);
  move_thread_kernel<D><<<(unsigned)std::max<int64_t>(blocks, 1), kThreads, 0, s>>>(P, L);
  LVG_LAUNCH();
}

// The degree classes are independent within a pass (each writes only its own
// vertices' decisions and atomically adds into the deltas), so the small-grid
// classes run on side streams, forked from and joined back into `s`.
void launch_moves(const LevelGraph& g, CommState& st, cudaStream_t s, const SideStreams* ss) {
  MoveArgs P = move_args(g, st);
  // batched runs: the block-per-item kernels are persistent and pull their
  // items from device counters (one per launch), zeroed before the fork
  unsigned long long* q = (st.gid && st.queue) ? st.queue : nullptr;
  if (q) LVG_CUDA(cudaMemsetAsync(q, 0, sizeof(unsigned long long) * kQueueSlots, s));
  cudaStream_t sh = s, sb = s, st2 = s;
  if (ss) {
    LVG_CUDA(cudaEventRecord(ss->fork, s));
    for (int k = 0; k < 3; ++k) LVG_CUDA(cudaStreamWaitEvent(ss->side[k], ss->fork, 0));
    sh = ss->side[0]; sb = ss->side[1]; st2 = ss->side[2];
  }
  const int64_t nhub = g.nbucket[kBHub];
  if (nhub > 0) {
    HubArgs H;
    H.hubs = g.blist + g.bstart[kBHub];
    H.chunk_hub = g.chunk_hub; H.chunk_beg = g.chunk_beg; H.chunk_cbo = g.chunk_cbo; H.chunk_stg = g.chunk_stg;
    H.hub_plog = g.hub_plog; H.hub_cb0 = g.hub_cb0; H.hub_bb0 = g.hub_bb0; H.bucket_hub = g.bucket_hub;
    H.cb_off = g.cb_off; H.stage = g.stage; H.sawown = g.hub_sawown; H.part = g.hub_part;
    H.nbucket = g.nhub_bucket;
    hub_part_kernel<<<(unsigned)g.nchunk, kHubPartThreads, 0, sh>>>(P, H);
    LVG_LAUNCH();
    const size_t smem = g.int_acc ? agg_smem_bytes<true>() : agg_smem_bytes<false>();
    const int per_sm = std::max(1, std::min(8, (int)((227u * 1024u) / (smem + 1024))));
    const int64_t grid = std::min<int64_t>(g.nhub_bucket, (int64_t)sm_count() * per_sm);
    MoveArgs PA = P;
    PA.queue = q ? q + 0 : nullptr;
    if (g.int_acc) hub_agg_kernel<true><<<(unsigned)grid, kThreads, smem, sh>>>(PA, H);
    else hub_agg_kernel<false><<<(unsigned)grid, kThreads, smem, sh>>>(PA, H);
    LVG_LAUNCH();
    hub_decide_kernel<<<grid_for(nhub, 128), 128, 0, sh>>>(P, H, nhub);
    LVG_LAUNCH();
  }
  if (g.nbucket[kBBlock] > 0) {
    MoveArgs Q = P;
    Q.list = g.blist + g.bstart[kBBlock];
    Q.n = g.nbucket[kBBlock];
    // degree bands (lo, hi], hi = 1024, 2048, ..., each with a table of 2 hi slots
    int64_t lo = 0;
    int band = 0;
    for (int64_t hi = 1024; lo < g.block_max; hi *= 2, ++band) {
      Q.queue = q ? q + 2 + std::min(band, kQueueSlots - 3) : nullptr;
      const int64_t h = std::min<int64_t>(hi, g.block_max);
      int lg = 5;
      while (((int64_t)1 << lg) < 2 * h) ++lg;
      const size_t slot = g.int_acc ? sizeof(int32_t) + sizeof(int32_t) : sizeof(double) + sizeof(int32_t);
      const size_t smem = ((size_t)1 << lg) * slot;
      const bool narrow = h <= 1024;
      const unsigned grid = (unsigned)std::min<int64_t>(Q.n, (int64_t)sm_count() * (narrow ? 16 : 8));
      if (g.int_acc && narrow) move_block_kernel<int, 128><<<grid, 128, smem, sb>>>(Q, lg, lo, h);
      else if (g.int_acc) move_block_kernel<int, 256><<<grid, 256, smem, sb>>>(Q, lg, lo, h);
      else if (narrow) move_block_kernel<double, 128><<<grid, 128, smem, sb>>>(Q, lg, lo, h);
      else move_block_kernel<double, 256><<<grid, 256, smem, sb>>>(Q, lg, lo, h);
      LVG_LAUNCH();
      lo = h;
    }
  }
  if (g.ntiles > 0) {
    MoveArgs Q = P;
    Q.list = g.blist + g.bstart[kBTile];
    Q.n = g.nbucket[kBTile];
    if (g.int_acc && g.V <= kTilePackedMaxComm) {
      Q.queue = q ? q + 1 : nullptr;
      const size_t smem = sizeof(TilePackedSmem);
      const int per_sm = std::max(1, std::min(8, (int)((227u * 1024u) / (smem + 1024))));
      const int64_t grid = std::min<int64_t>(g.ntiles, (int64_t)sm_count() * per_sm);
      move_tile_packed_kernel<<<(unsigned)std::max<int64_t>(grid, 1), kThreads, smem, st2>>>(Q, g.tile_start,
                                                                                            g.ntiles);
      LVG_LAUNCH();
    } else if (g.int_acc) {
      launch_tiles<int>(g, Q, st2);
    } else {
      launch_tiles<double>(g, Q, st2);
    }
  }
  launch_thread<32>(g, P, kB32, s);
  launch_thread<16>(g, P, kB16, s);
  launch_thread<8>(g, P, kB8, s);
  launch_thread<4>(g, P, kB4, s);
  if (ss) {
    for (int k = 0; k < 3; ++k) {
      LVG_CUDA(cudaEventRecord(ss->join[k], ss->side[k]));
      LVG_CUDA(cudaStreamWaitEvent(s, ss->join[k], 0));
    }
  }
}

template <int D>
static void launch_sp_thread(const LevelGraph& g, MoveArgs P, int bucket, cudaStream_t s) {
  EllArgs L;
  L.n = g.nbucket[bucket];
  if (L.n == 0) return;
  L.col = g.ell_col + g.ell_base[bucket];
  L.w = g.ell_w + g.ell_base[bucket];
  L.list = g.blist + g.bstart[bucket];
  L.info = g.ell_info + (g.bstart[bucket] - g.bstart[kB4]);
  const int64_t vper_block = (int64_t)kThreads / D;
  int64_t blocks = std::min<int64_t>((L.n + vper_block - 1) / vper_block, (int64_t)sm_count() * 16);
  sp_thread_kernel<D><<<(unsigned)std::max<int64_t>(blocks, 1), kThreads, 0, s>>>(P, L);
  LVG_LAUNCH();
}

void launch_moves_singleton(const LevelGraph& g, CommState& st, cudaStream_t s, const SideStreams* ss) {
  MoveArgs P = move_args(g, st);
  cudaStream_t sc = s;
  if (ss) {
    LVG_CUDA(cudaEventRecord(ss->fork, s));
    LVG_CUDA(cudaStreamWaitEvent(ss->side[0], ss->fork, 0));
    sc = ss->side[0];
  }
  if (g.sp_nchunk > 0) {
    const int64_t blocks = std::min<int64_t>((g.sp_nchunk + kThreads / 32 - 1) / (kThreads / 32),
                                             (int64_t)sm_count() * 16);
    sp_chunk_kernel<<<(unsigned)std::max<int64_t>(blocks, 1), kThreads, 0, sc>>>(P, g.sp_chunk, g.sp_nchunk,
                                                                                 g.sp_part);
    LVG_LAUNCH();
    if (g.sp_nmulti > 0) {
      sp_combine_kernel<<<sm_grid(g.sp_nmulti, kThreads), kThreads, 0, sc>>>(P, g.sp_multi, g.sp_nmulti, g.sp_part);
      LVG_LAUNCH();
    }
  }
  launch_sp_thread<32>(g, P, kB32, s);
  launch_sp_thread<16>(g, P, kB16, s);
  launch_sp_thread<8>(g, P, kB8, s);
  launch_sp_thread<4>(g, P, kB4, s);
  if (ss) {
    LVG_CUDA(cudaEventRecord(ss->join[0], ss->side[0]));
    LVG_CUDA(cudaStreamWaitEvent(s, ss->join[0], 0));
  }
}

void launch_pass(const LevelGraph& g, CommState& st, cudaStream_t s, const SideStreams* ss) {
  launch_moves(g, st, s, ss);
  launch_commit(g, st, s);
}

void launch_commit(const LevelGraph& g, CommState& st, cudaStream_t s) {
  commit_kernel<kCommitPass><<<(unsigned)st.ngroups, kRedThreads, 0, s>>>(
      g.V, g.m, st.comm, st.next, st.tot, st.in, st.size, st.delta, g.k, st.partials, st.ctl);
  LVG_LAUNCH();
  q_tail(st, nullptr, s, true);
}

void launch_merge(const LevelGraph& g, CommState& st, cudaStream_t s) {
  const int32_t V = g.V;
  if (V > 0) {
    merge_kernel<<<sm_grid(V, kThreads), kThreads, 0, s>>>(V, st.comm, st.next, st.cand, g.k, g.loopw, st.delta);
    LVG_LAUNCH();
  }
  commit_kernel<kCommitForce><<<(unsigned)st.ngroups, kRedThreads, 0, s>>>(
      V, g.m, st.comm, st.next, st.tot, st.in, st.size, st.delta, g.k, st.partials, st.ctl);
  LVG_LAUNCH();
  q_tail(st, &st.ctl->q_ret, s, false);
}

void set_state_from(const LevelGraph& g, CommState& st, const int32_t* d_comm, cudaStream_t s) {
  const int32_t V = g.V;
  if (V == 0) return;
  LVG_CUDA(cudaMemsetAsync(st.tot, 0, sizeof(double) * V, s));
  LVG_CUDA(cudaMemsetAsync(st.in, 0, sizeof(double) * V, s));
  LVG_CUDA(cudaMemsetAsync(st.size, 0, sizeof(int32_t) * V, s));
  set_state_kernel<<<sm_grid(V, kThreads), kThreads, 0, s>>>(V, d_comm, g.k, g.loopw, st.comm, st.next, st.tot,
                                                             st.in, st.size);
  LVG_LAUNCH();
  clear_deltas(g, st, s);
}

void reset_ctl(CommState& st, double lower, double pass_min, int32_t max_passes, cudaStream_t s) {
  ctl_init_kernel<<<1, 1, 0, s>>>(st.ctl, lower, pass_min, max_passes);
  LVG_LAUNCH();
}

void clear_deltas(const LevelGraph& g, CommState& st, cudaStream_t s) {
  if (g.V == 0) return;
  clear_deltas_kernel<<<sm_grid(g.V, kThreads), kThreads, 0, s>>>(g.V, st.delta, st.cand);
  LVG_LAUNCH();
}

int32_t renumber(const LevelGraph& g, const int32_t* comm, int32_t* part, Arena& a, cudaStream_t s) {
  const int32_t V = g.V;
  if (V == 0) return 0;
  HiScope hs(a);
  int32_t* minidx = a.hi_n<int32_t>(V);
  uint32_t* flag = a.hi_n<uint32_t>(V + 1);
  uint32_t* pos = a.hi_n<uint32_t>(V + 1);
  LVG_CUDA(cudaMemsetAsync(minidx, 0x7f, sizeof(int32_t) * V, s));
  min_member_kernel<<<sm_grid(V, kThreads), kThreads, 0, s>>>(V, comm, minidx);
  LVG_LAUNCH();
  head_flag_kernel<<<grid_for(V, kThreads), kThreads, 0, s>>>(V, comm, minidx, flag);
  LVG_LAUNCH();
  scan_u32(flag, pos, V, a, s);
  renumber_apply_kernel<<<sm_grid(V, kThreads), kThreads, 0, s>>>(V, comm, flag, pos, minidx);
  LVG_LAUNCH();
  gather_kernel<<<sm_grid(V, kThreads), kThreads, 0, s>>>(V, comm, minidx, part);
  LVG_LAUNCH();
  uint32_t C = 0;
  LVG_CUDA(cudaMemcpyAsync(&C, pos + V, sizeof C, cudaMemcpyDeviceToHost, s));
  LVG_CUDA(cudaStreamSynchronize(s));
  return (int32_t)C;
}

int64_t induce(const LevelGraph& g, const int32_t* part, int32_t C, int32_t** out_src, int32_t** out_dst,
               float** out_w, Arena& a, cudaStream_t s, PreCsr* next, int32_t mode) {
  const int64_t E = g.E;
  if (E >= ((int64_t)1 << 32)) throw Error(LVG_ERR_CAPACITY, "level edge list exceeds 2^32-1 entries");
  // the output stays in high scratch for the caller; temporaries are released below it
  int32_t* osrc = a.hi_n<int32_t>(E);
  int32_t* odst = a.hi_n<int32_t>(E);
  float* ow = a.hi_n<float>(E);
  int64_t cnt = 0;
  if (next) {
    *next = PreCsr();
    if (g.sorted_symmetric) {
      next->off = a.hi_n<int64_t>((int64_t)C + 1);
      next->col = a.hi_n<int32_t>(E);
      next->cw = a.hi_n<float>(E);
      next->k = a.hi_n<double>(C);
      next->loopw = a.hi_n<float>(C);
      next->has_loop = a.hi_n<uint8_t>(C);
    }
  }
  // automatic: by transposition (measured on one B200, R-MAT scale 25: level 0
  // 1.05 G -> 0.68 G entries 156 -> 106 ms; level 1, where most entries merge,
  // 46 -> 48 ms; the LFR n = 2^20 levels 2.2 -> 1.9 and 1.7 -> 1.5 ms)
  // (a sort-free method that lacks arena room declines, and the next one is tried)
  const bool by_tx = mode == kCoarsenTransposed || mode == kCoarsenAuto;
  if ((by_tx && induce_transposed(g, part, C, osrc, odst, ow, &cnt, next, a, s)) ||
      (mode != kCoarsenSort && induce_sorted(g, part, C, osrc, odst, ow, &cnt, next, a, s))) {
    *out_src = osrc;
    *out_dst = odst;
    *out_w = ow;
    return cnt;
  }
  {
    HiScope hs(a);
    const int B = std::max(1, bits_for(C));
    uint64_t* k0 = a.hi_n<uint64_t>(E);
    float* v0 = a.hi_n<float>(E);
    uint64_t* k1 = a.hi_n<uint64_t>(E);
    float* v1 = a.hi_n<float>(E);
    uint32_t* head = a.hi_n<uint32_t>(E + 1);
    uint32_t* pos = a.hi_n<uint32_t>(E + 1);
    double* wsum = a.hi_n<double>(E);
    if (E > 0) {
      induce_keys_kernel<<<sm_grid(E, kThreads), kThreads, 0, s>>>(g.src, g.dst, g.w, E, part, B, k0, v0);
      LVG_LAUNCH();
    }
    int which = radix_sort_pairs(k0, v0, k1, v1, E, 2 * B, a, s);   // InducedGraphKernel.cu:91
    uint64_t* keys = which ? k1 : k0;
    float* vals = which ? v1 : v0;
    if (E > 0) {
      run_head_kernel<<<sm_grid(E, kThreads), kThreads, 0, s>>>(keys, E, head);
      LVG_LAUNCH();
    }
    scan_u32(head, pos, E, a, s);
    uint32_t n_out = 0;
    LVG_CUDA(cudaMemcpyAsync(&n_out, pos + E, sizeof n_out, cudaMemcpyDeviceToHost, s));
    LVG_CUDA(cudaStreamSynchronize(s));
    cnt = n_out;
    LVG_CUDA(cudaMemsetAsync(wsum, 0, sizeof(double) * std::max<int64_t>(cnt, 1), s));
    if (E > 0) {
      run_sum_kernel<<<grid_for(E, kThreads), kThreads, 0, s>>>(keys, vals, E, B, pos, head, osrc, odst, wsum);
      LVG_LAUNCH();
    }
    if (cnt > 0) {
      to_float_kernel<<<sm_grid(cnt, kThreads), kThreads, 0, s>>>(wsum, ow, cnt);
      LVG_LAUNCH();
    }
    LVG_CUDA(cudaStreamSynchronize(s));
  }
  *out_src = osrc;
  *out_dst = odst;
  *out_w = ow;
  return cnt;
}

// Kc and Ain of a list known to be symmetric (every (u, v, w) has its
// (v, u, w)) and sorted by source: the destination side of Kc equals the
// source side, so each entry adds 2w to its source's community only, and 2w
// to Ain when both ends share a community.  Lanes holding entries of one
// source row add them by a segmented warp scan; the last lane of each row
// piece makes one atomic update of each sum -- a few updates per row instead
// of one per entry, and no shuffle loop over all 32 lanes.
//
// The row pieces then add into a small block-private table of communities in
// shared memory (open addressing, a few probes; a community that finds no
// slot adds to the global sums directly), flushed once per block.  The last
// levels leave a few very large communities, and one global atomic per row
// piece into those few addresses would serialise at the L2: with the table
// each block makes one global update per large community.  Each block takes
// one contiguous range of the list (whole 256-entry steps, so every warp
// stays converged), whose rows meet the same large communities again and
// again.
constexpr int kNmHotLog = 9;        // 512 slots: 10 KB, eight blocks per SM
constexpr int kNmHot = 1 << kNmHotLog;
constexpr int kNmHotProbes = 8;
constexpr int kNmSymBlocksPerSm = 8;

__device__ __forceinline__ void nm_hot_add(int32_t* hk, double* hK, double* hA, double* Kc, double* Ain, int32_t a,
                                           double kin, double ain) {
  uint32_t h = hash_c(a, kNmHotLog);
  for (int p = 0; p < kNmHotProbes; ++p) {
    const int32_t prev = atomicCAS(&hk[h], -1, a);
    if (prev == -1 || prev == a) {
      atomicAdd(&hK[h], kin);
      if (ain != 0.0) atomicAdd(&hA[h], ain);
      return;
    }
    h = (h + 1) & (kNmHot - 1);
  }
  atomicAdd(&Kc[a], kin);
  if (ain != 0.0) atomicAdd(&Ain[a], ain);
}

__global__ void __launch_bounds__(kThreads) nm_accum_sym_kernel(const int32_t* src, const int32_t* dst,
                                                                const float* w, int64_t E, const int32_t* part,
                                                                double* Kc, double* Ain) {
  __shared__ int32_t hk[kNmHot];
  __shared__ double hK[kNmHot], hA[kNmHot];
  for (int x = threadIdx.x; x < kNmHot; x += kThreads) { hk[x] = -1; hK[x] = 0.0; hA[x] = 0.0; }
  __syncthreads();
  const int64_t steps = (E + kThreads - 1) / kThreads;
  const int64_t per = (steps + gridDim.x - 1) / gridDim.x;
  const int64_t s0 = (int64_t)blockIdx.x * per;
  const int64_t s1 = min(steps, s0 + per);
  for (int64_t st = s0; st < s1; ++st) {
    const int64_t e = st * kThreads + threadIdx.x;
    const bool ok = e < E;
    const int32_t u = ok ? src[e] : -1;
    const double x = ok ? 2.0 * (double)w[e] : 0.0;
    const int32_t a = ok ? part[u] : -1, b = ok ? part[dst[e]] : -1;
    const double kin = seg_warp_sum<int32_t>(x, u);
    const double ain = seg_warp_sum<int32_t>(a == b ? x : 0.0, u);
    if (seg_warp_last<int32_t>(u, ok)) nm_hot_add(hk, hK, hA, Kc, Ain, a, kin, ain);
  }
  __syncthreads();
  for (int x = threadIdx.x; x < kNmHot; x += kThreads) {
    const int32_t a = hk[x];
    if (a >= 0) {
      atomicAdd(&Kc[a], hK[x]);
      if (hA[x] != 0.0) atomicAdd(&Ain[a], hA[x]);
    }
  }
}

// Raises the dynamic shared memory limit of nm_accum_smem_kernel on the
// current device to at least `smem` bytes.  The limit only ever grows, under
// one lock shared by every caller, so a launch never finds it lowered by a
// smaller request made in between.
static void nm_smem_attr(size_t smem) {
  if (smem <= 48 * 1024) return;
  constexpr int kDevs = 64;
  static std::mutex mu;
  static size_t attr[kDevs] = {};
  int dev = 0;
  LVG_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(mu);
  if (dev >= 0 && dev < kDevs && smem <= attr[dev]) return;
  LVG_CUDA(cudaFuncSetAttribute(nm_accum_smem_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  if (dev >= 0 && dev < kDevs) attr[dev] = smem;
}

// Kc and Ain of every community: shared-memory sums when they fit, else
// warp-aggregated global atomics.
static void nm_accum(const int32_t* src, const int32_t* dst, const float* w, int64_t E, int32_t C,
                     const int32_t* part, double* Kc, double* Ain, uint32_t* bad, cudaStream_t s) {
  if (E <= 0) return;
  if (C <= kNmSmemMax) {
    const size_t smem = sizeof(double) * 2 * (size_t)C;
    nm_smem_attr(smem);
    nm_accum_smem_kernel<<<sm_grid(E, kThreads), kThreads, smem, s>>>(src, dst, w, E, part, C, Kc, Ain, bad);
  } else {
    nm_accum_agg_kernel<<<sm_grid(E, kThreads), kThreads, 0, s>>>(src, dst, w, E, part, C, Kc, Ain, bad);
  }
  LVG_LAUNCH();
}

double modularity_fp64(const int32_t* src, const int32_t* dst, const float* w, int64_t E, int32_t C,
                       const int32_t* part, Arena& a, cudaStream_t s, bool symmetric) {
  HiScope hs(a);
  double* Kc = a.hi_n<double>(C);
  double* Ain = a.hi_n<double>(C);
  double* t = a.hi_n<double>(C);
  double* twoW = a.hi_n<double>(2);
  LVG_CUDA(cudaMemsetAsync(Kc, 0, sizeof(double) * std::max(C, 1), s));
  LVG_CUDA(cudaMemsetAsync(Ain, 0, sizeof(double) * std::max(C, 1), s));
  if (symmetric && E > 0 && C > kNmSmemMax) {
    const unsigned grid = std::min<unsigned>(grid_for(E, kThreads), (unsigned)(sm_count() * kNmSymBlocksPerSm));
    nm_accum_sym_kernel<<<grid, kThreads, 0, s>>>(src, dst, w, E, part, Kc, Ain);
    LVG_LAUNCH();
  } else {
    nm_accum(src, dst, w, E, C, part, Kc, Ain, nullptr, s);   // ids checked on the host
  }
  tree_sum_f64(Kc, C, twoW, a, s);
  nm_term_kernel<<<sm_grid(C, kThreads), kThreads, 0, s>>>(Kc, Ain, C, twoW, t);
  LVG_LAUNCH();
  tree_sum_f64(t, C, twoW + 1, a, s);
  double q = 0.0;
  LVG_CUDA(cudaMemcpyAsync(&q, twoW + 1, sizeof q, cudaMemcpyDeviceToHost, s));
  LVG_CUDA(cudaStreamSynchronize(s));
  return q;
}

// The modularity kernels of modularity_fp64 with every scratch array given by
// the caller (used by the allocation-free entry point).  C <= 2048 * 2048.
// Community ids outside [0, C) take no part in the sums and set *bad.
void modularity_fp64_scratch(const int32_t* src, const int32_t* dst, const float* w, int64_t E, int32_t C,
                             const int32_t* part, double* Kc, double* Ain, double* t, double* partials,
                             double* twoW_q, uint32_t* bad, cudaStream_t s) {
  LVG_CUDA(cudaMemsetAsync(Kc, 0, sizeof(double) * C, s));
  LVG_CUDA(cudaMemsetAsync(Ain, 0, sizeof(double) * C, s));
  nm_accum(src, dst, w, E, C, part, Kc, Ain, bad, s);
  // the fixed tree of tree_sum_f64, partials from the caller
  auto tree = [&](const double* x, double* out) {
    int64_t nb = ((int64_t)C + kGroup - 1) / kGroup;
    tree_level_ctl_kernel<<<(unsigned)nb, kRedThreads, 0, s>>>(x, C, nb == 1 ? out : partials, nullptr, 0);
    LVG_LAUNCH();
    if (nb > 1) {
      ctl_q_kernel<<<1, kRedThreads, 0, s>>>(partials, nb, out);
      LVG_LAUNCH();
    }
  };
  tree(Kc, twoW_q);
  nm_term_kernel<<<sm_grid(C, kThreads), kThreads, 0, s>>>(Kc, Ain, C, twoW_q, t);
  LVG_LAUNCH();
  tree(t, twoW_q + 1);
}

void iota(int32_t* x, int64_t n, cudaStream_t s) {
  if (n <= 0) return;
  iota_kernel<<<sm_grid(n, kThreads), kThreads, 0, s>>>(x, n);
  LVG_LAUNCH();
}

void compose(int32_t* composed, const int32_t* part_level, int64_t n, cudaStream_t s) {
  if (n <= 0) return;
  compose_kernel<<<sm_grid(n, kThreads), kThreads, 0, s>>>(composed, part_level, n);
  LVG_LAUNCH();
}

}  // namespace lvg

// ============================================================================
// Batched runs: many independent graphs as one disjoint-union level graph.
// Graphs occupy contiguous vertex ranges vbase[j]..vbase[j+1]; everything a
// single run keeps as a scalar (m, the pass control, Q, the level break) is
// kept per graph, and the Q of a graph is summed on the same fixed tree as a
// single run over its own communities.
namespace lvg {
namespace {

// Level-0 union list: graph g's entries come from its own arrays (psrc[g],
// pdst[g], pw[g]) and its ids are moved up by voff[g].
__global__ void batch_globalize_kernel(const int32_t* const* psrc, const int32_t* const* pdst,
                                       const float* const* pw, int64_t E, const int64_t* eoff, const int32_t* voff,
                                       int32_t G, int32_t* gsrc, int32_t* gdst, float* gw, uint32_t* bad) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < E; e += (int64_t)gridDim.x * blockDim.x) {
    int lo = 0, hi = G - 1;
    while (lo < hi) {  // last graph whose first entry is <= e
      int mid = (lo + hi + 1) >> 1;
      if (eoff[mid] <= e) lo = mid; else hi = mid - 1;
    }
    const int64_t j = e - eoff[lo];
    int32_t n = voff[lo + 1] - voff[lo];
    int32_t a = psrc[lo][j], b = pdst[lo][j];
    float x = pw[lo][j];
    if (a < 0 || a >= n || b < 0 || b >= n || !(x >= 0.0f) || isinf(x)) atomicOr(bad, 1u);
    gsrc[e] = a + voff[lo];
    gdst[e] = b + voff[lo];
    gw[e] = x;
  }
}

__global__ void vgid_fill_kernel(const int32_t* vbase, int32_t G, int32_t V, int32_t* vgid) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < V; i += (int64_t)gridDim.x * blockDim.x) {
    int lo = 0, hi = G - 1;
    while (lo < hi) {
      int mid = (lo + hi + 1) >> 1;
      if (vbase[mid] <= i) lo = mid; else hi = mid - 1;
    }
    vgid[i] = lo;
  }
}

// m of every graph: runs of entries of one graph inside a warp add once.
__global__ void local_ids_kernel(const int32_t* gid, const int32_t* voff, int32_t V, int32_t* local) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < V; i += (int64_t)gridDim.x * blockDim.x)
    local[i] = (int32_t)i - voff[gid[i]];
}

__global__ void batch_m_kernel(const int32_t* src, const float* w, int64_t E, const int32_t* vgid, double* gm) {
  int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  bool valid = e < E;
  int64_t g = valid ? vgid[src[e]] : -1;
  double x = seg_warp_sum<int64_t>(valid ? (double)w[e] : 0.0, g);
  if (seg_warp_last<int64_t>(g, valid)) atomicAdd(&gm[g], x);
}

__global__ void batch_init_kernel(int32_t V, const double* k, const float* loopw, int32_t* comm, int32_t* next,
                                  double* tot, double* in, int32_t* size, Delta* delta, int32_t* cand) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < V; i += (int64_t)gridDim.x * blockDim.x) {
    comm[i] = (int32_t)i;
    next[i] = (int32_t)i;
    tot[i] = k[i];
    in[i] = (double)loopw[i];
    size[i] = 1;
    delta_clear(delta[i]);
    cand[i] = -1;
  }
}

template <int MODE>
__global__ void __launch_bounds__(kRedThreads) batch_commit_kernel(
    const int32_t* blk_g, const int32_t* blk_c0, const int32_t* vbase, const double* gm, int32_t* comm,
    const int32_t* next, double* tot, double* in, int32_t* size, Delta* delta, const double* k,
    double* partials, BatchCtl C) {
  __shared__ double ws[8];
  const int32_t g = blk_g[blockIdx.x];
  const int64_t c0 = blk_c0[blockIdx.x];
  const int64_t cend = vbase[g + 1];
  const int64_t base = c0 + threadIdx.x;
  if (MODE == kCommitPass) {
    if (C.done[g]) return;
    bool stop = __dsub_rn(C.q_prev[g], C.cur[g]) < C.pass_min;
    bool capped = C.max_passes >= 0 && C.pass[g] >= C.max_passes;
    if (stop || capped) {
      for (int j = 0; j < 8; ++j) {
        int64_t c = base + (int64_t)j * 256;
        if (c < cend) delta_clear(delta[c]);
      }
      if (c0 == vbase[g] && threadIdx.x == 0) C.stop_now[g] = stop ? 1 : 2;
      return;
    }
  }
  const double m = gm[g];
  const double twom = __dmul_rn(2.0, m);
  double s = 0.0;
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    int64_t c = base + (int64_t)j * 256;
    if (c < cend) {
      double t, x;
      if (MODE != kCommitInit) {
        t = tot[c]; x = in[c];
        int32_t sz = size[c];
        delta_commit(delta[c], k[c], t, x, sz);
        tot[c] = t; in[c] = x; size[c] = sz;
        comm[c] = next[c];
      } else {
        t = tot[c]; x = in[c];
      }
      s = __dadd_rn(s, q_term(x, t, m, twom));
    }
  }
  double r = block_tree256(s, ws);
  if (threadIdx.x == 0) partials[blockIdx.x] = r;
}

enum { kBatchCtlPass = 0, kBatchCtlInit = 1, kBatchCtlRet = 2 };

template <int MODE>
__global__ void __launch_bounds__(kRedThreads) batch_ctl_kernel(const int32_t* gblk0, const double* partials,
                                                                BatchCtl C, int32_t G, PassCtl* ctl) {
  __shared__ double ws[8];
  __shared__ int flag;
  const int32_t g = blockIdx.x;
  if (MODE == kBatchCtlPass) {
    if (threadIdx.x == 0) flag = C.done[g] ? 2 : (C.stop_now[g] ? 1 : 0);
    __syncthreads();
    int f = flag;
    if (f == 2) return;
    if (f == 1) {
      if (threadIdx.x == 0) {
        C.status[g] = C.stop_now[g] == 2 ? LVG_ERR_NOT_CONVERGED : LVG_OK;
        C.passes[g] = C.pass[g];
        C.stop_now[g] = 0;
        C.done[g] = 1;
        __threadfence();
        if (atomicAdd(C.ndone, 1) + 1 == G) ctl->done = 1;
      }
      return;
    }
  }
  double q = group_sum_block<double>(partials + gblk0[g], gblk0[g + 1] - gblk0[g], ws);
  if (threadIdx.x == 0) {
    if (MODE == kBatchCtlPass) {
      double cur = C.q_prev[g];
      if (cur < C.lower[g]) cur = C.lower[g];
      C.cur[g] = cur;
      C.q_prev[g] = q;
      C.pass[g] += 1;
    } else if (MODE == kBatchCtlInit) {
      C.q_prev[g] = q;
    } else {
      C.q_ret[g] = q;
    }
  }
}

__global__ void batch_keys_kernel(const int32_t* src, const int32_t* dst, const float* w, int64_t E,
                                  const int32_t* part, const int32_t* vgid, const int32_t* shift, int B,
                                  uint64_t* keys, float* vals) {
  const uint64_t sentinel = (B >= 32) ? ~0ull : ((1ull << (2 * B)) - 1);
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < E; e += (int64_t)gridDim.x * blockDim.x) {
    int32_t j = vgid[src[e]];
    int32_t sh = shift[j];
    if (sh == INT_MIN) {            // graph finished at this level: dropped
      keys[e] = sentinel;
      vals[e] = 0.0f;
      continue;
    }
    uint64_t a = (uint32_t)(part[src[e]] + sh), b = (uint32_t)(part[dst[e]] + sh);
    keys[e] = (a << B) | b;
    float x = w[e];
    vals[e] = x == 0.0f ? 1.0f : x;   // InducedGraphKernel.cu:38-39
  }
}

__global__ void gather_u32_kernel(const uint32_t* pos, const int32_t* idx, int32_t n, int32_t* out) {
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x)
    out[j] = (int32_t)pos[idx[j]];
}

__global__ void batch_count_kernel(const int32_t* src, int64_t E, const int32_t* vgid, int64_t* cnt) {
  int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  bool valid = e < E;
  int64_t g = valid ? vgid[src[e]] : -1;
  double x = seg_warp_sum<int64_t>(valid ? 1.0 : 0.0, g);
  if (seg_warp_last<int64_t>(g, valid)) atomicAdd((unsigned long long*)&cnt[g], (unsigned long long)x);
}

__global__ void batch_compose_kernel(int32_t* local0, const int32_t* gid0, int64_t n, const int32_t* lidx,
                                     const int32_t* vbase, const int32_t* cbase, const int32_t* part) {
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
    int32_t j = lidx[gid0[v]];
    if (j >= 0) local0[v] = part[vbase[j] + local0[v]] - cbase[j];
  }
}

// Newman modularity per graph over its level-0 entries (global community
// ids coff[g] + local id).
__global__ void batch_nm_accum_kernel(const int32_t* src, const int32_t* dst, const float* w, int64_t E,
                                      const int32_t* gid0, const int32_t* local0, const int32_t* coff, double* Kc,
                                      double* Ain) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t e0 = blockIdx.x * (int64_t)blockDim.x; e0 < E; e0 += stride) {
    const int64_t e = e0 + threadIdx.x;
    const bool ok = e < E;
    double x = 0.0;
    int32_t a = -1, b = -1;
    if (ok) {
      const int32_t g = gid0[src[e]];
      x = (double)w[e];
      a = coff[g] + local0[src[e]];
      b = coff[g] + local0[dst[e]];
    }
    warp_group_add(Kc, a, x);
    warp_group_add(Kc, b, x);
    warp_group_add(Ain, (ok && a == b) ? a : -1, 2.0 * x);
  }
}

// Per-graph fixed-tree sums: block b sums x over communities blk_c0[b] ..
// min(+2048, end of its graph), the same tree as one graph's tree_sum_f64.
__global__ void __launch_bounds__(kRedThreads) batch_group_kernel(const double* x, const int32_t* blk_g,
                                                                  const int32_t* blk_c0, const int32_t* cbeg,
                                                                  double* partials) {
  __shared__ double ws[8];
  const int32_t g = blk_g[blockIdx.x];
  const int64_t c0 = blk_c0[blockIdx.x];
  double r = group_sum_block<double>(x + c0, (int64_t)cbeg[g + 1] - c0, ws);
  if (threadIdx.x == 0) partials[blockIdx.x] = r;
}

__global__ void __launch_bounds__(kRedThreads) batch_finish_kernel(const double* partials, const int32_t* gblk0,
                                                                   double* out) {
  __shared__ double ws[8];
  const int32_t g = blockIdx.x;
  const int32_t n = gblk0[g + 1] - gblk0[g];
  double r = n == 1 ? partials[gblk0[g]] : group_sum_block<double>(partials + gblk0[g], n, ws);
  if (threadIdx.x == 0) out[g] = n == 0 ? 0.0 : r;
}

__global__ void batch_nm_term_kernel(const double* Kc, const double* Ain, const int32_t* cg, int32_t C,
                                     const double* twoW, double* t) {
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < C; c += (int64_t)gridDim.x * blockDim.x) {
    double tw = twoW[cg[c]];
    double f = __ddiv_rn(Kc[c], tw);
    t[c] = tw > 0.0 ? __dsub_rn(__ddiv_rn(Ain[c], tw), __dmul_rn(f, f)) : 0.0;
  }
}

}  // namespace

void batch_globalize(const int32_t* const* psrc, const int32_t* const* pdst, const float* const* pw, int64_t E,
                     const int64_t* eoff, const int32_t* voff, int32_t G, int32_t* gsrc, int32_t* gdst, float* gw,
                     uint32_t* bad, cudaStream_t s) {
  if (E == 0) return;
  batch_globalize_kernel<<<sm_grid(E, kThreads), kThreads, 0, s>>>(psrc, pdst, pw, E, eoff, voff, G, gsrc, gdst, gw,
                                                                    bad);
  LVG_LAUNCH();
}

void batch_vgid(const int32_t* vbase, int32_t G, int32_t V, int32_t* vgid, cudaStream_t s) {
  if (V == 0) return;
  vgid_fill_kernel<<<sm_grid(V, kThreads), kThreads, 0, s>>>(vbase, G, V, vgid);
  LVG_LAUNCH();
}

void batch_local_ids(const int32_t* gid, const int32_t* voff, int32_t V, int32_t* local, cudaStream_t s) {
  if (V == 0) return;
  local_ids_kernel<<<sm_grid(V, kThreads), kThreads, 0, s>>>(gid, voff, V, local);
  LVG_LAUNCH();
}

void batch_m(const int32_t* src, const float* w, int64_t E, const int32_t* vgid, double* gm, int32_t G,
             cudaStream_t s) {
  LVG_CUDA(cudaMemsetAsync(gm, 0, sizeof(double) * std::max(G, 1), s));
  if (E == 0) return;
  batch_m_kernel<<<grid_for(E, kThreads), kThreads, 0, s>>>(src, w, E, vgid, gm);
  LVG_LAUNCH();
}

void batch_init(const LevelGraph& g, CommState& st, cudaStream_t s) {
  if (g.V == 0) return;
  batch_init_kernel<<<sm_grid(g.V, kThreads), kThreads, 0, s>>>(g.V, g.k, g.loopw, st.comm, st.next, st.tot, st.in,
                                                                st.size, st.delta, st.cand);
  LVG_LAUNCH();
}

void batch_commit(int mode, const BatchPlan& bp, const double* gm, const double* g_k, CommState& st,
                  const BatchCtl& C, cudaStream_t s) {
  const unsigned nb = (unsigned)bp.nblk;
  if (nb == 0) return;
  if (mode == kCommitInit)
    batch_commit_kernel<kCommitInit><<<nb, kRedThreads, 0, s>>>(bp.blk_g, bp.blk_c0, bp.vbase, gm, st.comm, st.next,
                                                                st.tot, st.in, st.size, st.delta, g_k,
                                                                st.partials, C);
  else if (mode == kCommitPass)
    batch_commit_kernel<kCommitPass><<<nb, kRedThreads, 0, s>>>(bp.blk_g, bp.blk_c0, bp.vbase, gm, st.comm, st.next,
                                                                st.tot, st.in, st.size, st.delta, g_k,
                                                                st.partials, C);
  else
    batch_commit_kernel<kCommitForce><<<nb, kRedThreads, 0, s>>>(bp.blk_g, bp.blk_c0, bp.vbase, gm, st.comm,
                                                                 st.next, st.tot, st.in, st.size, st.delta, g_k,
                                                                 st.partials, C);
  LVG_LAUNCH();
}

void batch_ctl(int mode, const BatchPlan& bp, const CommState& st, const BatchCtl& C, int32_t G, cudaStream_t s) {
  if (G == 0) return;
  if (mode == 0) batch_ctl_kernel<kBatchCtlPass><<<G, kRedThreads, 0, s>>>(bp.gblk0, st.partials, C, G, st.ctl);
  else if (mode == 1) batch_ctl_kernel<kBatchCtlInit><<<G, kRedThreads, 0, s>>>(bp.gblk0, st.partials, C, G, st.ctl);
  else batch_ctl_kernel<kBatchCtlRet><<<G, kRedThreads, 0, s>>>(bp.gblk0, st.partials, C, G, st.ctl);
  LVG_LAUNCH();
}

void launch_merge_deltas(const LevelGraph& g, CommState& st, cudaStream_t s) {
  if (g.V == 0) return;
  merge_kernel<<<sm_grid(g.V, kThreads), kThreads, 0, s>>>(g.V, st.comm, st.next, st.cand, g.k, g.loopw, st.delta);
  LVG_LAUNCH();
}

int32_t renumber_pos(const LevelGraph& g, const int32_t* comm, int32_t* part, uint32_t* pos, Arena& a,
                     cudaStream_t s) {
  const int32_t V = g.V;
  if (V == 0) return 0;
  HiScope hs(a);
  int32_t* minidx = a.hi_n<int32_t>(V);
  uint32_t* flag = a.hi_n<uint32_t>(V + 1);
  LVG_CUDA(cudaMemsetAsync(minidx, 0x7f, sizeof(int32_t) * V, s));
  min_member_kernel<<<sm_grid(V, kThreads), kThreads, 0, s>>>(V, comm, minidx);
  LVG_LAUNCH();
  head_flag_kernel<<<grid_for(V, kThreads), kThreads, 0, s>>>(V, comm, minidx, flag);
  LVG_LAUNCH();
  scan_u32(flag, pos, V, a, s);
  renumber_apply_kernel<<<sm_grid(V, kThreads), kThreads, 0, s>>>(V, comm, flag, pos, minidx);
  LVG_LAUNCH();
  gather_kernel<<<sm_grid(V, kThreads), kThreads, 0, s>>>(V, comm, minidx, part);
  LVG_LAUNCH();
  uint32_t C = 0;
  LVG_CUDA(cudaMemcpyAsync(&C, pos + V, sizeof C, cudaMemcpyDeviceToHost, s));
  LVG_CUDA(cudaStreamSynchronize(s));
  return (int32_t)C;
}

int64_t batch_induce(const LevelGraph& g, const int32_t* part, const int32_t* vgid, const int32_t* shift,
                     int32_t C_next, int64_t E_keep, int32_t** out_src, int32_t** out_dst, float** out_w, Arena& a,
                     cudaStream_t s) {
  const int64_t E = g.E;
  if (E >= ((int64_t)1 << 32)) throw Error(LVG_ERR_CAPACITY, "level edge list exceeds 2^32-1 entries");
  int32_t* osrc = a.hi_n<int32_t>(E_keep);
  int32_t* odst = a.hi_n<int32_t>(E_keep);
  float* ow = a.hi_n<float>(E_keep);
  int64_t cnt = 0;
  {
    HiScope hs(a);
    const int B = std::max(1, bits_for((int64_t)C_next + 1));
    uint64_t* k0 = a.hi_n<uint64_t>(E);
    float* v0 = a.hi_n<float>(E);
    uint64_t* k1 = a.hi_n<uint64_t>(E);
    float* v1 = a.hi_n<float>(E);
    uint32_t* head = a.hi_n<uint32_t>(E_keep + 1);
    uint32_t* pos = a.hi_n<uint32_t>(E_keep + 1);
    double* wsum = a.hi_n<double>(E_keep);
    if (E > 0) {
      batch_keys_kernel<<<sm_grid(E, kThreads), kThreads, 0, s>>>(g.src, g.dst, g.w, E, part, vgid, shift, B, k0, v0);
      LVG_LAUNCH();
    }
    int which = radix_sort_pairs(k0, v0, k1, v1, E, 2 * B, a, s);
    uint64_t* keys = which ? k1 : k0;
    float* vals = which ? v1 : v0;
    if (E_keep > 0) {
      run_head_kernel<<<sm_grid(E_keep, kThreads), kThreads, 0, s>>>(keys, E_keep, head);
      LVG_LAUNCH();
    }
    scan_u32(head, pos, E_keep, a, s);
    uint32_t n_out = 0;
    LVG_CUDA(cudaMemcpyAsync(&n_out, pos + E_keep, sizeof n_out, cudaMemcpyDeviceToHost, s));
    LVG_CUDA(cudaStreamSynchronize(s));
    cnt = n_out;
    LVG_CUDA(cudaMemsetAsync(wsum, 0, sizeof(double) * std::max<int64_t>(cnt, 1), s));
    if (E_keep > 0) {
      run_sum_kernel<<<grid_for(E_keep, kThreads), kThreads, 0, s>>>(keys, vals, E_keep, B, pos, head, osrc, odst,
                                                                       wsum);
      LVG_LAUNCH();
    }
    if (cnt > 0) {
      to_float_kernel<<<sm_grid(cnt, kThreads), kThreads, 0, s>>>(wsum, ow, cnt);
      LVG_LAUNCH();
    }
    LVG_CUDA(cudaStreamSynchronize(s));
  }
  *out_src = osrc;
  *out_dst = odst;
  *out_w = ow;
  return cnt;
}

void gather_u32(const uint32_t* pos, const int32_t* idx, int32_t n, int32_t* out, cudaStream_t s) {
  if (n == 0) return;
  gather_u32_kernel<<<sm_grid(n, kThreads), kThreads, 0, s>>>(pos, idx, n, out);
  LVG_LAUNCH();
}

void batch_count(const int32_t* src, int64_t E, const int32_t* vgid, int64_t* cnt, int32_t G, cudaStream_t s) {
  LVG_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int64_t) * std::max(G, 1), s));
  if (E == 0) return;
  batch_count_kernel<<<grid_for(E, kThreads), kThreads, 0, s>>>(src, E, vgid, cnt);
  LVG_LAUNCH();
}

void batch_compose(int32_t* local0, const int32_t* gid0, int64_t n, const int32_t* lidx, const int32_t* vbase,
                   const int32_t* cbase, const int32_t* part, cudaStream_t s) {
  if (n == 0) return;
  batch_compose_kernel<<<sm_grid(n, kThreads), kThreads, 0, s>>>(local0, gid0, n, lidx, vbase, cbase, part);
  LVG_LAUNCH();
}

void batch_modularity(const int32_t* src, const int32_t* dst, const float* w, int64_t E, const int32_t* gid0,
                      const int32_t* local0, const BatchPlan& cp, const int32_t* cg, int32_t Ctot, int32_t G,
                      double* q, Arena& a, cudaStream_t s) {
  HiScope hs(a);
  double* Kc = a.hi_n<double>(Ctot);
  double* Ain = a.hi_n<double>(Ctot);
  double* t = a.hi_n<double>(Ctot);
  double* partials = a.hi_n<double>(cp.nblk);
  double* twoW = a.hi_n<double>(G);
  LVG_CUDA(cudaMemsetAsync(Kc, 0, sizeof(double) * std::max(Ctot, 1), s));
  LVG_CUDA(cudaMemsetAsync(Ain, 0, sizeof(double) * std::max(Ctot, 1), s));
  if (E > 0) {
    batch_nm_accum_kernel<<<sm_grid(E, kThreads), kThreads, 0, s>>>(src, dst, w, E, gid0, local0, cp.vbase, Kc, Ain);
    LVG_LAUNCH();
  }
  if (cp.nblk > 0) {
    batch_group_kernel<<<(unsigned)cp.nblk, kRedThreads, 0, s>>>(Kc, cp.blk_g, cp.blk_c0, cp.vbase, partials);
    LVG_LAUNCH();
  }
  batch_finish_kernel<<<G, kRedThreads, 0, s>>>(partials, cp.gblk0, twoW);
  LVG_LAUNCH();
  if (Ctot > 0) {
    batch_nm_term_kernel<<<sm_grid(Ctot, kThreads), kThreads, 0, s>>>(Kc, Ain, cg, Ctot, twoW, t);
    LVG_LAUNCH();
    batch_group_kernel<<<(unsigned)cp.nblk, kRedThreads, 0, s>>>(t, cp.blk_g, cp.blk_c0, cp.vbase, partials);
    LVG_LAUNCH();
  }
  batch_finish_kernel<<<G, kRedThreads, 0, s>>>(partials, cp.gblk0, q);
  LVG_LAUNCH();
}

// ------------------------------------------------------------ degree statistics
__global__ void max_degree_kernel(const int64_t* off, int32_t V, unsigned long long* out) {
  unsigned long long m = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < V; i += (int64_t)gridDim.x * blockDim.x)
    m = max(m, (unsigned long long)(off[i + 1] - off[i]));
  for (int o = 16; o; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0 && m) atomicMax(out, m);
}

int64_t max_degree(const LevelGraph& g, Arena& a, cudaStream_t s) {
  if (g.V <= 0) return 0;
  HiScope hs(a);
  unsigned long long* d = a.hi_n<unsigned long long>(1);
  LVG_CUDA(cudaMemsetAsync(d, 0, sizeof *d, s));
  max_degree_kernel<<<sm_grid(g.V, kThreads), kThreads, 0, s>>>(g.off, g.V, d);
  LVG_LAUNCH();
  unsigned long long h = 0;
  LVG_CUDA(cudaMemcpyAsync(&h, d, sizeof h, cudaMemcpyDeviceToHost, s));
  LVG_CUDA(cudaStreamSynchronize(s));
  return (int64_t)h;
}

}  // namespace lvg
