// Coarsening of a level whose list is strictly sorted and symmetric (every
// level after the first, and a first level given in that form), without a
// device-wide sort of all its entries.
//
// The reference maps both endpoints of every entry to communities, sorts the
// (cu, cv) keys and sums equal keys (InducedGraphKernel.cu:28-48,84-113).
// Here the list's rows are laid out community by community instead: the
// members of each community (in vertex order) are found by a stable sort of
// the V community ids, and the rows of the members of one community, read in
// member order, form that community's segment -- entries already grouped by
// cu, at positions known from a scan of the row lengths.  The position range
// is cut into chunks of 4096 entries.  A 512-thread block takes a chunk:
// it reads cv = part[dst] of its entries (gathered once in list order by a
// streaming kernel), sorts (segment, cv) keys in
// shared memory (stable 8-bit LSD passes over only the bits the chunk needs),
// and sums equal keys in a fixed order.  A segment that lies inside one chunk
// is then final.  Segments that cross a chunk boundary (the large
// communities) leave one partial run per chunk and distinct cv; only those
// partial runs -- a fraction of the entries -- go through the device-wide
// radix sort, keyed by (open segment, cv), and are summed again.  A scan of
// the distinct counts of every community places each community's entries.
//
// A chunk that lies inside one segment continuing on both sides sends all its
// runs on, so it sums equal cv in a shared-memory hash table instead of
// sorting them.
//
// Output: the same list as the sort-based path (entries ordered by (cu, cv),
// weights 0 counted as 1, sums in FP64 rounded once to float).  Sums inside a
// sorted chunk run in a fixed order; the hash tables and the sums across
// chunks use FP64 atomics, whose order does not matter for integer weights
// (every partial sum is exact).
#include <algorithm>
#include <cstddef>
#include <mutex>

#include "louvain.cuh"
#include "prims.cuh"

namespace lvg {
namespace {

constexpr int kIcThreads = 512;
constexpr int kIcItems = 8;
constexpr int kIcChunk = kIcThreads * kIcItems;   // list positions per chunk
constexpr int kIcWarps = kIcThreads / 32;
constexpr int kIcRadix = 256;
constexpr int kIcRelBits = 13;                    // member index inside a chunk, 0..4096
constexpr uint32_t kIcRelMask = (1u << kIcRelBits) - 1u;
constexpr int kIcFlat = 256;                      // threads of the flat kernels

enum : uint32_t { kOpenL = 1u, kOpenR = 2u, kSingle = 4u };

int ic_sms() {
  static const int sms = [] {
    int dev = 0, n = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    return n > 0 ? n : 148;
  }();
  return sms;
}

unsigned ic_grid(int64_t n) {
  int64_t g = (n + kIcFlat - 1) / kIcFlat;
  const int64_t cap = (int64_t)ic_sms() * 16;
  if (g > cap) g = cap;
  return (unsigned)(g > 0 ? g : 1);
}

#define IC_FOR(i, n) \
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (n); i += (int64_t)gridDim.x * blockDim.x)

// ------------------------------------------------------------------ members
// Sort key of a vertex: its community, or C for a vertex without entries
// (those sort after every member and take no list positions).
__global__ void ic_member_keys_kernel(int32_t V, const int64_t* off, const uint8_t* has_loop, const int32_t* part,
                                      int32_t C, uint64_t* key, float* val, uint32_t* loops) {
  IC_FOR(i, V) {
    const int64_t rl = off[i + 1] - off[i] + has_loop[i];
    key[i] = rl > 0 ? (uint64_t)(uint32_t)part[i] : (uint64_t)(uint32_t)C;
    val[i] = __int_as_float((int32_t)i);
    loops[i] = has_loop[i];
  }
}

// Members in community order: vertex, community, row length; nz = members
// with entries (written by the last of them).
__global__ void ic_member_len_kernel(int32_t V, const uint64_t* skey, const float* sval, const int64_t* off,
                                     const uint8_t* has_loop, int32_t C, int32_t* mem, int32_t* mcomm,
                                     int64_t* mlen, int32_t* nz) {
  IC_FOR(i, V) {
    const int32_t u = __float_as_int(sval[i]);
    const int32_t c = (int32_t)skey[i];
    mem[i] = u;
    mcomm[i] = c;
    const bool has = c < C;
    mlen[i] = has ? off[u + 1] - off[u] + has_loop[u] : 0;
    if (has && (i + 1 == V || (int32_t)skey[i + 1] >= C)) *nz = (int32_t)(i + 1);
  }
}

// cv of every list entry, in list order: the one random gather of the
// coarsening, made by a streaming kernel (many loads in flight per SM) so
// that the chunk kernel reads cv coalesced along the rows.
__global__ void ic_cv_kernel(const int32_t* ldst, const int32_t* part, int64_t E, int32_t* cvl) {
  IC_FOR(e, E) cvl[e] = __ldg(part + __ldg(ldst + e));
}

// cfirst[c] = the member whose positions hold chunk c's first position.
__global__ void ic_chunk_first_kernel(const int64_t* mscan, const int32_t* nzp, int32_t* cfirst, int64_t nchunks) {
  const int32_t nz = *nzp;
  IC_FOR(i, nz) {
    const int64_t s = mscan[i], e = mscan[i + 1];
    const int64_t c0 = (s + kIcChunk - 1) / kIcChunk, c1 = (e + kIcChunk - 1) / kIcChunk;
    for (int64_t c = c0; c < c1; ++c) cfirst[c] = (int32_t)i;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) cfirst[nchunks] = nz;
}

// ------------------------------------------------------------------ chunks
struct IcSmem {
  union {
    uint64_t key[kIcChunk];          // sort keys (from the first ranking on)
    uint32_t mark[kIcChunk];         // per position: (local segment << 13) | member (gather)
  } a;
  union {
    struct {
      float val[kIcChunk];
      uint32_t wc[kIcWarps][kIcRadix + 1];
      uint32_t dstart[kIcRadix];
    } s;
    int64_t ebase[kIcChunk + 1];     // per member: list index minus list position (gather)
  } b;
  int32_t loc_a[kIcChunk + 1];       // community of each local segment
  uint32_t locfirst[kIcChunk + 2];   // first run of each local segment, then the run count
  uint32_t wmax[kIcWarps];
  uint32_t wflag[kIcWarps];
  double wsum[kIcWarps];
  uint32_t nloc, openL, openR;
};

// Exclusive max-scan of one value per thread over the 512-thread block.
__device__ __forceinline__ uint32_t ic_block_excl_max(uint32_t v, uint32_t* wmax) {
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  uint32_t inc = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t u = __shfl_up_sync(full, inc, o);
    if (lane >= o) inc = max(inc, u);
  }
  if (lane == 31) wmax[w] = inc;
  __syncthreads();
  uint32_t pre = 0;
  for (int ww = 0; ww < w; ++ww) pre = max(pre, wmax[ww]);
  uint32_t ex = __shfl_up_sync(full, inc, 1);
  if (lane == 0) ex = 0;
  __syncthreads();
  return max(pre, ex);
}

// Exclusive segmented scan over the block of (f, s) pairs: f says a run
// starts inside the thread's items, s is the sum of the thread's items after
// its last run start (all of them when f is 0).  The result is the sum of
// the run open at the thread's first item, over the earlier threads' items.
// Combine: (f1, s1) then (f2, s2) -> (f1 | f2, f2 ? s2 : s1 + s2), applied in
// a fixed tree, so the additions do not depend on timing.
__device__ __forceinline__ double ic_block_seg_carry(uint32_t f, double s, uint32_t* wflag, double* wsum) {
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  uint32_t fi = f;
  double si = s;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t fu = __shfl_up_sync(full, fi, o);
    const double su = __shfl_up_sync(full, si, o);
    if (lane >= o) {
      si = fi ? si : __dadd_rn(su, si);
      fi |= fu;
    }
  }
  if (lane == 31) { wflag[w] = fi; wsum[w] = si; }
  __syncthreads();
  // prefix of the earlier warps, left to right
  double ps = 0.0;
  for (int ww = 0; ww < w; ++ww) ps = wflag[ww] ? wsum[ww] : __dadd_rn(ps, wsum[ww]);
  uint32_t fe = __shfl_up_sync(full, fi, 1);
  double se = __shfl_up_sync(full, si, 1);
  if (lane == 0) { fe = 0; se = 0.0; }
  __syncthreads();
  return fe ? se : __dadd_rn(ps, se);
}

// Hash-table reduction of a chunk inside one segment (items in registers,
// keys = cv).  A table of 2 x kIcChunk slots over the shared memory of the
// sort layout: keys 32-bit (empty = all ones; cv < 2^31), sums FP64.  Lanes
// of a warp holding the same cv add first, then one shared atomic per cv.
// Writes the distinct (community, cv) runs in table order at p0.., and
// leaves the run count in S.nloc and the community in S.openL (after a
// barrier) for the caller's chunk summary.
constexpr int kIcHashSlots = 2 * kIcChunk;
constexpr uint32_t kIcEmpty = 0xffffffffu;
static_assert(sizeof(uint32_t) * kIcHashSlots + sizeof(double) * kIcHashSlots <=
                  offsetof(IcSmem, wmax), "hash table fits below the block's scalars");

__device__ __forceinline__ void ic_chunk_hash(IcSmem& S, unsigned char* raw, const uint64_t* k, const float* x,
                                              int n, int64_t p0, uint64_t* tkey, double* tsum, uint32_t* hl) {
  const unsigned full = 0xffffffffu;
  const int t = threadIdx.x, lane = t & 31;
  const int32_t a0 = S.loc_a[0];
  __syncthreads();   // the table overwrites the gather layout
  uint32_t* hk = reinterpret_cast<uint32_t*>(raw);
  double* hv = reinterpret_cast<double*>(raw + sizeof(uint32_t) * kIcHashSlots);
  for (int i = t; i < kIcHashSlots; i += kIcThreads) {
    hk[i] = kIcEmpty;
    hv[i] = 0.0;
  }
  __syncthreads();
#pragma unroll
  for (int jj = 0; jj < kIcItems; ++jj) {
    const uint32_t key = k[jj] == ~0ull ? kIcEmpty : (uint32_t)k[jj];
    double v = (double)x[jj];
    const unsigned peers = __match_any_sync(full, key);
    if (__any_sync(full, __popc(peers) > 1)) {
      double sum = 0.0;
#pragma unroll
      for (int l = 0; l < 32; ++l) {
        const double u = __shfl_sync(full, v, l);
        if ((peers >> l) & 1u) sum = __dadd_rn(sum, u);
      }
      v = sum;
    }
    if (key != kIcEmpty && lane == __ffs(peers) - 1) {
      uint32_t slot = (key * 0x9E3779B1u) >> (32 - 13);
      static_assert(kIcHashSlots == 1 << 13, "13-bit slots");
      while (true) {
        const uint32_t prev = atomicCAS(&hk[slot], kIcEmpty, key);
        if (prev == kIcEmpty || prev == key) break;
        slot = (slot + 1) & (kIcHashSlots - 1);
      }
      atomicAdd(&hv[slot], v);
    }
  }
  __syncthreads();
  constexpr int kPer = kIcHashSlots / kIcThreads;
  uint32_t cnt = 0;
#pragma unroll
  for (int i = 0; i < kPer; ++i) cnt += hk[t * kPer + i] != kIcEmpty;
  uint32_t tot;
  uint32_t o = block_exclusive_scan512<uint32_t>(cnt, &tot);
#pragma unroll
  for (int i = 0; i < kPer; ++i) {
    const int slot = t * kPer + i;
    if (hk[slot] != kIcEmpty) {
      tkey[p0 + o] = ((uint64_t)(uint32_t)a0 << 32) | hk[slot];
      tsum[p0 + o] = hv[slot];
      if (hk[slot] == (uint32_t)a0) hl[a0] = 1u;
      ++o;
    }
  }
  if (t == 0) {
    S.nloc = tot;
    S.openL = (uint32_t)a0;
  }
  __syncthreads();
}

// One chunk of kIcChunk list positions (see the file comment).  Writes its
// runs (sorted by (local segment, cv), one per distinct key) at tkey/tsum
// [p0, p0 + runs); for each segment that lies inside the chunk, its run count
// and first run; and the chunk's summary (runs, runs of the segment open to
// the left / right, flags, community of the last segment).
__global__ void __launch_bounds__(kIcThreads, 2) ic_chunk_kernel(
    int64_t E, int64_t nchunks, int Bb, const int32_t* mem, const int32_t* mcomm, const int64_t* mscan,
    const int32_t* cfirst, const int64_t* off, const uint32_t* lscan, const int32_t* cvl, const float* lw,
    uint64_t* tkey, double* tsum, uint32_t* dcount, uint32_t* firstrun, uint32_t* c_runs,
    uint32_t* c_nl, uint32_t* c_nr, uint32_t* c_flags, int32_t* c_ar, uint32_t* hl, uint32_t* notint) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  IcSmem& S = *reinterpret_cast<IcSmem*>(smem_raw);
  const unsigned full = 0xffffffffu;
  const int t = threadIdx.x, w = t >> 5, lane = t & 31;
  const int64_t j = blockIdx.x;
  const int64_t p0 = j * kIcChunk;
  const int n = (int)(E - p0 < kIcChunk ? E - p0 : (int64_t)kIcChunk);
  const int64_t p1 = p0 + n;
  const int32_t i0 = cfirst[j];
  const int32_t ihi = j + 1 < nchunks ? cfirst[j + 1] : cfirst[nchunks] - 1;
  const int m = ihi - i0;   // candidate members after i0 (each starts in (p0, p1])

  for (int q = t; q < kIcChunk; q += kIcThreads) S.a.mark[q] = 0u;
  if (t == 0) {
    const int32_t u0 = mem[i0];
    S.b.ebase[0] = off[u0] + (int64_t)lscan[u0] - mscan[i0];
    S.loc_a[0] = mcomm[i0];
  }
  __syncthreads();
  // members: local segment index by a scan of community changes
  {
    uint32_t heads = 0;
    int32_t cm[kIcItems];
    bool hd[kIcItems];
#pragma unroll
    for (int jj = 0; jj < kIcItems; ++jj) {
      const int r = 1 + t * kIcItems + jj;
      hd[jj] = false;
      cm[jj] = 0;
      if (r <= m) {
        const int32_t i = i0 + r;
        cm[jj] = mcomm[i];
        hd[jj] = mscan[i] < p1 && cm[jj] != mcomm[i - 1];
        heads += hd[jj];
      }
    }
    uint32_t tot;
    uint32_t loc = block_exclusive_scan512<uint32_t>(heads, &tot);
#pragma unroll
    for (int jj = 0; jj < kIcItems; ++jj) {
      const int r = 1 + t * kIcItems + jj;
      if (r <= m) {
        const int32_t i = i0 + r;
        const int64_t st = mscan[i];
        loc += hd[jj];
        if (st < p1) {
          const int32_t u = mem[i];
          S.a.mark[st - p0] = (loc << kIcRelBits) | (uint32_t)r;
          S.b.ebase[r] = off[u] + (int64_t)lscan[u] - st;
          if (hd[jj]) S.loc_a[loc] = cm[jj];
        }
      }
    }
    if (t == 0) S.nloc = tot + 1;
  }
  __syncthreads();
  // each position's member: inclusive max-scan of the marks (both fields grow)
  {
    uint32_t v[kIcItems];
    uint32_t run = 0;
#pragma unroll
    for (int jj = 0; jj < kIcItems; ++jj) {
      run = max(run, S.a.mark[t * kIcItems + jj]);
      v[jj] = run;
    }
    const uint32_t pre = ic_block_excl_max(run, S.wmax);
#pragma unroll
    for (int jj = 0; jj < kIcItems; ++jj) S.a.mark[t * kIcItems + jj] = max(pre, v[jj]);
  }
  const uint32_t nloc = S.nloc;
  if (t == 0) {
    const int32_t cl = mscan[i0] < p0 ? mcomm[i0] : (p0 > 0 ? mcomm[i0 - 1] : -1);
    S.openL = p0 > 0 && cl == S.loc_a[0];
    S.openR = p1 < E && mcomm[cfirst[j + 1]] == S.loc_a[nloc - 1];
  }
  __syncthreads();
  // gather (warp-striped positions: q = w*256 + jj*32 + lane)
  uint64_t k[kIcItems];
  float x[kIcItems];
  bool frac = false;   // a weight that is not an integer
  const uint64_t bmask = (Bb >= 64) ? ~0ull : ((1ull << Bb) - 1ull);
#pragma unroll
  for (int jj = 0; jj < kIcItems; ++jj) {
    const int q = w * (32 * kIcItems) + jj * 32 + lane;
    k[jj] = ~0ull;
    x[jj] = 0.0f;
    if (q < n) {
      const uint32_t pk = S.a.mark[q];
      const int64_t e = S.b.ebase[pk & kIcRelMask] + p0 + q;
      const uint32_t b = (uint32_t)__ldg(cvl + e);
      const float wv = __ldg(lw + e);
      k[jj] = ((uint64_t)(pk >> kIcRelBits) << Bb) | b;
      x[jj] = wv == 0.0f ? 1.0f : wv;     // InducedGraphKernel.cu:38-39
      frac |= wv != truncf(wv);
    }
  }
  if (__syncthreads_or(frac) && t == 0) atomicOr(notint, 1u);
  if (nloc == 1 && S.openL && S.openR) {
    // The chunk lies inside one segment that continues on both sides: its
    // runs all go on to the device-wide sort, so they need no order here.
    // Equal cv are summed in a shared-memory hash table instead of sorted.
    ic_chunk_hash(S, smem_raw, k, x, n, p0, tkey, tsum, hl);
    if (t == 0) {
      const uint32_t runs = S.nloc;   // set by ic_chunk_hash
      c_runs[j] = runs;
      c_nl[j] = runs;
      c_nr[j] = runs;
      c_flags[j] = kOpenL | kOpenR | kSingle;
      c_ar[j] = S.openL;               // community, set by ic_chunk_hash
    }
    return;
  }
  // stable LSD passes over the bits in use; items past n carry all-ones keys
  // and stay behind every real item
  int lb = 0;
  while ((1u << lb) < nloc) ++lb;
  const int bits = Bb + lb;
  const int npass = (bits + 7) / 8;
  const unsigned lt = (1u << lane) - 1u;
  for (int p = 0; p < npass; ++p) {
    const int shift = 8 * p;
    for (int i = t; i < kIcWarps * (kIcRadix + 1); i += kIcThreads) (&S.b.s.wc[0][0])[i] = 0u;
    __syncthreads();
    uint32_t rank[kIcItems];
#pragma unroll
    for (int jj = 0; jj < kIcItems; ++jj) {
      const unsigned d = (unsigned)(k[jj] >> shift) & (kIcRadix - 1);
      const unsigned peers = __match_any_sync(full, d);
      const uint32_t before = S.b.s.wc[w][d];
      rank[jj] = before + __popc(peers & lt);
      __syncwarp();
      if ((peers & lt) == 0) S.b.s.wc[w][d] = before + __popc(peers);
      __syncwarp();
    }
    __syncthreads();
    uint32_t cnt = 0;
    if (t < kIcRadix) {
#pragma unroll
      for (int ww = 0; ww < kIcWarps; ++ww) {
        const uint32_t c = S.b.s.wc[ww][t];
        S.b.s.wc[ww][t] = cnt;
        cnt += c;
      }
    }
    uint32_t tot;
    const uint32_t st = block_exclusive_scan512<uint32_t>(t < kIcRadix ? cnt : 0u, &tot);
    if (t < kIcRadix) S.b.s.dstart[t] = st;
    __syncthreads();
#pragma unroll
    for (int jj = 0; jj < kIcItems; ++jj) {
      const unsigned d = (unsigned)(k[jj] >> shift) & (kIcRadix - 1);
      const uint32_t pos = S.b.s.dstart[d] + S.b.s.wc[w][d] + rank[jj];
      S.a.key[pos] = k[jj];
      S.b.s.val[pos] = x[jj];
    }
    __syncthreads();
    if (p + 1 < npass) {
#pragma unroll
      for (int jj = 0; jj < kIcItems; ++jj) {
        const int q = w * (32 * kIcItems) + jj * 32 + lane;
        k[jj] = S.a.key[q];
        x[jj] = S.b.s.val[q];
      }
    }
  }
  if (npass == 0) {
#pragma unroll
    for (int jj = 0; jj < kIcItems; ++jj) {
      const int q = w * (32 * kIcItems) + jj * 32 + lane;
      S.a.key[q] = k[jj];
      S.b.s.val[q] = x[jj];
    }
    __syncthreads();
  }
  // runs of equal keys (blocked positions q = t*8 + jj): count, carry, sums
  uint32_t hc = 0, f = 0;
  double sp = 0.0;
#pragma unroll
  for (int jj = 0; jj < kIcItems; ++jj) {
    const int q = t * kIcItems + jj;
    if (q < n) {
      const uint64_t kk = S.a.key[q];
      const float xv = S.b.s.val[q];
      if (q == 0 || S.a.key[q - 1] != kk) {
        f = 1u;
        ++hc;
        sp = (double)xv;
      } else {
        sp = __dadd_rn(sp, (double)xv);
      }
    }
  }
  uint32_t nruns;
  const uint32_t hb = block_exclusive_scan512<uint32_t>(hc, &nruns);
  double acc = ic_block_seg_carry(f, sp, S.wflag, S.wsum);
  int64_t run = (int64_t)hb - 1;
#pragma unroll
  for (int jj = 0; jj < kIcItems; ++jj) {
    const int q = t * kIcItems + jj;
    if (q < n) {
      const uint64_t kk = S.a.key[q];
      const float xv = S.b.s.val[q];
      const bool head = q == 0 || S.a.key[q - 1] != kk;
      if (head) {
        ++run;
        acc = (double)xv;
        if (q == 0 || (S.a.key[q - 1] >> Bb) != (kk >> Bb)) S.locfirst[kk >> Bb] = (uint32_t)run;
      } else {
        acc = __dadd_rn(acc, (double)xv);
      }
      if (q + 1 == n || S.a.key[q + 1] != kk) {
        const int32_t a = S.loc_a[kk >> Bb];
        tkey[p0 + run] = ((uint64_t)(uint32_t)a << 32) | (kk & bmask);
        tsum[p0 + run] = acc;
        if ((kk & bmask) == (uint64_t)(uint32_t)a) hl[a] = 1u;   // the community's self loop
      }
    }
  }
  if (t == 0) S.locfirst[nloc] = nruns;
  __syncthreads();
  const bool oL = S.openL != 0, oR = S.openR != 0;
  for (uint32_t l = t; l < nloc; l += kIcThreads) {
    const bool open = (l == 0 && oL) || (l + 1 == nloc && oR);
    if (!open) {
      const int32_t a = S.loc_a[l];
      dcount[a] = S.locfirst[l + 1] - S.locfirst[l];
      firstrun[a] = (uint32_t)p0 + S.locfirst[l];
    }
  }
  if (t == 0) {
    c_runs[j] = nruns;
    c_nl[j] = oL ? S.locfirst[1] - S.locfirst[0] : 0u;
    c_nr[j] = oR ? nruns - S.locfirst[nloc - 1] : 0u;
    c_flags[j] = (oL ? kOpenL : 0u) | (oR ? kOpenR : 0u) | ((nloc == 1 && oL && oR) ? kSingle : 0u);
    c_ar[j] = S.loc_a[nloc - 1];
  }
}

// ------------------------------------------------------------------ open segments
// Per chunk: does its last segment start a new open segment, and how many of
// its runs belong to open segments.
__global__ void ic_open_count_kernel(int64_t nchunks, const uint32_t* c_runs, const uint32_t* c_nl,
                                     const uint32_t* c_nr, const uint32_t* c_flags, uint32_t* newr,
                                     uint32_t* nopen) {
  IC_FOR(j, nchunks) {
    const uint32_t fl = c_flags[j];
    const bool single = (fl & kSingle) != 0;
    newr[j] = ((fl & kOpenR) && !single) ? 1u : 0u;
    nopen[j] = single ? c_runs[j] : c_nl[j] + c_nr[j];
  }
}

// The runs of open segments, keyed (open segment, cv), with their slot in
// tkey/tsum as payload; oa = community of each open segment.  A warp per chunk.
__global__ void ic_open_gather_kernel(int64_t nchunks, int Bb, const uint32_t* c_runs, const uint32_t* c_nl,
                                      const uint32_t* c_nr, const uint32_t* c_flags, const int32_t* c_ar,
                                      const uint32_t* newr_x, const uint32_t* nopen_x, const uint64_t* tkey,
                                      uint64_t* okey, float* oval, int32_t* oa) {
  const int lane = threadIdx.x & 31;
  const uint64_t bmask = (1ull << Bb) - 1ull;
  const int64_t nw = (int64_t)gridDim.x * (blockDim.x / 32);
  for (int64_t j = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) / 32; j < nchunks; j += nw) {
    const uint32_t o0 = nopen_x[j], no = nopen_x[j + 1] - o0;
    if (no == 0) continue;
    const uint32_t fl = c_flags[j], runs = c_runs[j], nl = c_nl[j], nr = c_nr[j];
    const uint32_t nnew = newr_x[j + 1] - newr_x[j];
    const uint32_t orank_l = newr_x[j] - 1u, orank_r = newr_x[j] + nnew - 1u;
    if (lane == 0 && nnew) oa[orank_r] = c_ar[j];
    for (uint32_t k = lane; k < no; k += 32) {
      uint32_t r, orank;
      if (fl & kSingle) { r = k; orank = orank_r; }
      else if (k < nl) { r = k; orank = orank_l; }
      else { r = runs - nr + (k - nl); orank = orank_r; }
      const uint64_t tt = (uint64_t)j * kIcChunk + r;
      okey[o0 + k] = ((uint64_t)orank << Bb) | (tkey[tt] & bmask);
      oval[o0 + k] = __uint_as_float((uint32_t)tt);
    }
  }
}

__global__ void ic_head_kernel(const uint64_t* k, int64_t n, uint32_t* head) {
  IC_FOR(i, n) head[i] = (i == 0 || k[i - 1] != k[i]) ? 1u : 0u;
}

// Sums of the open runs by distinct (open segment, cv): lanes of a warp add
// equal keys first, one FP64 atomic per key and warp.  ofirst[o] = distinct
// rank of open segment o's first key.  Grid covers n in whole warps.
__global__ void ic_open_sum_kernel(const uint64_t* k, const float* v, int64_t n, int Bb, const uint32_t* pos,
                                   const uint32_t* head, const double* tsum, double* osum, uint32_t* ofirst,
                                   uint32_t n_open) {
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const bool valid = i < n;
  const int64_t g = valid ? (int64_t)pos[i] + (int64_t)head[i] - 1 : -1;
  double x = valid ? tsum[__float_as_uint(v[i])] : 0.0;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const double u = __shfl_up_sync(full, x, o);
    const int64_t gu = __shfl_up_sync(full, g, o);
    if (lane >= o && gu == g) x = __dadd_rn(x, u);
  }
  const int64_t gn = __shfl_down_sync(full, g, 1);
  const bool vn = __shfl_down_sync(full, valid, 1);
  if (valid && (lane == 31 || !vn || gn != g)) atomicAdd(&osum[g], x);
  if (valid) {
    const uint64_t o = k[i] >> Bb;
    if (i == 0 || (k[i - 1] >> Bb) != o) ofirst[o] = (uint32_t)g;
    if (i + 1 == n) ofirst[n_open] = (uint32_t)g + 1u;
  }
}

__global__ void ic_open_dcount_kernel(uint32_t n_open, const uint32_t* ofirst, const int32_t* oa, uint32_t* dcount) {
  IC_FOR(o, (int64_t)n_open) dcount[oa[o]] = ofirst[o + 1] - ofirst[o];
}

// ------------------------------------------------------------------ placement
// The next level's CSR, written with the list (what build_csr_fast would make
// of it): a non-loop entry at list position p of row a goes to p - (loops in
// rows before a) - (1 if row a's loop sorts before it); a loop sets the row's
// loop weight; degrees k sum f = (w == 0 ? 1 : w), doubled, twice for a loop
// (InitKernel.cu:154-194).
struct IcCsrOut {
  int32_t* col;
  float* cw;
  double* k;
  float* loopw;
  uint8_t* has_loop;
  const uint32_t* hl;      // [C] 1: the coarse list has (a, a)
  const uint32_t* loopx;   // [C + 1] exclusive scan of hl
};

__device__ __forceinline__ double ic_seg_sum(double v, int32_t seg) {
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const double u = __shfl_up_sync(full, v, o);
    const int32_t t = __shfl_up_sync(full, seg, o);
    if (lane >= o && t == seg) v = __dadd_rn(v, u);
  }
  return v;
}

// One coarse entry (a, b, wf) at list position p (when `emit`) into the CSR,
// and its row's degree: lanes of a warp with the same row add first.  All
// lanes of the warp call it; `row` is a for every lane holding an entry of
// the sorted order (emitting or not) and -1 past the end.
__device__ __forceinline__ void ic_emit_csr(const IcCsrOut& O, bool emit, int32_t row, int32_t b, float wf,
                                            uint64_t p) {
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const bool loop = emit && row == b;
  if (emit && !loop) {
    const uint64_t cp = p - O.loopx[row] - ((O.hl[row] && b > row) ? 1u : 0u);
    O.col[cp] = b;
    O.cw[cp] = __double2float_rn(__dadd_rn((double)wf, (double)wf));
  }
  if (loop) {
    O.loopw[row] = wf;
    O.has_loop[row] = 1;
  }
  float f = wf == 0.0f ? 1.0f : wf;
  if (loop) f *= 2.0f;
  const double sum = ic_seg_sum(emit ? __dadd_rn((double)f, (double)f) : 0.0, row);
  const int32_t nx = __shfl_down_sync(full, row, 1);
  if (row >= 0 && (lane == 31 || nx != row) && sum != 0.0) atomicAdd(&O.k[row], sum);
}

// Runs of the segments inside one chunk, to their final slots.  A block per chunk.
__global__ void ic_final_closed_kernel(const uint32_t* c_runs, const uint32_t* c_nl, const uint32_t* c_nr,
                                       const uint32_t* c_flags, const uint64_t* tkey, const double* tsum,
                                       const uint32_t* segoff, const uint32_t* firstrun, int32_t* osrc,
                                       int32_t* odst, float* ow, IcCsrOut O) {
  const int64_t j = blockIdx.x;
  if (c_flags[j] & kSingle) return;
  const uint32_t lo = c_nl[j], hi = c_runs[j] - c_nr[j];
  for (uint32_t r0 = lo; r0 < hi; r0 += blockDim.x) {   // whole warps every round
    const uint32_t r = r0 + threadIdx.x;
    const bool valid = r < hi;
    int32_t a = -1, b = 0;
    float wf = 0.0f;
    uint64_t p = 0;
    if (valid) {
      const uint64_t tt = (uint64_t)j * kIcChunk + r;
      const uint64_t kk = tkey[tt];
      a = (int32_t)(kk >> 32);
      b = (int32_t)(uint32_t)kk;
      p = (uint64_t)segoff[a] + (tt - firstrun[a]);
      wf = __double2float_rn(tsum[tt]);
      osrc[p] = a;
      odst[p] = b;
      ow[p] = wf;
    }
    if (O.col) ic_emit_csr(O, valid, a, b, wf, p);
  }
}

// Distinct keys of the open segments, to their final slots.  Grid-stride
// over whole warps.
__global__ void ic_final_open_kernel(const uint64_t* k, int64_t n, int Bb, const uint32_t* pos,
                                     const uint32_t* head, const uint32_t* ofirst, const int32_t* oa,
                                     const uint32_t* segoff, const double* osum, int32_t* osrc, int32_t* odst,
                                     float* ow, IcCsrOut O) {
  const uint64_t bmask = (1ull << Bb) - 1ull;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i0 = blockIdx.x * (int64_t)blockDim.x; i0 < n; i0 += stride) {
    const int64_t i = i0 + threadIdx.x;
    const bool in = i < n;
    const bool emit = in && head[i];
    int32_t a = -1, b = 0;
    float wf = 0.0f;
    uint64_t p = 0;
    if (in) {
      const uint64_t kk = k[i];
      const uint32_t o = (uint32_t)(kk >> Bb);
      a = oa[o];
      b = (int32_t)(kk & bmask);
      if (emit) {
        const uint32_t g = pos[i];
        p = (uint64_t)segoff[a] + (g - ofirst[o]);
        wf = __double2float_rn(osum[g]);
        osrc[p] = a;
        odst[p] = b;
        ow[p] = wf;
      }
    }
    if (O.col) ic_emit_csr(O, emit, a, b, wf, p);
  }
}

// CSR row offsets of the next level: list row start minus the loops before.
__global__ void ic_csr_off_kernel(int32_t C, const uint32_t* segoff, const uint32_t* loopx, int64_t* off) {
  IC_FOR(a, (int64_t)C + 1) off[a] = (int64_t)segoff[a] - (int64_t)loopx[a];
}

// Bytes of scratch induce_sorted may take, at most (the open runs can be all
// runs in the worst case).
size_t induce_sorted_scratch(int64_t V, int64_t E, int64_t C) {
  const int64_t nchunks = (E + kIcChunk - 1) / kIcChunk;
  const int64_t slots = nchunks * kIcChunk;
  size_t b = 0;
  b += (size_t)V * (2 * 12 + 4 + 4 + 4 + 8) + 8 * 256 * (size_t)(V / 4096 + 2);   // member sort, scans
  b += (size_t)E * 4 + (size_t)slots * 16 + (size_t)nchunks * 28 + (size_t)C * 20;   // cv, runs, chunk facts
  b += (size_t)E * (2 * 12 + 4 + 4 + 8 + 4) + 8 * 256 * (size_t)(E / 4096 + 2); // open runs, worst case
  return b + ((size_t)64 << 10) * 32;                                            // alignment slack
}

void ic_attributes() {
  constexpr int kDevs = 64;
  static std::mutex mu;
  static bool done[kDevs] = {};
  int dev = 0;
  LVG_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(mu);
  if (dev >= 0 && dev < kDevs && done[dev]) return;
  LVG_CUDA(cudaFuncSetAttribute(ic_chunk_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(IcSmem)));
  if (dev >= 0 && dev < kDevs) done[dev] = true;
}

template <typename T>
T read_back(const T* d, cudaStream_t s) {
  T h{};
  LVG_CUDA(cudaMemcpyAsync(&h, d, sizeof(T), cudaMemcpyDeviceToHost, s));
  LVG_CUDA(cudaStreamSynchronize(s));
  return h;
}

// ------------------------------------------------------------ by transposition
// The members' rows read in community order (the segment layout above) list
// every entry (u, d) grouped by part[u], ascending.  The list is symmetric
// with bitwise-equal weights, so (d, u, w) is an entry as well, and the same
// positions therefore list every coarse key (part[d], part[u]) grouped by its
// SECOND community, ascending.  One stable sort by the first community alone
// then leaves the keys in (first, second) order with equal keys adjacent:
// 8-bit passes over one community width instead of two, and no sort inside
// the segments.
constexpr int kTxThreads = 256;
constexpr int kTxItems = kIcChunk / kTxThreads;   // 16 consecutive positions (entries) per thread

// Per member of a chunk: start relative to the chunk (0 for the member
// holding the chunk's first position), list index of its first position
// minus its start, community.
struct TxSmem {
  int32_t rs[kIcChunk + 2];
  int64_t eb[kIcChunk + 1];
  int32_t yc[kIcChunk + 1];
};

// Keys (dense community of d << Bb | community of u: the caller passes the
// dense ids of the vertices as `part`) and weights (0 counted as 1) of the
// entries
// in segment order, a block per 4096 positions.  The chunk's members are
// staged in shared memory; a thread takes 16 positions 256 apart, finds the
// member of each by a binary search, then issues all 16 list loads and all
// 16 community gathers before it uses any of them.
__global__ void __launch_bounds__(kTxThreads) tx_layout_kernel(
    int64_t E, int32_t nz, int Bb, const int32_t* mem, const int32_t* mcomm, const int64_t* mscan,
    const int32_t* cfirst, const int64_t* off, const uint32_t* lscan, const int32_t* ldst, const float* lw,
    const int32_t* part, uint64_t* keys, float* vals, uint32_t* notint) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  TxSmem& S = *reinterpret_cast<TxSmem*>(smem_raw);
  const int64_t c = blockIdx.x;
  const int64_t p0 = c * (int64_t)kIcChunk;
  const int n = (int)min((int64_t)kIcChunk, E - p0);
  // members j0 .. jend - 1 cover [p0, p0 + n); at most kIcChunk of them start
  // inside the chunk, so nm <= kIcChunk + 1
  const int32_t j0 = cfirst[c];
  const int32_t jend = min(cfirst[c + 1] + 1, nz);
  const int nm = jend - j0;
  {   // stage the members: every thread's loads issued before any is used
    constexpr int kStage = (kIcChunk + 2 + kTxThreads - 1) / kTxThreads;
    int64_t st[kStage];
    int32_t uu[kStage], yy[kStage];
#pragma unroll
    for (int x = 0; x < kStage; ++x) {
      const int t = threadIdx.x + x * kTxThreads;
      st[x] = t <= nm ? mscan[j0 + t] : 0;
      uu[x] = t < nm ? mem[j0 + t] : 0;
      yy[x] = t < nm ? mcomm[j0 + t] : 0;
    }
    int64_t ob[kStage];
#pragma unroll
    for (int x = 0; x < kStage; ++x) {
      const int t = threadIdx.x + x * kTxThreads;
      ob[x] = t < nm ? off[uu[x]] + (int64_t)lscan[uu[x]] : 0;
    }
#pragma unroll
    for (int x = 0; x < kStage; ++x) {
      const int t = threadIdx.x + x * kTxThreads;
      if (t <= nm) {
        const int64_t r = st[x] - p0;
        S.rs[t] = (int32_t)(r < 0 ? 0 : (r > kIcChunk ? kIcChunk : r));
      }
      if (t < nm) {
        S.eb[t] = ob[x] - st[x];
        S.yc[t] = yy[x];
      }
    }
  }
  __syncthreads();
  // position q = i * 256 + thread: a warp's loads and stores are contiguous
  // along the rows; the member of each position by a branch-free binary
  // search over the staged starts (all 16 searches independent)
  bool frac = false;
  int64_t e[kTxItems];
  int32_t y[kTxItems];
#pragma unroll
  for (int i = 0; i < kTxItems; ++i) {
    const int q = i * kTxThreads + threadIdx.x;
    int lo = 0;
#pragma unroll
    for (int b = 12; b >= 0; --b) {   // nm <= kIcChunk + 1 < 2^13
      const int cand = lo + (1 << b);
      if (cand < nm && S.rs[cand] <= q) lo = cand;
    }
    e[i] = q < n ? S.eb[lo] + p0 + q : 0;
    y[i] = S.yc[lo];
  }
  int32_t d[kTxItems];
  float wv[kTxItems];
#pragma unroll
  for (int i = 0; i < kTxItems; ++i) {
    const bool ok = i * kTxThreads + (int)threadIdx.x < n;
    d[i] = ok ? __ldg(ldst + e[i]) : 0;
    wv[i] = ok ? __ldg(lw + e[i]) : 1.0f;
  }
#pragma unroll
  for (int i = 0; i < kTxItems; ++i) d[i] = __ldg(part + d[i]);
#pragma unroll
  for (int i = 0; i < kTxItems; ++i) {
    const int q = i * kTxThreads + threadIdx.x;
    if (q < n) {
      keys[p0 + q] = ((uint64_t)(uint32_t)d[i] << Bb) | (uint32_t)y[i];
      vals[p0 + q] = wv[i] == 0.0f ? 1.0f : wv[i];   // InducedGraphKernel.cu:38-39
      frac |= wv[i] != truncf(wv[i]);
    }
  }
  if (__syncthreads_or(frac) && threadIdx.x == 0) atomicOr(notint, 1u);
}

// The 16 sorted keys and weights of a thread (16-byte loads when whole).
__device__ __forceinline__ int tx_load16(const uint64_t* k, const float* v, int64_t i0, int64_t n,
                                         uint64_t (&kk)[kTxItems], float (&vv)[kTxItems]) {
  const int m = (int)max((int64_t)0, min((int64_t)kTxItems, n - i0));
  if (m == kTxItems) {
#pragma unroll
    for (int i = 0; i < kTxItems; i += 2) {
      const ulonglong2 x = reinterpret_cast<const ulonglong2*>(k + i0)[i / 2];
      kk[i] = x.x;
      kk[i + 1] = x.y;
    }
    if (v) {
#pragma unroll
      for (int i = 0; i < kTxItems; i += 4) {
        const float4 x = reinterpret_cast<const float4*>(v + i0)[i / 4];
        vv[i] = x.x; vv[i + 1] = x.y; vv[i + 2] = x.z; vv[i + 3] = x.w;
      }
    }
  } else {
#pragma unroll
    for (int i = 0; i < kTxItems; ++i) {
      kk[i] = i < m ? k[i0 + i] : ~0ull;
      if (v) vv[i] = i < m ? v[i0 + i] : 0.0f;
    }
  }
  return m;
}

// Runs of equal keys (dense first community << Bb | second community), per
// 4096-entry tile of the sorted keys: the number of run heads (first entries;
// low 32 bits) and of heads that are coarse self loops (high 32 bits), so
// that one scan gives every run its distinct index and the self loops before
// it.
__global__ void __launch_bounds__(kTxThreads) tx_count_kernel(const uint64_t* k, int64_t n, int Bb,
                                                              const int32_t* und, int64_t* tcount) {
  const uint64_t mask = (1ull << Bb) - 1ull;
  const int64_t i0 = blockIdx.x * (int64_t)kIcChunk + (int64_t)threadIdx.x * kTxItems;
  uint64_t kk[kTxItems];
  float unused[kTxItems];
  const int m = tx_load16(k, nullptr, i0, n, kk, unused);
  uint64_t prev = (i0 > 0 && m > 0) ? k[i0 - 1] : ~0ull;
  unsigned long long cnt = 0;
#pragma unroll
  for (int i = 0; i < kTxItems; ++i) {
    if (i < m && (i0 + i == 0 || kk[i] != prev))
      cnt += ((uint64_t)und[(int32_t)(kk[i] >> Bb)] == (kk[i] & mask)) ? (1ull << 32) + 1ull : 1ull;
    prev = kk[i];
  }
  unsigned long long tot;
  block_exclusive_scan256<unsigned long long>(cnt, &tot);
  if (threadIdx.x == 0) tcount[blockIdx.x] = (int64_t)tot;
}

__device__ __forceinline__ double tx_seg_sum(double v, int64_t seg) {
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const double u = __shfl_up_sync(full, v, o);
    const int64_t t = __shfl_up_sync(full, seg, o);
    if (lane >= o && t == seg) v = __dadd_rn(v, u);
  }
  return v;
}

__device__ __forceinline__ bool tx_seg_last(int64_t seg, bool valid) {
  const unsigned full = 0xffffffffu;
  const int64_t nx = __shfl_down_sync(full, seg, 1);
  const bool nvalid = __shfl_down_sync(full, valid, 1);
  return valid && ((threadIdx.x & 31) == 31 || !nvalid || nx != seg);
}

struct TxEmitSmem {
  uint64_t key[kIcChunk];     // key of the tile's i-th distinct entry
  double sum[kIcChunk];       // its summed weight; -1: the run is still open at the tile's end
  uint16_t lp[kIcChunk];      // coarse self loops among the tile's distinct entries before it
  double lead[kTxThreads];    // sum of a thread's entries before its first head
  uint8_t anyhead[kTxThreads];
};

__device__ __forceinline__ uint32_t tx_lo(int64_t x) { return (uint32_t)((uint64_t)x & 0xffffffffull); }
__device__ __forceinline__ uint32_t tx_hi(int64_t x) { return (uint32_t)((uint64_t)x >> 32); }

// One coarse entry (row a, column b, float weight wf) at distinct index r
// with `lb` self loops before it into the next level's CSR: a loop sets the
// row's loop weight, any other entry goes to position r - lb (weight doubled:
// the merged doubled list holds each entry twice).  The row's degree, summed
// over the lanes of the warp with the same row, is added by the caller.
__device__ __forceinline__ double tx_csr_entry(const IcCsrOut& O, int32_t a, int32_t b, float wf, int64_t r,
                                               int64_t lb) {
  const bool loop = a == b;
  if (loop) {
    O.loopw[a] = wf;
    O.has_loop[a] = 1;
  } else {
    O.col[r - lb] = b;
    O.cw[r - lb] = __double2float_rn(__dadd_rn((double)wf, (double)wf));
  }
  float f = wf == 0.0f ? 1.0f : wf;   // InitKernel.cu:154-179: weight 0 counts 1, a loop twice
  if (loop) f *= 2.0f;
  return __dadd_rn((double)f, (double)f);
}

// Each run of equal keys (dense first community, mapped back by und; the
// second community as it is) once, a block per 4096-entry tile, 16 consecutive
// entries per thread.  A thread sums the runs that start in its entries in
// entry order (FP64); a run that goes on past the thread is finished by the
// thread holding its head, which adds the leading pieces of the threads after
// it.  The tile's distinct entries are staged in shared memory and written in
// order: (osrc, odst), the float weight, the coarse self loops (hl), the
// distinct entries per row (dcount) and, with O.col, the next level's CSR
// entry and the row degrees.  The tile's last run, when it goes on into the
// next tiles, is summed with atomics into opensum[tile] (its continuations
// find the tile by a binary search) and finished by tx_open_kernel.
__global__ void __launch_bounds__(kTxThreads) tx_emit_kernel(const uint64_t* k, const float* v, int64_t n, int Bb,
                                                             const int64_t* tscan, const int32_t* und,
                                                             int32_t* osrc, int32_t* odst, float* ow, double* opensum,
                                                             uint32_t* openflag, uint32_t* hl, uint32_t* dcount,
                                                             IcCsrOut O) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  TxEmitSmem& S = *reinterpret_cast<TxEmitSmem*>(smem_raw);
  const uint64_t mask = (1ull << Bb) - 1ull;
  const int t = threadIdx.x;
  const int64_t tile = blockIdx.x;
  const int64_t i0 = tile * kIcChunk + (int64_t)t * kTxItems;
  uint64_t kk[kTxItems];
  float vv[kTxItems];
  const int m = tx_load16(k, v, i0, n, kk, vv);
  uint64_t prev = (i0 > 0 && m > 0) ? k[i0 - 1] : ~0ull;
  uint32_t hmask = 0, nloop = 0;
#pragma unroll
  for (int i = 0; i < kTxItems; ++i) {
    if (i < m && (i0 + i == 0 || kk[i] != prev)) {
      hmask |= 1u << i;
      nloop += (uint64_t)und[(int32_t)(kk[i] >> Bb)] == (kk[i] & mask) ? 1u : 0u;
    }
    prev = kk[i];
  }
  unsigned long long both;
  const unsigned long long ex =
      block_exclusive_scan256<unsigned long long>(((unsigned long long)nloop << 32) | (uint32_t)__popc(hmask), &both);
  const uint32_t tot = (uint32_t)both;
  int loc = (int)(uint32_t)ex - 1;
  uint32_t lc = (uint32_t)(ex >> 32);   // self loops among the tile's distinct entries before the next head
  double s = 0.0;
  bool started = false;
#pragma unroll
  for (int i = 0; i < kTxItems; ++i) {
    if (i < m) {
      if ((hmask >> i) & 1u) {
        if (started) S.sum[loc] = s;   // a run that began and ended in this thread
        else S.lead[t] = s;
        started = true;
        ++loc;
        S.key[loc] = kk[i];
        S.lp[loc] = (uint16_t)lc;
        lc += (uint64_t)und[(int32_t)(kk[i] >> Bb)] == (kk[i] & mask) ? 1u : 0u;
        s = (double)vv[i];
      } else {
        s = __dadd_rn(s, (double)vv[i]);
      }
    }
  }
  if (!started) S.lead[t] = s;
  S.anyhead[t] = started ? 1 : 0;
  __syncthreads();
  const int64_t tb = tx_lo(tscan[tile]);
  if (t == 0 && m > 0 && !(hmask & 1u)) {
    // entries before the tile's first head continue the last run of an
    // earlier tile h: the run with distinct index tb - 1
    double x = 0.0;
    for (int u = 0; u < kTxThreads; ++u) {
      x = __dadd_rn(x, S.lead[u]);
      if (S.anyhead[u]) break;
    }
    int64_t lo = tile - 1, hi = tile - 1;   // last tile whose first distinct index is <= tb - 1
    if ((int64_t)tx_lo(tscan[lo]) > tb - 1) lo = 0;   // the previous tile holds no head: search
    while (lo < hi) {
      const int64_t mid = (lo + hi + 1) >> 1;
      if ((int64_t)tx_lo(tscan[mid]) <= tb - 1) lo = mid; else hi = mid - 1;
    }
    atomicAdd(&opensum[lo], x);
  }
  if (started) {   // the thread's last run takes the leading pieces after it
    double x = s;
    bool open = true;
    for (int u = t + 1; u < kTxThreads; ++u) {
      x = __dadd_rn(x, S.lead[u]);
      if (S.anyhead[u]) { open = false; break; }
    }
    if (open && i0 + kIcChunk - (int64_t)t * kTxItems < n) {   // goes on into the next tile
      atomicAdd(&opensum[tile], x);
      openflag[tile] = 1u;
      S.sum[loc] = -1.0;
    } else {
      S.sum[loc] = x;
    }
  }
  __syncthreads();
  // the tile's distinct entries, in order
  const int64_t lt = tx_hi(tscan[tile]);
  const int lane = t & 31;
  for (uint32_t l0 = 0; l0 < tot; l0 += kTxThreads) {
    const uint32_t l = l0 + t;
    const bool valid = l < tot;
    const int64_t r = tb + l;
    int32_t a = -1, b = 0;
    double x = -1.0;
    if (valid) {
      const uint64_t key = S.key[l];
      a = und[(int32_t)(key >> Bb)];
      b = (int32_t)(key & mask);
      x = S.sum[l];
      osrc[r] = a;
      odst[r] = b;
      if (a == b) hl[a] = 1u;
    }
    const bool closed = valid && x >= 0.0;
    const float wf = closed ? __double2float_rn(x) : 0.0f;
    if (closed) ow[r] = wf;
    // distinct entries per row: lanes of one row are consecutive
    const int32_t ap = __shfl_up_sync(0xffffffffu, a, 1);
    const unsigned starts = __ballot_sync(0xffffffffu, valid && (lane == 0 || ap != a));
    const bool last = tx_seg_last(a, valid);
    if (last) {
      const int first = 31 - __clz(starts & (0xffffffffu >> (31 - lane)));
      atomicAdd(&dcount[a], (uint32_t)(lane - first + 1));
    }
    if (O.col) {
      const double kd = closed ? tx_csr_entry(O, a, b, wf, r, lt + (valid ? S.lp[l] : 0)) : 0.0;
      const double ks = tx_seg_sum(kd, a);
      if (last && ks != 0.0) atomicAdd(&O.k[a], ks);
    }
  }
}

// The runs left open at a tile's end: their final sums, float weights and
// CSR entries (one thread per tile).
__global__ void tx_open_kernel(int64_t ntiles, const int64_t* tscan, const double* opensum, const uint32_t* openflag,
                               const int32_t* osrc, const int32_t* odst, float* ow, IcCsrOut O) {
  IC_FOR(h, ntiles) {
    if (!openflag[h]) continue;
    const int64_t r = (int64_t)tx_lo(tscan[h + 1]) - 1;   // the tile's last run
    const float wf = __double2float_rn(opensum[h]);
    ow[r] = wf;
    if (O.col) {
      const int32_t a = osrc[r], b = odst[r];
      const int64_t lb = (int64_t)tx_hi(tscan[h + 1]) - (a == b ? 1 : 0);
      atomicAdd(&O.k[a], tx_csr_entry(O, a, b, wf, r, lb));
    }
  }
}

// Dense ids of the communities that have entries (members 0 .. nz - 1 are
// sorted by community), mapped both ways.
// Sorting by dense ids needs bits for these communities only; the first
// level of a graph with many isolated vertices has far fewer of them than
// communities.
__global__ void tx_dense_flag_kernel(int32_t nz, const int32_t* mcomm, uint32_t* flag) {
  IC_FOR(i, nz) flag[i] = (i == 0 || mcomm[i] != mcomm[i - 1]) ? 1u : 0u;
}

__global__ void tx_dense_kernel(int32_t nz, const int32_t* mcomm, const uint32_t* ex, int32_t* dn, int32_t* und) {
  IC_FOR(i, nz) {
    if (i == 0 || mcomm[i] != mcomm[i - 1]) {
      dn[mcomm[i]] = (int32_t)ex[i];
      und[ex[i]] = mcomm[i];
    }
  }
}

// Dense community id of every vertex with entries (the only vertices that
// appear as a neighbour); 0 for the others, which are never read.
__global__ void tx_vdense_kernel(int32_t V, const int32_t* part, const int64_t* off, const uint8_t* has_loop,
                                 const int32_t* dn, int32_t* pd) {
  IC_FOR(v, V) pd[v] = (off[v + 1] > off[v] || has_loop[v]) ? dn[part[v]] : 0;
}

void tx_attributes() {
  constexpr int kDevs = 64;
  static std::mutex mu;
  static bool done[kDevs] = {};
  int dev = 0;
  LVG_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(mu);
  if (dev >= 0 && dev < kDevs && done[dev]) return;
  LVG_CUDA(cudaFuncSetAttribute(tx_layout_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(TxSmem)));
  LVG_CUDA(cudaFuncSetAttribute(tx_emit_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)sizeof(TxEmitSmem)));
  if (dev >= 0 && dev < kDevs) done[dev] = true;
}

}  // namespace

// Bytes of scratch induce_transposed may take, at most.
size_t induce_transposed_scratch(int64_t V, int64_t E, int64_t C) {
  const int64_t nchunks = (E + kIcChunk - 1) / kIcChunk;
  size_t b = 0;
  b += (size_t)V * (2 * 12 + 4 + 4 + 4 + 8) + 8 * 256 * (size_t)(V / 4096 + 2);   // member sort, scans
  b += (size_t)(nchunks + 1) * 4;                                                  // chunk first members
  b += (size_t)E * (2 * 12) + 8 * 256 * (size_t)(E / 4096 + 2);                   // keys, weights, look-back
  b += 32 * (size_t)(E / 4096 + 2);                                                // tile counts, open runs
  b += (size_t)V * 16 + (size_t)C * 8;                                             // dense community ids
  b += (size_t)C * 16 + 64;                                                        // loops, counts, offsets
  return b + ((size_t)64 << 10) * 32;                                              // alignment slack
}

bool induce_transposed(const LevelGraph& g, const int32_t* part, int32_t C, int32_t* osrc, int32_t* odst, float* ow,
                       int64_t* count, PreCsr* next, Arena& a, cudaStream_t s) {
  const int32_t V = g.V;
  const int64_t E = g.E;
  if (!g.sorted_symmetric || V <= 0 || C <= 0) return false;
  if (E + 2 * (int64_t)kIcChunk >= ((int64_t)1 << 32)) return false;   // heads and positions are 32-bit
  if (a.hi < a.lo || a.hi - a.lo < induce_transposed_scratch(V, E, C)) return false;
  if (E == 0) { *count = 0; return true; }
  HiScope hs(a);
  const int64_t nchunks = (E + kIcChunk - 1) / kIcChunk;
  // members in community order (stable: vertex order inside a community)
  uint64_t* mk0 = a.hi_n<uint64_t>(V);
  float* mv0 = a.hi_n<float>(V);
  uint64_t* mk1 = a.hi_n<uint64_t>(V);
  float* mv1 = a.hi_n<float>(V);
  uint32_t* lscan = a.hi_n<uint32_t>(V + 1);
  ic_member_keys_kernel<<<ic_grid(V), kIcFlat, 0, s>>>(V, g.off, g.has_loop, part, C, mk0, mv0, lscan);
  LVG_LAUNCH();
  const int which = radix_sort_pairs(mk0, mv0, mk1, mv1, V, bits_for((int64_t)C + 1), a, s);
  scan_u32(lscan, lscan, V, a, s);   // self loops before each vertex: list row start = off + lscan
  int32_t* mem = a.hi_n<int32_t>(V);
  int32_t* mcomm = a.hi_n<int32_t>(V);
  int64_t* mscan = a.hi_n<int64_t>(V + 1);
  int32_t* nz = a.hi_n<int32_t>(1);
  LVG_CUDA(cudaMemsetAsync(nz, 0, sizeof(int32_t), s));
  ic_member_len_kernel<<<ic_grid(V), kIcFlat, 0, s>>>(V, which ? mk1 : mk0, which ? mv1 : mv0, g.off, g.has_loop,
                                                      C, mem, mcomm, mscan, nz);
  LVG_LAUNCH();
  scan_i64(mscan, mscan, V, a, s);
  int64_t h_rows = 0;
  int32_t h_nz = 0;
  LVG_CUDA(cudaMemcpyAsync(&h_rows, mscan + V, sizeof h_rows, cudaMemcpyDeviceToHost, s));
  LVG_CUDA(cudaMemcpyAsync(&h_nz, nz, sizeof h_nz, cudaMemcpyDeviceToHost, s));
  LVG_CUDA(cudaStreamSynchronize(s));   // both values with one wait
  if (h_rows != E) throw Error(LVG_ERR_CUDA, "coarsening: list rows disagree with the CSR");
  int32_t* cfirst = a.hi_n<int32_t>(nchunks + 1);
  ic_chunk_first_kernel<<<ic_grid(V), kIcFlat, 0, s>>>(mscan, nz, cfirst, nchunks);
  LVG_LAUNCH();
  // dense ids of the communities with entries: the sort needs their bits only
  uint32_t* dflag = a.hi_n<uint32_t>(h_nz + 1);
  int32_t* dn = a.hi_n<int32_t>(C);
  int32_t* und = a.hi_n<int32_t>(C);
  int32_t* pd = a.hi_n<int32_t>(V);
  tx_dense_flag_kernel<<<ic_grid(h_nz), kIcFlat, 0, s>>>(h_nz, mcomm, dflag);
  LVG_LAUNCH();
  scan_u32(dflag, dflag, h_nz, a, s);
  tx_dense_kernel<<<ic_grid(h_nz), kIcFlat, 0, s>>>(h_nz, mcomm, dflag, dn, und);
  LVG_LAUNCH();
  tx_vdense_kernel<<<ic_grid(V), kIcFlat, 0, s>>>(V, part, g.off, g.has_loop, dn, pd);
  LVG_LAUNCH();
  const int64_t ndense = read_back(dflag + h_nz, s);
  const int Bb = std::max(1, bits_for(C));            // second community, as it is
  const int Bd = std::max(1, bits_for(ndense));       // first community, dense: the sort key
  // keys in segment order, then one stable sort by the first community
  uint64_t* k0 = a.hi_n<uint64_t>(E);
  float* v0 = a.hi_n<float>(E);
  uint64_t* k1 = a.hi_n<uint64_t>(E);
  float* v1 = a.hi_n<float>(E);
  uint32_t* flags = a.hi_n<uint32_t>(1);   // a weight not integral
  LVG_CUDA(cudaMemsetAsync(flags, 0, sizeof(uint32_t), s));
  tx_attributes();
  tx_layout_kernel<<<(unsigned)nchunks, kTxThreads, sizeof(TxSmem), s>>>(E, h_nz, Bb, mem, mcomm, mscan, cfirst,
                                                                         g.off, lscan, g.dst, g.w, pd, k0, v0,
                                                                         flags);
  LVG_LAUNCH();
  const int w2 = radix_sort_pairs_range(k0, v0, k1, v1, E, Bb, Bd, a, s);
  const uint64_t* keys = w2 ? k1 : k0;
  const float* vals = w2 ? v1 : v0;
  // runs of equal keys: heads (and self-loop heads) per 4096-entry tile,
  // their scan, then every run once
  int64_t* tscan = a.hi_n<int64_t>(nchunks + 1);
  tx_count_kernel<<<(unsigned)nchunks, kTxThreads, 0, s>>>(keys, E, Bb, und, tscan);
  LVG_LAUNCH();
  scan_i64(tscan, tscan, nchunks, a, s);
  int64_t h_tot = 0;
  uint32_t h_frac = 0;
  LVG_CUDA(cudaMemcpyAsync(&h_tot, tscan + nchunks, sizeof h_tot, cudaMemcpyDeviceToHost, s));
  LVG_CUDA(cudaMemcpyAsync(&h_frac, flags, sizeof h_frac, cudaMemcpyDeviceToHost, s));
  LVG_CUDA(cudaStreamSynchronize(s));   // both values with one wait
  const int64_t cnt = (int64_t)((uint64_t)h_tot & 0xffffffffull);
  const bool int_weights = h_frac == 0u;
  double* opensum = a.hi_n<double>(nchunks);
  uint32_t* openflag = a.hi_n<uint32_t>(nchunks);
  uint32_t* hl = a.hi_n<uint32_t>((int64_t)C + 1);
  uint32_t* dcount = a.hi_n<uint32_t>((int64_t)C + 1);
  LVG_CUDA(cudaMemsetAsync(opensum, 0, sizeof(double) * (size_t)nchunks, s));
  LVG_CUDA(cudaMemsetAsync(openflag, 0, sizeof(uint32_t) * (size_t)nchunks, s));
  LVG_CUDA(cudaMemsetAsync(hl, 0, sizeof(uint32_t) * ((size_t)C + 1), s));
  LVG_CUDA(cudaMemsetAsync(dcount, 0, sizeof(uint32_t) * ((size_t)C + 1), s));
  // The CSR is written only for integral weights: then every sum is exact,
  // so the coarse list is exactly symmetric, as the CSR written from one
  // direction assumes.
  IcCsrOut O{};
  const bool csr = next && next->col && int_weights;
  if (csr) {
    LVG_CUDA(cudaMemsetAsync(next->k, 0, sizeof(double) * (size_t)C, s));
    LVG_CUDA(cudaMemsetAsync(next->loopw, 0, sizeof(float) * (size_t)C, s));
    LVG_CUDA(cudaMemsetAsync(next->has_loop, 0, (size_t)C, s));
    O = IcCsrOut{next->col, next->cw, next->k, next->loopw, next->has_loop, hl, nullptr};
  }
  tx_emit_kernel<<<(unsigned)nchunks, kTxThreads, sizeof(TxEmitSmem), s>>>(keys, vals, E, Bb, tscan, und, osrc,
                                                                           odst, ow, opensum, openflag, hl, dcount,
                                                                           O);
  LVG_LAUNCH();
  tx_open_kernel<<<ic_grid(nchunks), kIcFlat, 0, s>>>(nchunks, tscan, opensum, openflag, osrc, odst, ow, O);
  LVG_LAUNCH();
  if (csr) {   // the rest of the next level's CSR: row offsets, entry count, m
    uint32_t* segoff = a.hi_n<uint32_t>((int64_t)C + 1);
    uint32_t* loopx = a.hi_n<uint32_t>((int64_t)C + 1);
    scan_u32(dcount, segoff, C, a, s);
    scan_u32(hl, loopx, C, a, s);
    ic_csr_off_kernel<<<ic_grid((int64_t)C + 1), kIcFlat, 0, s>>>(C, segoff, loopx, next->off);
    LVG_LAUNCH();
    double* d_m = a.hi_n<double>(1);
    tree_sum_f32(ow, cnt, d_m, a, s);   // as build_level's m over the list (NeighbourCompute.cu:46)
    LVG_CUDA(cudaMemcpyAsync(&next->m, d_m, sizeof(double), cudaMemcpyDeviceToHost, s));
    const int64_t loops = read_back(loopx + C, s);
    next->nnz = cnt - loops;
    next->valid = true;
  }
  LVG_CUDA(cudaStreamSynchronize(s));
  *count = cnt;
  return true;
}

bool induce_sorted(const LevelGraph& g, const int32_t* part, int32_t C, int32_t* osrc, int32_t* odst, float* ow,
                   int64_t* count, PreCsr* next, Arena& a, cudaStream_t s) {
  const int32_t V = g.V;
  const int64_t E = g.E;
  if (!g.sorted_symmetric || V <= 0 || C <= 0) return false;
  if (E + 2 * (int64_t)kIcChunk >= ((int64_t)1 << 32)) return false;   // slots and counts are 32-bit
  if (a.hi < a.lo || a.hi - a.lo < induce_sorted_scratch(V, E, C)) return false;
  if (E == 0) { *count = 0; return true; }
  HiScope hs(a);
  const int64_t nchunks = (E + kIcChunk - 1) / kIcChunk;
  const int Bb = bits_for(C);
  // members in community order (stable: vertex order inside a community)
  uint64_t* mk0 = a.hi_n<uint64_t>(V);
  float* mv0 = a.hi_n<float>(V);
  uint64_t* mk1 = a.hi_n<uint64_t>(V);
  float* mv1 = a.hi_n<float>(V);
  uint32_t* lscan = a.hi_n<uint32_t>(V + 1);
  ic_member_keys_kernel<<<ic_grid(V), kIcFlat, 0, s>>>(V, g.off, g.has_loop, part, C, mk0, mv0, lscan);
  LVG_LAUNCH();
  const int which = radix_sort_pairs(mk0, mv0, mk1, mv1, V, bits_for((int64_t)C + 1), a, s);
  scan_u32(lscan, lscan, V, a, s);   // self loops before each vertex: list row start = off + lscan
  int32_t* mem = a.hi_n<int32_t>(V);
  int32_t* mcomm = a.hi_n<int32_t>(V);
  int64_t* mscan = a.hi_n<int64_t>(V + 1);
  int32_t* nz = a.hi_n<int32_t>(1);
  LVG_CUDA(cudaMemsetAsync(nz, 0, sizeof(int32_t), s));
  ic_member_len_kernel<<<ic_grid(V), kIcFlat, 0, s>>>(V, which ? mk1 : mk0, which ? mv1 : mv0, g.off, g.has_loop,
                                                      C, mem, mcomm, mscan, nz);
  LVG_LAUNCH();
  scan_i64(mscan, mscan, V, a, s);
  if (read_back(mscan + V, s) != E) throw Error(LVG_ERR_CUDA, "coarsening: list rows disagree with the CSR");
  int32_t* cfirst = a.hi_n<int32_t>(nchunks + 1);
  ic_chunk_first_kernel<<<ic_grid(V), kIcFlat, 0, s>>>(mscan, nz, cfirst, nchunks);
  LVG_LAUNCH();
  // chunks
  uint64_t* tkey = a.hi_n<uint64_t>(nchunks * kIcChunk);
  double* tsum = a.hi_n<double>(nchunks * kIcChunk);
  uint32_t* dcount = a.hi_n<uint32_t>((int64_t)C + 1);
  uint32_t* hl = a.hi_n<uint32_t>((int64_t)C + 2);   // coarse self loops; [C + 1]: a weight not integral
  uint32_t* notint = hl + C + 1;
  LVG_CUDA(cudaMemsetAsync(hl, 0, sizeof(uint32_t) * ((size_t)C + 2), s));
  uint32_t* firstrun = a.hi_n<uint32_t>(C);
  uint32_t* c_runs = a.hi_n<uint32_t>(nchunks);
  uint32_t* c_nl = a.hi_n<uint32_t>(nchunks);
  uint32_t* c_nr = a.hi_n<uint32_t>(nchunks);
  uint32_t* c_flags = a.hi_n<uint32_t>(nchunks);
  int32_t* c_ar = a.hi_n<int32_t>(nchunks);
  LVG_CUDA(cudaMemsetAsync(dcount, 0, sizeof(uint32_t) * ((size_t)C + 1), s));
  ic_attributes();
  int32_t* cvl = a.hi_n<int32_t>(E);
  ic_cv_kernel<<<ic_grid(E), kIcFlat, 0, s>>>(g.dst, part, E, cvl);
  LVG_LAUNCH();
  ic_chunk_kernel<<<(unsigned)nchunks, kIcThreads, sizeof(IcSmem), s>>>(
      E, nchunks, Bb, mem, mcomm, mscan, cfirst, g.off, lscan, cvl, g.w, tkey, tsum, dcount, firstrun, c_runs,
      c_nl, c_nr, c_flags, c_ar, hl, notint);
  LVG_LAUNCH();
  // segments open across chunk boundaries
  uint32_t* newr = a.hi_n<uint32_t>(nchunks + 1);
  uint32_t* nopen = a.hi_n<uint32_t>(nchunks + 1);
  ic_open_count_kernel<<<ic_grid(nchunks), kIcFlat, 0, s>>>(nchunks, c_runs, c_nl, c_nr, c_flags, newr, nopen);
  LVG_LAUNCH();
  scan_u32(newr, newr, nchunks, a, s);
  scan_u32(nopen, nopen, nchunks, a, s);
  const uint32_t n_open = read_back(newr + nchunks, s);
  // The CSR is written only for integral weights: then every sum is exact,
  // so the coarse list is exactly symmetric, as the CSR written from one
  // direction assumes.
  const bool int_weights = read_back(notint, s) == 0u;
  const int64_t n_orun = read_back(nopen + nchunks, s);
  uint64_t* okeys = nullptr;
  uint32_t *ohead = nullptr, *opos = nullptr, *ofirst = nullptr;
  int32_t* oa = nullptr;
  double* osum = nullptr;
  if (n_orun > 0) {
    uint64_t* ok0 = a.hi_n<uint64_t>(n_orun);
    float* ov0 = a.hi_n<float>(n_orun);
    uint64_t* ok1 = a.hi_n<uint64_t>(n_orun);
    float* ov1 = a.hi_n<float>(n_orun);
    oa = a.hi_n<int32_t>(n_open);
    ic_open_gather_kernel<<<ic_grid(nchunks * 32), kIcFlat, 0, s>>>(nchunks, Bb, c_runs, c_nl, c_nr, c_flags, c_ar,
                                                                     newr, nopen, tkey, ok0, ov0, oa);
    LVG_LAUNCH();
    const int w2 = radix_sort_pairs(ok0, ov0, ok1, ov1, n_orun, bits_for(n_open) + Bb, a, s);
    okeys = w2 ? ok1 : ok0;
    const float* ovals = w2 ? ov1 : ov0;
    ohead = a.hi_n<uint32_t>(n_orun + 1);
    opos = a.hi_n<uint32_t>(n_orun + 1);
    ic_head_kernel<<<ic_grid(n_orun), kIcFlat, 0, s>>>(okeys, n_orun, ohead);
    LVG_LAUNCH();
    scan_u32(ohead, opos, n_orun, a, s);
    const uint32_t n_odist = read_back(opos + n_orun, s);
    osum = a.hi_n<double>(n_odist);
    ofirst = a.hi_n<uint32_t>((int64_t)n_open + 1);
    LVG_CUDA(cudaMemsetAsync(osum, 0, sizeof(double) * std::max<uint32_t>(n_odist, 1), s));
    ic_open_sum_kernel<<<grid_for(n_orun, kIcFlat), kIcFlat, 0, s>>>(okeys, ovals, n_orun, Bb, opos, ohead, tsum,
                                                                      osum, ofirst, n_open);
    LVG_LAUNCH();
    ic_open_dcount_kernel<<<ic_grid(n_open), kIcFlat, 0, s>>>(n_open, ofirst, oa, dcount);
    LVG_LAUNCH();
  }
  // every community's first slot, then the entries
  uint32_t* segoff = a.hi_n<uint32_t>((int64_t)C + 1);
  scan_u32(dcount, segoff, C, a, s);
  const int64_t cnt = read_back(segoff + C, s);
  IcCsrOut O{};
  uint32_t* loopx = a.hi_n<uint32_t>((int64_t)C + 1);
  if (next && next->col && int_weights) {
    scan_u32(hl, loopx, C, a, s);
    LVG_CUDA(cudaMemsetAsync(next->k, 0, sizeof(double) * (size_t)C, s));
    LVG_CUDA(cudaMemsetAsync(next->loopw, 0, sizeof(float) * (size_t)C, s));
    LVG_CUDA(cudaMemsetAsync(next->has_loop, 0, (size_t)C, s));
    O = IcCsrOut{next->col, next->cw, next->k, next->loopw, next->has_loop, hl, loopx};
  }
  ic_final_closed_kernel<<<(unsigned)nchunks, kIcFlat, 0, s>>>(c_runs, c_nl, c_nr, c_flags, tkey, tsum, segoff,
                                                               firstrun, osrc, odst, ow, O);
  LVG_LAUNCH();
  if (n_orun > 0) {
    ic_final_open_kernel<<<ic_grid(n_orun), kIcFlat, 0, s>>>(okeys, n_orun, Bb, opos, ohead, ofirst, oa, segoff,
                                                             osum, osrc, odst, ow, O);
    LVG_LAUNCH();
  }
  if (O.col) {   // the rest of the next level's CSR: row offsets, entry count, m
    ic_csr_off_kernel<<<ic_grid((int64_t)C + 1), kIcFlat, 0, s>>>(C, segoff, loopx, next->off);
    LVG_LAUNCH();
    double* d_m = a.hi_n<double>(1);
    tree_sum_f32(ow, cnt, d_m, a, s);   // as build_level's m over the list (NeighbourCompute.cu:46)
    LVG_CUDA(cudaMemcpyAsync(&next->m, d_m, sizeof(double), cudaMemcpyDeviceToHost, s));
    const int64_t loops = read_back(loopx + C, s);
    next->nnz = cnt - loops;
    next->valid = true;
  }
  LVG_CUDA(cudaStreamSynchronize(s));
  *count = cnt;
  return true;
}

}  // namespace lvg
