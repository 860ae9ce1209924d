// Device-wide primitives: scans, fixed-tree sums, stable LSD radix sort.
//
// Radix sort (replaces thrust::sort_by_key on zip keys, NeighbourCompute.cu:82,
// InducedGraphKernel.cu:91): stable LSD, 8-bit digits.  One upfront pass over
// the keys counts every digit position; then one kernel per digit: a
// 4096-key tile (taken in launch order from a counter) ranks its keys stably
// in shared memory (warp __match_any_sync multisplit), learns the counts of
// its digits in all earlier tiles by decoupled look-back (bounded spin, error
// flag), and writes its keys out digit run by digit run.
#include <algorithm>
#include <atomic>
#include <mutex>

#include "prims.cuh"

namespace lvg {
namespace {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

template <typename T>
__device__ __forceinline__ T block_exclusive_scan(T v, T* total) {
  static_assert(kScanThreads == 256, "block scan assumes 256 threads");
  return block_exclusive_scan256<T>(v, total);
}

template <typename T>
__global__ void __launch_bounds__(kScanThreads) scan_reduce_kernel(const T* in, int64_t n, T* bsum) {
  int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
  T s = 0;
#pragma unroll
  for (int j = 0; j < kScanItems; ++j)
    if (base + j < n) s += in[base + j];
  T tot;
  block_exclusive_scan(s, &tot);
  if (threadIdx.x == 0) bsum[blockIdx.x] = tot;
}

template <typename T>
__global__ void __launch_bounds__(kScanThreads) scan_apply_kernel(const T* in, T* out, int64_t n,
                                                                  const T* bscan) {
  int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
  T v[kScanItems];
  T s = 0;
#pragma unroll
  for (int j = 0; j < kScanItems; ++j) {
    v[j] = base + j < n ? in[base + j] : T(0);
    s += v[j];
  }
  T tot;
  T pre = block_exclusive_scan(s, &tot);
  T off = (bscan ? bscan[blockIdx.x] : T(0)) + pre;
#pragma unroll
  for (int j = 0; j < kScanItems; ++j) {
    if (base + j < n) out[base + j] = off;
    off += v[j];
  }
  if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0)
    out[n] = (bscan ? bscan[blockIdx.x] : T(0)) + tot;
}

template <typename T>
void scan_impl(const T* in, T* out, int64_t n, Arena& a, cudaStream_t s) {
  if (n <= 0) {
    LVG_CUDA(cudaMemsetAsync(out, 0, sizeof(T), s));
    return;
  }
  HiScope hs(a);
  int64_t nb = (n + kScanTile - 1) / kScanTile;
  T* bscan = nullptr;
  if (nb > 1) {
    T* bsum = a.hi_n<T>(nb + 1);
    scan_reduce_kernel<T><<<(unsigned)nb, kScanThreads, 0, s>>>(in, n, bsum);
    LVG_LAUNCH();
    scan_impl<T>(bsum, bsum, nb, a, s);
    bscan = bsum;
  }
  scan_apply_kernel<T><<<(unsigned)nb, kScanThreads, 0, s>>>(in, out, n, bscan);
  LVG_LAUNCH();
}

// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(kRedThreads) tree_group_kernel(const T* x, int64_t n, double* out) {
  __shared__ double ws[8];
  int64_t b = blockIdx.x;
  int64_t len = n - b * kGroup;
  if (len > kGroup) len = kGroup;
  double r = group_sum_block<T>(x + b * kGroup, len, ws);
  if (threadIdx.x == 0) out[b] = r;
}

void finish_impl(const double* p, int64_t n, double* d_out, Arena& a, cudaStream_t s) {
  HiScope hs(a);
  while (n > 1) {
    int64_t nb = (n + kGroup - 1) / kGroup;
    double* q = nb == 1 ? d_out : a.hi_n<double>(nb);
    tree_group_kernel<double><<<(unsigned)nb, kRedThreads, 0, s>>>(p, n, q);
    LVG_LAUNCH();
    p = q;
    n = nb;
  }
}

// ---------------------------------------------------------------------------
constexpr int kRsThreads = 256;
constexpr int kRsItems = 16;
constexpr int kRsTile = kRsThreads * kRsItems;  // 4096 keys
constexpr int kRsWarps = kRsThreads / 32;
constexpr int kRadix = 256;

// One pass over the keys gives the global histogram of every digit position.
constexpr int kRsMaxPasses = 8;

__global__ void __launch_bounds__(kRsThreads) rs_upfront_kernel(const uint64_t* keys, int64_t n, int lo, int npass,
                                                                uint32_t* ghist) {
  __shared__ uint32_t h[kRsMaxPasses][kRadix];
  for (int i = threadIdx.x; i < kRsMaxPasses * kRadix; i += kRsThreads) (&h[0][0])[i] = 0;
  __syncthreads();
  for (int64_t i = blockIdx.x * (int64_t)kRsThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kRsThreads) {
    const uint64_t k = keys[i] >> lo;
    for (int p = 0; p < npass; ++p) atomicAdd(&h[p][(unsigned)(k >> (8 * p)) & (kRadix - 1)], 1u);
  }
  __syncthreads();
  for (int p = 0; p < npass; ++p) {
    const uint32_t c = h[p][threadIdx.x];
    if (c) atomicAdd(&ghist[p * kRadix + threadIdx.x], c);
  }
}

// Exclusive scan of each pass's global histogram (one block, thread = digit).
__global__ void __launch_bounds__(kRsThreads) rs_gscan_kernel(uint32_t* ghist, int npass) {
  for (int p = 0; p < npass; ++p) {
    uint32_t tot;
    const uint32_t v = ghist[p * kRadix + threadIdx.x];
    const uint32_t x = block_exclusive_scan<uint32_t>(v, &tot);
    __syncthreads();
    ghist[p * kRadix + threadIdx.x] = x;
    __syncthreads();
  }
}

struct RsSmem {
  uint64_t key[kRsTile];
  float val[kRsTile];
  uint32_t wc[kRsWarps][kRadix + 1];
  uint32_t dstart[kRadix];
  uint32_t gbase[kRadix];
  uint32_t tile;
};

// Look-back words, one per (tile, digit): code in bits 56..63 (2p+1: this
// tile's count, 2p+2: count of every tile up to this one, for pass p; codes of
// earlier passes read as "not yet"), count in bits 0..31.
constexpr int kRsSpinLimit = 1 << 22;
// Test hook (lvg_debug_radix_hold): a smaller spin limit and one tile that
// never publishes, so that the bounded wait of its successors runs out.
std::atomic<int> g_rs_spin_limit{kRsSpinLimit};
std::atomic<int64_t> g_rs_hold_tile{-1};

__device__ __forceinline__ void rs_publish(unsigned long long* w, unsigned code, uint32_t count) {
  atomicExch(w, ((unsigned long long)code << 56) | count);
}

// One LSD pass: a tile (taken in launch order from a counter) ranks its keys
// by digit in shared memory, learns the keys of its digits in all earlier
// tiles by decoupled look-back, and writes its keys out digit run by digit
// run.  Stable: ranks follow key order inside a tile and tiles in order.
__global__ void __launch_bounds__(kRsThreads) rs_onesweep_kernel(const uint64_t* kin, const float* vin,
                                                                 uint64_t* kout, float* vout, int64_t n,
                                                                 int shift, int pass, const uint32_t* gstart,
                                                                 unsigned long long* look, uint32_t* counter,
                                                                 uint32_t* err, int spin_limit, int64_t hold) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  RsSmem& S = *reinterpret_cast<RsSmem*>(smem_raw);
  const unsigned full = 0xffffffffu;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) S.tile = atomicAdd(counter, 1u);
  for (int i = threadIdx.x; i < kRsWarps * (kRadix + 1); i += kRsThreads) (&S.wc[0][0])[i] = 0;
  __syncthreads();
  const int64_t tile = S.tile;
  const int64_t tile0 = tile * kRsTile;
  const int64_t base = tile0 + (int64_t)w * (32 * kRsItems);
  uint64_t k[kRsItems];
  float v[kRsItems];
  uint32_t rank[kRsItems];
  uint16_t dg[kRsItems];
  const unsigned lt = (1u << lane) - 1u;
#pragma unroll
  for (int j = 0; j < kRsItems; ++j) {
    const int64_t idx = base + j * 32 + lane;
    const bool ok = idx < n;
    k[j] = ok ? kin[idx] : 0ull;
    v[j] = ok ? vin[idx] : 0.0f;
  }
#pragma unroll
  for (int j = 0; j < kRsItems; ++j) {
    const int64_t idx = base + j * 32 + lane;
    const unsigned d = idx < n ? (unsigned)(k[j] >> shift) & (kRadix - 1) : (unsigned)kRadix;
    dg[j] = (uint16_t)d;
    const unsigned peers = __match_any_sync(full, d);
    const uint32_t before = S.wc[w][d];
    rank[j] = before + __popc(peers & lt);
    __syncwarp();
    if ((peers & lt) == 0) S.wc[w][d] = before + __popc(peers);
    __syncwarp();
  }
  __syncthreads();
  // thread = digit: prefix over warps, tile count, look-back across tiles
  const int d = threadIdx.x;
  uint32_t cnt = 0;
#pragma unroll
  for (int ww = 0; ww < kRsWarps; ++ww) {
    const uint32_t t = S.wc[ww][d];
    S.wc[ww][d] = cnt;
    cnt += t;
  }
  const unsigned agg = 2u * (unsigned)pass + 1u, inc = agg + 1u;
  unsigned long long* mine = look + tile * kRadix + d;
  const bool publish = tile != hold;   // hold: a test makes this tile's successors wait out their limit
  uint32_t excl = 0;
  if (tile == 0) {
    if (publish) rs_publish(mine, inc, cnt);
  } else {
    if (publish) rs_publish(mine, agg, cnt);
    int64_t j = tile - 1;
    int spins = 0;
    while (j >= 0) {
      const unsigned long long x = *reinterpret_cast<volatile unsigned long long*>(look + j * kRadix + d);
      const unsigned code = (unsigned)(x >> 56);
      if (code == inc) { excl += (uint32_t)x; break; }
      if (code == agg) { excl += (uint32_t)x; --j; continue; }
      if (++spins > spin_limit) { atomicOr(err, 1u); break; }   // bounded wait: report, never hang
    }
    if (publish) rs_publish(mine, inc, excl + cnt);
  }
  uint32_t tot;
  const uint32_t start = block_exclusive_scan<uint32_t>(cnt, &tot);
  S.dstart[d] = start;
  S.gbase[d] = gstart[d] + excl;
  __syncthreads();
#pragma unroll
  for (int j = 0; j < kRsItems; ++j) {
    const unsigned dd = dg[j];
    if (dd < (unsigned)kRadix) {
      const uint32_t pos = S.dstart[dd] + S.wc[w][dd] + rank[j];
      S.key[pos] = k[j];
      S.val[pos] = v[j];
    }
  }
  __syncthreads();
  int64_t tn = n - tile0;
  if (tn > kRsTile) tn = kRsTile;
  for (int p = threadIdx.x; p < tn; p += kRsThreads) {
    const uint64_t kk = S.key[p];
    const unsigned dd = (unsigned)(kk >> shift) & (kRadix - 1);
    const uint32_t o = S.gbase[dd] + ((uint32_t)p - S.dstart[dd]);
    kout[o] = kk;
    vout[o] = S.val[p];
  }
}

}  // namespace

void scan_u32(const uint32_t* in, uint32_t* out, int64_t n, Arena& a, cudaStream_t s) {
  scan_impl<uint32_t>(in, out, n, a, s);
}
void scan_i64(const int64_t* in, int64_t* out, int64_t n, Arena& a, cudaStream_t s) {
  scan_impl<int64_t>(in, out, n, a, s);
}

void tree_sum_f64(const double* x, int64_t n, double* d_out, Arena& a, cudaStream_t s) {
  if (n <= 0) { LVG_CUDA(cudaMemsetAsync(d_out, 0, sizeof(double), s)); return; }
  HiScope hs(a);
  int64_t nb = (n + kGroup - 1) / kGroup;
  double* p = nb == 1 ? d_out : a.hi_n<double>(nb);
  tree_group_kernel<double><<<(unsigned)nb, kRedThreads, 0, s>>>(x, n, p);
  LVG_LAUNCH();
  if (nb > 1) finish_impl(p, nb, d_out, a, s);
}

void tree_sum_f32(const float* x, int64_t n, double* d_out, Arena& a, cudaStream_t s) {
  if (n <= 0) { LVG_CUDA(cudaMemsetAsync(d_out, 0, sizeof(double), s)); return; }
  HiScope hs(a);
  int64_t nb = (n + kGroup - 1) / kGroup;
  double* p = nb == 1 ? d_out : a.hi_n<double>(nb);
  tree_group_kernel<float><<<(unsigned)nb, kRedThreads, 0, s>>>(x, n, p);
  LVG_LAUNCH();
  if (nb > 1) finish_impl(p, nb, d_out, a, s);
}

void tree_finish(const double* partials, int64_t n, double* d_out, Arena& a, cudaStream_t s) {
  if (n <= 1) {
    if (n == 1) LVG_CUDA(cudaMemcpyAsync(d_out, partials, sizeof(double), cudaMemcpyDeviceToDevice, s));
    else LVG_CUDA(cudaMemsetAsync(d_out, 0, sizeof(double), s));
    return;
  }
  finish_impl(partials, n, d_out, a, s);
}

int radix_sort_pairs(uint64_t* k0, float* v0, uint64_t* k1, float* v1, int64_t n, int bits, Arena& a,
                     cudaStream_t s) {
  return radix_sort_pairs_range(k0, v0, k1, v1, n, 0, bits, a, s);
}

int radix_sort_pairs_range(uint64_t* k0, float* v0, uint64_t* k1, float* v1, int64_t n, int lo, int bits, Arena& a,
                           cudaStream_t s) {
  if (n >= ((int64_t)1 << 32)) throw Error(LVG_ERR_CAPACITY, "radix sort limited to 2^32-1 entries");
  if (lo < 0 || lo >= 64) throw Error(LVG_ERR_INVALID_ARG, "radix sort: first key bit out of range");
  bits = std::min(bits, 64 - lo);
  if (n <= 1 || bits <= 0) return 0;
  static std::once_flag attr_once;
  std::call_once(attr_once, [] {
    LVG_CUDA(cudaFuncSetAttribute(rs_onesweep_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)sizeof(RsSmem)));
  });
  const int npass = (bits + 7) / 8;
  HiScope hs(a);
  const int64_t ntiles = (n + kRsTile - 1) / kRsTile;
  unsigned long long* look = a.hi_n<unsigned long long>(ntiles * kRadix);
  uint32_t* ghist = a.hi_n<uint32_t>(kRsMaxPasses * kRadix + kRsMaxPasses + 1);
  uint32_t* counters = ghist + kRsMaxPasses * kRadix;
  uint32_t* err = counters + kRsMaxPasses;
  LVG_CUDA(cudaMemsetAsync(look, 0, sizeof(unsigned long long) * ntiles * kRadix, s));
  LVG_CUDA(cudaMemsetAsync(ghist, 0, sizeof(uint32_t) * (kRsMaxPasses * kRadix + kRsMaxPasses + 1), s));
  const int64_t ublocks = std::min<int64_t>((n + kRsThreads - 1) / kRsThreads, 148 * 8);
  rs_upfront_kernel<<<(unsigned)ublocks, kRsThreads, 0, s>>>(k0, n, lo, npass, ghist);
  LVG_LAUNCH();
  rs_gscan_kernel<<<1, kRsThreads, 0, s>>>(ghist, npass);
  LVG_LAUNCH();
  int cur = 0;
  uint64_t* K[2] = {k0, k1};
  float* Vv[2] = {v0, v1};
  for (int p = 0; p < npass; ++p) {
    rs_onesweep_kernel<<<(unsigned)ntiles, kRsThreads, sizeof(RsSmem), s>>>(
        K[cur], Vv[cur], K[cur ^ 1], Vv[cur ^ 1], n, lo + 8 * p, p, ghist + p * kRadix, look, counters + p, err,
        g_rs_spin_limit.load(), g_rs_hold_tile.load());
    LVG_LAUNCH();
    cur ^= 1;
  }
  uint32_t h = 0;
  LVG_CUDA(cudaMemcpyAsync(&h, err, sizeof h, cudaMemcpyDeviceToHost, s));
  LVG_CUDA(cudaStreamSynchronize(s));
  if (h) throw Error(LVG_ERR_CUDA, "radix sort look-back did not complete");
  return cur;
}

}  // namespace lvg

extern "C" lvg_status lvg_debug_radix_hold(int32_t spin_limit, int64_t hold_tile) {
  if (spin_limit < 1) return LVG_ERR_INVALID_ARG;
  lvg::g_rs_spin_limit.store(spin_limit);
  lvg::g_rs_hold_tile.store(hold_tile);
  return LVG_OK;
}
