// Device-wide primitives: scans, fixed-tree sums, stable LSD radix sort.
//
// Radix sort (replaces thrust::sort_by_key on zip keys, NeighbourCompute.cu:82,
// InducedGraphKernel.cu:91): 8-bit digits, reduce-then-scan.  Per digit pass a
// histogram kernel counts digits per 2048-key tile, an exclusive scan over the
// digit-major [256][tiles] table yields every tile's global digit offsets, and
// a scatter kernel ranks the tile's keys stably in shared memory (warp
// __match_any_sync multisplit) and writes them to their global positions.
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
constexpr int kRsItems = 8;
constexpr int kRsTile = kRsThreads * kRsItems;  // 2048 keys
constexpr int kRsWarps = kRsThreads / 32;
constexpr int kRadix = 256;

__global__ void __launch_bounds__(kRsThreads) rs_hist_kernel(const uint64_t* keys, int64_t n, int shift,
                                                             uint32_t* hist, int64_t ntiles) {
  __shared__ uint32_t h[kRsWarps][kRadix];
  for (int i = threadIdx.x; i < kRsWarps * kRadix; i += kRsThreads) (&h[0][0])[i] = 0;
  __syncthreads();
  int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int64_t base = (int64_t)blockIdx.x * kRsTile + (int64_t)w * (32 * kRsItems);
#pragma unroll 4
  for (int j = 0; j < kRsItems; ++j) {
    int64_t idx = base + j * 32 + lane;
    if (idx < n) atomicAdd(&h[w][(unsigned)(keys[idx] >> shift) & (kRadix - 1)], 1u);
  }
  __syncthreads();
  uint32_t c = 0;
#pragma unroll
  for (int k = 0; k < kRsWarps; ++k) c += h[k][threadIdx.x];
  hist[(int64_t)threadIdx.x * ntiles + blockIdx.x] = c;
}

struct RsSmem {
  uint64_t key[kRsTile];
  float val[kRsTile];
  uint32_t wc[kRsWarps][kRadix + 1];
  uint32_t dstart[kRadix];
  uint32_t gbase[kRadix];
};

__global__ void __launch_bounds__(kRsThreads) rs_scatter_kernel(const uint64_t* kin, const float* vin,
                                                                uint64_t* kout, float* vout, int64_t n,
                                                                int shift, const uint32_t* offs,
                                                                int64_t ntiles) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  RsSmem& S = *reinterpret_cast<RsSmem*>(smem_raw);
  const unsigned full = 0xffffffffu;
  int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int i = threadIdx.x; i < kRsWarps * (kRadix + 1); i += kRsThreads) (&S.wc[0][0])[i] = 0;
  __syncthreads();
  int64_t tile0 = (int64_t)blockIdx.x * kRsTile;
  int64_t base = tile0 + (int64_t)w * (32 * kRsItems);
  uint64_t k[kRsItems];
  float v[kRsItems];
  uint32_t rank[kRsItems];
  uint16_t dg[kRsItems];
  unsigned lt = (1u << lane) - 1u;
#pragma unroll
  for (int j = 0; j < kRsItems; ++j) {
    int64_t idx = base + j * 32 + lane;
    bool ok = idx < n;
    k[j] = ok ? kin[idx] : 0ull;
    v[j] = ok ? vin[idx] : 0.0f;
    unsigned d = ok ? (unsigned)(k[j] >> shift) & (kRadix - 1) : (unsigned)kRadix;
    dg[j] = (uint16_t)d;
    unsigned peers = __match_any_sync(full, d);
    uint32_t before = S.wc[w][d];
    rank[j] = before + __popc(peers & lt);
    __syncwarp();
    if ((peers & lt) == 0) S.wc[w][d] = before + __popc(peers);
    __syncwarp();
  }
  __syncthreads();
  // per digit (thread = digit): exclusive prefix over warps, tile count
  uint32_t cnt = 0;
  {
    int d = threadIdx.x;
#pragma unroll
    for (int ww = 0; ww < kRsWarps; ++ww) {
      uint32_t t = S.wc[ww][d];
      S.wc[ww][d] = cnt;
      cnt += t;
    }
  }
  uint32_t tot;
  uint32_t start = block_exclusive_scan<uint32_t>(cnt, &tot);
  S.dstart[threadIdx.x] = start;
  S.gbase[threadIdx.x] = offs[(int64_t)threadIdx.x * ntiles + blockIdx.x];
  __syncthreads();
#pragma unroll
  for (int j = 0; j < kRsItems; ++j) {
    unsigned d = dg[j];
    if (d < (unsigned)kRadix) {
      uint32_t pos = S.dstart[d] + S.wc[w][d] + rank[j];
      S.key[pos] = k[j];
      S.val[pos] = v[j];
    }
  }
  __syncthreads();
  int64_t tn = n - tile0;
  if (tn > kRsTile) tn = kRsTile;
  for (int p = threadIdx.x; p < tn; p += kRsThreads) {
    uint64_t kk = S.key[p];
    unsigned d = (unsigned)(kk >> shift) & (kRadix - 1);
    uint32_t o = S.gbase[d] + ((uint32_t)p - S.dstart[d]);
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
  if (n >= ((int64_t)1 << 32)) throw Error(LVG_ERR_CAPACITY, "radix sort limited to 2^32-1 entries");
  if (n <= 1 || bits <= 0) return 0;
  static std::once_flag attr_once;
  std::call_once(attr_once, [] {
    LVG_CUDA(cudaFuncSetAttribute(rs_scatter_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)sizeof(RsSmem)));
  });
  HiScope hs(a);
  int64_t ntiles = (n + kRsTile - 1) / kRsTile;
  uint32_t* hist = a.hi_n<uint32_t>(kRadix * ntiles + 1);
  int cur = 0;
  uint64_t* K[2] = {k0, k1};
  float* Vv[2] = {v0, v1};
  for (int shift = 0; shift < bits; shift += 8) {
    rs_hist_kernel<<<(unsigned)ntiles, kRsThreads, 0, s>>>(K[cur], n, shift, hist, ntiles);
    LVG_LAUNCH();
    scan_u32(hist, hist, kRadix * ntiles, a, s);
    rs_scatter_kernel<<<(unsigned)ntiles, kRsThreads, sizeof(RsSmem), s>>>(K[cur], Vv[cur], K[cur ^ 1],
                                                                           Vv[cur ^ 1], n, shift, hist,
                                                                           ntiles);
    LVG_LAUNCH();
    cur ^= 1;
  }
  return cur;
}

}  // namespace lvg
