// Internal definitions shared by the CUDA translation units of liblvg.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>

#include "../../include/lvg.h"

namespace lvg {

// Error carried from the point of failure to the C ABI, where it becomes an
// lvg_status and the context's last-error string.
struct Error : std::runtime_error {
  lvg_status status;
  Error(lvg_status s, const std::string& m) : std::runtime_error(m), status(s) {}
};

inline void cuda_check(cudaError_t e, const char* what, const char* file, int line) {
  if (e != cudaSuccess) {
    char buf[512];
    std::snprintf(buf, sizeof buf, "%s failed at %s:%d: %s", what, file, line, cudaGetErrorString(e));
    throw Error(e == cudaErrorMemoryAllocation ? LVG_ERR_OOM : LVG_ERR_CUDA, buf);
  }
}
#define LVG_CUDA(x) ::lvg::cuda_check((x), #x, __FILE__, __LINE__)
// Every kernel launch site is followed by LVG_LAUNCH(), which checks the launch
// and counts it (lvg_kernel_launches).
void count_launch();
#define LVG_LAUNCH() (::lvg::count_launch(), ::lvg::cuda_check(cudaGetLastError(), "kernel launch", __FILE__, __LINE__))

// Device arena: one cudaMalloc slab, allocated from both ends.  The low end
// holds level-lifetime data (level input list, CSR, community state); the high
// end holds phase scratch (sort buffers, hub tables) released when the phase
// ends.  Replaces the reference's three slabs (LouvainCPP.cpp:136-205) and
// Thrust's cached_allocator (cached_allocator.h:12-108).
struct Arena {
  char* base = nullptr;
  size_t cap = 0, lo = 0, hi = 0, peak = 0;
  static constexpr size_t kAlign = 256;
  void reserve(size_t bytes) {
    bytes = (bytes + ((size_t)2 << 20) - 1) & ~(((size_t)2 << 20) - 1);  // both ends stay 256-aligned
    if (bytes <= cap) { lo = 0; hi = cap; return; }
    release();
    LVG_CUDA(cudaMalloc(&base, bytes));
    cap = bytes; lo = 0; hi = cap;
  }
  void release() {
    if (base) cudaFree(base);
    base = nullptr; cap = lo = hi = 0;
  }
  static size_t up(size_t x) { return (x + kAlign - 1) & ~(kAlign - 1); }
  void* alloc_lo(size_t bytes) {
    size_t b = up(bytes ? bytes : 1);
    if (lo + b > hi) oom(bytes);
    void* p = base + lo;
    lo += b;
    track();
    return p;
  }
  void* alloc_hi(size_t bytes) {
    size_t b = up(bytes ? bytes : 1);
    if (hi < lo + b) oom(bytes);
    hi -= b;
    track();
    return base + hi;
  }
  template <typename T> T* lo_n(int64_t n) { return (T*)alloc_lo(sizeof(T) * (size_t)(n > 0 ? n : 1)); }
  template <typename T> T* hi_n(int64_t n) { return (T*)alloc_hi(sizeof(T) * (size_t)(n > 0 ? n : 1)); }
  void track() { size_t used = lo + (cap - hi); if (used > peak) peak = used; }
  [[noreturn]] void oom(size_t bytes) {
    char buf[256];
    std::snprintf(buf, sizeof buf, "device arena exhausted: need %zu more bytes (capacity %zu, in use %zu)",
                  bytes, cap, lo + (cap - hi));
    throw Error(LVG_ERR_OOM, buf);
  }
};

struct HiScope {  // releases high-end scratch on scope exit
  Arena& a;
  size_t mark;
  explicit HiScope(Arena& ar) : a(ar), mark(ar.hi) {}
  ~HiScope() { a.hi = mark; }
};

inline int bits_for(int64_t n) {  // bits needed to hold values 0..n-1
  int b = 0;
  while (b < 63 && ((int64_t)1 << b) < n) ++b;
  return b;
}

inline unsigned grid_for(int64_t n, int per_block) {
  int64_t g = (n + per_block - 1) / per_block;
  return (unsigned)(g > 0 ? g : 1);
}

// ---------------------------------------------------------------------------
// Fixed-shape FP64 sum shared with the oracle: groups of 2048 values; thread t
// of a 256-thread block sums x[t], x[256+t], ..., x[1792+t] left to right; the
// thread sums are added by eight 32-lane shuffle-down trees and the eight warp
// sums by one more (zero padded).  Group sums are reduced again the same way.
constexpr int kGroup = 2048;
constexpr int kRedThreads = 256;

__device__ __forceinline__ double block_tree256(double s, double* ws /*[8] smem*/) {
  const unsigned full = 0xffffffffu;
  for (int o = 16; o >= 1; o >>= 1) s = __dadd_rn(s, __shfl_down_sync(full, s, o));
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) ws[w] = s;
  __syncthreads();
  double r = 0.0;
  if (w == 0) {
    double v = lane < 8 ? ws[lane] : 0.0;
    for (int o = 16; o >= 1; o >>= 1) v = __dadd_rn(v, __shfl_down_sync(full, v, o));
    r = v;
  }
  __syncthreads();
  return r;  // valid in thread 0
}

// Sum of one group x[0..n), n <= 2048, by a 256-thread block; result in thread 0.
template <typename T>
__device__ __forceinline__ double group_sum_block(const T* x, int64_t n, double* ws) {
  double s = 0.0;
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    int64_t idx = (int64_t)j * 256 + threadIdx.x;
    if (idx < n) s = __dadd_rn(s, (double)x[idx]);
  }
  return block_tree256(s, ws);
}

// Warp inclusive scan and block (256-thread) exclusive scan of one value per thread.
template <typename T>
__device__ __forceinline__ T warp_inclusive_scan(T v) {
  const unsigned full = 0xffffffffu;
  int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    T u = __shfl_up_sync(full, v, o);
    if (lane >= o) v += u;
  }
  return v;
}

template <typename T>
__device__ __forceinline__ T block_exclusive_scan256(T v, T* total) {
  __shared__ T wsum[8];
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  T inc = warp_inclusive_scan(v);
  if (lane == 31) wsum[w] = inc;
  __syncthreads();
  if (w == 0) {
    T x = lane < 8 ? wsum[lane] : T(0);
    x = warp_inclusive_scan(x);
    if (lane < 8) wsum[lane] = x;
  }
  __syncthreads();
  T base = w > 0 ? wsum[w - 1] : T(0);
  *total = wsum[7];
  __syncthreads();
  return base + inc - v;
}

// Block (512-thread) exclusive scan of one value per thread.
template <typename T>
__device__ __forceinline__ T block_exclusive_scan512(T v, T* total) {
  __shared__ T wsum[16];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const T inc = warp_inclusive_scan(v);
  if (lane == 31) wsum[w] = inc;
  __syncthreads();
  if (w == 0) {
    T x = lane < 16 ? wsum[lane] : T(0);
    x = warp_inclusive_scan(x);
    if (lane < 16) wsum[lane] = x;
  }
  __syncthreads();
  const T base = w > 0 ? wsum[w - 1] : T(0);
  *total = wsum[15];
  __syncthreads();
  return base + inc - v;
}

// Counter-based random numbers (splitmix64 finaliser), identical on host and
// device so that generated graphs do not depend on where they are generated.
__host__ __device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
__host__ __device__ __forceinline__ uint64_t rng_at(uint64_t seed, uint64_t stream, uint64_t i) {
  return mix64(mix64(seed ^ mix64(stream + 0x632BE59BD9B4E019ull)) + i);
}
__host__ __device__ __forceinline__ double u01(uint64_t r) {  // [0,1) with 53 bits
  return (double)(r >> 11) * (1.0 / 9007199254740992.0);
}

}  // namespace lvg
