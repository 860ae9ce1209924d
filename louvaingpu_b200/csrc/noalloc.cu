// Allocation-free FP64 modularity.
//
// Some callers cannot allocate device memory at the moment they need a
// modularity value: a serving process whose caching allocator has already
// reserved all free HBM for its own pool (a cudaMalloc would fail or force
// that pool to shrink), and latency-bound loops that run beside work on other
// streams and cannot take the device-wide synchronisation that cudaMalloc and
// cudaFree imply.  lvg_modularity_fp64_noalloc serves them: its scratch is the
// file-scope array below, allocated once when the module is loaded on a device
// and kept until the process exits.
#include <cstring>
#include <mutex>

#include "louvain.cuh"

namespace {

constexpr int64_t kMaxComms = LVG_NOALLOC_MAX_COMMS;
constexpr int64_t kPartials = (kMaxComms + lvg::kGroup - 1) / lvg::kGroup;
// Kc | Ain | t (kMaxComms each) | tree partials | 2W, Q | bad-id flag
constexpr int64_t kScratch = 3 * kMaxComms + kPartials + 3;
static_assert(kScratch * sizeof(double) == LVG_NOALLOC_SCRATCH_BYTES, "header states the array size");

static __device__ __align__(256) double g_noalloc_scratch[kScratch];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
double* g_addr[kMaxDevices] = {};

// Device address of the scratch array for the current device, looked up once
// per device with that device current.  Host code only holds the symbol's
// host-side stand-in, which must never reach a kernel.
double* scratch_for_current_device() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return nullptr;
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_addr[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess) return nullptr;
    g_addr[dev] = static_cast<double*>(p);
  }
  return g_addr[dev];
}

}  // namespace

extern "C" lvg_status lvg_modularity_fp64_noalloc(const int32_t* d_src, const int32_t* d_dst, const float* d_w,
                                                  int64_t n_entries, const int32_t* d_part, int32_t n_comms,
                                                  void* stream, double* q) {
  if (!q || n_entries < 0 || n_comms < 1) return LVG_ERR_INVALID_ARG;
  if (n_entries > 0 && (!d_src || !d_dst || !d_w || !d_part)) return LVG_ERR_INVALID_ARG;
  if (n_comms > kMaxComms) return LVG_ERR_CAPACITY;
  double* base = scratch_for_current_device();
  if (!base) return LVG_ERR_CUDA;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  double* Kc = base;
  double* Ain = base + kMaxComms;
  double* t = base + 2 * kMaxComms;
  double* partials = base + 3 * kMaxComms;
  double* out = partials + kPartials;                       // 2W, Q
  uint32_t* bad = reinterpret_cast<uint32_t*>(out + 2);     // set by a community id outside [0, n_comms)
  try {
    LVG_CUDA(cudaMemsetAsync(bad, 0, sizeof(double), s));
    lvg::modularity_fp64_scratch(d_src, d_dst, d_w, n_entries, n_comms, d_part, Kc, Ain, t, partials, out, bad, s);
    double h[3];
    LVG_CUDA(cudaMemcpyAsync(h, out, sizeof h, cudaMemcpyDeviceToHost, s));
    LVG_CUDA(cudaStreamSynchronize(s));
    uint32_t flag = 0;
    std::memcpy(&flag, &h[2], sizeof flag);
    if (flag) return LVG_ERR_INVALID_ARG;
    *q = h[1];
  } catch (const lvg::Error& e) {
    return e.status;
  }
  return LVG_OK;
}
