// Seeded synthetic graphs generated straight into HBM (R-MAT, batched SBM).
// The random stream is the counter-based construction of lvg_internal.cuh, so
// an R-MAT graph generated here equals the host generator's entry for entry.
#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "../../include/lvg_gen.h"
#include "prims.cuh"

struct lvg_dgraph {
  int32_t device = 0;
  int32_t n_graphs = 0;
  int64_t n_entries = 0;
  int64_t n_vertices = 0;
  int32_t* src = nullptr;
  int32_t* dst = nullptr;
  float* w = nullptr;
  std::vector<int64_t> eoff;
  std::vector<int32_t> voff;
  ~lvg_dgraph() {
    cudaFree(src);
    cudaFree(dst);
    cudaFree(w);
  }
};

namespace lvg {
namespace {

thread_local std::string g_gen_err;
constexpr int kT = 256;

__host__ __device__ __forceinline__ float int_weight(uint64_t r, int32_t lo, int32_t hi) {
  if (hi <= lo) return (float)lo;
  return (float)(lo + (int32_t)(r % (uint64_t)(hi - lo + 1)));
}

unsigned sm_blocks(int64_t n) {
  int64_t g = (n + kT - 1) / kT;
  return (unsigned)std::max<int64_t>(1, std::min<int64_t>(g, 148 * 16));
}

// ------------------------------------------------------------------ R-MAT
// Edge e: `scale` quadrant draws u01(rng_at(seed, 16 + level, e)); weight from
// rng_at(seed, 3, e).  Key (min << scale) | max; self loops get the sentinel
// key, which sorts after every edge.
__global__ void rmat_kernel(int64_t M, int scale, double a, double ab, double abc, int32_t w_lo, int32_t w_hi,
                            uint64_t seed, uint64_t sentinel, uint64_t* keys, float* vals,
                            unsigned long long* loops) {
  unsigned long long nl = 0;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < M; e += (int64_t)gridDim.x * blockDim.x) {
    uint32_t u = 0, v = 0;
    for (int l = 0; l < scale; ++l) {
      double x = u01(rng_at(seed, (uint64_t)l + 16, (uint64_t)e));
      uint32_t bu = x >= ab ? 1u : 0u;
      uint32_t bv = ((x >= a && x < ab) || x >= abc) ? 1u : 0u;
      u = (u << 1) | bu;
      v = (v << 1) | bv;
    }
    if (u == v) {
      keys[e] = sentinel;
      vals[e] = 0.0f;
      ++nl;
    } else {
      uint64_t lo = u < v ? u : v, hi = u < v ? v : u;
      keys[e] = (lo << scale) | hi;
      vals[e] = int_weight(rng_at(seed, 3, (uint64_t)e), w_lo, w_hi);
    }
  }
  if (nl) atomicAdd(loops, nl);
}

__global__ void head_kernel(const uint64_t* keys, int64_t n, uint32_t* head) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    head[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1u : 0u;
}

// Unique keys and their summed weights (small integers: exact in float).
__global__ void unique_kernel(const uint64_t* keys, const float* vals, int64_t n, const uint32_t* head,
                              const uint32_t* pos, uint64_t* ukeys, float* uw) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    uint32_t j = pos[i] + head[i] - 1;
    if (head[i]) ukeys[j] = keys[i];
    atomicAdd(&uw[j], vals[i]);
  }
}

// Both directions of every undirected edge (u < v) as (src << B) | dst keys.
__global__ void symmetrise_kernel(const uint64_t* ukeys, const float* uw, int64_t U, int B, uint64_t* keys,
                                  float* vals) {
  const uint64_t mask = (1ull << B) - 1;
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < U; j += (int64_t)gridDim.x * blockDim.x) {
    uint64_t k = ukeys[j];
    uint64_t lo = k >> B, hi = k & mask;
    keys[2 * j] = k;
    keys[2 * j + 1] = (hi << B) | lo;
    vals[2 * j] = uw[j];
    vals[2 * j + 1] = uw[j];
  }
}

// Sorted keys -> src, dst (minus the owning graph's first vertex), w.
__global__ void emit_kernel(const uint64_t* keys, const float* vals, int64_t n, int B, const int32_t* voff,
                            int32_t G, int32_t* src, int32_t* dst, float* w) {
  const uint64_t mask = (1ull << B) - 1;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    int32_t s = (int32_t)(keys[i] >> B), d = (int32_t)(keys[i] & mask);
    int32_t base = 0;
    if (voff) {
      int lo = 0, hi = G - 1;
      while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (voff[mid] <= s) lo = mid; else hi = mid - 1;
      }
      base = voff[lo];
    }
    src[i] = s - base;
    dst[i] = d - base;
    w[i] = vals[i];
  }
}

// entry_off[g] = number of keys whose source is below voff[g].
__global__ void graph_bounds_kernel(const uint64_t* keys, int64_t n, int B, const int32_t* voff, int32_t G,
                                    int64_t* eoff) {
  for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g <= G; g += (int64_t)gridDim.x * blockDim.x) {
    uint64_t k = (uint64_t)voff[g] << B;
    int64_t lo = 0, hi = n;
    while (lo < hi) {
      int64_t mid = (lo + hi) >> 1;
      if (keys[mid] < k) lo = mid + 1; else hi = mid;
    }
    eoff[g] = lo;
  }
}

// --------------------------------------------------------------- batched SBM
// Every graph is sampled as segments: the inter-block segment is the ordered
// n x n square with p_out, keeping u < v in different blocks; intra segment k
// is block k's square with p_in, keeping u < v.  A segment is cut into chunks
// of K positions (about 256 expected samples each); chunk c of segment s of
// graph g draws a geometric skip sequence from rng_at(seed_g, s << 32 | c, i).
struct Seg {
  int64_t chunk0;   // first global chunk of the segment
  int64_t K;        // positions per chunk
  int64_t LL;       // positions (L * L)
  double lq;        // log1p(-p), 0 when p >= 1
  int32_t g;        // graph
  int32_t sid;      // 0 inter, 1 + k intra block k
  int32_t base;     // first vertex of the square (local)
  int32_t L;        // side
};

struct SbmGraph {
  int32_t n, blocks, voff;
  int32_t pad;
  uint64_t seed;
};

__device__ __forceinline__ int32_t block_of(int64_t u, int64_t n, int64_t B) {
  return (int32_t)(((u + 1) * B - 1) / n);   // largest k with floor(n*k/B) <= u
}

template <bool WRITE>
__global__ void sbm_chunks_kernel(const Seg* segs, int64_t nseg, int64_t nchunks, const SbmGraph* graphs,
                                  int32_t w_lo, int32_t w_hi, uint32_t* cnt, unsigned long long* total,
                                  const uint32_t* off, uint64_t* keys, float* vals, int B) {
  unsigned long long mine = 0;
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < nchunks;
       c += (int64_t)gridDim.x * blockDim.x) {
    int64_t lo = 0, hi = nseg - 1;
    while (lo < hi) {
      int64_t mid = (lo + hi + 1) >> 1;
      if (segs[mid].chunk0 <= c) lo = mid; else hi = mid - 1;
    }
    const Seg S = segs[lo];
    const SbmGraph G = graphs[S.g];
    const int64_t cl = c - S.chunk0;
    const int64_t beg = cl * S.K;
    const int64_t end = min(beg + S.K, S.LL);
    const uint64_t stream = ((uint64_t)S.sid << 32) | (uint64_t)cl;
    uint64_t i = 0;
    int64_t idx = beg - 1;
    uint32_t k = 0;
    const uint64_t vbase = (uint64_t)G.voff;
    for (;;) {
      if (S.lq == 0.0) {
        idx += 1;
      } else {
        double x = u01(rng_at(G.seed, stream, i++));
        double sk = floor(log1p(-x) / S.lq);
        if (sk >= (double)(end - idx)) break;
        idx += 1 + (int64_t)sk;
      }
      if (idx >= end) break;
      int64_t u = S.base + idx / S.L, v = S.base + idx % S.L;
      if (u >= v) continue;
      if (S.sid == 0 && block_of(u, G.n, G.blocks) == block_of(v, G.n, G.blocks)) continue;
      if (WRITE) {
        if (k >= cnt[c]) break;   // never more than the counting pass found
        float wt = int_weight(rng_at(G.seed, stream, (1ull << 63) | (uint64_t)idx), w_lo, w_hi);
        int64_t p = 2 * ((int64_t)off[c] + k);
        keys[p] = ((vbase + u) << B) | (vbase + v);
        keys[p + 1] = ((vbase + v) << B) | (vbase + u);
        vals[p] = wt;
        vals[p + 1] = wt;
      }
      ++k;
    }
    if (!WRITE) cnt[c] = k;
    mine += k;
  }
  if (!WRITE && mine) atomicAdd(total, mine);
}

template <typename F>
lvg_status gen_guard(F&& f) {
  try {
    f();
    return LVG_OK;
  } catch (const Error& e) {
    g_gen_err = e.what();
    return e.status;
  } catch (const std::bad_alloc&) {
    g_gen_err = "host allocation failed";
    return LVG_ERR_OOM;
  } catch (const std::exception& e) {
    g_gen_err = e.what();
    return LVG_ERR_CUDA;
  }
}

void req(bool ok, lvg_status s, const char* msg) {
  if (!ok) throw Error(s, msg);
}

template <typename T>
T* dmalloc(int64_t n) {
  void* p = nullptr;
  LVG_CUDA(cudaMalloc(&p, sizeof(T) * (size_t)std::max<int64_t>(n, 1)));
  return (T*)p;
}

// Scratch device memory of one generator call, freed on every exit.
struct Scratch {
  std::vector<void*> bufs;
  std::vector<Arena*> arenas;
  template <typename T> T* get(int64_t n) {
    T* p = dmalloc<T>(n);
    bufs.push_back(p);
    return p;
  }
  Arena& arena(size_t bytes) {
    arenas.push_back(new Arena());
    arenas.back()->reserve(bytes);
    return *arenas.back();
  }
  ~Scratch() {
    for (void* p : bufs) cudaFree(p);
    for (Arena* a : arenas) { a->release(); delete a; }
  }
};

// Sort scratch bytes of radix_sort_pairs / scan_u32 for n keys.
size_t sort_scratch(int64_t n) {
  return (size_t)256 * 4 * (size_t)(n / 2048 + 2) * 2 + ((size_t)16 << 20);
}

}  // namespace
}  // namespace lvg

using namespace lvg;

extern "C" {

const char* lvg_gen_last_error(void) { return g_gen_err.c_str(); }

lvg_status lvg_gen_rmat(int32_t device, void* stream, int32_t scale, int32_t edge_factor, double a, double b,
                        double c, int32_t w_lo, int32_t w_hi, uint64_t seed, lvg_dgraph** out) {
  return gen_guard([&] {
    req(out != nullptr, LVG_ERR_INVALID_ARG, "null output");
    *out = nullptr;
    req(scale >= 1 && scale <= 30 && edge_factor >= 1, LVG_ERR_INVALID_ARG, "scale must be 1..30");
    const int64_t M = (int64_t)edge_factor << scale;
    req(2 * M < ((int64_t)1 << 32), LVG_ERR_CAPACITY, "edge_factor * 2^scale must stay below 2^31");
    LVG_CUDA(cudaSetDevice(device));
    cudaStream_t s = (cudaStream_t)stream;
    const int B = scale;
    const uint64_t sentinel = (2 * B >= 64) ? ~0ull : ((1ull << (2 * B)) - 1);
    Scratch scr;
    Arena& ar = scr.arena((size_t)M * 2 * 24 + (size_t)(M + 1) * 8 + sort_scratch(2 * M) + ((size_t)64 << 20));
    uint64_t* K0 = ar.lo_n<uint64_t>(2 * M);
    uint64_t* K1 = ar.lo_n<uint64_t>(2 * M);
    float* V0 = ar.lo_n<float>(2 * M);
    float* V1 = ar.lo_n<float>(2 * M);
    unsigned long long* loops = ar.lo_n<unsigned long long>(1);
    LVG_CUDA(cudaMemsetAsync(loops, 0, sizeof(unsigned long long), s));
    const double ab = a + b, abc = a + b + c;
    rmat_kernel<<<sm_blocks(M), kT, 0, s>>>(M, scale, a, ab, abc, w_lo, w_hi, seed, sentinel, K0, V0, loops);
    LVG_LAUNCH();
    int which = radix_sort_pairs(K0, V0, K1, V1, M, 2 * B, ar, s);
    uint64_t* Ks = which ? K1 : K0;
    float* Vs = which ? V1 : V0;
    uint64_t* Ko = which ? K0 : K1;
    float* Vo = which ? V0 : V1;
    unsigned long long nl = 0;
    LVG_CUDA(cudaMemcpyAsync(&nl, loops, sizeof nl, cudaMemcpyDeviceToHost, s));
    LVG_CUDA(cudaStreamSynchronize(s));
    const int64_t Mv = M - (int64_t)nl;
    uint32_t U = 0;
    {
      HiScope hs(ar);
      uint32_t* head = ar.hi_n<uint32_t>(Mv + 1);
      uint32_t* pos = ar.hi_n<uint32_t>(Mv + 1);
      if (Mv > 0) {
        head_kernel<<<sm_blocks(Mv), kT, 0, s>>>(Ks, Mv, head);
        LVG_LAUNCH();
      }
      scan_u32(head, pos, Mv, ar, s);
      LVG_CUDA(cudaMemcpyAsync(&U, pos + Mv, sizeof U, cudaMemcpyDeviceToHost, s));
      LVG_CUDA(cudaStreamSynchronize(s));
      LVG_CUDA(cudaMemsetAsync(Vo, 0, sizeof(float) * std::max<int64_t>(U, 1), s));
      if (Mv > 0) {
        unique_kernel<<<sm_blocks(Mv), kT, 0, s>>>(Ks, Vs, Mv, head, pos, Ko, Vo);
        LVG_LAUNCH();
      }
    }
    const int64_t E = 2 * (int64_t)U;
    if (U > 0) {
      symmetrise_kernel<<<sm_blocks(U), kT, 0, s>>>(Ko, Vo, U, B, Ks, Vs);
      LVG_LAUNCH();
    }
    int w2 = radix_sort_pairs(Ks, Vs, Ko, Vo, E, 2 * B, ar, s);
    uint64_t* Kf = w2 ? Ko : Ks;
    float* Vf = w2 ? Vo : Vs;
    auto* g = new lvg_dgraph();
    try {
      g->device = device;
      g->n_graphs = 1;
      g->n_entries = E;
      g->n_vertices = (int64_t)1 << scale;
      g->src = dmalloc<int32_t>(E);
      g->dst = dmalloc<int32_t>(E);
      g->w = dmalloc<float>(E);
      if (E > 0) {
        emit_kernel<<<sm_blocks(E), kT, 0, s>>>(Kf, Vf, E, B, nullptr, 1, g->src, g->dst, g->w);
        LVG_LAUNCH();
      }
      LVG_CUDA(cudaStreamSynchronize(s));
      g->eoff = {0, E};
      g->voff = {0, (int32_t)g->n_vertices};
    } catch (...) {
      delete g;
      throw;
    }
    *out = g;
  });
}

lvg_status lvg_gen_sbm_batch(int32_t device, void* stream, int32_t n_graphs, const int32_t* n,
                             const int32_t* blocks, const double* p_in, const double* p_out, int32_t w_lo,
                             int32_t w_hi, const uint64_t* seeds, lvg_dgraph** out) {
  return gen_guard([&] {
    req(out != nullptr, LVG_ERR_INVALID_ARG, "null output");
    *out = nullptr;
    req(n_graphs >= 1 && n && blocks && p_in && p_out && seeds, LVG_ERR_INVALID_ARG, "bad arguments");
    LVG_CUDA(cudaSetDevice(device));
    cudaStream_t s = (cudaStream_t)stream;
    std::vector<SbmGraph> gs(n_graphs);
    std::vector<Seg> segs;
    std::vector<int32_t> voff(n_graphs + 1, 0);
    int64_t chunks = 0;
    auto add = [&](int32_t g, int32_t sid, int32_t base, int32_t L, double p) {
      if (!(p > 0.0) || L < 2) return;
      Seg S;
      S.g = g;
      S.sid = sid;
      S.base = base;
      S.L = L;
      S.LL = (int64_t)L * L;
      S.lq = p >= 1.0 ? 0.0 : std::log1p(-p);
      const double kd = p >= 1.0 ? 1024.0 : std::max(1024.0, std::ceil(256.0 / p));
      S.K = kd >= (double)S.LL ? S.LL : (int64_t)kd;
      S.chunk0 = chunks;
      chunks += (S.LL + S.K - 1) / S.K;
      segs.push_back(S);
    };
    for (int32_t g = 0; g < n_graphs; ++g) {
      req(n[g] >= 1 && blocks[g] >= 1 && blocks[g] <= n[g], LVG_ERR_INVALID_ARG, "need 1 <= blocks <= n");
      req(p_in[g] >= 0.0 && p_out[g] >= 0.0, LVG_ERR_INVALID_ARG, "probabilities must be >= 0");
      req((int64_t)voff[g] + n[g] < ((int64_t)1 << 31), LVG_ERR_CAPACITY, "more than 2^31-1 vertices");
      voff[g + 1] = voff[g] + n[g];
      gs[g] = SbmGraph{n[g], blocks[g], voff[g], 0, seeds[g]};
      add(g, 0, 0, n[g], p_out[g]);
      for (int32_t k = 0; k < blocks[g]; ++k) {
        int32_t b0 = (int32_t)((int64_t)n[g] * k / blocks[g]), b1 = (int32_t)((int64_t)n[g] * (k + 1) / blocks[g]);
        add(g, 1 + k, b0, b1 - b0, p_in[g]);
      }
    }
    req(chunks < ((int64_t)1 << 32), LVG_ERR_CAPACITY, "too many sample chunks");
    const int64_t Vtot = voff[n_graphs];
    const int B = std::max(1, bits_for(Vtot));
    req(2 * B <= 64, LVG_ERR_CAPACITY, "vertex ids too wide");
    const int64_t nseg = (int64_t)segs.size();
    // pass 1: samples per chunk
    Scratch scr;
    Seg* d_segs = scr.get<Seg>(nseg);
    SbmGraph* d_graphs = scr.get<SbmGraph>(n_graphs);
    int32_t* d_voff = scr.get<int32_t>(n_graphs + 1);
    uint32_t* cnt = scr.get<uint32_t>(chunks + 1);
    uint32_t* off = scr.get<uint32_t>(chunks + 1);
    unsigned long long* total = scr.get<unsigned long long>(1);
    LVG_CUDA(cudaMemcpyAsync(d_segs, segs.data(), sizeof(Seg) * std::max<int64_t>(nseg, 1), cudaMemcpyHostToDevice,
                             s));
    LVG_CUDA(cudaMemcpyAsync(d_graphs, gs.data(), sizeof(SbmGraph) * n_graphs, cudaMemcpyHostToDevice, s));
    LVG_CUDA(cudaMemcpyAsync(d_voff, voff.data(), sizeof(int32_t) * (n_graphs + 1), cudaMemcpyHostToDevice, s));
    LVG_CUDA(cudaMemsetAsync(total, 0, sizeof(unsigned long long), s));
    unsigned long long U = 0;
    if (chunks > 0) {
      sbm_chunks_kernel<false><<<sm_blocks(chunks), kT, 0, s>>>(d_segs, nseg, chunks, d_graphs, w_lo, w_hi, cnt,
                                                                total, nullptr, nullptr, nullptr, B);
      LVG_LAUNCH();
    }
    LVG_CUDA(cudaMemcpyAsync(&U, total, sizeof U, cudaMemcpyDeviceToHost, s));
    LVG_CUDA(cudaStreamSynchronize(s));
    // the 32-bit chunk offsets below are exact only under this bound
    req(2 * U < ((unsigned long long)1 << 31), LVG_ERR_CAPACITY,
        "the packed list would exceed 2^31-1 entries; split the batch");
    const int64_t E = 2 * (int64_t)U;
    Arena& ar = scr.arena((size_t)E * 24 + sort_scratch(std::max<int64_t>(E, chunks)) + ((size_t)64 << 20));
    scan_u32(cnt, off, chunks, ar, s);
    uint64_t* K0 = ar.lo_n<uint64_t>(E);
    uint64_t* K1 = ar.lo_n<uint64_t>(E);
    float* V0 = ar.lo_n<float>(E);
    float* V1 = ar.lo_n<float>(E);
    int64_t* d_eoff = ar.lo_n<int64_t>(n_graphs + 1);
    // pass 2: the same draws, written at the chunk offsets
    if (chunks > 0) {
      sbm_chunks_kernel<true><<<sm_blocks(chunks), kT, 0, s>>>(d_segs, nseg, chunks, d_graphs, w_lo, w_hi, cnt,
                                                               nullptr, off, K0, V0, B);
      LVG_LAUNCH();
    }
    int which = radix_sort_pairs(K0, V0, K1, V1, E, 2 * B, ar, s);
    uint64_t* Kf = which ? K1 : K0;
    float* Vf = which ? V1 : V0;
    auto* g = new lvg_dgraph();
    try {
      g->device = device;
      g->n_graphs = n_graphs;
      g->n_entries = E;
      g->n_vertices = Vtot;
      g->src = dmalloc<int32_t>(E);
      g->dst = dmalloc<int32_t>(E);
      g->w = dmalloc<float>(E);
      if (E > 0) {
        emit_kernel<<<sm_blocks(E), kT, 0, s>>>(Kf, Vf, E, B, d_voff, n_graphs, g->src, g->dst, g->w);
        LVG_LAUNCH();
      }
      graph_bounds_kernel<<<sm_blocks(n_graphs + 1), kT, 0, s>>>(Kf, E, B, d_voff, n_graphs, d_eoff);
      LVG_LAUNCH();
      g->eoff.resize(n_graphs + 1);
      LVG_CUDA(cudaMemcpyAsync(g->eoff.data(), d_eoff, sizeof(int64_t) * (n_graphs + 1), cudaMemcpyDeviceToHost, s));
      LVG_CUDA(cudaStreamSynchronize(s));
      g->voff = voff;
    } catch (...) {
      delete g;
      throw;
    }
    *out = g;
  });
}

lvg_status lvg_dgraph_info(const lvg_dgraph* g, int32_t* n_graphs, int64_t* n_entries, int64_t* n_vertices) {
  if (!g) return LVG_ERR_INVALID_ARG;
  if (n_graphs) *n_graphs = g->n_graphs;
  if (n_entries) *n_entries = g->n_entries;
  if (n_vertices) *n_vertices = g->n_vertices;
  return LVG_OK;
}

lvg_status lvg_dgraph_arrays(const lvg_dgraph* g, const int32_t** src, const int32_t** dst, const float** w) {
  if (!g) return LVG_ERR_INVALID_ARG;
  if (src) *src = g->src;
  if (dst) *dst = g->dst;
  if (w) *w = g->w;
  return LVG_OK;
}

lvg_status lvg_dgraph_offsets(const lvg_dgraph* g, int64_t* entry_off, int32_t* vertex_off) {
  if (!g) return LVG_ERR_INVALID_ARG;
  if (entry_off) std::copy(g->eoff.begin(), g->eoff.end(), entry_off);
  if (vertex_off) std::copy(g->voff.begin(), g->voff.end(), vertex_off);
  return LVG_OK;
}

lvg_status lvg_dgraph_copy_to_host(const lvg_dgraph* g, int32_t* src, int32_t* dst, float* w) {
  if (!g) return LVG_ERR_INVALID_ARG;
  return gen_guard([&] {
    LVG_CUDA(cudaSetDevice(g->device));
    const size_t n = (size_t)g->n_entries;
    if (n == 0) return;
    if (src) LVG_CUDA(cudaMemcpy(src, g->src, 4 * n, cudaMemcpyDeviceToHost));
    if (dst) LVG_CUDA(cudaMemcpy(dst, g->dst, 4 * n, cudaMemcpyDeviceToHost));
    if (w) LVG_CUDA(cudaMemcpy(w, g->w, 4 * n, cudaMemcpyDeviceToHost));
  });
}

void lvg_dgraph_free(lvg_dgraph* g) { delete g; }

}  // extern "C"
