// Seeded synthetic graph generators (host).  The random stream is the same
// counter-based splitmix64 construction as the device generator, so R-MAT
// graphs generated here and on the GPU are identical.
#include "gen_host.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <vector>

namespace {

inline uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
inline uint64_t rng_at(uint64_t seed, uint64_t stream, uint64_t i) {
  return mix64(mix64(seed ^ mix64(stream + 0x632BE59BD9B4E019ull)) + i);
}
inline double u01(uint64_t r) { return (double)(r >> 11) * (1.0 / 9007199254740992.0); }

struct Rng {  // sequential stream
  uint64_t seed, stream, i = 0;
  Rng(uint64_t s, uint64_t st) : seed(s), stream(st) {}
  uint64_t next() { return rng_at(seed, stream, i++); }
  double uni() { return u01(next()); }
  uint64_t below(uint64_t n) { return n ? next() % n : 0; }
};

struct UEdge {
  int32_t u, v;
  float w;
};

}  // namespace

struct lvggen_graph {
  int32_t n = 0;
  std::vector<int32_t> src, dst;
  std::vector<float> w;
  std::vector<int32_t> truth;
};

namespace {

template <typename T>
inline T fetch_add(T* x, T v) { return __atomic_fetch_add(x, v, __ATOMIC_RELAXED); }

// Undirected edges (u < v; u < 0 marks a dropped entry) -> merged, symmetric
// list sorted by (src, dst), built in parallel.  Row i holds its partners
// below i (edges (u, i)) and then those above i (edges (i, v)), each part in
// increasing partner order; duplicate edges are merged (weights summed, or the
// first kept).  The list is unique: parts are sorted by partner, and equal
// (u, v) weights are integers, whose sums are exact in any order.
void finish(lvggen_graph* g, std::vector<UEdge>& ue, bool sum_dups) {
  const int32_t n = g->n;
  const int64_t M = (int64_t)ue.size();
  // 1. bucket by the smaller endpoint
  std::vector<int64_t> off((size_t)n + 1, 0);
#pragma omp parallel for schedule(static)
  for (int64_t e = 0; e < M; ++e)
    if (ue[e].u >= 0) fetch_add<int64_t>(&off[(size_t)ue[e].u + 1], 1);
  for (int32_t i = 0; i < n; ++i) off[i + 1] += off[i];
  std::vector<UEdge> b((size_t)off[n]);
  {
    std::vector<int64_t> cur(off.begin(), off.end() - 1);
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < M; ++e)
      if (ue[e].u >= 0) b[(size_t)fetch_add<int64_t>(&cur[ue[e].u], 1)] = ue[e];
  }
  std::vector<UEdge>().swap(ue);
  // 2. each bucket sorted by partner, duplicates merged in place
  std::vector<int64_t> mcnt(n, 0), tcnt(n, 0);
#pragma omp parallel for schedule(dynamic, 1024)
  for (int32_t u = 0; u < n; ++u) {
    UEdge* lo = b.data() + off[u];
    UEdge* hi = b.data() + off[u + 1];
    std::sort(lo, hi, [](const UEdge& x, const UEdge& y) { return x.v != y.v ? x.v < y.v : x.w < y.w; });
    int64_t k = 0;
    for (UEdge* it = lo; it != hi; ++it) {
      if (k > 0 && lo[k - 1].v == it->v) {
        if (sum_dups) lo[k - 1].w += it->w;
      } else {
        lo[k++] = *it;
      }
    }
    mcnt[u] = k;
    for (int64_t j = 0; j < k; ++j) fetch_add<int64_t>(&tcnt[lo[j].v], 1);
  }
  // 3. rows of the symmetric list
  std::vector<int64_t> row((size_t)n + 1, 0);
  for (int32_t i = 0; i < n; ++i) row[i + 1] = row[i] + tcnt[i] + mcnt[i];
  const int64_t E = row[n];
  g->src.resize(E); g->dst.resize(E); g->w.resize(E);
  {
    std::vector<int64_t> cur(row.begin(), row.end() - 1);
#pragma omp parallel for schedule(dynamic, 1024)
    for (int32_t u = 0; u < n; ++u) {
      const UEdge* lo = b.data() + off[u];
      for (int64_t j = 0; j < mcnt[u]; ++j) {   // (u, v) seen from v: partner u below v
        const int64_t p = fetch_add<int64_t>(&cur[lo[j].v], 1);
        g->src[p] = lo[j].v; g->dst[p] = u; g->w[p] = lo[j].w;
      }
      const int64_t q = row[u] + tcnt[u];       // partners above u, already in order
      for (int64_t j = 0; j < mcnt[u]; ++j) {
        g->src[q + j] = u; g->dst[q + j] = lo[j].v; g->w[q + j] = lo[j].w;
      }
    }
  }
  // 4. the lower part of every row in partner order (partners are distinct)
#pragma omp parallel
  {
    std::vector<std::pair<int32_t, float>> tmp;
#pragma omp for schedule(dynamic, 1024)
    for (int32_t i = 0; i < n; ++i) {
      const int64_t lo = row[i], k = tcnt[i];
      if (k < 2) continue;
      tmp.resize(k);
      for (int64_t j = 0; j < k; ++j) tmp[j] = {g->dst[lo + j], g->w[lo + j]};
      std::sort(tmp.begin(), tmp.end(), [](const std::pair<int32_t, float>& x, const std::pair<int32_t, float>& y) {
        return x.first < y.first;
      });
      for (int64_t j = 0; j < k; ++j) { g->dst[lo + j] = tmp[j].first; g->w[lo + j] = tmp[j].second; }
    }
  }
}

float int_weight(uint64_t r, int32_t lo, int32_t hi) {
  if (hi <= lo) return (float)lo;
  return (float)(lo + (int32_t)(r % (uint64_t)(hi - lo + 1)));
}

double powerlaw(double u, double g, double lo, double hi) {
  double a = std::pow(lo, 1.0 - g), b = std::pow(hi, 1.0 - g);
  return std::pow(a + (b - a) * u, 1.0 / (1.0 - g));
}

}  // namespace

extern "C" {

lvggen_graph* lvggen_sbm(int32_t n, int32_t blocks, double p_in, double p_out, int32_t w_lo, int32_t w_hi,
                         uint64_t seed) {
  if (n <= 0 || blocks <= 0 || blocks > n) return nullptr;
  auto* g = new lvggen_graph();
  g->n = n;
  g->truth.resize(n);
  std::vector<int32_t> bstart(blocks + 1);
  for (int32_t b = 0; b <= blocks; ++b) bstart[b] = (int32_t)((int64_t)n * b / blocks);
  for (int32_t b = 0; b < blocks; ++b)
    for (int32_t v = bstart[b]; v < bstart[b + 1]; ++v) g->truth[v] = b;
  std::vector<UEdge> ue;
  uint64_t pair_id = 0;
  for (int32_t A = 0; A < blocks; ++A) {
    for (int32_t B = A; B < blocks; ++B, ++pair_id) {
      double p = A == B ? p_in : p_out;
      if (p <= 0.0) continue;
      int64_t sa = bstart[A + 1] - bstart[A], sb = bstart[B + 1] - bstart[B];
      int64_t S = sa * sb;  // ordered square; intra keeps u < v only
      Rng r(seed, pair_id);
      double lq = p < 1.0 ? std::log1p(-p) : 0.0;
      int64_t idx = -1;
      for (;;) {
        if (p >= 1.0) idx += 1;
        else {
          double u = r.uni();
          idx += 1 + (int64_t)std::floor(std::log1p(-u) / lq);
        }
        if (idx >= S || idx < 0) break;
        int32_t u = bstart[A] + (int32_t)(idx / sb), v = bstart[B] + (int32_t)(idx % sb);
        if (A == B && u >= v) continue;
        ue.push_back({u, v, int_weight(r.next(), w_lo, w_hi)});
      }
    }
  }
  finish(g, ue, true);
  return g;
}

lvggen_graph* lvggen_lfr(int32_t n, double deg_exp, int32_t d_min, int32_t d_max, double com_exp, int32_t c_min,
                         int32_t c_max, double mu, uint64_t seed) {
  if (n <= 0 || d_min <= 0 || d_max < d_min || c_min <= 1 || c_max < c_min) return nullptr;
  auto* g = new lvggen_graph();
  g->n = n;
  Rng r(seed, 1);
  std::vector<int32_t> deg(n);
  for (int32_t i = 0; i < n; ++i) {
    double x = powerlaw(r.uni(), deg_exp, d_min, d_max + 1.0);
    deg[i] = std::min(d_max, std::max(d_min, (int32_t)std::floor(x)));
  }
  // community sizes; the remainder that does not fill a community joins the smallest one
  std::vector<int32_t> cs;
  int64_t total = 0;
  while (total < n) {
    int32_t s = std::min(c_max, std::max(c_min, (int32_t)std::floor(powerlaw(r.uni(), com_exp, c_min, c_max + 1.0))));
    if (total + s > n) {
      int32_t rest = (int32_t)(n - total);
      if (rest >= c_min || cs.empty()) cs.push_back(rest);
      else *std::min_element(cs.begin(), cs.end()) += rest;
      total = n;
      break;
    }
    cs.push_back(s);
    total += s;
  }
  const int32_t K = (int32_t)cs.size();
  // internal degree and assignment (largest internal degree first)
  std::vector<int32_t> din(n), order(n), freeslots(cs), comm(n, -1);
  for (int32_t i = 0; i < n; ++i) din[i] = (int32_t)std::lround((1.0 - mu) * deg[i]);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) { return din[a] > din[b]; });
  std::vector<int64_t> cum(K + 1, 0);
  for (int32_t k = 0; k < K; ++k) cum[k + 1] = cum[k] + cs[k];
  for (int32_t v : order) {
    int32_t pick = -1;
    for (int t = 0; t < 64 && pick < 0; ++t) {
      int64_t x = (int64_t)r.below((uint64_t)cum[K]);
      int32_t k = (int32_t)(std::upper_bound(cum.begin(), cum.end(), x) - cum.begin()) - 1;
      if (freeslots[k] > 0 && cs[k] > din[v]) pick = k;
    }
    if (pick < 0) {
      int32_t bestk = -1;
      for (int32_t k = 0; k < K; ++k)
        if (freeslots[k] > 0 && (bestk < 0 || cs[k] > cs[bestk])) bestk = k;
      pick = bestk;
    }
    comm[v] = pick;
    freeslots[pick]--;
    din[v] = std::min(din[v], cs[pick] - 1);
  }
  g->truth = comm;
  std::vector<std::vector<int32_t>> members(K);
  for (int32_t v = 0; v < n; ++v) members[comm[v]].push_back(v);
  std::vector<UEdge> ue;
  ue.reserve((size_t)std::accumulate(deg.begin(), deg.end(), (int64_t)0) / 2 + 16);
  std::vector<int32_t> stubs;
  for (int32_t k = 0; k < K; ++k) {
    stubs.clear();
    for (int32_t v : members[k])
      for (int32_t j = 0; j < din[v]; ++j) stubs.push_back(v);
    Rng rk(seed, 1000 + (uint64_t)k);
    for (size_t i = stubs.size(); i > 1; --i) std::swap(stubs[i - 1], stubs[rk.below(i)]);
    for (size_t i = 0; i + 1 < stubs.size(); i += 2) {
      int32_t a = stubs[i], b = stubs[i + 1];
      if (a != b) ue.push_back({std::min(a, b), std::max(a, b), 1.0f});
    }
  }
  stubs.clear();
  for (int32_t v = 0; v < n; ++v)
    for (int32_t j = 0; j < deg[v] - din[v]; ++j) stubs.push_back(v);
  Rng rx(seed, 2);
  for (size_t i = stubs.size(); i > 1; --i) std::swap(stubs[i - 1], stubs[rx.below(i)]);
  for (size_t i = 0; i + 1 < stubs.size(); i += 2) {
    int32_t a = stubs[i], b = stubs[i + 1];
    if (a != b) ue.push_back({std::min(a, b), std::max(a, b), 1.0f});
  }
  finish(g, ue, false);
  return g;
}

lvggen_graph* lvggen_rmat(int32_t scale, int32_t edge_factor, double a, double b, double c, int32_t w_lo,
                          int32_t w_hi, uint64_t seed) {
  if (scale <= 0 || scale > 30 || edge_factor <= 0) return nullptr;
  auto* g = new lvggen_graph();
  g->n = (int32_t)1 << scale;
  g->truth.assign(g->n, -1);
  const int64_t M = (int64_t)edge_factor << scale;
  std::vector<UEdge> ue((size_t)M);
  const double ab = a + b, abc = a + b + c;
#pragma omp parallel for schedule(static)
  for (int64_t e = 0; e < M; ++e) {
    uint32_t u = 0, v = 0;
    for (int l = 0; l < scale; ++l) {
      double x = u01(rng_at(seed, (uint64_t)l + 16, (uint64_t)e));
      uint32_t bu = x >= ab ? 1u : 0u;
      uint32_t bv = (x >= a && x < ab) || x >= abc ? 1u : 0u;
      u = (u << 1) | bu;
      v = (v << 1) | bv;
    }
    if (u == v) { ue[e] = {-1, -1, 0.0f}; continue; }   // self loop: dropped
    float w = int_weight(rng_at(seed, 3, (uint64_t)e), w_lo, w_hi);
    ue[e] = {(int32_t)std::min(u, v), (int32_t)std::max(u, v), w};
  }
  finish(g, ue, true);
  return g;
}

int32_t lvggen_n_vertices(const lvggen_graph* g) { return g ? g->n : 0; }
int64_t lvggen_n_entries(const lvggen_graph* g) { return g ? (int64_t)g->src.size() : 0; }
void lvggen_copy(const lvggen_graph* g, int32_t* src, int32_t* dst, float* w) {
  if (src) std::memcpy(src, g->src.data(), sizeof(int32_t) * g->src.size());
  if (dst) std::memcpy(dst, g->dst.data(), sizeof(int32_t) * g->dst.size());
  if (w) std::memcpy(w, g->w.data(), sizeof(float) * g->w.size());
}
void lvggen_truth(const lvggen_graph* g, int32_t* m) {
  if (m) std::memcpy(m, g->truth.data(), sizeof(int32_t) * g->truth.size());
}
void lvggen_free(lvggen_graph* g) { delete g; }

}  // extern "C"
