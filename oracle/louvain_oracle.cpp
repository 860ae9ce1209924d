// CPU oracle for the Louvain hot path of LouvainGPU -- TEST INFRASTRUCTURE ONLY.
//
// Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference
// legs load this library, always as the checker or the timed CPU baseline.
//
// PARITY UNPINNED: the reference cannot be built or run here (CUDPP 2.3 and
// Boost.Python absent, Thrust API drift against CUDA 12.9, pre-Volta
// __shfl_down undefined on sm_100a) and it ships no test or golden vector.
// The restatement below is pinned by hand-derived known answers and by
// networkx modularity instead.
//
// Every function cites the reference file:line it restates.  Compile with
// -ffp-contract=off: the FP64 gain and Q expressions must round exactly as the
// CUDA kernels do (they use __dmul_rn/__dsub_rn/__ddiv_rn).
#include "oracle.h"

#include <omp.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <memory>
#include <numeric>
#include <type_traits>
#include <vector>

namespace {

double tree_sum(const double* x, int64_t n);
template <typename T>
double tree_sum_of(const T* x, int64_t n);

// One entry of a source-grouped list: neighbour (or coarse target) and weight.
struct Ent {
  int32_t c;
  float w;
};
inline bool ent_less(const Ent& x, const Ent& y) { return x.c < y.c; }

// Stable sort by c.  Short runs take an insertion sort in place (no buffer
// allocation per run); a stable sort's result is unique, so both give the
// same order.
inline void stable_sort_ents(Ent* b, Ent* e) {
  if (e - b > 48) {
    std::stable_sort(b, e, ent_less);
    return;
  }
  for (Ent* i = b + 1; i < e; ++i) {
    Ent x = *i;
    Ent* j = i;
    for (; j > b && x.c < (j - 1)->c; --j) *j = *(j - 1);
    *j = x;
  }
}

// Stable counting sort of items 0..n-1 by key(i) in [0, K): bucket k receives
// its items in index order at positions [off[k], off[k+1]), put(pos, i) writes
// one.  Threads count and place contiguous index ranges; a thread's items of a
// bucket go after those of every lower-ranked thread, so the order is the
// same as one thread's.
template <typename KeyF, typename PutF>
void stable_scatter(int64_t n, int32_t K, KeyF key, PutF put, std::vector<int64_t>& off) {
  off.assign((size_t)K + 1, 0);
  int want = n < (1 << 16) ? 1 : std::min(omp_get_max_threads(), 32);
  std::unique_ptr<int64_t[]> cnt;
  int nth = 1;
#pragma omp parallel num_threads(want)
  {
#pragma omp single
    {
      nth = omp_get_num_threads();
      cnt.reset(new int64_t[(size_t)nth * (size_t)K + 1]);
    }
    const int t = omp_get_thread_num();
    const int64_t lo = n * t / nth, hi = n * (t + 1) / nth;
    int64_t* c = cnt.get() + (size_t)t * (size_t)K;
    std::fill(c, c + K, (int64_t)0);
    for (int64_t i = lo; i < hi; ++i) c[key(i)]++;
#pragma omp barrier
#pragma omp for schedule(static)
    for (int32_t k = 0; k < K; ++k) {
      int64_t run = 0;
      for (int tt = 0; tt < nth; ++tt) {
        int64_t& x = cnt[(size_t)tt * (size_t)K + k];
        const int64_t v = x;
        x = run;
        run += v;
      }
      off[(size_t)k + 1] = run;
    }
#pragma omp single
    for (int32_t k = 0; k < K; ++k) off[(size_t)k + 1] += off[k];
    for (int64_t i = lo; i < hi; ++i) {
      const int32_t k = key(i);
      put(off[k] + c[k]++, i);
    }
  }
}

struct Csr {
  int32_t V = 0;
  int64_t nnz = 0;
  std::vector<int64_t> off;
  std::vector<int32_t> col;
  std::vector<float> w;
  std::vector<double> k;      // FP64 degree (InitKernel.cu:154-179)
  std::vector<float> kf32;    // float degree, the reference's gdegrees
  std::vector<float> loopw;   // weight of the last self-loop entry (InitKernel.cu:181-194)
  std::vector<uint8_t> has_loop;
  std::vector<uint8_t> active;  // vertex owns at least one entry of the doubled list
  double m = 0.0;               // sum of input weights (NeighbourCompute.cu:46)
};

// Doubled list D = input ++ reversed(input) (NeighbourCompute.cu:66-68), sorted
// by (src, dst) keeping D-order among equal keys (NeighbourCompute.cu:82, a
// merge sort), then per source: degree, last self-loop weight, and the merged
// weight of every distinct non-loop neighbour.
Csr* build_csr(int32_t V, int64_t E, const int32_t* src, const int32_t* dst, const float* w) {
  if (V < 0 || E < 0) return nullptr;
  bool bad = false;
#pragma omp parallel for schedule(static) reduction(|| : bad)
  for (int64_t e = 0; e < E; ++e) {
    if (src[e] < 0 || src[e] >= V || dst[e] < 0 || dst[e] >= V) bad = true;
    if (!(w[e] >= 0.0f) || std::isinf(w[e])) bad = true;
  }
  if (bad) return nullptr;
  auto* g = new Csr();
  g->V = V;
  g->m = tree_sum_of(w, E);   // m = sum of weights (NeighbourCompute.cu:46) on the fixed tree
  // stable counting sort of D by source: D-order index d < E is input entry d,
  // d >= E the reversed copy of entry d - E
  std::vector<int64_t> roff;
  std::unique_ptr<Ent[]> D(new Ent[2 * E]);   // uninitialised: the scattering threads touch it first
  stable_scatter(
      2 * E, V, [&](int64_t d) { return d < E ? src[d] : dst[d - E]; },
      [&](int64_t pos, int64_t d) { D[pos] = d < E ? Ent{dst[d], w[d]} : Ent{src[d - E], w[d - E]}; }, roff);
  g->k.assign(V, 0.0);
  g->kf32.assign(V, 0.0f);
  g->loopw.assign(V, 0.0f);
  g->has_loop.assign(V, 0);
  g->active.assign(V, 0);
  std::vector<int64_t> cnt(V + 1, 0);
#pragma omp parallel for schedule(dynamic, 256)
  for (int32_t i = 0; i < V; ++i) {
    Ent* b = D.get() + roff[i];
    Ent* e = D.get() + roff[i + 1];
    stable_sort_ents(b, e);
    double kd = 0.0;
    float kf = 0.0f;
    int64_t distinct = 0;
    for (Ent* it = b; it != e; ++it) {
      float v = it->w == 0.0f ? 1.0f : it->w;   // InitKernel.cu:165-167
      if (it->c == i) v *= 2.0f;                 // InitKernel.cu:169-170
      kd += (double)v;
      kf += v;
      if (it->c == i) { g->loopw[i] = it->w; g->has_loop[i] = 1; }
      else if (it == b || (it - 1)->c != it->c) distinct++;
    }
    g->k[i] = kd;
    g->kf32[i] = kf;
    g->active[i] = (b != e);
    cnt[i + 1] = distinct;
  }
  for (int32_t i = 0; i < V; ++i) cnt[i + 1] += cnt[i];
  g->off = cnt;
  g->nnz = cnt[V];
  g->col.resize(g->nnz);
  g->w.resize(g->nnz);
#pragma omp parallel for schedule(dynamic, 256)
  for (int32_t i = 0; i < V; ++i) {
    int64_t o = g->off[i];
    int64_t p = roff[i], q = roff[i + 1];
    while (p < q) {
      int32_t j = D[p].c;
      double s = 0.0;
      int64_t r = p;
      while (r < q && D[r].c == j) s += (double)D[r++].w;
      if (j != i) { g->col[o] = j; g->w[o] = (float)s; ++o; }
      p = r;
    }
  }
  return g;
}

// Fixed summation tree shared with the device reduction (tree_sum in the
// package's reduce.cuh).  Values are taken in groups of 2048; inside a group,
// thread t of 256 sums x[t], x[256+t], ..., x[1792+t] left to right, the 256
// thread sums are added as eight 32-lane shuffle-down trees (offsets
// 16,8,4,2,1) and the eight warp sums by one more 32-lane tree (zero padded).
// Group sums are reduced the same way until one value remains.
double tree32(const double* v, int n) {
  double s[32];
  for (int l = 0; l < 32; ++l) s[l] = l < n ? v[l] : 0.0;
  for (int o = 16; o >= 1; o >>= 1)
    for (int l = 0; l < o; ++l) s[l] = s[l] + s[l + o];
  return s[0];
}
template <typename T>
double group_sum(const T* x, int64_t n) {  // values are widened to double as read
  double ts[256];
  for (int t = 0; t < 256; ++t) {
    double s = 0.0;
    for (int j = 0; j < 8; ++j) {
      int64_t idx = (int64_t)j * 256 + t;
      if (idx < n) s = s + (double)x[idx];
    }
    ts[t] = s;
  }
  double ws[8];
  for (int wi = 0; wi < 8; ++wi) ws[wi] = tree32(ts + wi * 32, 32);
  return tree32(ws, 8);
}
template <typename T>
double tree_sum_of(const T* x, int64_t n) {
  if (n <= 0) return 0.0;
  const int64_t nb0 = (n + 2047) / 2048;
  std::vector<double> cur(nb0), nxt;
#pragma omp parallel for schedule(static) if (nb0 >= 64)
  for (int64_t b = 0; b < nb0; ++b) cur[b] = group_sum(x + b * 2048, std::min<int64_t>(2048, n - b * 2048));
  while (cur.size() > 1) {
    int64_t nn = (int64_t)cur.size();
    int64_t nb = (nn + 2047) / 2048;
    nxt.assign(nb, 0.0);
    for (int64_t b = 0; b < nb; ++b) nxt[b] = group_sum(cur.data() + b * 2048, std::min<int64_t>(2048, nn - b * 2048));
    cur.swap(nxt);
  }
  return cur[0];
}
double tree_sum(const double* x, int64_t n) { return tree_sum_of(x, n); }

double q_terms_fp64(const double* tot, const double* in, int32_t n, double m) {
  // OneLevelKernel.cu:427-451 in FP64: in/m - (tot/2m)^2, zero when m == 0.
  std::vector<double> t(n, 0.0);
  if (m > 0.0) {
    double twom = 2.0 * m;
    for (int32_t c = 0; c < n; ++c) {
      double a = in[c] / m;
      double b = tot[c] / twom;
      t[c] = a - b * b;
    }
  }
  return tree_sum(t.data(), n);
}

float q_terms_ref32(const int32_t* tot, const int32_t* in, int32_t n, float m) {
  // OneLevelKernel.cu:443-448: float terms; the device-wide float reduction is
  // stood in for by an FP64 sum rounded once.
  double s = 0.0;
  if (m > 0.0f) {
    for (int32_t c = 0; c < n; ++c) {
      float a = (float)in[c] / m;
      float b = (float)tot[c] / (2.0f * m);
      s += (double)(a - b * b);
    }
  }
  return (float)s;
}

// Per-thread scratch for neighbour-community aggregation.
template <typename W>
struct Scratch {
  std::vector<W> acc;
  std::vector<int32_t> stamp;
  std::vector<int32_t> touched;
  explicit Scratch(int32_t V) : acc(V, W(0)), stamp(V, -1) { touched.reserve(1024); }
};

// One synchronous decision for vertex i (OneLevelKernel.cu:248-386 for the
// best-community search, :388-422 for the singleton-pair rule, :138-171 for the
// merge candidate).  The chunked warp reduction of the reference is restated
// as the argmax it implements: highest gain among neighbour communities with
// non-zero summed weight, ties to the lower community id, accepted only when
// strictly positive.
template <bool REF32>
struct Decision {
  int32_t next, cand, nseg;
  double wbest;  // summed weight to the chosen community
};

template <bool REF32, typename TotT>
inline Decision<REF32> decide(const Csr& g, int32_t i, const int32_t* comm, const TotT* tot,
                              const int32_t* size, double kfrac, float degc32,
                              Scratch<typename std::conditional<REF32, float, double>::type>& s) {
  using W = typename std::conditional<REF32, float, double>::type;
  Decision<REF32> d;
  int32_t own = comm[i];
  if (!g.active[i]) { d.next = own; d.cand = -1; d.nseg = 0; d.wbest = 0.0; return d; }
  s.touched.clear();
  for (int64_t e = g.off[i]; e < g.off[i + 1]; ++e) {
    int32_t c = comm[g.col[e]];
    if (s.stamp[c] != i) { s.stamp[c] = i; s.acc[c] = W(0); s.touched.push_back(c); }
    s.acc[c] += (W)g.w[e];
  }
  int32_t nseg = (int32_t)s.touched.size();
  if (g.has_loop[i] && s.stamp[own] != i) nseg++;  // self-loop entry keyed by own community
  int32_t best = own;
  W bg = W(0), bw = W(0);
  for (int32_t c : s.touched) {
    W wc = s.acc[c];
    if (wc == W(0)) continue;                                   // OneLevelKernel.cu:303,327
    W gain;
    if constexpr (REF32) {
      gain = std::fma(-(float)tot[c], degc32, wc);              // weight - degree * degcTotW
    } else {
      double t = (double)tot[c] * kfrac;
      gain = wc - t;
    }
    if (gain > bg || (gain == bg && bg != W(0) && c < best)) {  // OneLevelKernel.cu:330,358
      best = c; bg = gain; bw = wc;
    }
  }
  for (int32_t c : s.touched) s.stamp[c] = -1;                  // scratch reused by the next vertex/pass
  int32_t raw = best;
  if (size[own] == 1 && size[best] == 1 && best > own) best = own;  // OneLevelKernel.cu:407-410
  d.next = best;
  d.nseg = nseg;
  d.wbest = (double)bw;
  d.cand = (size[own] == 1 && nseg == 1 && raw != own && own < raw) ? raw : -1;  // :147-169
  return d;
}

struct LevelRec {
  int32_t V = 0;
  int64_t E = 0, nnz = 0;
  int32_t C = 0, passes = 0;
  double q_start = 0.0, q_level = 0.0;
  std::vector<int32_t> part, labels;
  std::vector<double> qtrace;
};

struct RunState {
  int32_t status = 0;
  std::vector<LevelRec> levels;
  double seconds = 0.0;
  int64_t pass_entries = 0;
};

// oneLevelCUDA (OneLevelKernel.cu:518-954) in FP64.
template <bool REF32>
int32_t one_level(const Csr& g, double lower, const orc_config& cfg, std::vector<int32_t>& comm,
                  double& q_start, double& q_ret, int32_t& passes, std::vector<double>& qtrace) {
  const int32_t V = g.V;
  using TotT = typename std::conditional<REF32, int32_t, double>::type;
  using W = typename std::conditional<REF32, float, double>::type;
  std::vector<TotT> tot(V), in(V), dtot(V, TotT(0)), din(V, TotT(0));
  std::vector<int32_t> size(V, 1), dsize(V, 0), next(V), cand(V), nseg(V);
  std::vector<double> wbest(V), kfrac(V);
  std::vector<float> degc(V);
  const double twom = 2.0 * g.m;
  const float m32 = (float)g.m;
  comm.resize(V);
  for (int32_t i = 0; i < V; ++i) {
    comm[i] = i;                                            // InitKernel.cu:196-216
    if constexpr (REF32) {
      tot[i] = (int32_t)g.kf32[i];                          // InitKernel.cu:236 (float->int)
      in[i] = (int32_t)g.loopw[i];                          // InitKernel.cu:241-242
      degc[i] = g.kf32[i] / (m32 * 2.0f);                   // OneLevelKernel.cu:307
    } else {
      tot[i] = g.k[i];
      in[i] = (double)g.loopw[i];
      kfrac[i] = g.m > 0.0 ? g.k[i] / twom : 0.0;
    }
  }
  auto qcur = [&]() -> double {
    if constexpr (REF32) return (double)q_terms_ref32(tot.data(), in.data(), V, m32);
    else return q_terms_fp64(tot.data(), in.data(), V, g.m);
  };
  double qs = qcur();
  q_start = qs;
  int nt = cfg.n_threads > 0 ? cfg.n_threads : omp_get_max_threads();
  std::vector<std::unique_ptr<Scratch<W>>> scr(nt);
  for (int t = 0; t < nt; ++t) scr[t].reset(new Scratch<W>(V));
  auto decide_all = [&]() {
#pragma omp parallel for num_threads(nt) schedule(dynamic, 512)
    for (int32_t i = 0; i < V; ++i) {
      auto d = decide<REF32>(g, i, comm.data(), tot.data(), size.data(), kfrac[i], degc[i],
                             *scr[omp_get_thread_num()]);
      next[i] = d.next; cand[i] = d.cand; nseg[i] = d.nseg; wbest[i] = d.wbest;
    }
  };
  // remove/insert (OneLevelKernel.cu:52-78): accumulate into the *Upd buffers.
  auto move_vertex = [&](int32_t i, int32_t from, int32_t to, double wgt) {
    if constexpr (REF32) {
      int32_t kd = (int32_t)g.kf32[i];
      int32_t iw = (int32_t)((float)wgt + g.loopw[i]);
      dtot[from] -= kd; dtot[to] += (int32_t)(long long)g.kf32[i];
      din[from] -= iw; din[to] += iw;
    } else {
      dtot[from] -= g.k[i]; dtot[to] += g.k[i];
      double iw = wgt + (double)g.loopw[i];
      din[from] -= iw; din[to] += iw;
    }
    dsize[from] -= 1; dsize[to] += 1;
  };
  auto commit = [&]() {  // communitySetKernel (OneLevelKernel.cu:93-107)
    for (int32_t c = 0; c < V; ++c) {
      tot[c] += dtot[c]; in[c] += din[c]; size[c] += dsize[c];
      dtot[c] = TotT(0); din[c] = TotT(0); dsize[c] = 0;
    }
  };
  double cur = -1.0;
  float cur32 = -1.0f;
  int32_t pass = 0, status = 0;
  for (;;) {
    ++pass;
    decide_all();
    double newmod = qs;
    qtrace.push_back(newmod);
    bool stop;
    if constexpr (REF32) stop = (double)((float)newmod - cur32) < cfg.pass_min_gain;
    else stop = (newmod - cur) < cfg.pass_min_gain;          // OneLevelKernel.cu:889
    if (stop) break;
    if (cfg.max_passes >= 0 && pass >= cfg.max_passes) { status = 4; break; }
    if constexpr (REF32) { cur32 = (float)newmod; if (cur32 < (float)lower) cur32 = (float)lower; }
    else { cur = newmod; if (cur < lower) cur = lower; }    // :894-896
    for (int32_t i = 0; i < V; ++i)
      if (next[i] != comm[i]) move_vertex(i, comm[i], next[i], wbest[i]);
    commit();
    comm.swap(next);
    qs = qcur();
  }
  // Isolated-vertex merge (OneLevelKernel.cu:921-928, :138-171) on the committed
  // state, then adopt the last pass's decisions (:934-937).
  for (int32_t c = 0; c < V; ++c) { dtot[c] = TotT(0); din[c] = TotT(0); dsize[c] = 0; }
  for (int32_t i = 0; i < V; ++i) {
    if (cand[i] >= 0) { move_vertex(i, comm[i], cand[i], 0.0); next[i] = cand[i]; }
  }
  commit();
  comm.swap(next);
  q_ret = qcur();
  passes = pass;
  return status;
}

int32_t renumber(int32_t V, const int32_t* comm, int32_t* newid) {
  // RenumberKernel.cu:94-191: communities numbered by their smallest member index.
  std::vector<int32_t> id(V, -1);
  int32_t C = 0;
  for (int32_t i = 0; i < V; ++i) {
    int32_t c = comm[i];
    if (id[c] < 0) id[c] = C++;
    newid[i] = id[c];
  }
  return C;
}

struct Edges {
  std::vector<int32_t> s, t;
  std::vector<float> w;
};

void induce(int64_t E, const int32_t* src, const int32_t* dst, const float* w, const int32_t* part,
            int32_t C, Edges& out) {
  // InducedGraphKernel.cu:28-113: map both endpoints, weight 0 -> 1, sort by
  // (cu, cv) and sum the weights of equal keys (FP64 sum, rounded once).
  // Entries grouped by cu in input order, then each group sorted stably by
  // cv; groups are independent, so they sort and sum in parallel and write
  // their distinct keys at offsets from a scan of the per-group counts.
  std::vector<int64_t> cnt;
  std::unique_ptr<Ent[]> R(new Ent[E]);
  stable_scatter(
      E, C, [&](int64_t e) { return part[src[e]]; },
      [&](int64_t pos, int64_t e) { R[pos] = Ent{part[dst[e]], w[e] == 0.0f ? 1.0f : w[e]}; }, cnt);
  std::vector<int64_t> dcnt((size_t)C + 1, 0);
#pragma omp parallel for schedule(dynamic, 64)
  for (int32_t a = 0; a < C; ++a) {
    Ent* b = R.get() + cnt[a];
    Ent* e = R.get() + cnt[a + 1];
    stable_sort_ents(b, e);
    int64_t d = 0;
    for (Ent* it = b; it != e; ++it)
      if (it == b || (it - 1)->c != it->c) ++d;
    dcnt[(size_t)a + 1] = d;
  }
  for (int32_t a = 0; a < C; ++a) dcnt[(size_t)a + 1] += dcnt[a];
  const int64_t n_out = dcnt[C];
  out.s.assign(n_out, 0); out.t.assign(n_out, 0); out.w.assign(n_out, 0.0f);
#pragma omp parallel for schedule(dynamic, 64)
  for (int32_t a = 0; a < C; ++a) {
    int64_t o = dcnt[a];
    const Ent* b = R.get() + cnt[a];
    const Ent* e = R.get() + cnt[a + 1];
    for (const Ent* it = b; it != e;) {
      int32_t v = it->c;
      double s = 0.0;
      while (it != e && it->c == v) { s += (double)it->w; ++it; }
      out.s[o] = a; out.t[o] = v; out.w[o] = (float)s;
      ++o;
    }
  }
}

}  // namespace

struct orc_csr { Csr g; };
struct orc_run { RunState st; };

extern "C" {

orc_csr* orc_csr_build(int32_t V, int64_t E, const int32_t* src, const int32_t* dst, const float* w) {
  Csr* g = build_csr(V, E, src, dst, w);
  if (!g) return nullptr;
  auto* h = new orc_csr();
  h->g = std::move(*g);
  delete g;
  return h;
}
void orc_csr_free(orc_csr* h) { delete h; }
int64_t orc_csr_nnz(const orc_csr* h) { return h->g.nnz; }
double orc_csr_m(const orc_csr* h) { return h->g.m; }
void orc_csr_get(const orc_csr* h, int64_t* off, int32_t* col, float* w, double* k, float* loopw,
                 uint8_t* has_loop) {
  const Csr& g = h->g;
  if (off) std::copy(g.off.begin(), g.off.end(), off);
  if (col) std::copy(g.col.begin(), g.col.end(), col);
  if (w) std::copy(g.w.begin(), g.w.end(), w);
  if (k) std::copy(g.k.begin(), g.k.end(), k);
  if (loopw) std::copy(g.loopw.begin(), g.loopw.end(), loopw);
  if (has_loop) std::copy(g.has_loop.begin(), g.has_loop.end(), has_loop);
}

void orc_move_decide(const orc_csr* h, const int32_t* comm, const double* tot, const int32_t* size,
                     int32_t* next, int32_t* cand, int32_t* nseg, int n_threads) {
  const Csr& g = h->g;
  int nt = n_threads > 0 ? n_threads : omp_get_max_threads();
  std::vector<std::unique_ptr<Scratch<double>>> scr(nt);
  for (int t = 0; t < nt; ++t) scr[t].reset(new Scratch<double>(g.V));
  const double twom = 2.0 * g.m;
#pragma omp parallel for num_threads(nt) schedule(dynamic, 512)
  for (int32_t i = 0; i < g.V; ++i) {
    double kf = g.m > 0.0 ? g.k[i] / twom : 0.0;
    auto d = decide<false>(g, i, comm, tot, size, kf, 0.0f, *scr[omp_get_thread_num()]);
    if (next) next[i] = d.next;
    if (cand) cand[i] = d.cand;
    if (nseg) nseg[i] = d.nseg;
  }
}

// orc_move_decide for the listed vertices only (a bounded sample of one
// decision pass): outputs are written at the listed positions.  Returns the
// seconds of the decisions alone (the per-thread scratch is set up first, as
// a whole run sets it up once per level).
double orc_move_decide_subset(const orc_csr* h, const int32_t* comm, const double* tot, const int32_t* size,
                            const int32_t* verts, int64_t n_verts, int32_t* next, int32_t* cand, int32_t* nseg,
                            int n_threads) {
  const Csr& g = h->g;
  int nt = n_threads > 0 ? n_threads : omp_get_max_threads();
  std::vector<std::unique_ptr<Scratch<double>>> scr(nt);
#pragma omp parallel num_threads(nt)
  scr[omp_get_thread_num()].reset(new Scratch<double>(g.V));   // first touch by the thread that uses it
  const double twom = 2.0 * g.m;
  const auto t0 = std::chrono::steady_clock::now();
#pragma omp parallel for num_threads(nt) schedule(dynamic, 512)
  for (int64_t j = 0; j < n_verts; ++j) {
    const int32_t i = verts[j];
    double kf = g.m > 0.0 ? g.k[i] / twom : 0.0;
    auto d = decide<false>(g, i, comm, tot, size, kf, 0.0f, *scr[omp_get_thread_num()]);
    if (next) next[i] = d.next;
    if (cand) cand[i] = d.cand;
    if (nseg) nseg[i] = d.nseg;
  }
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

double orc_tree_sum(const double* x, int64_t n) { return tree_sum(x, n); }

double orc_q_totals(const double* tot, const double* in, int32_t n, double m) {
  return q_terms_fp64(tot, in, n, m);
}

int32_t orc_renumber(int32_t V, const int32_t* comm, int32_t* newid) { return renumber(V, comm, newid); }

int64_t orc_induce(int32_t V, int64_t E, const int32_t* src, const int32_t* dst, const float* w,
                   const int32_t* part, int32_t* out_src, int32_t* out_dst, float* out_w) {
  int32_t C = 0;
  for (int32_t i = 0; i < V; ++i) C = std::max(C, part[i] + 1);
  Edges o;
  induce(E, src, dst, w, part, C, o);
  if (out_src) {
    std::copy(o.s.begin(), o.s.end(), out_src);
    std::copy(o.t.begin(), o.t.end(), out_dst);
    std::copy(o.w.begin(), o.w.end(), out_w);
  }
  return (int64_t)o.s.size();
}

// generate_dendogram (LouvainCPP.cpp:209-553).
orc_run* orc_run_louvain(int32_t V, int64_t E, const int32_t* src, const int32_t* dst, const float* w,
                         const orc_config* cfgp) {
  orc_config cfg = *cfgp;
  auto* h = new orc_run();
  RunState& st = h->st;
  auto t0 = std::chrono::steady_clock::now();
  if (cfg.n_threads > 0) omp_set_num_threads(cfg.n_threads);
  const bool ref32 = cfg.mode == ORC_REF32;
  if (E == 0) {  // LouvainCPP.cpp:211-230: one identity partition
    LevelRec r;
    r.V = V; r.C = V; r.part.resize(V); r.labels.resize(V);
    std::iota(r.part.begin(), r.part.end(), 0);
    std::iota(r.labels.begin(), r.labels.end(), 0);
    st.levels.push_back(r);
    return h;
  }
  Edges cur;
  cur.s.assign(src, src + E); cur.t.assign(dst, dst + E); cur.w.assign(w, w + E);
  int32_t nv = V;
  double mod = 0.0;
  for (int32_t level = 0;; ++level) {
    std::unique_ptr<Csr> g(build_csr(nv, (int64_t)cur.s.size(), cur.s.data(), cur.t.data(), cur.w.data()));
    if (!g) { st.status = 1; break; }
    LevelRec r;
    r.V = nv; r.E = (int64_t)cur.s.size(); r.nnz = g->nnz;
    std::vector<int32_t> comm;
    double qs = 0.0, qr = 0.0;
    int32_t passes = 0;
    double lower = mod;
    if (level == 0) {
      // modularityCUDA of the singleton state (LouvainCPP.cpp:356) is the lower bound.
      if (ref32) {
        std::vector<int32_t> t(nv), in(nv);
        for (int32_t i = 0; i < nv; ++i) { t[i] = (int32_t)g->kf32[i]; in[i] = (int32_t)g->loopw[i]; }
        lower = (double)q_terms_ref32(t.data(), in.data(), nv, (float)g->m);
      } else {
        std::vector<double> in(nv);
        for (int32_t i = 0; i < nv; ++i) in[i] = (double)g->loopw[i];
        lower = q_terms_fp64(g->k.data(), in.data(), nv, g->m);
      }
    }
    int32_t s = ref32 ? one_level<true>(*g, lower, cfg, comm, qs, qr, passes, r.qtrace)
                      : one_level<false>(*g, lower, cfg, comm, qs, qr, passes, r.qtrace);
    if (ref32) qr = (double)(float)qr;
    r.q_start = qs; r.q_level = qr; r.passes = passes;
    r.labels = comm;
    r.part.resize(nv);
    r.C = renumber(nv, comm.data(), r.part.data());
    st.pass_entries += g->nnz * (int64_t)passes;
    st.levels.push_back(std::move(r));
    if (s != 0) { st.status = s; break; }
    if (level > 0) {
      bool stop = ref32 ? (double)((float)qr - (float)mod) < cfg.level_min_gain
                        : (qr - mod) < cfg.level_min_gain;   // LouvainCPP.cpp:466
      if (stop) break;
    }
    if (cfg.max_levels >= 0 && level + 1 >= cfg.max_levels) { st.status = 4; break; }
    mod = ref32 ? (double)(float)qr : qr;
    Edges nxt;
    const LevelRec& lr = st.levels.back();
    induce((int64_t)cur.s.size(), cur.s.data(), cur.t.data(), cur.w.data(), lr.part.data(), lr.C, nxt);
    cur = std::move(nxt);
    nv = lr.C;
  }
  st.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return h;
}

void orc_run_free(orc_run* h) { delete h; }
int32_t orc_run_status(const orc_run* h) { return h->st.status; }
int32_t orc_run_levels(const orc_run* h) { return (int32_t)h->st.levels.size(); }
void orc_run_level_info(const orc_run* h, int32_t l, int32_t* V, int64_t* E, int64_t* nnz, int32_t* C,
                        int32_t* passes, double* q_start, double* q_level) {
  const LevelRec& r = h->st.levels[l];
  if (V) *V = r.V;
  if (E) *E = r.E;
  if (nnz) *nnz = r.nnz;
  if (C) *C = r.C;
  if (passes) *passes = r.passes;
  if (q_start) *q_start = r.q_start;
  if (q_level) *q_level = r.q_level;
}
void orc_run_level_partition(const orc_run* h, int32_t l, int32_t* part) {
  const LevelRec& r = h->st.levels[l];
  std::copy(r.part.begin(), r.part.end(), part);
}
void orc_run_level_labels(const orc_run* h, int32_t l, int32_t* labels) {
  const LevelRec& r = h->st.levels[l];
  std::copy(r.labels.begin(), r.labels.end(), labels);
}
int32_t orc_run_level_qtrace(const orc_run* h, int32_t l, double* q, int32_t cap) {
  const LevelRec& r = h->st.levels[l];
  int32_t n = (int32_t)r.qtrace.size();
  for (int32_t i = 0; i < n && i < cap; ++i) q[i] = r.qtrace[i];
  return n;
}
void orc_run_partition(const orc_run* h, int32_t level, int32_t* part) {
  // partitionAtLevel (LouvainCPP.cpp:82-106) as a composition of dense maps.
  const auto& L = h->st.levels;
  int32_t V = L[0].V;
  for (int32_t i = 0; i < V; ++i) {
    int32_t p = L[0].part[i];
    for (int32_t t = 1; t <= level && t < (int32_t)L.size(); ++t) p = L[t].part[p];
    part[i] = p;
  }
}
double orc_run_seconds(const orc_run* h) { return h->st.seconds; }
int64_t orc_run_pass_entries(const orc_run* h) { return h->st.pass_entries; }

double orc_modularity_fp64(int32_t V, int64_t E, const int32_t* src, const int32_t* dst, const float* w,
                           const int32_t* part) {
  // Newman modularity over the doubled list D = input ++ reversed(input):
  // Q = sum_c [ A_in(c) / 2W - (K_c / 2W)^2 ],  2W = sum of all D weights.
  int32_t C = 0;
  for (int32_t i = 0; i < V; ++i) C = std::max(C, part[i] + 1);
  std::vector<double> Kc(C, 0.0), Ain(C, 0.0);
  double twoW = 0.0;
  for (int64_t e = 0; e < E; ++e) {
    double x = (double)w[e];
    int32_t a = part[src[e]], b = part[dst[e]];
    Kc[a] += x; Kc[b] += x;      // the entry and its reversed copy
    twoW += 2.0 * x;
    if (a == b) Ain[a] += 2.0 * x;
  }
  if (twoW <= 0.0) return 0.0;
  double q = 0.0;
  for (int32_t c = 0; c < C; ++c) q += Ain[c] / twoW - (Kc[c] / twoW) * (Kc[c] / twoW);
  return q;
}

}  // extern "C"
