/*
 * lvg_reference_api.h -- the reference's C++ host API over liblvg.
 *
 * Header-only.  Keeps the names, argument order and meaning of the phase API
 * the reference's level driver links against (LouvainCUDA/LouvainCPP.cpp:129-134)
 * and of its host types (Graph.h, CUDAGraph.h, StatusCUDA.h, partition.h,
 * community.h, Edge.h), so a driver written against the reference relinks
 * against liblvg.so.  Differences a caller sees:
 *   - the CUDPPHandle parameter is the liblvg context (no CUDPP);
 *   - StatusCUDA carries the context instead of raw device slabs;
 *   - errors throw lvg_ref::Error (the reference checked nothing).
 * Node ids of the level-0 Graph may be arbitrary ints; they are mapped to
 * dense indices on load, as the reference's id->index hash did
 * (InitKernel.cu:276-306).
 */
#ifndef LVG_REFERENCE_API_H
#define LVG_REFERENCE_API_H

#include <algorithm>
#include <cerrno>
#include <cstdint>
#include <cstdlib>
#include <fstream>
#include <map>
#include <numeric>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <utility>
#include <vector>

#include "lvg.h"

namespace lvg_ref {

struct Error : std::runtime_error {
  lvg_status status;
  Error(lvg_status s, const std::string& m) : std::runtime_error(m), status(s) {}
};

inline void check(lvg_ctx* ctx, lvg_status s) {
  if (s != LVG_OK) throw Error(s, std::string(lvg_status_string(s)) + ": " + (ctx ? lvg_last_error(ctx) : ""));
}

/* Edge.h:65-69 */
struct Edge {
  int target, source;
  float weight;
};

/* Edge.h:26-63 (SoA edge list) */
struct EdgeContainer {
  std::vector<int> source, target;
  std::vector<float> weight;
  int count = 0;
};

/* community.h:16-20 */
struct Community {
  int* node = nullptr;
  int* community = nullptr;
};

/* partition.h:14-29: (node, community) pairs owned by the caller */
struct Partition {
  int count = 0;
  Community partition;
  void Deallocate() {
    delete[] partition.node;
    delete[] partition.community;
    partition.node = partition.community = nullptr;
  }
};

/* Graph.h:39-130 (the parts the level driver uses) */
class Graph {
 public:
  int setNodes(const int* nodes, int size) {               /* Graph.cpp:122-137 */
    nodes_.assign(nodes, nodes + size);
    index_.clear();
    for (int i = 0; i < size; ++i) index_[nodes_[i]] = i;
    return 0;
  }
  int setEdges(const Edge* edges, int size) {              /* Graph.cpp:139-160 */
    edges_.source.resize(size);
    edges_.target.resize(size);
    edges_.weight.resize(size);
    for (int i = 0; i < size; ++i) {
      edges_.source[i] = edges[i].source;
      edges_.target[i] = edges[i].target;
      edges_.weight[i] = edges[i].weight;
    }
    edges_.count = size;
    return 0;
  }
  int* getNodes() { return nodes_.data(); }
  int getNodeAt(int i) const { return nodes_[i]; }
  int getNodeSize() const { return (int)nodes_.size(); }
  int getEdgeSize() const { return edges_.count; }
  EdgeContainer& getEdgeContainer() { return edges_; }
  int getIdxOfNode(int id) const {
    auto it = index_.find(id);
    if (it == index_.end()) throw Error(LVG_ERR_INVALID_ARG, "edge names a node missing from the node list");
    return it->second;
  }

 private:
  std::vector<int> nodes_;
  EdgeContainer edges_;
  std::unordered_map<int, int> index_;
};

/* CUDAGraph.h:14-28: sizes of the current level (the arrays live in the context) */
struct CUDAGraph {
  int nodesSize = 0, edgeSize = 0;
  int nrOfAllNeighbours = 0;
};

/* StatusCUDA.h:19-87: the device state of a run is the liblvg context */
struct StatusCUDA {
  lvg_ctx* ctx = nullptr;
  float totalWeight = 0.0f;
  int keys = 0;
  std::vector<int> level_nodes;   /* node ids of the current level's vertices */
};

typedef lvg_ctx* CUDPPHandle;

/* AllocateMemory (LouvainCPP.cpp:136-198): context + device arena, loads the graph. */
inline void AllocateMemory(StatusCUDA& status, Graph& graph, CUDAGraph& cuGraph, const lvg_config* cfg = nullptr) {
  if (!status.ctx) check(nullptr, lvg_create(cfg, &status.ctx));
  EdgeContainer& e = graph.getEdgeContainer();
  std::vector<int32_t> s(e.count), d(e.count);
  for (int i = 0; i < e.count; ++i) {
    s[i] = graph.getIdxOfNode(e.source[i]);
    d[i] = graph.getIdxOfNode(e.target[i]);
  }
  check(status.ctx, lvg_load_edges(status.ctx, s.data(), d.data(), e.weight.data(), e.count, graph.getNodeSize()));
  status.keys = graph.getNodeSize();
  status.level_nodes.assign(graph.getNodes(), graph.getNodes() + graph.getNodeSize());
  cuGraph.nodesSize = graph.getNodeSize();
  cuGraph.edgeSize = e.count;
  cuGraph.nrOfAllNeighbours = 2 * e.count;
}

/* DeAllocateMemory (LouvainCPP.cpp:200-205) */
inline void DeAllocateMemory(StatusCUDA& status) {
  if (status.ctx) lvg_destroy(status.ctx);
  status.ctx = nullptr;
}

/* CalculateNeighbour (NeighbourCompute.cu:42-117) and initCUDA (InitKernel.cu:128-221):
 * the CSR, degrees and loops of a level are built when its edge list arrives
 * (AllocateMemory for level 0, inducedGraphCUDA for the next ones); these
 * report its total weight and sizes. */
inline void CalculateNeighbour(StatusCUDA& status, CUDAGraph& cuGraph) {
  int32_t V = 0;
  int64_t nnz = 0;
  double m = 0.0;
  check(status.ctx, lvg_get_csr(status.ctx, &V, &nnz, &m, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr));
  status.totalWeight = (float)m;
  cuGraph.nrOfAllNeighbours = 2 * cuGraph.edgeSize;
}
inline void initCUDA(StatusCUDA& status, CUDAGraph& cuGraph) { status.keys = cuGraph.nodesSize; }

/* modularityCUDA (OneLevelKernel.cu:965-980) */
inline float modularityCUDA(StatusCUDA& status, int /*nodeCount*/) {
  double q = 0.0;
  check(status.ctx, lvg_modularity(status.ctx, &q));
  return (float)q;
}

/* oneLevelCUDA (OneLevelKernel.cu:518-954) */
inline float oneLevelCUDA(StatusCUDA& status, int /*nodeCount*/, int /*neighboursCount*/,
                          int /*neighbourComputeCount*/, float& lower) {
  double q = 0.0;
  int32_t passes = 0;
  check(status.ctx, lvg_one_level(status.ctx, (double)lower, &q, &passes));
  return (float)q;
}

/* renumberCUDA (RenumberKernel.cu:63-221): (node id, new community) pairs in
 * the reference's order -- grouped by the community label before renumbering,
 * ascending vertex index inside a group. */
inline Partition renumberCUDA(CUDPPHandle& /*handle*/, StatusCUDA& status) {
  const int V = status.keys;
  std::vector<int32_t> part(V), labels(V);
  int32_t C = 0, level = 0;
  check(status.ctx, lvg_renumber(status.ctx, part.data(), &C));
  check(status.ctx, lvg_num_levels(status.ctx, &level));
  check(status.ctx, lvg_get_level_labels(status.ctx, level - 1, labels.data()));
  std::vector<int> order(V);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return labels[a] < labels[b]; });
  Partition p;
  p.count = V;
  p.partition.node = new int[V];
  p.partition.community = new int[V];
  for (int k = 0; k < V; ++k) {
    p.partition.node[k] = status.level_nodes[order[k]];
    p.partition.community[k] = part[order[k]];
  }
  return p;
}

/* inducedGraphCUDA (InducedGraphKernel.cu:50-113) */
inline void inducedGraphCUDA(CUDPPHandle& /*handle*/, StatusCUDA& status, CUDAGraph& cuGraph,
                             Partition& /*partition*/) {
  check(status.ctx, lvg_induce(status.ctx));
  int32_t V = 0;
  int64_t nnz = 0;
  double m = 0.0;
  check(status.ctx, lvg_get_csr(status.ctx, &V, &nnz, &m, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr));
  int32_t L = 0;
  lvg_level_info info;
  check(status.ctx, lvg_num_levels(status.ctx, &L));
  check(status.ctx, lvg_get_level_info(status.ctx, L - 1, &info));
  cuGraph.nodesSize = V;
  status.keys = V;
  status.level_nodes.resize(V);
  std::iota(status.level_nodes.begin(), status.level_nodes.end(), 0);   /* InducedGraphKernel.cu:57-60 */
  (void)info;
}

/* generate_dendogram (LouvainCPP.cpp:209-553): one Partition per level. */
inline std::vector<Partition> generate_dendogram(Graph& graph, std::map<int, std::pair<int, float>>& /*part_init*/,
                                                 const lvg_config* cfg = nullptr) {
  StatusCUDA status;
  CUDAGraph cuGraph;
  std::vector<Partition> out;
  AllocateMemory(status, graph, cuGraph, cfg);
  try {
    lvg_result res;
    check(status.ctx, lvg_run(status.ctx, &res));
    for (int l = 0; l < res.n_levels; ++l) {
      lvg_level_info info;
      check(status.ctx, lvg_get_level_info(status.ctx, l, &info));
      const int V = info.n_vertices;
      std::vector<int32_t> part(V), labels(V);
      check(status.ctx, lvg_get_level_partition(status.ctx, l, part.data()));
      check(status.ctx, lvg_get_level_labels(status.ctx, l, labels.data()));
      std::vector<int> order(V);
      std::iota(order.begin(), order.end(), 0);
      std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return labels[a] < labels[b]; });
      Partition p;
      p.count = V;
      p.partition.node = new int[V];
      p.partition.community = new int[V];
      for (int k = 0; k < V; ++k) {
        p.partition.node[k] = l == 0 ? graph.getNodeAt(order[k]) : order[k];
        p.partition.community[k] = part[order[k]];
      }
      out.push_back(p);
    }
  } catch (...) {
    DeAllocateMemory(status);
    throw;
  }
  DeAllocateMemory(status);
  return out;
}

/* partitionAtLevel (LouvainCPP.cpp:82-106): compose levels 0..level.  The
 * returned Partition owns fresh arrays (the reference aliased level 0's). */
inline Partition partitionAtLevel(std::vector<Partition>& dendogram, int level) {
  const Partition& p0 = dendogram[0];
  Partition out;
  out.count = p0.count;
  out.partition.node = new int[p0.count];
  out.partition.community = new int[p0.count];
  std::copy(p0.partition.node, p0.partition.node + p0.count, out.partition.node);
  std::copy(p0.partition.community, p0.partition.community + p0.count, out.partition.community);
  for (int i = 1; i <= level && i < (int)dendogram.size(); ++i) {
    std::unordered_map<int, int> m;
    for (int k = 0; k < dendogram[i].count; ++k) m[dendogram[i].partition.node[k]] = dendogram[i].partition.community[k];
    for (int j = 0; j < out.count; ++j) {
      auto it = m.find(out.partition.community[j]);
      out.partition.community[j] = it == m.end() ? -1 : it->second;
    }
  }
  return out;
}

/* getPartitions (LouvainCPP.cpp:108-114).  The reference rejects a level
 * outside [0, size-1], then evaluates `level || dendogram.size() - 1`, a
 * bool, so it always returns level 1 when there are two or more levels;
 * reference_quirk = true keeps both behaviours, false returns the requested
 * level (the last level for level < 0). */
inline Partition getPartitions(std::vector<Partition>& dendogram, int level = 0, bool reference_quirk = true) {
  if (level >= (int)dendogram.size() || (reference_quirk && level < 0))
    throw Error(LVG_ERR_INVALID_ARG, "Invalid argument: level is not between 1 and len(dendogram) - 1 included.");
  if (reference_quirk) return partitionAtLevel(dendogram, (level != 0 || dendogram.size() - 1 != 0) ? 1 : 0);
  return partitionAtLevel(dendogram, level < 0 ? (int)dendogram.size() - 1 : level);
}

/* countPartitions (LouvainCPP.cpp:116-127) */
inline int countPartitions(const Partition& p) {
  int mx = 0;
  for (int i = 0; i < p.count; ++i) mx = std::max(mx, p.partition.community[i]);
  return 1 + mx;
}

/* Whitespace-separated tokens of a text file after its leading count.  The
 * reference parses them with atoi/atof (a corrupt token becomes 0) and writes
 * past its count-sized array when the file holds more values than the count
 * (LouvainCPP.cpp:660-737); here a token that is not entirely a number, a
 * count that is not a non-negative integer, or a value count that differs
 * from `count * per_record` throws Error. */
namespace detail {
inline std::vector<std::string> counted_tokens(const std::string& path, size_t per_record, long long& count) {
  std::ifstream f(path);
  if (!f) throw Error(LVG_ERR_INVALID_ARG, "cannot open " + path);
  std::string tok;
  if (!(f >> tok)) throw Error(LVG_ERR_INVALID_ARG, path + ": empty file (no count)");
  char* end = nullptr;
  errno = 0;
  count = std::strtoll(tok.c_str(), &end, 10);
  if (errno || *end != '\0' || count < 0) throw Error(LVG_ERR_INVALID_ARG, path + ": bad count '" + tok + "'");
  std::vector<std::string> out;
  out.reserve((size_t)count * per_record);
  while (f >> tok) {
    if (out.size() == (size_t)count * per_record)
      throw Error(LVG_ERR_INVALID_ARG, path + ": more values than the count " + std::to_string(count) + " gives");
    out.push_back(tok);
  }
  if (out.size() != (size_t)count * per_record)
    throw Error(LVG_ERR_INVALID_ARG, path + ": truncated: " + std::to_string(out.size()) + " values, " +
                                         std::to_string((size_t)count * per_record) + " expected");
  return out;
}
inline int to_int(const std::string& path, const std::string& t) {
  char* end = nullptr;
  errno = 0;
  long v = std::strtol(t.c_str(), &end, 10);
  if (errno || *end != '\0' || t.empty() || v < INT32_MIN || v > INT32_MAX)
    throw Error(LVG_ERR_INVALID_ARG, path + ": not an integer id: '" + t + "'");
  return (int)v;
}
inline float to_float(const std::string& path, const std::string& t) {
  char* end = nullptr;
  errno = 0;
  float v = std::strtof(t.c_str(), &end);
  if (errno || *end != '\0' || t.empty()) throw Error(LVG_ERR_INVALID_ARG, path + ": not a weight: '" + t + "'");
  return v;
}
}  // namespace detail

/* loadNodes (LouvainCPP.cpp:660-701): "count id id id ...". */
inline std::vector<int> loadNodes(const std::string& path = "nodes.txt") {
  long long count = 0;
  std::vector<std::string> tok = detail::counted_tokens(path, 1, count);
  std::vector<int> ids(tok.size());
  for (size_t i = 0; i < tok.size(); ++i) ids[i] = detail::to_int(path, tok[i]);
  return ids;
}

/* loadEdges (LouvainCPP.cpp:703-737): "count src tgt w src tgt w ...". */
inline std::vector<Edge> loadEdges(const std::string& path = "edges.txt") {
  long long count = 0;
  std::vector<std::string> tok = detail::counted_tokens(path, 3, count);
  std::vector<Edge> edges((size_t)count);
  for (size_t i = 0; i < edges.size(); ++i) {
    edges[i].source = detail::to_int(path, tok[3 * i]);
    edges[i].target = detail::to_int(path, tok[3 * i + 1]);
    edges[i].weight = detail::to_float(path, tok[3 * i + 2]);
  }
  return edges;
}

}  // namespace lvg_ref

#endif
