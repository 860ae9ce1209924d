// Drives liblvg through lvg_reference_api.h the way the reference's main()
// and generate_dendogram do (LouvainCPP.cpp:209-553, 739-806).
//   reference_driver <dir> run    -> whole dendrogram through generate_dendogram
//   reference_driver <dir> steps  -> the phase functions called one by one
//   reference_driver <dir> float  -> the same through the shim's float phase
//                                    functions, as a relinked reference driver
//                                    calls them (LouvainCPP.cpp:356-470)
// Reads <dir>/nodes.txt and <dir>/edges.txt; prints one line per level:
//   level <l> <count> then "node:community" pairs, and "communities <n>".
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "lvg_reference_api.h"

using namespace lvg_ref;

static void print_partition(int level, const Partition& p) {
  std::printf("level %d %d", level, p.count);
  for (int k = 0; k < p.count; ++k) std::printf(" %d:%d", p.partition.node[k], p.partition.community[k]);
  std::printf("\n");
}

int main(int argc, char** argv) {
  if (argc < 3) return 2;
  std::string dir = argv[1];
  std::vector<int> nodes = loadNodes(dir + "/nodes.txt");
  std::vector<Edge> edges = loadEdges(dir + "/edges.txt");
  Graph graph;
  graph.setNodes(nodes.data(), (int)nodes.size());
  graph.setEdges(edges.data(), (int)edges.size());
  std::vector<Partition> dendogram;
  if (std::strcmp(argv[2], "run") == 0) {
    std::map<int, std::pair<int, float>> init;
    dendogram = generate_dendogram(graph, init);
  } else if (std::strcmp(argv[2], "float") == 0) {
    // modularity values as floats end to end: the floor handed to each
    // one-level phase and the level break are the float ones
    StatusCUDA status;
    CUDAGraph cuGraph;
    CUDPPHandle handle = nullptr;
    AllocateMemory(status, graph, cuGraph);
    handle = status.ctx;
    CalculateNeighbour(status, cuGraph);
    initCUDA(status, cuGraph);
    float mod = modularityCUDA(status, graph.getNodeSize());
    float next = oneLevelCUDA(status, cuGraph.nodesSize, cuGraph.nrOfAllNeighbours, cuGraph.edgeSize * 2, mod);
    Partition first = renumberCUDA(handle, status);
    dendogram.push_back(first);
    mod = next;
    inducedGraphCUDA(handle, status, cuGraph, first);
    for (;;) {
      CalculateNeighbour(status, cuGraph);
      initCUDA(status, cuGraph);
      next = oneLevelCUDA(status, cuGraph.nodesSize, cuGraph.nrOfAllNeighbours, cuGraph.edgeSize * 2, mod);
      Partition p = renumberCUDA(handle, status);
      dendogram.push_back(p);
      if (next - mod < 1e-7f) break;
      mod = next;
      inducedGraphCUDA(handle, status, cuGraph, p);
    }
    DeAllocateMemory(status);
  } else {
    // LouvainCPP.cpp:334-507 with the reference's call sequence
    StatusCUDA status;
    CUDAGraph cuGraph;
    CUDPPHandle handle = nullptr;
    AllocateMemory(status, graph, cuGraph);
    handle = status.ctx;
    CalculateNeighbour(status, cuGraph);
    initCUDA(status, cuGraph);
    // modularityCUDA / oneLevelCUDA return float like the reference; the
    // FP64 values are taken from the C ABI so that this sequence reproduces
    // lvg_run bit for bit.
    float mod32 = modularityCUDA(status, graph.getNodeSize());
    double mod = 0.0;
    check(status.ctx, lvg_modularity(status.ctx, &mod));
    if ((double)mod32 != (double)(float)mod) return 3;
    double q = 0.0;
    int32_t passes = 0;
    check(status.ctx, lvg_one_level(status.ctx, mod, &q, &passes));
    Partition p2 = renumberCUDA(handle, status);
    dendogram.push_back(p2);
    mod = q;
    inducedGraphCUDA(handle, status, cuGraph, p2);
    for (;;) {
      CalculateNeighbour(status, cuGraph);
      initCUDA(status, cuGraph);
      check(status.ctx, lvg_one_level(status.ctx, mod, &q, &passes));
      Partition p = renumberCUDA(handle, status);
      dendogram.push_back(p);
      if (q - mod < 1e-7) break;           // LouvainCPP.cpp:466 in FP64
      mod = q;
      inducedGraphCUDA(handle, status, cuGraph, p);
    }
    DeAllocateMemory(status);
  }
  for (size_t l = 0; l < dendogram.size(); ++l) print_partition((int)l, dendogram[l]);
  Partition last = partitionAtLevel(dendogram, (int)dendogram.size() - 1);
  std::printf("communities %d\n", countPartitions(last));
  Partition quirk = getPartitions(dendogram);
  std::printf("getPartitions_level1_communities %d\n", countPartitions(quirk));
  for (auto& p : dendogram) p.Deallocate();
  last.Deallocate();
  quirk.Deallocate();
  return 0;
}
