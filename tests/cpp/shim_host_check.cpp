// Host-only checks of the reference-API shim (no device call): dendrogram
// composition, the getPartitions level quirk, countPartitions and the text
// loaders, against answers worked out by hand from the reference's
// partitionAtLevel / getPartitions / countPartitions (LouvainCPP.cpp:82-127)
// and loaders (LouvainCPP.cpp:660-737).  Usage: shim_host_check <scratch dir>.
#include <cstdio>
#include <fstream>
#include <string>
#include <vector>

#include "lvg_reference_api.h"

using lvg_ref::Partition;

static int failures = 0;

static void expect(bool ok, const char* what) {
  if (!ok) {
    std::printf("FAIL %s\n", what);
    ++failures;
  }
}

static Partition make(const std::vector<int>& node, const std::vector<int>& comm) {
  Partition p;
  p.count = (int)node.size();
  p.partition.node = new int[p.count];
  p.partition.community = new int[p.count];
  for (int i = 0; i < p.count; ++i) {
    p.partition.node[i] = node[i];
    p.partition.community[i] = comm[i];
  }
  return p;
}

static std::vector<int> comms(Partition p) {
  std::vector<int> c(p.partition.community, p.partition.community + p.count);
  p.Deallocate();
  return c;
}

int main(int argc, char** argv) {
  if (argc < 2) return 2;
  // level 0: original node ids -> level-0 communities; later levels list their
  // (node, community) pairs in any order
  std::vector<Partition> d;
  d.push_back(make({10, 11, 12, 13, 14}, {0, 1, 0, 2, 1}));
  d.push_back(make({2, 0, 1}, {0, 0, 1}));
  d.push_back(make({1, 0}, {0, 0}));
  expect(comms(lvg_ref::partitionAtLevel(d, 0)) == std::vector<int>({0, 1, 0, 2, 1}), "partitionAtLevel 0");
  expect(comms(lvg_ref::partitionAtLevel(d, 1)) == std::vector<int>({0, 1, 0, 0, 1}), "partitionAtLevel 1");
  expect(comms(lvg_ref::partitionAtLevel(d, 2)) == std::vector<int>({0, 0, 0, 0, 0}), "partitionAtLevel 2");
  // `level || size - 1` is a bool: level 1 whenever there are two or more levels
  expect(comms(lvg_ref::getPartitions(d)) == std::vector<int>({0, 1, 0, 0, 1}), "getPartitions default");
  expect(comms(lvg_ref::getPartitions(d, 2)) == std::vector<int>({0, 1, 0, 0, 1}), "getPartitions 2 (quirk)");
  expect(comms(lvg_ref::getPartitions(d, 2, false)) == std::vector<int>({0, 0, 0, 0, 0}), "getPartitions 2");
  expect(comms(lvg_ref::getPartitions(d, -1, false)) == std::vector<int>({0, 0, 0, 0, 0}), "getPartitions last");
  bool threw = false;
  try { comms(lvg_ref::getPartitions(d, 3)); } catch (const lvg_ref::Error&) { threw = true; }
  expect(threw, "getPartitions rejects level 3");
  threw = false;
  try { comms(lvg_ref::getPartitions(d, -1)); } catch (const lvg_ref::Error&) { threw = true; }
  expect(threw, "getPartitions rejects level -1 (reference check)");
  // one level only: `0 || 0` is level 0
  std::vector<Partition> one;
  one.push_back(make({7, 8}, {1, 0}));
  expect(comms(lvg_ref::getPartitions(one)) == std::vector<int>({1, 0}), "getPartitions single level");
  // a community missing from the next level composes to -1 (newCom = -1)
  std::vector<Partition> gap;
  gap.push_back(make({0, 1, 2}, {0, 1, 2}));
  gap.push_back(make({0, 2}, {5, 6}));
  expect(comms(lvg_ref::partitionAtLevel(gap, 1)) == std::vector<int>({5, -1, 6}), "missing node -> -1");
  // countPartitions: 1 + max, with the maximum starting at 0
  Partition p = make({0, 1, 2, 3}, {0, 3, 1, 3});
  expect(lvg_ref::countPartitions(p) == 4, "countPartitions");
  p.Deallocate();
  p = make({0, 1}, {-1, -1});
  expect(lvg_ref::countPartitions(p) == 1, "countPartitions of -1s");
  p.Deallocate();
  for (auto& x : d) x.Deallocate();
  for (auto& x : one) x.Deallocate();
  for (auto& x : gap) x.Deallocate();
  // loaders: "count v v v" and "count s t w s t w"
  const std::string dir = argv[1];
  { std::ofstream f(dir + "/nodes.txt"); f << "4\n1000 -3\n77 5\n"; }
  { std::ofstream f(dir + "/edges.txt"); f << "3\n1000 -3 1.5\n77 5 2\n5 1000 0.25\n"; }
  std::vector<int> nodes = lvg_ref::loadNodes(dir + "/nodes.txt");
  expect(nodes == std::vector<int>({1000, -3, 77, 5}), "loadNodes");
  std::vector<lvg_ref::Edge> e = lvg_ref::loadEdges(dir + "/edges.txt");
  expect(e.size() == 3 && e[0].source == 1000 && e[0].target == -3 && e[0].weight == 1.5f && e[1].source == 77 &&
             e[1].target == 5 && e[1].weight == 2.0f && e[2].source == 5 && e[2].target == 1000 &&
             e[2].weight == 0.25f,
         "loadEdges");
  threw = false;
  try { lvg_ref::loadNodes(dir + "/absent.txt"); } catch (const lvg_ref::Error&) { threw = true; }
  expect(threw, "loadNodes on a missing file");
  // truncated and corrupt files are errors, not short or garbage lists
  // (the reference reads them with atoi/atof and writes past its arrays)
  const char* bad_nodes[] = {"", "4\n1000 -3\n77\n", "3\n1 2 3 4\n", "x\n1 2\n", "-2\n", "2\n1 2x\n",
                             "2\n1 99999999999\n"};
  for (const char* text : bad_nodes) {
    { std::ofstream f(dir + "/bad_nodes.txt"); f << text; }
    threw = false;
    try { lvg_ref::loadNodes(dir + "/bad_nodes.txt"); } catch (const lvg_ref::Error&) { threw = true; }
    expect(threw, (std::string("loadNodes rejects: ") + text).c_str());
  }
  const char* bad_edges[] = {"2\n1 2 1.0\n", "2\n1 2 1.0\n3 4\n", "1\n1 2 1.0 5\n", "1\n1 2 heavy\n",
                             "1\n1 two 1.0\n", "1\n1.5 2 1.0\n", "1 1 2\n"};
  for (const char* text : bad_edges) {
    { std::ofstream f(dir + "/bad_edges.txt"); f << text; }
    threw = false;
    try { lvg_ref::loadEdges(dir + "/bad_edges.txt"); } catch (const lvg_ref::Error&) { threw = true; }
    expect(threw, (std::string("loadEdges rejects: ") + text).c_str());
  }
  { std::ofstream f(dir + "/empty_edges.txt"); f << "0\n"; }
  expect(lvg_ref::loadEdges(dir + "/empty_edges.txt").empty(), "loadEdges of count 0");
  std::printf(failures ? "%d FAILED\n" : "ok\n", failures);
  return failures ? 1 : 0;
}
