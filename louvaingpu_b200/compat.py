"""start(): the reference's Python entry point, over liblvg.

The reference exports one Python function from its Boost.Python module,
start(nodeList, edgeList, part_init) (LouvainCUDA/LouvainCPP.cpp:808-951).
This module keeps its arguments, result and side effects for callers that
switch to this library:

  nodeList   list of dicts with an "id" (any int; Graph.cpp:57-75 maps ids to
             indices in list order)
  edgeList   list of dicts with "source", "target" (node ids) and "weight"
             (Edge.h:40-56), passed on as given: the library appends the
             reversed copy of every entry, as the reference does
             (NeighbourCompute.cu:66-68)
  part_init  list of dicts with "node", "community", "weight"; the reference
             reads and renumbers them (LouvainCPP.cpp:828-849) but its
             generate_dendogram never uses them (:209-553), so they are
             checked the same way and not used

Returns {"size": number of communities, node id: community, ...} and writes
"cluster" and "my_community" into every node dict (LouvainCPP.cpp:897-915).
The partition is getPartitions(dendogram) (LouvainCPP.cpp:108-114), which
composes levels 0 and 1 only, whatever the dendrogram's depth; pass
reference_quirk=False for the partition of the last level.  The reference's
circle layout ("x", "y", LouvainCPP.cpp:555-651) is not computed.

Where the reference reads uninitialised memory or loops forever this
module raises instead: a node id listed twice, an edge naming an unknown id
(the reference's CUDPP lookup would return garbage), a missing key.
"""
import numpy as np

from .louvain import Louvain


def lists_to_arrays(nodeList, edgeList):
    """(ids, src, dst, w): node ids in list order and the edge list as dense
    indices into them (host-side replacement of the reference's CUDPP
    id -> index table, InitKernel.cu:159-191)."""
    ids = [int(nd["id"]) for nd in nodeList]
    index = {}
    for i, v in enumerate(ids):
        if v in index:
            raise ValueError(f"node id {v} is listed twice")
        index[v] = i
    E = len(edgeList)
    src = np.empty(E, np.int32)
    dst = np.empty(E, np.int32)
    w = np.empty(E, np.float32)
    for k, e in enumerate(edgeList):
        try:
            src[k] = index[int(e["source"])]
            dst[k] = index[int(e["target"])]
        except KeyError as err:
            if isinstance(err.args[0], str):
                raise
            raise ValueError(f"edge {k} names node id {err.args[0]}, which is not in nodeList") from None
        w[k] = float(e["weight"])
    return np.array(ids, np.int64), src, dst, w


def check_part_init(part_init):
    """The reference extracts node, community and weight of every entry and
    renumbers the communities (LouvainCPP.cpp:828-849); the result is not
    used by its level loop.  Returns the renumbered {node: (community, weight)}."""
    recomm, out = {}, {}
    for p in part_init:
        c = recomm.setdefault(int(p["community"]), len(recomm))
        out[int(p["node"])] = (c, float(p["weight"]))
    return out


def start(nodeList, edgeList, part_init=(), reference_quirk=True, device=0):
    ids, src, dst, w = lists_to_arrays(nodeList, edgeList)
    check_part_init(part_init)
    n = len(ids)
    with Louvain(device=device) as lv:
        lv.load_edges(src, dst, w, n)
        res = lv.run()
        if reference_quirk:
            level = 1 if res.n_levels > 1 else 0
        else:
            level = res.n_levels - 1
        part = lv.partition(level)
    size = int(part.max()) + 1 if n else 0        # countPartitions (LouvainCPP.cpp:116-127)
    out = {"size": size}
    for i, v in enumerate(ids.tolist()):
        out[v] = int(part[i])
    for i, nd in enumerate(nodeList):
        nd["cluster"] = int(part[i])
        nd["my_community"] = int(part[i])
    return out
