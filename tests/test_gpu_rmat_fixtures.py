"""GPU parity at the R-MAT scales where hub degrees reach 10^5..10^6: the
CUDA path against the oracle's committed fixtures (written on the CPU by
tests/golden/make_workload_goldens.py).

  rmat22_seed2.json         -- the whole dendrogram of the R-MAT scale-22
                               graph, plus its level-0 CSR and the decisions
                               of a pass from the singleton state and of the
                               pass after it;
  rmat25_seed2_level0.json  -- level 0 of the R-MAT scale-25 graph (1.07e9
                               entries): CSR, both pass decision vectors, the
                               one-level phase, the renumbered partition and
                               the coarse level-1 list and CSR.

The graphs are generated on the device (equal to the host generator the
fixtures were made from; the input fingerprint checks it).  Integer weights
make every sum exact, so everything is compared bit for bit.
"""
import hashlib
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def sha(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def csr_sha(c):
    return sha(c["off"], c["col"], c["w"], c["k"], c["loopw"], c["has_loop"])


@pytest.fixture(scope="module")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for gpu tests")
    return torch


def device_graph(scale):
    from louvaingpu_b200 import graphgen
    return graphgen.rmat_device(scale)


def check_pass_decisions(lv, V, g):
    """Hashing kernels from the singleton state and from the state after it:
    the same decision vectors as the oracle's."""
    lv.set_communities(np.arange(V, dtype=np.int32))
    first, _ = lv.move_decide()
    assert sha(first) == g["pass1_decisions_sha256"]
    lv.set_communities(first)
    second, _ = lv.move_decide()
    assert sha(second) == g["pass2_decisions_sha256"]


def test_rmat22_dendrogram_fixture(cuda):
    from louvaingpu_b200 import Louvain
    with open(os.path.join(GOLDEN, "rmat22_seed2.json")) as f:
        g = json.load(f)
    dg = device_graph(22)
    try:
        assert (dg.n_vertices, dg.n_entries) == (g["n_vertices"], g["n_entries"])
        assert sha(*dg.to_host()) == g["input_sha256"]
        with Louvain() as lv:
            lv.load_edges_device(dg.src, dg.dst, dg.w, dg.n_entries, dg.n_vertices)
            assert csr_sha(lv.csr()) == g["csr_sha256"]
            check_pass_decisions(lv, dg.n_vertices, g)
            res = lv.run()
            assert res.n_levels == len(g["levels"])
            for l, x in enumerate(g["levels"]):
                li = lv.level_info(l)
                assert (li.n_vertices, li.nnz, li.passes, li.n_comms) == \
                       (x["n_vertices"], x["nnz"], x["passes"], x["n_comms"]), f"level {l}"
                assert li.q_start.hex() == x["q_start"] and li.q_level.hex() == x["q_level"], f"level {l}"
            assert sha(np.ascontiguousarray(lv.partition(), np.int32)) == g["final_partition_sha256"]
            assert res.q_final == pytest.approx(float.fromhex(g["final_modularity_fp64"]), abs=1e-9)
    finally:
        dg.close()


def test_rmat25_level0_fixture(cuda):
    from louvaingpu_b200 import Louvain
    with open(os.path.join(GOLDEN, "rmat25_seed2_level0.json")) as f:
        g = json.load(f)
    dg = device_graph(25)
    try:
        V = dg.n_vertices
        assert (V, dg.n_entries) == (g["n_vertices"], g["n_entries"])
        assert sha(*dg.to_host()) == g["input_sha256"]
        with Louvain() as lv:
            lv.load_edges_device(dg.src, dg.dst, dg.w, dg.n_entries, V)
            c = lv.csr()
            assert (c["nnz"], c["m"].hex()) == (g["nnz"], g["m"])
            assert csr_sha(c) == g["csr_sha256"]
            del c
            check_pass_decisions(lv, V, g)
            lv.set_communities(np.arange(V, dtype=np.int32))   # the level's initial state
            q0 = lv.modularity()
            q, passes = lv.one_level(q0)
            assert (passes, q0.hex(), q.hex()) == (g["passes"], g["q_start"], g["q_level"])
            part, C = lv.renumber()
            assert C == g["n_comms"]
            assert sha(part) == g["partition_sha256"]
            assert sha(lv.level_labels(0)) == g["labels_sha256"]
            lv.induce()
            cs, cd, cw = lv.level_edges()
            assert len(cs) == g["coarse_entries"]
            assert sha(cs, cd, cw) == g["coarse_list_sha256"]
            c = lv.csr()
            assert c["nnz"] == g["coarse_nnz"]
            assert csr_sha(c) == g["coarse_csr_sha256"]
    finally:
        dg.close()
