"""CPU tests of the oracle against hand-derived known answers and networkx.

The reference ships no test or golden vector and cannot be built here, so the
oracle is pinned by answers derived by hand from its kernels
(tests/golden/two_triangles.json) and by networkx's FP64 modularity.
"""
import json
import os

import numpy as np
import pytest

from conftest import undirected_to_lists

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def load_golden(name):
    with open(os.path.join(GOLDEN, name)) as f:
        return json.load(f)


def test_two_triangles_known_answer(oracle):
    g = load_golden("two_triangles.json")
    src, dst, w = undirected_to_lists(g["undirected_edges"])
    r = oracle.Run(g["n_vertices"], src, dst, w)
    assert r.status == 0
    assert len(r.levels) == len(g["levels"])
    for lv, exp in zip(r.levels, g["levels"]):
        assert lv.n_vertices == exp["n_vertices"]
        assert lv.n_entries == exp["n_entries"]
        assert lv.nnz == exp["nnz"]
        assert lv.n_comms == exp["n_comms"]
        assert lv.passes == exp["passes"]
        assert lv.q_start == pytest.approx(exp["q_start"], abs=1e-12)
        assert lv.q == pytest.approx(exp["q_level"], abs=1e-12)
        assert lv.labels.tolist() == exp["labels"]
        assert lv.part.tolist() == exp["part"]
    assert r.final.tolist() == g["final_partition"]
    q = oracle.modularity_fp64(g["n_vertices"], src, dst, w, r.final)
    assert q == pytest.approx(g["final_modularity_fp64"], abs=1e-12)


def test_two_triangles_coarse_level(oracle):
    g = load_golden("two_triangles.json")
    src, dst, w = undirected_to_lists(g["undirected_edges"])
    part = np.array(g["levels"][0]["part"], np.int32)
    s, d, ww = oracle.induce(6, src, dst, w, part)
    exp = g["level1_input"]
    assert s.tolist() == exp["src"] and d.tolist() == exp["dst"] and ww.tolist() == exp["w"]
    csr = oracle.Csr(3, s, d, ww)
    assert csr.k.tolist() == g["level1_degree"]
    assert csr.loopw.tolist() == g["level1_loop"]
    assert csr.has_loop.tolist() == [1, 0, 1]


def test_singleton_pair_rule_and_merge_candidate(oracle):
    # one edge 0-1 from singletons: 0's best (1) is a higher-id singleton -> 0 stays
    # but becomes the isolated-merge candidate; 1 moves to 0 (OneLevelKernel.cu:407-410, :159-169)
    src, dst, w = undirected_to_lists([(0, 1)])
    csr = oracle.Csr(2, src, dst, w)
    nxt, cand, nseg = csr.decide([0, 1], csr.k, [1, 1])
    assert nxt.tolist() == [0, 0]
    assert cand.tolist() == [1, -1]
    assert nseg.tolist() == [1, 1]


def test_tie_goes_to_lower_community(oracle):
    # vertex 0 joined to 1 and 2 with equal weights and degrees: equal gains -> community 1
    src, dst, w = undirected_to_lists([(0, 1), (0, 2), (1, 3), (2, 4)])
    csr = oracle.Csr(5, src, dst, w)
    nxt, cand, nseg = csr.decide(np.arange(5), csr.k, np.ones(5))
    assert nxt[0] == 0          # best is 1 > 0, both singletons -> stays
    comm = np.array([3, 1, 2, 3, 4], np.int32)   # 0 no longer a singleton's owner
    tot = np.zeros(5); size = np.zeros(5, np.int32)
    for i, c in enumerate(comm):
        tot[c] += csr.k[i]; size[c] += 1
    nxt, cand, nseg = csr.decide(comm, tot, size)
    assert nxt[0] == 1


def test_zero_weight_edges_and_self_loops(oracle):
    # weight 0 counts 1 in the degree (InitKernel.cu:165-167), a self loop twice
    src = np.array([0, 1, 1, 1, 2], np.int32)
    dst = np.array([1, 0, 1, 2, 1], np.int32)
    w = np.array([0, 0, 3, 2, 2], np.float32)
    csr = oracle.Csr(3, src, dst, w)
    # doubled list rows: 0:{(0,1,0)x2} 1:{(1,0,0)x2,(1,1,3)x2,(1,2,2)x2} 2:{(2,1,2)x2}
    assert csr.k.tolist() == [2.0, 2.0 + 12.0 + 4.0, 4.0]
    assert csr.loopw.tolist() == [0.0, 3.0, 0.0]
    assert csr.off.tolist() == [0, 1, 3, 4]
    assert csr.col.tolist() == [1, 0, 2, 1]
    assert csr.w.tolist() == [0.0, 0.0, 4.0, 4.0]
    assert csr.m == 7.0


def test_renumber_by_smallest_member(oracle):
    comm = np.array([5, 5, 2, 6, 2, 6, 5], np.int32)
    part, C = oracle.renumber(comm)
    assert C == 3
    assert part.tolist() == [0, 0, 1, 2, 1, 2, 0]


def test_induce_maps_zero_weight_to_one(oracle):
    src = np.array([0, 1, 2, 3], np.int32)
    dst = np.array([1, 0, 3, 2], np.int32)
    w = np.array([0, 0, 2.5, 2.5], np.float32)
    s, d, ww = oracle.induce(4, src, dst, w, np.array([0, 0, 1, 1], np.int32))
    assert list(zip(s.tolist(), d.tolist(), ww.tolist())) == [(0, 0, 2.0), (1, 1, 5.0)]


def test_tree_sum_matches_exact_sum_for_integers(oracle):
    x = np.arange(1, 100001, dtype=np.float64)
    assert oracle.tree_sum(x) == x.sum()
    assert oracle.tree_sum(np.array([])) == 0.0
    assert oracle.tree_sum(np.array([3.5])) == 3.5


def test_modularity_matches_networkx(oracle, gen):
    nx = pytest.importorskip("networkx")
    n, s, d, w, truth = gen.sbm(600, 6, 0.2, 0.01, 1, 4, seed=5, with_truth=True)
    G = nx.Graph()
    G.add_nodes_from(range(n))
    for a, b, x in zip(s, d, w):
        if a < b:
            G.add_edge(int(a), int(b), weight=float(x))
    comms = [set(np.nonzero(truth == c)[0].tolist()) for c in range(truth.max() + 1)]
    q_nx = nx.community.modularity(G, comms, weight="weight")
    q = oracle.modularity_fp64(n, s, d, w, truth)
    assert q == pytest.approx(q_nx, abs=1e-12)
    r = oracle.Run(n, s, d, w)
    comms = [set(np.nonzero(r.final == c)[0].tolist()) for c in range(r.final.max() + 1)]
    assert oracle.modularity_fp64(n, s, d, w, r.final) == pytest.approx(
        nx.community.modularity(G, comms, weight="weight"), abs=1e-12)


def test_ref32_and_fp64_agree_on_sbm(oracle, gen):
    # the reference's float/int arithmetic vs the FP64 method: final Q within 1e-3
    n, s, d, w = gen.sbm_10k(seed=0)
    a = oracle.Run(n, s, d, w, mode=oracle.FP64, level_min_gain=1e-6)
    b = oracle.Run(n, s, d, w, mode=oracle.REF32, level_min_gain=1e-6)
    qa = oracle.modularity_fp64(n, s, d, w, a.final)
    qb = oracle.modularity_fp64(n, s, d, w, b.final)
    assert abs(qa - qb) <= 1e-3


def test_empty_and_isolated(oracle):
    r = oracle.Run(4, np.zeros(0, np.int32), np.zeros(0, np.int32), np.zeros(0, np.float32))
    assert len(r.levels) == 1 and r.final.tolist() == [0, 1, 2, 3]
    # vertex 1 and 4 isolated: they stay singletons
    src, dst, w = undirected_to_lists([(0, 2), (2, 3), (0, 3)])
    r = oracle.Run(5, src, dst, w)
    f = r.final
    assert f[0] == f[2] == f[3]
    assert len({f[1], f[4], f[0]}) == 3


def test_sbm_golden_regression(oracle, gen):
    g = load_golden("sbm10k_seed0.json")
    n, s, d, w = gen.sbm_10k(seed=0)
    assert len(s) == g["n_entries"]
    r = oracle.Run(n, s, d, w, level_min_gain=1e-6)
    assert [lv.passes for lv in r.levels] == g["passes"]
    assert [lv.n_comms for lv in r.levels] == g["n_comms"]
    assert [lv.q for lv in r.levels] == g["q_level"]
    assert int(np.bincount(r.final).max()) == g["largest_community"]
    assert oracle.modularity_fp64(n, s, d, w, r.final) == g["final_modularity_fp64"]


def test_hand_graph_known_answers(oracle):
    """Two K4 joined by one edge: in pass 1 (m = 26) vertex 0's best gains
    tie between 1 and 2 (1 - 9/52), the tie goes to 1 and the singleton-pair
    rule keeps 0; 1, 2, 3 join 0; 4's best is 5 and it stays; 6, 7 join 5 and
    5 stays.  In pass 2 vertex 4 has W = 3 to {5,6,7} (gain 3 - 9*4/52 > 0)
    and W = 1 to {0..3} (gain 1 - 13*4/52 = 0), so it joins 5: two communities,
    the K4s.  Star: every leaf's only candidate is the centre (gain 1/2), the
    centre's tie over the leaves goes to leaf 1 and the singleton-pair rule
    keeps it, so all join community 0.  Ring of 8 K5: the cliques."""
    from conftest import hand_graph
    r = oracle.Run(*hand_graph("k4k4"))
    assert r.final.tolist() == [0, 0, 0, 0, 1, 1, 1, 1]
    assert r.levels[0].passes == 2
    r = oracle.Run(*hand_graph("star"))
    assert r.final.tolist() == [0] * 10
    r = oracle.Run(*hand_graph("ring_k5"))
    assert r.final.tolist() == [i // 5 for i in range(40)]
    r = oracle.Run(*hand_graph("path"))
    assert len(r.levels) >= 1 and r.final.max() < 12


def test_results_do_not_depend_on_thread_count(oracle):
    """The CSR build and the coarsening sort per thread; a shuffled list with
    repeated (src, dst) entries and fractional weights of wide range makes
    the summation order visible, so every output is compared bit for bit."""
    rng = np.random.default_rng(12)
    n, m = 3000, 150000
    s = rng.integers(0, n, m).astype(np.int32)
    d = rng.integers(0, n, m).astype(np.int32)
    w = (rng.random(m) * 3.7 + 1e-3).astype(np.float32)
    w[::7] *= 1e5
    runs = {}
    for th in (1, 3, 8):
        runs[th] = oracle.Run(n, s, d, w, n_threads=th)
    part = rng.integers(0, 400, n).astype(np.int32)
    ind = oracle.induce(n, s, d, w, part)
    for th in (3, 8):
        a, b = runs[1], runs[th]
        assert len(a.levels) == len(b.levels)
        for la, lb in zip(a.levels, b.levels):
            assert (la.nnz, la.n_comms, la.passes) == (lb.nnz, lb.n_comms, lb.passes)
            assert la.q.hex() == lb.q.hex() and la.q_start.hex() == lb.q_start.hex()
            np.testing.assert_array_equal(la.labels, lb.labels)
        np.testing.assert_array_equal(a.final, b.final)
    # `ind` ran on the thread count the last Run set (8); now one thread
    oracle.Run(n, s[:10], d[:10], w[:10], n_threads=1)
    ind8, ind1 = ind, oracle.induce(n, s, d, w, part)
    for x, y in zip(ind1, ind8):
        assert x.tobytes() == y.tobytes()


def _golden_sha(*arrays):
    import hashlib
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


@pytest.mark.parametrize("name,make", [("lfr_seed1.json", "lfr"), ("rmat16_seed2.json", "rmat16")])
def test_workload_golden_regression(oracle, gen, name, make):
    """The generators and the oracle reproduce the committed fixtures of the
    LFR n=2^20 and R-MAT 16 graphs bit for bit (make_workload_goldens.py)."""
    g = load_golden(name)
    n, s, d, w = gen.lfr() if make == "lfr" else gen.rmat(16)
    assert (n, len(s)) == (g["n_vertices"], g["n_entries"])
    assert _golden_sha(s, d, w) == g["input_sha256"]
    r = oracle.Run(n, s, d, w)
    assert len(r.levels) == len(g["levels"])
    for lv, x in zip(r.levels, g["levels"]):
        assert (lv.n_vertices, lv.nnz, lv.passes, lv.n_comms) == (x["n_vertices"], x["nnz"], x["passes"], x["n_comms"])
        assert lv.q_start.hex() == x["q_start"] and lv.q.hex() == x["q_level"]
    assert _golden_sha(r.final.astype(np.int32)) == g["final_partition_sha256"]
    assert oracle.modularity_fp64(n, s, d, w, r.final).hex() == g["final_modularity_fp64"]
