"""GPU parity: every phase of the CUDA path against the CPU oracle.

Integer-valued weights make every sum exact, so the CUDA path must agree with
the oracle bit for bit: CSR, degrees, loop weights, single-pass decisions,
renumbered partitions, coarse graphs, pass counts and the FP64 Q values.
"""
import json
import os

import numpy as np
import pytest

from conftest import undirected_to_lists

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def Louvain():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for gpu tests")
    from louvaingpu_b200 import Louvain as L
    return L


def csr_equal(lv, oc):
    c = lv.csr()
    assert c["V"] == oc.V
    assert c["nnz"] == oc.nnz
    assert c["m"] == oc.m
    np.testing.assert_array_equal(c["off"], oc.off)
    np.testing.assert_array_equal(c["col"], oc.col)
    np.testing.assert_array_equal(c["w"], oc.w)
    np.testing.assert_array_equal(c["k"], oc.k)
    np.testing.assert_array_equal(c["loopw"], oc.loopw)
    np.testing.assert_array_equal(c["has_loop"], oc.has_loop)


def run_equal(lv, res, orun, n, src, dst, w, oracle):
    assert res.n_levels == len(orun.levels)
    for l, ol in enumerate(orun.levels):
        li = lv.level_info(l)
        assert (li.n_vertices, li.n_entries, li.nnz, li.n_comms, li.passes) == \
               (ol.n_vertices, ol.n_entries, ol.nnz, ol.n_comms, ol.passes), f"level {l}"
        assert li.q_start == ol.q_start, f"level {l}"
        assert li.q_level == ol.q, f"level {l}"
        np.testing.assert_array_equal(lv.level_labels(l), ol.labels)
        np.testing.assert_array_equal(lv.level_partition(l), ol.part)
    np.testing.assert_array_equal(lv.partition(), orun.final)
    q = oracle.modularity_fp64(n, src, dst, w, orun.final)
    assert res.q_final == pytest.approx(q, abs=1e-9)


def test_two_triangles_known_answer(Louvain, oracle):
    with open(os.path.join(GOLDEN, "two_triangles.json")) as f:
        g = json.load(f)
    src, dst, w = undirected_to_lists(g["undirected_edges"])
    with Louvain() as lv:
        lv.load_edges(src, dst, w, g["n_vertices"])
        res = lv.run()
        assert res.n_levels == 2
        for l, exp in enumerate(g["levels"]):
            li = lv.level_info(l)
            assert li.passes == exp["passes"] and li.n_comms == exp["n_comms"] and li.nnz == exp["nnz"]
            assert li.q_level == pytest.approx(exp["q_level"], abs=1e-12)
            assert lv.level_labels(l).tolist() == exp["labels"]
            assert lv.level_partition(l).tolist() == exp["part"]
        assert lv.partition().tolist() == g["final_partition"]
        assert res.q_final == pytest.approx(g["final_modularity_fp64"], abs=1e-12)


@pytest.mark.parametrize("case", ["sbm_small", "weighted", "loops_zeros_isolated", "odd_sizes", "hub"])
def test_csr_build_bit_exact(Louvain, oracle, gen, case):
    n, s, d, w = make_case(gen, case)
    oc = oracle.Csr(n, s, d, w)
    with Louvain() as lv:
        lv.load_edges(s, d, w, n)
        csr_equal(lv, oc)


def make_case(gen, case):
    rng = np.random.default_rng(7)
    if case == "sbm_small":
        return gen.sbm(2000, 20, 0.05, 0.002, 1, 1, seed=1)
    if case == "weighted":
        return gen.sbm(3000, 30, 0.05, 0.002, 1, 4, seed=2)
    if case == "loops_zeros_isolated":
        n = 500
        m = 3000
        s = rng.integers(0, n - 50, m).astype(np.int32)   # vertices >= 450 isolated
        d = rng.integers(0, n - 50, m).astype(np.int32)
        w = rng.integers(0, 4, m).astype(np.float32)       # zero weights and self loops included
        return n, s, d, w
    if case == "odd_sizes":
        n = 1001
        m = 2999
        s = rng.integers(0, n, m).astype(np.int32)
        d = rng.integers(0, n, m).astype(np.int32)
        w = rng.integers(1, 6, m).astype(np.float32)
        return n, s, d, w
    if case == "hub":
        # a star hub of degree 12000 (global-table path) plus a block-bucket hub and SBM background
        n, s, d, w = gen.sbm(20000, 40, 0.01, 0.0002, 1, 3, seed=3)
        leaves = np.arange(1, 12001, dtype=np.int32)
        mid = np.arange(13000, 13600, dtype=np.int32)
        hs = np.concatenate([np.zeros(12000, np.int32), leaves, np.full(600, 12500, np.int32), mid])
        hd = np.concatenate([leaves, np.zeros(12000, np.int32), mid, np.full(600, 12500, np.int32)])
        hw = np.ones(len(hs), np.float32) * 2
        return n, np.concatenate([s, hs]), np.concatenate([d, hd]), np.concatenate([w, hw])
    if case == "bighub":
        # a hub of degree 400,000 (512 aggregation buckets: a thread per
        # bucket slice) over leaves on a ring, integer weights 1..3
        n = 450000
        rng = np.random.default_rng(8)
        leaves = np.arange(1, 400001, dtype=np.int32)
        ring = np.roll(leaves, 1)
        u = np.concatenate([np.zeros(len(leaves), np.int32), leaves])
        v = np.concatenate([leaves, ring])
        w = rng.integers(1, 4, len(u)).astype(np.float32)
        return n, np.concatenate([u, v]), np.concatenate([v, u]), np.concatenate([w, w])
    raise ValueError(case)


@pytest.mark.parametrize("case", ["sbm_small", "weighted", "loops_zeros_isolated", "odd_sizes", "hub", "bighub"])
def test_move_decisions_bit_exact(Louvain, oracle, gen, case):
    n, s, d, w = make_case(gen, case)
    oc = oracle.Csr(n, s, d, w)
    rng = np.random.default_rng(11)
    with Louvain() as lv:
        lv.load_edges(s, d, w, n)
        # singleton state, then a random clustered state
        for comm in (np.arange(n, dtype=np.int32), rng.integers(0, n // 10, n).astype(np.int32)):
            tot = np.zeros(n)
            size = np.zeros(n, np.int32)
            np.add.at(tot, comm, oc.k)
            np.add.at(size, comm, 1)
            exp_next, exp_cand, _ = oc.decide(comm, tot, size)
            lv.set_communities(comm)
            nxt, cand = lv.move_decide()
            np.testing.assert_array_equal(nxt, exp_next)
            np.testing.assert_array_equal(cand, exp_cand)


@pytest.mark.parametrize("case", ["sbm_small", "weighted", "loops_zeros_isolated", "odd_sizes", "hub"])
def test_full_run_bit_exact(Louvain, oracle, gen, case):
    n, s, d, w = make_case(gen, case)
    orun = oracle.Run(n, s, d, w)
    with Louvain() as lv:
        lv.load_edges(s, d, w, n)
        res = lv.run()
        run_equal(lv, res, orun, n, s, d, w, oracle)


@pytest.mark.parametrize("name", ["k4k4", "ring_k5", "star", "path"])
def test_hand_graphs_bit_exact(Louvain, oracle, name):
    from conftest import hand_graph
    n, s, d, w = hand_graph(name)
    orun = oracle.Run(n, s, d, w)
    with Louvain() as lv:
        lv.load_edges(s, d, w, n)
        res = lv.run()
        run_equal(lv, res, orun, n, s, d, w, oracle)


@pytest.mark.parametrize("case", ["weighted", "hub"])
def test_fractional_weights_within_tolerance(Louvain, oracle, gen, case):
    """Non-integral weights take the f64 accumulators (tile, block, hub
    tables); sums may round in another order than the oracle's, so the
    check is the north-star tolerance on the final modularity."""
    n, s, d, w = make_case(gen, case)
    w = (w * 0.37 + 0.05).astype(np.float32)
    orun = oracle.Run(n, s, d, w)
    q_oracle = oracle.modularity_fp64(n, s, d, w, orun.final)
    with Louvain() as lv:
        lv.load_edges(s, d, w, n)
        res = lv.run()
        part = lv.partition()
        assert part.min() >= 0 and part.max() < n
        assert res.q_final == pytest.approx(oracle.modularity_fp64(n, s, d, w, part), abs=1e-9)
        assert abs(res.q_final - q_oracle) <= 1e-3


def test_sbm_10k_config(Louvain, oracle, gen):
    """SBM n=10,000 config: level gain threshold 1e-6, bit-exact dendrogram."""
    n, s, d, w = gen.sbm_10k(seed=0)
    orun = oracle.Run(n, s, d, w, level_min_gain=1e-6)
    with open(os.path.join(GOLDEN, "sbm10k_seed0.json")) as f:
        g = json.load(f)
    with Louvain(level_min_gain=1e-6) as lv:
        lv.load_edges(s, d, w, n)
        res = lv.run()
        run_equal(lv, res, orun, n, s, d, w, oracle)
        assert [lv.level_info(l).passes for l in range(res.n_levels)] == g["passes"]
        assert res.q_final == pytest.approx(g["final_modularity_fp64"], abs=1e-9)


def test_step_api_matches_run(Louvain, oracle, gen):
    """modularity / one_level / renumber / induce called one by one as the
    reference's driver does (LouvainCPP.cpp:334-501)."""
    n, s, d, w = gen.sbm(3000, 30, 0.05, 0.002, 1, 1, seed=4)
    orun = oracle.Run(n, s, d, w)
    with Louvain() as lv:
        lv.load_edges(s, d, w, n)
        q0 = lv.modularity()
        assert q0 == orun.levels[0].q_start
        q, passes = lv.one_level(q0)
        assert (q, passes) == (orun.levels[0].q, orun.levels[0].passes)
        part, C = lv.renumber()
        np.testing.assert_array_equal(part, orun.levels[0].part)
        lv.induce()
        q1, p1 = lv.one_level(q)
        assert (q1, p1) == (orun.levels[1].q, orun.levels[1].passes)


@pytest.mark.parametrize("mode", [0, 1, 2, 3])
def test_lfr_full_size(Louvain, oracle, gen, mode):
    """LFR-style n=2^20 config: the dendrogram matches the oracle bit for bit
    and the final Q lies within 1e-3, whichever method coarsens the sorted
    symmetric levels (0 automatic, 1 segment chunks, 2 by transposition, 3
    sort of all keys)."""
    n, s, d, w = gen.lfr()
    orun = oracle.Run(n, s, d, w)
    with Louvain(coarsen_mode=mode) as lv:
        lv.load_edges(s, d, w, n)
        res = lv.run()
        run_equal(lv, res, orun, n, s, d, w, oracle)


@pytest.mark.parametrize("use_graphs,passes_per_sync", [(False, 1), (True, 1), (True, 7)])
def test_graph_replay_and_sync_interval_do_not_change_results(Louvain, oracle, gen, use_graphs, passes_per_sync):
    n, s, d, w = gen.sbm(4000, 40, 0.05, 0.002, 1, 2, seed=6)
    orun = oracle.Run(n, s, d, w)
    with Louvain(use_graphs=use_graphs, passes_per_sync=passes_per_sync) as lv:
        lv.load_edges(s, d, w, n)
        res = lv.run()
        run_equal(lv, res, orun, n, s, d, w, oracle)


def test_unsorted_input_matches_sorted(Louvain, gen):
    """The sort-free CSR build (sorted symmetric list) and the sorting build
    (the same list shuffled) give the same CSR and dendrogram."""
    n, s, d, w = gen.sbm(3000, 30, 0.05, 0.002, 1, 3, seed=8)
    perm = np.random.default_rng(1).permutation(len(s))
    with Louvain() as a, Louvain() as b:
        a.load_edges(s, d, w, n)
        b.load_edges(s[perm], d[perm], w[perm], n)
        ca, cb = a.csr(), b.csr()
        for key in ("off", "col", "w", "k", "loopw", "has_loop"):
            np.testing.assert_array_equal(ca[key], cb[key])
        ra, rb = a.run(), b.run()
        assert ra.n_levels == rb.n_levels
        np.testing.assert_array_equal(a.partition(), b.partition())


@pytest.mark.parametrize("change", ["one_weight", "one_direction", "extra_entry"])
def test_sorted_but_not_symmetric_takes_the_sorting_build(Louvain, oracle, gen, change):
    """Sorted lists that are not symmetric (a weight differing between the two
    directions, an edge listed one way, an entry without its mirror) must not
    take the sort-free build: the CSR equals the oracle's."""
    n, s, d, w = gen.sbm(2000, 20, 0.05, 0.002, 1, 3, seed=9)
    s, d, w = s.copy(), d.copy(), w.copy()
    e = int(np.flatnonzero(s < d)[len(s) // 5])
    if change == "one_weight":
        w[e] += 1.0
    elif change == "one_direction":
        keep = np.ones(len(s), bool)
        keep[e] = False
        s, d, w = s[keep], d[keep], w[keep]
    else:
        u, v = int(s[e]), int(d[e])
        free = np.setdiff1d(np.arange(n), d[s == u])
        x = int(free[free > u][0]) if np.any(free > u) else int(free[0])
        s, d, w = np.append(s, u), np.append(d, x), np.append(w, 2.0)
        order = np.lexsort((d, s))
        s, d, w = s[order], d[order], w[order]
    oc = oracle.Csr(n, s, d, w)
    with Louvain() as lv:
        lv.load_edges(s, d, w, n)
        csr_equal(lv, oc)
        res = lv.run()
        r = oracle.Run(n, s, d, w)
        np.testing.assert_array_equal(lv.partition(), r.final)
        assert res.n_levels == len(r.levels)


def test_invalid_input_is_an_error(Louvain):
    from louvaingpu_b200 import LvgError
    with Louvain() as lv:
        with pytest.raises(LvgError):
            lv.load_edges([0, 5], [5, 0], [1.0, 1.0], 3)        # id out of range
        with pytest.raises(LvgError):
            lv.load_edges([0, 1], [1, 0], [-1.0, 1.0], 3)       # negative weight
        with pytest.raises(LvgError):
            lv.load_edges([0, 1], [1, 0], [np.nan, 1.0], 3)     # non-finite weight
        with pytest.raises(LvgError):
            lv.one_level(0.0)                                   # nothing loaded


def test_empty_graph(Louvain):
    with Louvain() as lv:
        lv.load_edges([], [], [], 5)
        res = lv.run()
        assert res.n_levels == 1
        assert lv.partition().tolist() == [0, 1, 2, 3, 4]


def test_pass_cap_reports_not_converged(Louvain, gen):
    from louvaingpu_b200 import LvgError
    n, s, d, w = gen.sbm(2000, 20, 0.05, 0.002, 1, 1, seed=1)
    with Louvain(max_passes=1) as lv:
        lv.load_edges(s, d, w, n)
        with pytest.raises(LvgError) as e:
            lv.run()
        assert e.value.status == 4


@pytest.mark.parametrize("name", ["lfr_seed1.json", "rmat16_seed2.json"])
def test_committed_workload_fixtures(Louvain, gen, name):
    """The CUDA path reproduces the committed fixtures of the LFR n=2^20 and
    R-MAT 16 graphs (tests/golden/make_workload_goldens.py): level sizes,
    passes, community counts and per-level Q bit for bit, the final partition
    by its hash, and the final FP64 Q within the tolerance of the other tests."""
    import hashlib
    with open(os.path.join(GOLDEN, name)) as f:
        g = json.load(f)
    n, s, d, w = gen.lfr() if name.startswith("lfr") else gen.rmat(16)
    assert (n, len(s)) == (g["n_vertices"], g["n_entries"])
    with Louvain() as lv:
        lv.load_edges(s, d, w, n)
        res = lv.run()
        assert res.n_levels == len(g["levels"])
        for l, x in enumerate(g["levels"]):
            li = lv.level_info(l)
            assert (li.n_vertices, li.nnz, li.passes, li.n_comms) == \
                   (x["n_vertices"], x["nnz"], x["passes"], x["n_comms"]), f"level {l}"
            assert li.q_start.hex() == x["q_start"] and li.q_level.hex() == x["q_level"], f"level {l}"
        part = np.ascontiguousarray(lv.partition(), np.int32)
        assert hashlib.sha256(part.tobytes()).hexdigest() == g["final_partition_sha256"]
        assert res.q_final == pytest.approx(float.fromhex(g["final_modularity_fp64"]), abs=1e-9)


def coarsening_partitions(oracle, gen, case, n, s, d, w):
    """Partitions (community ids as vertex indices) to coarsen under: the
    oracle's level-0 labels, or the planted communities for the LFR graph,
    and random labels over a seventh of the ids."""
    rng = np.random.default_rng(23)
    if case == "lfr":
        _, _, _, _, truth = gen.lfr(with_truth=True)
        first = truth.astype(np.int32)
    else:
        first = oracle.Run(n, s, d, w, max_levels=1).levels[0].labels
    return [first, rng.integers(0, max(1, n // 7), n).astype(np.int32)]


def sorted_symmetric(oracle, n, s, d, w):
    """The list as a strictly sorted, symmetric one (each entry mirrored,
    duplicates merged by the oracle's coarsening under the identity map), with
    weight 0 on a symmetric fifth of the entries: the form every coarse level
    has, which takes the sort-free coarsening."""
    loops = s == d
    s2, d2, w2 = np.r_[s, d[~loops]], np.r_[d, s[~loops]], np.r_[w, w[~loops]]
    ss, sd, sw = oracle.induce(n, s2, d2, w2, np.arange(n, dtype=np.int32))
    sw = np.where((ss.astype(np.int64) + sd) % 5 == 0, np.float32(0), sw).astype(np.float32)
    return ss, sd, sw


@pytest.mark.parametrize("form,mode", [("as_given", 0), ("sorted_symmetric", 1), ("sorted_symmetric", 2),
                                       ("sorted_symmetric", 3)])
@pytest.mark.parametrize("case", ["weighted", "loops_zeros_isolated", "odd_sizes", "hub", "lfr"])
def test_coarsening_bit_exact(Louvain, oracle, gen, case, form, mode):
    """renumber + induce from a given partition: the vertex map
    (RenumberKernel.cu:121-133), the coarse list -- one entry per distinct
    (cu, cv) key in key order, weight 0 counted as 1 (InducedGraphKernel.cu:28-48)
    and equal keys summed (:84-101) -- and the CSR built from it equal the
    oracle's entry for entry.  A list given strictly sorted and symmetric is
    coarsened without the device-wide sort (communities of up to ~10^5 entries
    here, so segments cross many 4096-entry chunks) by each coarsening method:
    segment chunks (1), by transposition (2) and the sort of all keys (3)."""
    n, s, d, w = gen.lfr() if case == "lfr" else make_case(gen, case)
    if form == "sorted_symmetric":
        s, d, w = sorted_symmetric(oracle, n, s, d, w)
    with Louvain(coarsen_mode=mode) as lv:
        for comm in coarsening_partitions(oracle, gen, case, n, s, d, w):
            lv.load_edges(s, d, w, n)
            lv.set_communities(comm)
            part, C = lv.renumber()
            exp_part, exp_C = oracle.renumber(comm)
            assert C == exp_C
            np.testing.assert_array_equal(part, exp_part)
            lv.induce()
            es, ed, ew = lv.level_edges()
            os_, od, ow = oracle.induce(n, s, d, w, exp_part)
            np.testing.assert_array_equal(es, os_)
            np.testing.assert_array_equal(ed, od)
            np.testing.assert_array_equal(ew, ow)
            csr_equal(lv, oracle.Csr(C, os_, od, ow))


def test_run_after_steps_matches_a_fresh_run(Louvain, oracle, gen):
    """lvg_run after one_level / set_communities / renumber calls on the same
    load restarts from the loaded level 0: same levels, Q and partition as
    the oracle's run (the singleton Q is the first level's floor)."""
    n, s, d, w = gen.sbm(3000, 30, 0.05, 0.002, 1, 4, seed=2)
    orun = oracle.Run(n, s, d, w)
    with Louvain() as lv:
        lv.load_edges(s, d, w, n)
        q0 = lv.modularity()
        lv.one_level(q0)
        lv.one_level(q0)
        res = lv.run()
        run_equal(lv, res, orun, n, s, d, w, oracle)
        lv.load_edges(s, d, w, n)
        lv.set_communities(np.random.default_rng(3).integers(0, n // 5, n).astype(np.int32))
        lv.renumber()
        res = lv.run()
        run_equal(lv, res, orun, n, s, d, w, oracle)


def test_partition_into_caller_buffers(Louvain, gen):
    """partition(out=...) fills a numpy array or a pinned host tensor with the
    same labels as partition(); a buffer of the wrong size or type is refused."""
    import torch
    n, s, d, w = make_case(gen, "weighted")
    with Louvain() as lv:
        lv.load_edges(s, d, w, n)
        lv.run()
        ref = lv.partition()
        a = np.full(n, -1, np.int32)
        assert lv.partition(out=a) is a
        np.testing.assert_array_equal(a, ref)
        t = torch.full((n,), -1, dtype=torch.int32).pin_memory()
        lv.partition(out=t)
        np.testing.assert_array_equal(t.numpy(), ref)
        with pytest.raises(ValueError):
            lv.partition(out=np.zeros(n - 1, np.int32))
        with pytest.raises(ValueError):
            lv.partition(out=np.zeros(n, np.int64))


@pytest.mark.parametrize("form", ["sorted_symmetric", "as_given"])
def test_chunked_host_load(Louvain, oracle, gen, form):
    """A host list copied in chunks (load_chunk_entries) while the level-0 CSR
    is built from the chunks already on the device: the CSR, two whole runs
    on one load, and the refusal of an out-of-range id or a negative weight in
    a late chunk equal what the whole-list load gives.  A list that is not
    sorted and symmetric falls back to the sorting build."""
    from louvaingpu_b200._lib import LvgError
    n, s, d, w = make_case(gen, "hub")
    if form == "sorted_symmetric":
        s, d, w = sorted_symmetric(oracle, n, s, d, w)
    assert len(s) > 4 * 4096
    oc = oracle.Csr(n, s, d, w)
    orun = oracle.Run(n, s, d, w)
    with Louvain(load_chunk_entries=4096) as lv:
        lv.load_edges(s, d, w, n)
        csr_equal(lv, oc)
        for _ in range(2):
            res = lv.run()
            run_equal(lv, res, orun, n, s, d, w, oracle)
        bad = d.copy()
        bad[len(bad) * 2 // 3] = n
        with pytest.raises(LvgError):
            lv.load_edges(s, bad, w, n)
        neg = w.copy()
        neg[len(neg) - 5] = -1.0
        with pytest.raises(LvgError):
            lv.load_edges(s, d, neg, n)
        lv.load_edges(s, d, w, n)
        csr_equal(lv, oc)
