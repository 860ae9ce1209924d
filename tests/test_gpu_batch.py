"""Batched runs (lvg_batch_run): many independent graphs in shared launches.

Every graph of a batch must get exactly what its own run gives: the same
final partition (bit for bit), level count, community count and status, and
the same FP64 modularity (the per-graph sums use the single-graph tree).
Integer-valued weights keep every sum exact, so the oracle's results are the
target as well.
"""
import numpy as np
import pytest

from conftest import undirected_to_lists
from test_gpu_parity import make_case

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def Louvain():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for gpu tests")
    from louvaingpu_b200 import Louvain as L
    return L


def mixed_graphs(gen):
    rng = np.random.default_rng(11)
    graphs = [make_case(gen, c) for c in ("sbm_small", "weighted", "loops_zeros_isolated", "odd_sizes", "hub")]
    graphs.append((5, np.zeros(0, np.int32), np.zeros(0, np.int32), np.zeros(0, np.float32)))   # no entries
    s, d, w = undirected_to_lists([(0, 1), (1, 2), (0, 2), (3, 4), (4, 5), (3, 5), (2, 3)])
    graphs.append((6, s, d, w))                                                                  # two triangles
    graphs.append((2, np.array([0], np.int32), np.array([1], np.int32), np.array([3.0], np.float32)))
    for k in range(24):                                                                          # small SBMs
        n = int(rng.integers(40, 3000))
        graphs.append(gen.sbm(n, max(2, n // 60), 0.15, 0.004, 1, 4, seed=100 + k))
    return graphs


def single_runs(Louvain, graphs, **cfg):
    out = []
    with Louvain(**cfg) as lv:
        for n, s, d, w in graphs:
            lv.load_edges(s, d, w, n)
            try:
                res = lv.run()
                status = 0
            except Exception as e:   # a capped run reports NOT_CONVERGED
                status = getattr(e, "status", -1)
                res = None
            out.append((res, lv.partition().copy() if lv.n_levels else None, status, lv.n_levels))
    return out


def test_batch_equals_single_runs(Louvain, gen):
    graphs = mixed_graphs(gen)
    ref = single_runs(Louvain, graphs)
    with Louvain() as lv:
        b = lv.run_batch(graphs)
    assert len(b) == len(graphs)
    for g, (res, part, status, nlev) in enumerate(ref):
        assert status == 0
        np.testing.assert_array_equal(b.part(g), part, err_msg=f"graph {g}")
        assert b.n_levels[g] == res.n_levels, g
        assert b.n_comms[g] == res.n_comms, g
        assert b.status[g] == 0, g
        assert b.q_final[g] == res.q_final, g          # same fixed tree: bit-identical


def test_batch_persistent_kernels_at_low_thresholds(Louvain, gen):
    """Tile, block and hub thresholds of 32 / 64 send most rows of the batch
    to the persistent block-per-item kernels (items pulled from device
    counters); every graph still gets its own run's result bit for bit."""
    graphs = mixed_graphs(gen)
    ref = single_runs(Louvain, graphs, tile_max_degree=32, block_max_degree=64)
    with Louvain(tile_max_degree=32, block_max_degree=64) as lv:
        b = lv.run_batch(graphs)
    for g, (res, part, status, nlev) in enumerate(ref):
        np.testing.assert_array_equal(b.part(g), part, err_msg=f"graph {g}")
        assert b.q_final[g] == res.q_final, g


def test_batch_matches_oracle(Louvain, oracle, gen):
    graphs = mixed_graphs(gen)
    with Louvain() as lv:
        b = lv.run_batch(graphs)
    for g, (n, s, d, w) in enumerate(graphs):
        if len(s) == 0:
            assert b.n_levels[g] == 1 and b.part(g).tolist() == list(range(n))
            continue
        r = oracle.Run(n, s, d, w)
        np.testing.assert_array_equal(b.part(g), r.final, err_msg=f"graph {g}")
        assert b.n_levels[g] == len(r.levels), g
        assert b.n_comms[g] == r.levels[-1].n_comms, g
        assert b.q_final[g] == pytest.approx(oracle.modularity_fp64(n, s, d, w, r.final), abs=1e-9), g


def test_batch_order_does_not_matter(Louvain, gen):
    graphs = mixed_graphs(gen)
    perm = np.random.default_rng(5).permutation(len(graphs))
    with Louvain() as lv:
        a = lv.run_batch(graphs)
        b = lv.run_batch([graphs[i] for i in perm])
    for j, i in enumerate(perm):
        np.testing.assert_array_equal(a.part(i), b.part(j))
        assert a.q_final[i] == b.q_final[j]
        assert a.n_levels[i] == b.n_levels[j]


def test_many_tiny_graphs(Louvain, oracle, gen):
    rng = np.random.default_rng(3)
    graphs = []
    for k in range(600):
        n = int(rng.integers(8, 200))
        graphs.append(gen.sbm(n, max(2, n // 20), 0.4, 0.02, 1, 4, seed=1000 + k))
    with Louvain() as lv:
        b = lv.run_batch(graphs)
    for g in range(0, len(graphs), 7):
        n, s, d, w = graphs[g]
        r = oracle.Run(n, s, d, w)
        np.testing.assert_array_equal(b.part(g), r.final, err_msg=f"graph {g}")
        assert b.n_levels[g] == len(r.levels)


def test_batch_caps_are_per_graph(Louvain, gen):
    graphs = mixed_graphs(gen)[:8]
    ref = single_runs(Louvain, graphs, max_levels=1)
    with Louvain(max_levels=1) as lv:
        b = lv.run_batch(graphs)
    for g, (res, part, status, nlev) in enumerate(ref):
        np.testing.assert_array_equal(b.part(g), part)
        assert b.status[g] == status
        assert b.n_levels[g] == nlev


def test_batch_invalid_input(Louvain):
    from louvaingpu_b200 import LvgError
    good = (3, np.array([0, 1], np.int32), np.array([1, 2], np.int32), np.ones(2, np.float32))
    bad = (3, np.array([0, 3], np.int32), np.array([1, 2], np.int32), np.ones(2, np.float32))  # id 3 >= n
    neg = (3, np.array([0, 1], np.int32), np.array([1, 2], np.int32), np.array([1, -1], np.float32))
    with Louvain() as lv:
        for graphs in ([good, bad], [neg, good]):
            with pytest.raises(LvgError):
                lv.run_batch(graphs)
        b = lv.run_batch([good, good])        # the context stays usable
        assert b.part(0).tolist() == b.part(1).tolist()
