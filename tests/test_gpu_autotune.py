"""GPU checks of the degree-threshold autotuner (lvg_autotune).

The thresholds route vertices to the thread, tile, block and hub kernels; the
decisions must not depend on them.  Runs with explicit extreme thresholds and
with the tuner's choice are compared with the oracle bit for bit."""
import numpy as np
import pytest

from test_gpu_parity import make_case, run_equal

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def Louvain():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for gpu tests")
    from louvaingpu_b200 import Louvain as L
    return L


@pytest.fixture(scope="module")
def rmat16(gen):
    return gen.rmat(16)


@pytest.mark.parametrize("tile,block", [(32, 32), (64, 256), (256, 1024), (512, 8192)])
def test_thresholds_do_not_change_results(Louvain, oracle, rmat16, tile, block):
    """(32, 32) sends every row above 32 entries to the global hub tables,
    (512, 8192) gives the block kernel its largest shared table."""
    n, s, d, w = rmat16
    orun = oracle.Run(n, s, d, w)
    with Louvain(tile_max_degree=tile, block_max_degree=block) as lv:
        assert lv.thresholds() == (tile, block)
        lv.load_edges(s, d, w, n)
        res = lv.run()
        run_equal(lv, res, orun, n, s, d, w, oracle)


def test_autotune_picks_a_measured_pair_and_keeps_results(Louvain, oracle, rmat16):
    from louvaingpu_b200 import tune_pick
    n, s, d, w = rmat16
    orun = oracle.Run(n, s, d, w)
    tiles, blocks = [32, 64, 256, 512], [256, 1024, 4096, 8192]
    with Louvain() as lv:
        lv.load_edges(s, d, w, n)
        best, pts = lv.autotune(tiles, blocks, reps=2)
        pairs = [(t, b) for t in tiles for b in blocks if b >= t]
        assert [(p[0], p[1]) for p in pts] == pairs
        assert all(p[2] > 0.0 and p[3] > 0.0 for p in pts)
        i = tune_pick(pts, pref=(512, 4096))
        assert i >= 0 and (best[0], best[1]) == (pts[i][0], pts[i][1])
        assert lv.thresholds() == (best[0], best[1])
        res = lv.run()                     # later levels are built with the chosen pair
        run_equal(lv, res, orun, n, s, d, w, oracle)


def test_autotune_cache_hit_measures_nothing(Louvain, rmat16):
    from louvaingpu_b200 import _lib
    n, s, d, w = rmat16
    _lib.load().lvg_tune_cache_clear()
    with Louvain() as a:
        a.load_edges(s, d, w, n)
        best, pts = a.autotune([64, 512], [1024, 4096], reps=1, use_cache=True)
        assert len(pts) == 4
    with Louvain() as b:
        b.load_edges(s, d, w, n)
        hit, pts2 = b.autotune([64, 512], [1024, 4096], reps=1, use_cache=True)
        assert pts2 == [] and (hit[0], hit[1]) == (best[0], best[1])
        assert b.thresholds() == (best[0], best[1])
        res = b.run()
        assert res.n_levels > 1


def test_autotuned_batched_run_equals_default(Louvain, gen):
    graphs = [gen.sbm(1500 + 300 * k, 10 + k, 0.05, 0.003, 1, 4, seed=20 + k) for k in range(6)]
    graphs.append(make_case(gen, "hub"))
    with Louvain() as ref:
        r0 = ref.run_batch(graphs)
    with Louvain() as lv:
        n, s, d, w = graphs[-1]
        lv.load_edges(s, d, w, n)
        lv.autotune([32, 128], [64, 1024], reps=1)
        r1 = lv.run_batch(graphs)
    np.testing.assert_array_equal(r0.partition, r1.partition)
    np.testing.assert_array_equal(r0.q_final, r1.q_final)
    np.testing.assert_array_equal(r0.n_levels, r1.n_levels)


def test_autotune_empty_graph_keeps_configured_pair(Louvain):
    with Louvain(tile_max_degree=256, block_max_degree=2048) as lv:
        lv.load_edges([], [], [], 7)
        best, pts = lv.autotune()
        assert pts == [] and (best[0], best[1]) == (256, 2048)
        assert lv.thresholds() == (256, 2048)
        lv.run()
        assert lv.partition().tolist() == list(range(7))
