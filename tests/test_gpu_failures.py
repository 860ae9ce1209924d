"""Failure paths on the GPU, made on the host or by a bounded wait that a test
runs out -- never by a device fault:

  * an arena too small for the graph: the load returns LVG_ERR_OOM from the
    arena's own check, and the same context then loads and runs a graph that
    fits (the reference rethrows Thrust's allocation failure,
    cached_allocator.h:56-59, and has no way back);
  * a radix-sort look-back wait that never ends (a tile held from publishing
    by the test hook, with a short poll limit): the sort returns its error
    flag as LVG_ERR_CUDA instead of hanging, and the context works after it.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

OOM, CUDA_ERR = 2, 5


@pytest.fixture(scope="module")
def lvmod():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for gpu tests")
    import louvaingpu_b200 as L
    return L


def run_equal_oracle(lv, oracle, n, s, d, w):
    res = lv.run()
    ref = oracle.Run(n, s, d, w)
    assert res.n_levels == len(ref.levels)
    np.testing.assert_array_equal(lv.partition(), ref.final)


def test_arena_cap_returns_oom_and_the_context_recovers(lvmod, oracle, gen):
    n, s, d, w = gen.sbm(20000, 40, 0.02, 0.0005, 1, 3, seed=4)
    small = gen.sbm(300, 3, 0.1, 0.01, 1, 2, seed=5)
    with lvmod.Louvain(arena_bytes=4 << 20) as lv:
        with pytest.raises(lvmod.LvgError) as e:
            lv.load_edges(s, d, w, n)
        assert e.value.status == OOM
        assert "arena exhausted" in str(e.value)
        with pytest.raises(lvmod.LvgError):
            lv.run()                       # nothing is loaded after the failed load
        lv.load_edges(*small[1:], small[0])
        run_equal_oracle(lv, oracle, *small)


def test_radix_lookback_wait_runs_out_and_reports(lvmod, oracle, gen):
    from louvaingpu_b200 import _lib
    L = _lib.load()
    n, s, d, w = gen.sbm(3000, 30, 0.05, 0.002, 1, 4, seed=2)
    perm = np.random.default_rng(1).permutation(len(s))
    s, d, w = s[perm], d[perm], w[perm]     # unsorted: the build sorts the doubled list
    assert 2 * len(s) > 4 * 4096            # several radix tiles
    try:
        assert L.lvg_debug_radix_hold(4096, 0) == 0
        with lvmod.Louvain() as lv:
            with pytest.raises(lvmod.LvgError) as e:
                lv.load_edges(s, d, w, n)
            assert e.value.status == CUDA_ERR
            assert "look-back did not complete" in str(e.value)
            assert L.lvg_debug_radix_hold(1 << 22, -1) == 0
            lv.load_edges(s, d, w, n)
            c = lv.csr()
            oc = oracle.Csr(n, s, d, w)
            np.testing.assert_array_equal(c["off"], oc.off)
            np.testing.assert_array_equal(c["col"], oc.col)
            np.testing.assert_array_equal(c["w"], oc.w)
            run_equal_oracle(lv, oracle, n, s, d, w)
    finally:
        L.lvg_debug_radix_hold(1 << 22, -1)
