"""Device generators (include/lvg_gen.h): R-MAT equals the host generator
entry for entry; batched SBMs are valid symmetric sorted lists with the
planted densities, deterministic and independent of their batch; batched
runs over device-resident lists equal per-graph runs."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for gpu tests")
    return torch


@pytest.mark.parametrize("scale,ef", [(10, 16), (14, 8)])
def test_rmat_device_equals_host(torch_cuda, gen, scale, ef):
    n, s, d, w = gen.rmat(scale, edge_factor=ef, seed=5)
    dg = gen.rmat_device(scale, edge_factor=ef, seed=5)
    assert dg.n_vertices == n and dg.n_entries == len(s)
    ds, dd, dw = dg.to_host()
    np.testing.assert_array_equal(ds, s)
    np.testing.assert_array_equal(dd, d)
    np.testing.assert_array_equal(dw, w)
    dg.close()


def check_sbm(n, blocks, p_in, p_out, s, d, w):
    assert len(s) % 2 == 0
    assert s.min(initial=0) >= 0 and s.max(initial=0) < n and d.min(initial=0) >= 0 and d.max(initial=0) < n
    assert np.all(s != d)
    key = s.astype(np.int64) * n + d
    assert np.all(np.diff(key) > 0)                                   # sorted, no duplicates
    rkey = np.sort(d.astype(np.int64) * n + s)
    np.testing.assert_array_equal(rkey, key)                          # symmetric
    assert set(np.unique(w).tolist()) <= {1.0, 2.0, 3.0, 4.0}
    b = (np.arange(n, dtype=np.int64) + 1) * blocks - 1
    blk = b // n
    sizes = np.bincount(blk, minlength=blocks).astype(np.float64)
    pairs_in = float((sizes * (sizes - 1) / 2).sum())
    pairs_out = n * (n - 1) / 2 - pairs_in
    up = s < d
    same = blk[s[up]] == blk[d[up]]
    for cnt, pairs, p in ((same.sum(), pairs_in, p_in), ((~same).sum(), pairs_out, p_out)):
        mean = pairs * min(p, 1.0)
        sd = np.sqrt(max(pairs * p * (1 - p), 1.0))
        assert abs(cnt - mean) <= 6 * sd + 1, (cnt, mean, sd)


def test_sbm_batch_device_valid_and_deterministic(torch_cuda, gen):
    params = gen.batched_sbm_params(40, seed=9, n_lo=20, n_hi=20000)
    a = gen.sbm_batch_device(params)
    b = gen.sbm_batch_device(params)
    sa, da, wa = a.to_host()
    sb, db, wb = b.to_host()
    np.testing.assert_array_equal(sa, sb)
    np.testing.assert_array_equal(da, db)
    np.testing.assert_array_equal(wa, wb)
    np.testing.assert_array_equal(a.entry_off, b.entry_off)
    for g, p in enumerate(params):
        e0, e1 = a.entry_off[g], a.entry_off[g + 1]
        assert a.vertex_off[g + 1] - a.vertex_off[g] == p["n"]
        check_sbm(p["n"], p["blocks"], p["p_in"], p["p_out"], sa[e0:e1], da[e0:e1], wa[e0:e1])
    # a graph does not depend on the rest of its batch
    for g in (0, 7, 39):
        one = gen.sbm_batch_device([params[g]])
        s1, d1, w1 = one.to_host()
        e0, e1 = a.entry_off[g], a.entry_off[g + 1]
        np.testing.assert_array_equal(s1, sa[e0:e1])
        np.testing.assert_array_equal(d1, da[e0:e1])
        np.testing.assert_array_equal(w1, wa[e0:e1])


def test_batch_run_device_equals_single_runs(torch_cuda, gen):
    from louvaingpu_b200 import Louvain
    params = gen.batched_sbm_params(60, seed=4, n_lo=64, n_hi=30000)
    dg = gen.sbm_batch_device(params)
    with Louvain() as lv:
        b = lv.run_batch_device(dg.src, dg.dst, dg.w, dg.entry_off, dg.vertex_off)
    s, d, w = dg.to_host()
    with Louvain() as lv:
        for g in range(len(params)):
            sp, dp, wp, e, n = dg.graph_ptrs(g)
            lv.load_edges_device(sp, dp, wp, e, n)
            res = lv.run()
            np.testing.assert_array_equal(b.part(g), lv.partition(), err_msg=f"graph {g}")
            assert b.q_final[g] == res.q_final
            assert b.n_levels[g] == res.n_levels
    with Louvain() as lv:   # the host-buffer entry point gives the same
        c = lv.run_batch(packed=(s, d, w, dg.entry_off, dg.vertex_off))
    np.testing.assert_array_equal(c.partition, b.partition)
    np.testing.assert_array_equal(c.q_final, b.q_final)
