"""CPU checks of the batched form's host side: the packing of many graphs
into one list (pack_graphs), the batched workload's per-graph parameters
against the configured shape, and the bench's split into sub-batches."""
import numpy as np


def test_pack_graphs_offsets_and_order():
    from louvaingpu_b200 import pack_graphs
    g0 = (3, np.array([0, 1], np.int32), np.array([1, 0], np.int32), np.array([2.0, 2.0], np.float32))
    g1 = (2, np.array([], np.int32), np.array([], np.int32), np.array([], np.float32))
    g2 = (4, np.array([0, 3, 3], np.int32), np.array([3, 0, 1], np.int32), np.array([1, 1, 5], np.float32))
    s, d, w, eoff, voff = pack_graphs([g0, g1, g2])
    assert eoff.tolist() == [0, 2, 2, 5] and voff.tolist() == [0, 3, 5, 9]
    assert s.tolist() == [0, 1, 0, 3, 3] and d.tolist() == [1, 0, 3, 0, 1]   # ids stay local to each graph
    assert w.tolist() == [2.0, 2.0, 1.0, 1.0, 5.0]
    assert s.dtype == np.int32 and w.dtype == np.float32 and eoff.dtype == np.int64 and voff.dtype == np.int32


def test_batched_params_follow_the_configured_shape():
    """n log-uniform in [64, 200000], 4-400 blocks, expected average degree
    uniform in [8, 32] with 70 % of it inside blocks, weights 1..4."""
    from louvaingpu_b200 import graphgen
    ps = graphgen.batched_sbm_params(8192, seed=3)
    n = np.array([p["n"] for p in ps])
    assert n.min() >= 64 and n.max() <= 200000
    lg = np.log(n)
    # log-uniform: mean and spread of log n match the uniform law on [log 64, log 200000]
    a, b = np.log(64), np.log(200000)
    assert abs(lg.mean() - (a + b) / 2) < 0.05 * (b - a)
    assert abs(lg.std() - (b - a) / np.sqrt(12)) < 0.05 * (b - a)
    blocks = np.array([p["blocks"] for p in ps])
    assert blocks.min() >= 4 and blocks.max() <= 400
    degs, intra = [], []
    for p in ps:
        s = p["n"] / p["blocks"]
        din, dout = p["p_in"] * (s - 1), p["p_out"] * (p["n"] - s)
        if p["p_in"] < 1.0:                        # not clipped by a tiny block
            degs.append(din + dout)
            intra.append(din / (din + dout))
        assert (p["w_lo"], p["w_hi"]) == (1, 4)
    degs, intra = np.array(degs), np.array(intra)
    # only graphs too small for 4 blocks of 0.7 d + 1 vertices take p_in = 1
    assert len(degs) > 0.98 * len(ps)
    assert max(p["n"] for p in ps if p["p_in"] >= 1.0) < 4 * (0.7 * 32 + 1)
    assert degs.min() > 7.99 and degs.max() < 32.01
    assert abs(degs.mean() - 20.0) < 0.5
    assert np.allclose(intra, 0.7, atol=0.01)


def test_generated_batched_graphs_have_the_shape(gen):
    """A few graphs drawn with those parameters: symmetric lists, no self
    loops, integer weights 1..4, average degree and intra-block share near
    the targets."""
    from louvaingpu_b200 import graphgen
    ps = [p for p in graphgen.batched_sbm_params(400, seed=5) if 5000 <= p["n"] <= 40000 and p["p_in"] < 1.0][:4]
    assert ps
    for p in ps:
        n, s, d, w, truth = gen.sbm(p["n"], p["blocks"], p["p_in"], p["p_out"], p["w_lo"], p["w_hi"], seed=p["seed"],
                                     with_truth=True)
        assert n == p["n"] and not np.any(s == d)
        assert set(np.unique(w).tolist()) <= {1.0, 2.0, 3.0, 4.0}
        fwd = set(zip(s.tolist(), d.tolist()))
        assert all((b, a) in fwd for a, b in list(fwd)[:2000])
        size = n / p["blocks"]
        target = p["p_in"] * (size - 1) + p["p_out"] * (n - size)
        assert abs(len(s) / n - target) < 0.1 * target
        share = np.mean(truth[s] == truth[d])
        exp = p["p_in"] * (size - 1) / target
        assert abs(share - exp) < 0.05


def test_bench_sub_batches_cover_every_graph_in_order():
    import bench
    params, groups = bench.batched_plan(600, 3, 2.0e6)
    flat = [p for g in groups for p in g]
    assert flat == params
    for g in groups:
        n_exp = 0.0
        for p in g:
            n_, B = p["n"], p["blocks"]
            k = np.arange(B + 1, dtype=np.int64)
            sizes = np.diff(n_ * k // B).astype(np.float64)
            pin = float((sizes * (sizes - 1) / 2).sum())
            n_exp += 2.0 * (pin * min(p["p_in"], 1.0) + (n_ * (n_ - 1) / 2 - pin) * min(p["p_out"], 1.0))
        assert len(g) == 1 or n_exp <= 2.0e6
