"""Request server: host-side behaviour on the CPU (argument checks; slots
that cannot start fail the queued requests instead of hanging), and on the
GPU every request's result is the same alone and in the mix."""
import time

import numpy as np
import pytest


def test_server_argument_errors():
    import ctypes
    from louvaingpu_b200 import _lib
    L = _lib.load()
    h = ctypes.c_void_p()
    assert L.lvg_server_create(None, 0, 1 << 30, 1000, 10, ctypes.byref(h)) == 1
    assert L.lvg_server_create(None, 2, 0, 1000, 10, ctypes.byref(h)) == 1
    assert L.lvg_server_create(None, 2, 1 << 30, 1000, 10, None) == 1
    assert L.lvg_server_submit(None, None, None, None, 0, 0, None, 0, None) == 1
    assert L.lvg_server_drain(None, 0) == 1
    assert L.lvg_server_destroy(None) == 1


def test_dead_slots_fail_queued_requests_without_a_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("needs a host without a usable GPU: every slot must fail to start")
    from louvaingpu_b200 import LvgError
    from louvaingpu_b200.serving import Server
    with Server(n_slots=2, hbm_budget=1 << 30, max_batch_entries=1000, max_batch_graphs=8) as srv:
        ids = []
        for k in range(3):
            try:
                ids.append(srv.submit(0, 0, 0, 0, 5, tag=k))
            except LvgError as e:          # every slot already gone: refused at once
                assert e.status == 6
        srv.drain(timeout_ms=10000)
        res = srv.poll()
        assert sorted(r.id for r in res) == sorted(ids)
        assert all(r.status != 0 for r in res)
        st = srv.stats()
        assert st["submitted"] == st["completed"] == len(ids)


@pytest.mark.gpu
def test_results_same_alone_and_in_the_mix(gen, oracle):
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for gpu tests")
    from louvaingpu_b200 import Louvain, LvgError
    from louvaingpu_b200.serving import Server
    params = gen.batched_sbm_params(150, seed=21, n_lo=32, n_hi=40000)
    dg = gen.sbm_batch_device(params)
    giants = [gen.rmat_device(13, seed=s) for s in (1, 2)]
    reqs = [dg.graph_ptrs(g) for g in range(dg.n_graphs)] + \
           [(x.src, x.dst, x.w, x.n_entries, x.n_vertices) for x in giants]
    order = np.random.default_rng(0).permutation(len(reqs))
    torch.cuda.synchronize()
    alone = {}
    with Louvain() as lv:
        for i in range(len(reqs)):
            s, d, w, e, n = reqs[i]
            lv.load_edges_device(s, d, w, e, n)
            res = lv.run()
            alone[i] = (lv.partition(), res.q_final, res.n_levels, res.n_comms)
    with Server(n_slots=3, hbm_budget=12e9, max_batch_entries=2_000_000, max_batch_graphs=64) as srv:
        rng = np.random.default_rng(1)
        for i in order:
            s, d, w, e, n = reqs[i]
            srv.submit(s, d, w, e, n, part_out=np.empty(n, np.int32), tag=int(i))
            if rng.random() < 0.3:
                time.sleep(0.002)       # arrivals spread while earlier batches run
        srv.drain(timeout_ms=300000)
        out = srv.poll(len(reqs) + 10)
        st = srv.stats()
        with pytest.raises(LvgError) as e:      # larger than one slot's share of the budget
            srv.submit(giants[0].src, giants[0].dst, giants[0].w, 10 ** 9, 10 ** 7)
        assert e.value.status == 3
    assert len(out) == len(reqs) and st["completed"] == len(reqs)
    assert st["batches"] < len(reqs)                      # requests were batched
    assert max(r.batch_graphs for r in out) > 1
    for r in out:
        part, q, nl, nc = alone[r.tag]
        assert r.status == 0, r
        np.testing.assert_array_equal(r.part, part, err_msg=f"request {r.tag}")
        assert r.q_final == q and r.n_levels == nl and r.n_comms == nc
        assert r.t_submit <= r.t_start <= r.t_done
    # a sample of the served results against the oracle (both giants included)
    hs, hd, hw = dg.to_host()
    host = {}
    for g in range(dg.n_graphs):
        e0, e1 = int(dg.entry_off[g]), int(dg.entry_off[g + 1])
        host[g] = (int(dg.vertex_off[g + 1] - dg.vertex_off[g]), hs[e0:e1], hd[e0:e1], hw[e0:e1])
    for k, x in enumerate(giants):
        host[dg.n_graphs + k] = (x.n_vertices, *x.to_host())
    by_tag = {r.tag: r for r in out}
    sample = list(np.random.default_rng(2).choice(dg.n_graphs, 10, replace=False)) + [dg.n_graphs, dg.n_graphs + 1]
    for t in sample:
        n, s_, d_, w_ = host[int(t)]
        ref = oracle.Run(n, s_, d_, w_)
        r = by_tag[int(t)]
        np.testing.assert_array_equal(r.part, ref.final, err_msg=f"request {t}")
        assert r.n_levels == len(ref.levels)
        assert r.q_final == pytest.approx(oracle.modularity_fp64(n, s_, d_, w_, ref.final), abs=1e-9)
