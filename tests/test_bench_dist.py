"""The N>1 bench path on the CPU: world_size-2 gloo ranks check the
max-over-ranks timing and the whole-job rate the JSON line reports, and that
batched/serving ranks draw different graphs (sharding by graph, no
collective on the data path)."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        t = bench.max_over_ranks([10.0 + rank, 5.0 - rank], dist)
        rate = bench.whole_job_rate(1000.0, world, t[0])
        params, _ = bench.batched_plan(16, 3 + rank, 1e7)
        out[rank] = (t, rate, [p["seed"] for p in params])
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_time():
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(2, port, out), nprocs=2, join=True)
        r0, r1 = out[0], out[1]
    assert r0[0] == r1[0] == [11.0, 5.0]
    assert r0[1] == r1[1] == pytest.approx(1000.0 * 2 / 0.011)
    assert r0[2] != r1[2]      # each rank runs its own graphs


def test_single_process_needs_no_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks([3.0, 4.0], None) == [3.0, 4.0]
    assert bench.whole_job_rate(10.0, 1, 1000.0) == 10.0
