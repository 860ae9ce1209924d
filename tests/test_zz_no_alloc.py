"""lvg_modularity_fp64_noalloc: the FP64 modularity for callers that cannot
allocate device memory when they need the value -- a serving process whose
caching allocator already holds all free HBM, or a latency-bound loop that
cannot take the device-wide synchronisation of cudaMalloc/cudaFree.  It must
give the oracle's value and the allocating entry point lvg_modularity_fp64's,
call after call, without changing the device's free memory.  Collected last
on purpose: a failure here leaves every other test already run."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-9          # the Q tolerance of the other GPU tests
MAX_COMMS = 1 << 18  # LVG_NOALLOC_MAX_COMMS
OK, INVALID_ARG, CAPACITY = 0, 1, 3


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _noalloc(L, ds, dd, dw, E, dp, C, stream):
    q = ctypes.c_double()
    st = L.lvg_modularity_fp64_noalloc(_ptr(ds), _ptr(dd), _ptr(dw), E, _ptr(dp), int(C), stream, ctypes.byref(q))
    return st, q.value


def test_noalloc_modularity_matches_allocating_entry_point(gen, oracle):
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for gpu tests")
    from louvaingpu_b200 import Louvain, _lib
    n, s, d, w, truth = gen.sbm(20000, 50, 0.02, 0.0005, 1, 3, seed=12, with_truth=True)
    rng = np.random.default_rng(5)
    lv = Louvain()
    try:
        lv.load_edges(s, d, w, n)
        lv.run()
        found = lv.partition()
        # singletons (20000 communities: global atomics), the found partition,
        # the planted one, 3500 communities (shared-memory sums above 48 KB)
        # and 4096 (the largest shared-memory case)
        parts = [np.arange(n, dtype=np.int32), found, truth.astype(np.int32),
                 (np.arange(n) % 3500).astype(np.int32), rng.integers(0, 4096, n).astype(np.int32)]
        parts[4][:4096] = np.arange(4096)
        expected = [oracle.modularity_fp64(n, s, d, w, p) for p in parts]
        for p, q in zip(parts, expected):
            assert abs(lv.modularity_fp64(p) - q) <= TOL
        L = _lib.load()
        ds, dd, dw = (torch.from_numpy(x).cuda() for x in (s, d, w))
        dparts = [torch.from_numpy(p).cuda() for p in parts]
        torch.cuda.synchronize()
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        free_before = None
        for k, (p, dp) in enumerate(zip(parts, dparts)):
            st, q = _noalloc(L, ds, dd, dw, len(s), dp, int(p.max()) + 1, stream)
            assert st == OK, st
            assert abs(q - expected[k]) <= TOL, (k, q, expected[k])
            free_now = torch.cuda.mem_get_info()[0]
            if free_before is not None:     # after the first call nothing more is allocated
                assert free_now == free_before
            free_before = free_now
        # two calls in a row give the same value (the shared array is cleared per call)
        for k in (1, 3):
            a = _noalloc(L, ds, dd, dw, len(s), dparts[k], int(parts[k].max()) + 1, stream)
            b = _noalloc(L, ds, dd, dw, len(s), dparts[k], int(parts[k].max()) + 1, stream)
            assert a == b and a[0] == OK
        # alternating with the allocating entry point at more communities: the
        # shared-memory limit one path raised is never lowered by the other
        for _ in range(2):
            assert abs(lv.modularity_fp64(parts[4]) - expected[4]) <= TOL
            st, q = _noalloc(L, ds, dd, dw, len(s), dparts[3], 3500, stream)
            assert st == OK and abs(q - expected[3]) <= TOL
            assert abs(lv.modularity_fp64(parts[4]) - expected[4]) <= TOL
        # ids outside [0, n_comms) are skipped by the kernels and reported
        st, _ = _noalloc(L, ds, dd, dw, len(s), dparts[3], 3000, stream)
        assert st == INVALID_ARG
        bad = parts[1].copy()
        bad[7] = -1
        st, _ = _noalloc(L, ds, dd, dw, len(s), torch.from_numpy(bad).cuda(), int(parts[1].max()) + 1, stream)
        assert st == INVALID_ARG
        # the next valid call is unaffected by the flag of the last one
        st, q = _noalloc(L, ds, dd, dw, len(s), dparts[1], int(parts[1].max()) + 1, stream)
        assert st == OK and abs(q - expected[1]) <= TOL
        # more communities than the fixed array holds: a clear error, no launch
        st, _ = _noalloc(L, ds, dd, dw, len(s), dparts[0], MAX_COMMS + 1, stream)
        assert st == CAPACITY
    finally:
        lv.close()
