"""lvg_modularity_fp64_noalloc: the FP64 modularity for callers that cannot
allocate device memory when they need it (code inside a CUDA-graph stream
capture, serving loops that own all free HBM, paths that cannot take the
synchronisation of cudaMalloc/cudaFree).  It must give the same value as the
allocating entry point lvg_modularity_fp64, call after call, without
changing the device's free memory.  Collected last on purpose: a failure here
leaves every other test already run."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-9          # the Q tolerance of the other GPU tests
MAX_COMMS = 1 << 18  # LVG_NOALLOC_MAX_COMMS


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def test_noalloc_modularity_matches_allocating_entry_point(gen):
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for gpu tests")
    from louvaingpu_b200 import Louvain, _lib
    n, s, d, w, truth = gen.sbm(20000, 50, 0.02, 0.0005, 1, 3, seed=12, with_truth=True)
    with Louvain() as lv:
        lv.load_edges(s, d, w, n)
        lv.run()
        found = lv.partition()
        parts = [np.arange(n, dtype=np.int32), found, truth.astype(np.int32)]
        expected = [lv.modularity_fp64(p) for p in parts]
    L = _lib.load()
    ds, dd, dw = (torch.from_numpy(x).cuda() for x in (s, d, w))
    dparts = [torch.from_numpy(p).cuda() for p in parts]
    torch.cuda.synchronize()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    free_before = None
    for k, (p, dp) in enumerate(zip(parts, dparts)):
        q = ctypes.c_double()
        st = L.lvg_modularity_fp64_noalloc(_ptr(ds), _ptr(dd), _ptr(dw), len(s), _ptr(dp), int(p.max()) + 1,
                                           stream, ctypes.byref(q))
        assert st == 0, st
        assert abs(q.value - expected[k]) <= TOL, (k, q.value, expected[k])
        free_now = torch.cuda.mem_get_info()[0]
        if free_before is not None:     # after the first call nothing more is allocated
            assert free_now == free_before
        free_before = free_now
    # the same partition twice in a row gives the same value (the shared array is cleared per call)
    q1, q2 = ctypes.c_double(), ctypes.c_double()
    for q in (q1, q2):
        assert L.lvg_modularity_fp64_noalloc(_ptr(ds), _ptr(dd), _ptr(dw), len(s), _ptr(dparts[1]),
                                             int(parts[1].max()) + 1, stream, ctypes.byref(q)) == 0
    assert q1.value == q2.value
    # more communities than the fixed array holds: a clear error, no launch
    q = ctypes.c_double()
    assert L.lvg_modularity_fp64_noalloc(_ptr(ds), _ptr(dd), _ptr(dw), len(s), _ptr(dparts[0]), MAX_COMMS + 1,
                                         stream, ctypes.byref(q)) == 3
