"""Seeded synthetic graphs of the benchmark shapes (host generators in C++).

Each function returns (n_vertices, src, dst, w) as numpy arrays: a symmetric
edge list (both directions), no self loops, duplicates merged, sorted.
"""
import ctypes
import os

import numpy as np

from ._lib import GEN_PATH

_gen = None


def _load():
    global _gen
    if _gen is None:
        if not os.path.exists(GEN_PATH):
            from .build import build_gen
            build_gen()
        L = ctypes.CDLL(GEN_PATH)
        P, i32, i64, dbl, u64 = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_double, ctypes.c_uint64
        L.lvggen_sbm.restype = P
        L.lvggen_sbm.argtypes = [i32, i32, dbl, dbl, i32, i32, u64]
        L.lvggen_lfr.restype = P
        L.lvggen_lfr.argtypes = [i32, dbl, i32, i32, dbl, i32, i32, dbl, u64]
        L.lvggen_rmat.restype = P
        L.lvggen_rmat.argtypes = [i32, i32, dbl, dbl, dbl, i32, i32, u64]
        L.lvggen_n_vertices.restype = i32
        L.lvggen_n_vertices.argtypes = [P]
        L.lvggen_n_entries.restype = i64
        L.lvggen_n_entries.argtypes = [P]
        L.lvggen_copy.argtypes = [P, P, P, P]
        L.lvggen_truth.argtypes = [P, P]
        L.lvggen_free.argtypes = [P]
        _gen = L
    return _gen


def _take(h, with_truth=False):
    L = _load()
    if not h:
        raise ValueError("generator rejected its parameters")
    try:
        n = L.lvggen_n_vertices(h)
        E = L.lvggen_n_entries(h)
        src = np.zeros(E, np.int32)
        dst = np.zeros(E, np.int32)
        w = np.zeros(E, np.float32)
        c = lambda a: a.ctypes.data_as(ctypes.c_void_p)
        L.lvggen_copy(h, c(src), c(dst), c(w))
        truth = None
        if with_truth:
            truth = np.zeros(n, np.int32)
            L.lvggen_truth(h, c(truth))
    finally:
        L.lvggen_free(h)
    return (n, src, dst, w, truth) if with_truth else (n, src, dst, w)


def sbm(n, blocks, p_in, p_out, w_lo=1, w_hi=1, seed=0, with_truth=False):
    """Planted-partition SBM with near-equal blocks."""
    return _take(_load().lvggen_sbm(int(n), int(blocks), float(p_in), float(p_out), int(w_lo), int(w_hi),
                                    int(seed)), with_truth)


def sbm_10k(seed=0):
    """n=10,000 in 100 blocks of 100, p_in=0.1, p_out=0.0006, unit weights."""
    return sbm(10000, 100, 0.1, 0.0006, 1, 1, seed)


def lfr(n=1 << 20, deg_exp=2.5, d_min=5, d_max=5000, com_exp=1.5, c_min=50, c_max=50000, mu=0.3, seed=1,
        with_truth=False):
    """LFR-style power-law graph (defaults: the n=2^20 benchmark shape)."""
    return _take(_load().lvggen_lfr(int(n), float(deg_exp), int(d_min), int(d_max), float(com_exp), int(c_min),
                                    int(c_max), float(mu), int(seed)), with_truth)


def rmat(scale, edge_factor=16, a=0.57, b=0.19, c=0.19, w_lo=1, w_hi=16, seed=2):
    """R-MAT graph (host generator; large scales use the device generator)."""
    return _take(_load().lvggen_rmat(int(scale), int(edge_factor), float(a), float(b), float(c), int(w_lo),
                                     int(w_hi), int(seed)))


def batched_sbm_params(count, seed=3, n_lo=64, n_hi=200000):
    """Per-graph SBM parameters of the batched shape: n log-uniform in
    [n_lo, n_hi], 4-400 blocks, average degree uniform in [8, 32], 70% intra
    edges, integer weights 1..4.

    The block count drawn in [4, 400] is capped so that a block holds at least
    0.7 d + 1 vertices: then 70 % of the degree fits inside the block
    (p_in <= 1).  Graphs too small for 4 such blocks (n < 4 (0.7 d + 1), at
    most 94 vertices) keep 4 blocks and take p_in = 1, below the target."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        n = int(round(np.exp(rng.uniform(np.log(n_lo), np.log(n_hi)))))
        drawn = int(rng.integers(4, 401))
        d = float(rng.uniform(8, 32))
        cap = int(n // (0.7 * d + 1.0))
        blocks = max(min(4, max(1, n // 4)), min(drawn, cap))
        s = n / blocks
        p_in = min(1.0, 0.7 * d / max(s - 1, 1))
        p_out = min(1.0, 0.3 * d / max(n - s, 1))
        out.append(dict(n=n, blocks=blocks, p_in=p_in, p_out=p_out, w_lo=1, w_hi=4,
                        seed=int(rng.integers(0, 2**62))))
    return out


# ---------------------------------------------------------------- device side
class DeviceGraphs:
    """Graph(s) generated into device memory by liblvg (include/lvg_gen.h).

    src/dst/w are device pointers (ints) of the packed list; entry_off and
    vertex_off are host arrays (n_graphs + 1).  Freed by close() or on
    garbage collection."""

    def __init__(self, handle):
        from . import _lib
        self._L = _lib.load()
        self._h = handle
        g, e, v = ctypes.c_int32(), ctypes.c_int64(), ctypes.c_int64()
        self._L.lvg_dgraph_info(self._h, ctypes.byref(g), ctypes.byref(e), ctypes.byref(v))
        self.n_graphs, self.n_entries, self.n_vertices = g.value, e.value, v.value
        s, d, w = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
        self._L.lvg_dgraph_arrays(self._h, ctypes.byref(s), ctypes.byref(d), ctypes.byref(w))
        self.src, self.dst, self.w = s.value or 0, d.value or 0, w.value or 0
        self.entry_off = np.zeros(self.n_graphs + 1, np.int64)
        self.vertex_off = np.zeros(self.n_graphs + 1, np.int32)
        self._L.lvg_dgraph_offsets(self._h, self.entry_off.ctypes.data_as(ctypes.c_void_p),
                                   self.vertex_off.ctypes.data_as(ctypes.c_void_p))

    def close(self):
        if getattr(self, "_h", None):
            self._L.lvg_dgraph_free(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def graph_ptrs(self, g):
        """(src, dst, w, n_entries, n_vertices) of graph g: device pointers."""
        e0, e1 = int(self.entry_off[g]), int(self.entry_off[g + 1])
        return (self.src + 4 * e0, self.dst + 4 * e0, self.w + 4 * e0, e1 - e0,
                int(self.vertex_off[g + 1] - self.vertex_off[g]))

    def to_host(self):
        """Copy the packed list back: (src, dst, w) numpy arrays."""
        src, dst = np.zeros(self.n_entries, np.int32), np.zeros(self.n_entries, np.int32)
        w = np.zeros(self.n_entries, np.float32)
        vp = lambda x: x.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
        _gen_check(self._L.lvg_dgraph_copy_to_host(self._h, vp(src), vp(dst), vp(w)))
        return src, dst, w


def _gen_check(status):
    from . import _lib
    if status != 0:
        raise _lib.LvgError(status, _lib.load().lvg_gen_last_error().decode())


def rmat_device(scale, edge_factor=16, a=0.57, b=0.19, c=0.19, w_lo=1, w_hi=16, seed=2, device=0, stream=None):
    """R-MAT generated on the device; equals rmat() with the same arguments."""
    from . import _lib
    h = ctypes.c_void_p()
    _gen_check(_lib.load().lvg_gen_rmat(int(device), ctypes.c_void_p(stream or 0), int(scale), int(edge_factor),
                                        float(a), float(b), float(c), int(w_lo), int(w_hi), int(seed),
                                        ctypes.byref(h)))
    return DeviceGraphs(h)


def sbm_batch_device(params, w_lo=1, w_hi=4, device=0, stream=None):
    """Packed batch of SBMs on the device; params as batched_sbm_params gives
    them (dicts with n, blocks, p_in, p_out, seed)."""
    from . import _lib
    G = len(params)
    n = np.array([p["n"] for p in params], np.int32)
    bl = np.array([p["blocks"] for p in params], np.int32)
    pi = np.array([p["p_in"] for p in params], np.float64)
    po = np.array([p["p_out"] for p in params], np.float64)
    sd = np.array([p["seed"] for p in params], np.uint64)
    h = ctypes.c_void_p()
    vp = lambda x: x.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    _gen_check(_lib.load().lvg_gen_sbm_batch(int(device), ctypes.c_void_p(stream or 0), G, vp(n), vp(bl), vp(pi),
                                             vp(po), int(w_lo), int(w_hi), vp(sd), ctypes.byref(h)))
    return DeviceGraphs(h)
