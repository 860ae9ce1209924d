"""ctypes binding of the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Loaded only by tests/, __graft_entry__.smoke() and bench.py's CPU legs, as the
checker or as the timed CPU baseline; the product never imports it.

PARITY UNPINNED: the reference cannot be built or run here and ships no golden
vectors; see the header of louvain_oracle.cpp.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liblvg_oracle.so")
_lib = None

FP64 = 0
REF32 = 1


class OrcConfig(ctypes.Structure):
    _fields_ = [
        ("mode", ctypes.c_int32),
        ("n_threads", ctypes.c_int32),
        ("pass_min_gain", ctypes.c_double),
        ("level_min_gain", ctypes.c_double),
        ("max_passes", ctypes.c_int32),
        ("max_levels", ctypes.c_int32),
    ]


def build():
    subprocess.check_call(["make", "-s", "-C", _HERE])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            build()
        L = ctypes.CDLL(_LIB)
        P = ctypes.c_void_p
        i32, i64, dbl = ctypes.c_int32, ctypes.c_int64, ctypes.c_double
        L.orc_csr_build.restype = P
        L.orc_csr_build.argtypes = [i32, i64, P, P, P]
        L.orc_csr_free.argtypes = [P]
        L.orc_csr_nnz.restype = i64
        L.orc_csr_nnz.argtypes = [P]
        L.orc_csr_m.restype = dbl
        L.orc_csr_m.argtypes = [P]
        L.orc_csr_get.argtypes = [P, P, P, P, P, P, P]
        L.orc_move_decide.argtypes = [P, P, P, P, P, P, P, ctypes.c_int]
        L.orc_move_decide_subset.restype = dbl
        L.orc_move_decide_subset.argtypes = [P, P, P, P, P, i64, P, P, P, ctypes.c_int]
        L.orc_tree_sum.restype = dbl
        L.orc_tree_sum.argtypes = [P, i64]
        L.orc_q_totals.restype = dbl
        L.orc_q_totals.argtypes = [P, P, i32, dbl]
        L.orc_renumber.restype = i32
        L.orc_renumber.argtypes = [i32, P, P]
        L.orc_induce.restype = i64
        L.orc_induce.argtypes = [i32, i64, P, P, P, P, P, P, P]
        L.orc_run_louvain.restype = P
        L.orc_run_louvain.argtypes = [i32, i64, P, P, P, ctypes.POINTER(OrcConfig)]
        L.orc_run_free.argtypes = [P]
        L.orc_run_status.restype = i32
        L.orc_run_status.argtypes = [P]
        L.orc_run_levels.restype = i32
        L.orc_run_levels.argtypes = [P]
        L.orc_run_level_info.argtypes = [P, i32, P, P, P, P, P, P, P]
        L.orc_run_level_partition.argtypes = [P, i32, P]
        L.orc_run_level_labels.argtypes = [P, i32, P]
        L.orc_run_level_qtrace.restype = i32
        L.orc_run_level_qtrace.argtypes = [P, i32, P, i32]
        L.orc_run_partition.argtypes = [P, i32, P]
        L.orc_run_seconds.restype = dbl
        L.orc_run_seconds.argtypes = [P]
        L.orc_run_pass_entries.restype = i64
        L.orc_run_pass_entries.argtypes = [P]
        L.orc_modularity_fp64.restype = dbl
        L.orc_modularity_fp64.argtypes = [i32, i64, P, P, P, P]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _edges(src, dst, w):
    return (np.ascontiguousarray(src, dtype=np.int32), np.ascontiguousarray(dst, dtype=np.int32),
            np.ascontiguousarray(w, dtype=np.float32))


class Csr:
    """Level CSR (NeighbourCompute.cu:42-117 + InitKernel.cu:154-243)."""

    def __init__(self, n_vertices, src, dst, w, arrays=True):
        """arrays=False copies out only off and k (large graphs: the
        entry arrays stay inside the library)."""
        s, d, ww = _edges(src, dst, w)
        self.V = int(n_vertices)
        self.h = lib().orc_csr_build(self.V, len(s), _p(s), _p(d), _p(ww))
        if not self.h:
            raise ValueError("oracle rejected the edge list")
        self.nnz = lib().orc_csr_nnz(self.h)
        self.m = lib().orc_csr_m(self.h)
        self.off = np.zeros(self.V + 1, np.int64)
        self.k = np.zeros(self.V, np.float64)
        if arrays:
            self.col = np.zeros(self.nnz, np.int32)
            self.w = np.zeros(self.nnz, np.float32)
            self.loopw = np.zeros(self.V, np.float32)
            self.has_loop = np.zeros(self.V, np.uint8)
            lib().orc_csr_get(self.h, _p(self.off), _p(self.col), _p(self.w), _p(self.k),
                              _p(self.loopw), _p(self.has_loop))
        else:
            lib().orc_csr_get(self.h, _p(self.off), None, None, _p(self.k), None, None)

    def decide(self, comm, tot, size, n_threads=0):
        comm = np.ascontiguousarray(comm, np.int32)
        tot = np.ascontiguousarray(tot, np.float64)
        size = np.ascontiguousarray(size, np.int32)
        nxt = np.zeros(self.V, np.int32)
        cand = np.zeros(self.V, np.int32)
        nseg = np.zeros(self.V, np.int32)
        lib().orc_move_decide(self.h, _p(comm), _p(tot), _p(size), _p(nxt), _p(cand), _p(nseg), n_threads)
        return nxt, cand, nseg

    def decide_subset(self, comm, tot, size, verts, n_threads=0):
        """decide() for the listed vertices only; returns the seconds the
        decisions took (timed inside the library, scratch set-up excluded)
        and next[] (entries of unlisted vertices are 0)."""
        comm = np.ascontiguousarray(comm, np.int32)
        tot = np.ascontiguousarray(tot, np.float64)
        size = np.ascontiguousarray(size, np.int32)
        verts = np.ascontiguousarray(verts, np.int32)
        nxt = np.zeros(self.V, np.int32)
        secs = lib().orc_move_decide_subset(self.h, _p(comm), _p(tot), _p(size), _p(verts), len(verts), _p(nxt),
                                            None, None, n_threads)
        return secs, nxt

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_csr_free(self.h)
            self.h = None


def tree_sum(x):
    x = np.ascontiguousarray(x, np.float64)
    return lib().orc_tree_sum(_p(x), len(x))


def q_totals(tot, inn, m):
    tot = np.ascontiguousarray(tot, np.float64)
    inn = np.ascontiguousarray(inn, np.float64)
    return lib().orc_q_totals(_p(tot), _p(inn), len(tot), float(m))


def renumber(comm):
    comm = np.ascontiguousarray(comm, np.int32)
    out = np.zeros(len(comm), np.int32)
    c = lib().orc_renumber(len(comm), _p(comm), _p(out))
    return out, int(c)


def induce(n_vertices, src, dst, w, part):
    s, d, ww = _edges(src, dst, w)
    part = np.ascontiguousarray(part, np.int32)
    n = lib().orc_induce(int(n_vertices), len(s), _p(s), _p(d), _p(ww), _p(part), None, None, None)
    os_, od, ow = np.zeros(n, np.int32), np.zeros(n, np.int32), np.zeros(n, np.float32)
    lib().orc_induce(int(n_vertices), len(s), _p(s), _p(d), _p(ww), _p(part), _p(os_), _p(od), _p(ow))
    return os_, od, ow


def modularity_fp64(n_vertices, src, dst, w, part):
    s, d, ww = _edges(src, dst, w)
    part = np.ascontiguousarray(part, np.int32)
    return lib().orc_modularity_fp64(int(n_vertices), len(s), _p(s), _p(d), _p(ww), _p(part))


class Level:
    pass


class Run:
    """Full dendrogram run (LouvainCPP.cpp:209-553)."""

    def __init__(self, n_vertices, src, dst, w, mode=FP64, n_threads=0, pass_min_gain=1e-7,
                 level_min_gain=1e-7, max_passes=-1, max_levels=-1):
        s, d, ww = _edges(src, dst, w)
        cfg = OrcConfig(mode, n_threads, pass_min_gain, level_min_gain, max_passes, max_levels)
        L = lib()
        h = L.orc_run_louvain(int(n_vertices), len(s), _p(s), _p(d), _p(ww), ctypes.byref(cfg))
        try:
            self.status = L.orc_run_status(h)
            self.seconds = L.orc_run_seconds(h)
            self.pass_entries = L.orc_run_pass_entries(h)
            self.levels = []
            for l in range(L.orc_run_levels(h)):
                V, E, nnz, C, P = (ctypes.c_int32(), ctypes.c_int64(), ctypes.c_int64(),
                                   ctypes.c_int32(), ctypes.c_int32())
                qs, ql = ctypes.c_double(), ctypes.c_double()
                L.orc_run_level_info(h, l, ctypes.byref(V), ctypes.byref(E), ctypes.byref(nnz),
                                     ctypes.byref(C), ctypes.byref(P), ctypes.byref(qs), ctypes.byref(ql))
                lv = Level()
                lv.n_vertices, lv.n_entries, lv.nnz = V.value, E.value, nnz.value
                lv.n_comms, lv.passes, lv.q_start, lv.q = C.value, P.value, qs.value, ql.value
                lv.part = np.zeros(lv.n_vertices, np.int32)
                L.orc_run_level_partition(h, l, _p(lv.part))
                lv.labels = np.zeros(lv.n_vertices, np.int32)
                L.orc_run_level_labels(h, l, _p(lv.labels))
                qt = np.zeros(lv.passes + 1, np.float64)
                n = L.orc_run_level_qtrace(h, l, _p(qt), len(qt))
                lv.qtrace = qt[:n]
                self.levels.append(lv)
            self.final = np.zeros(int(n_vertices), np.int32)
            if self.levels:
                L.orc_run_partition(h, len(self.levels) - 1, _p(self.final))
            self._compose = []
            for l in range(len(self.levels)):
                p = np.zeros(int(n_vertices), np.int32)
                L.orc_run_partition(h, l, _p(p))
                self._compose.append(p)
        finally:
            L.orc_run_free(h)

    def partition(self, level):
        return self._compose[level]
