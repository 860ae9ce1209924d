"""Host-side API over liblvg: the reference's phase functions as methods.

    lv = Louvain()                       # one context = one device arena + stream
    lv.load_edges(src, dst, w, n)        # CalculateNeighbour + initCUDA
    res = lv.run()                       # generate_dendogram
    part = lv.partition()                # partitionAtLevel(last level)

The per-phase methods keep the reference's names and argument meaning
(LouvainCUDA/LouvainCPP.cpp:129-134): modularity (modularityCUDA),
one_level (oneLevelCUDA), renumber (renumberCUDA), induce (inducedGraphCUDA).
"""
import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


@dataclass
class LevelInfo:
    n_vertices: int
    n_entries: int
    nnz: int
    n_comms: int
    passes: int
    q_start: float
    q_level: float
    ms_passes: float
    ms_build: float = 0.0
    ms_renumber: float = 0.0
    ms_induce: float = 0.0


@dataclass
class RunResult:
    n_levels: int
    n_comms: int
    q_final: float
    pass_entries: int
    status: int


@dataclass
class BatchResult:
    """Per-graph results of a batched run (graph g owns vertices
    vertex_off[g]..vertex_off[g+1] of `partition`, ids local to the graph)."""
    partition: np.ndarray
    vertex_off: np.ndarray
    q_final: np.ndarray
    n_levels: np.ndarray
    n_comms: np.ndarray
    status: np.ndarray

    def __len__(self):
        return len(self.q_final)

    def part(self, g):
        return self.partition[self.vertex_off[g]:self.vertex_off[g + 1]]


def pack_graphs(graphs):
    """[(n, src, dst, w), ...] -> concatenated src, dst, w (local ids) and the
    entry and vertex offsets lvg_batch_run takes."""
    n = np.array([int(g[0]) for g in graphs], np.int64)
    cnt = np.array([len(g[1]) for g in graphs], np.int64)
    voff = np.zeros(len(graphs) + 1, np.int64)
    eoff = np.zeros(len(graphs) + 1, np.int64)
    np.cumsum(n, out=voff[1:])
    np.cumsum(cnt, out=eoff[1:])
    if voff[-1] >= 2 ** 31:
        raise ValueError("a batch holds at most 2^31-1 vertices")
    cat = (lambda k, t: np.concatenate([np.asarray(g[k], t) for g in graphs]) if graphs else np.zeros(0, t))
    return cat(1, np.int32), cat(2, np.int32), cat(3, np.float32), eoff, voff.astype(np.int32)


class Louvain:
    def __init__(self, device=0, pass_min_gain=1e-7, level_min_gain=1e-7, max_passes=-1, max_levels=-1,
                 arena_bytes=0, tile_max_degree=0, block_max_degree=0, passes_per_sync=0, use_graphs=True, l2_persist=True,
                 load_chunk_entries=0, coarsen_mode=0):
        L = _lib.load()
        cfg = _lib.LvgConfig()
        L.lvg_config_default(ctypes.byref(cfg))
        cfg.device = device
        cfg.pass_min_gain = pass_min_gain
        cfg.level_min_gain = level_min_gain
        cfg.max_passes = max_passes
        cfg.max_levels = max_levels
        cfg.arena_bytes = arena_bytes
        if tile_max_degree:
            cfg.tile_max_degree = tile_max_degree
        if block_max_degree:
            cfg.block_max_degree = block_max_degree
        if passes_per_sync:
            cfg.passes_per_sync = passes_per_sync
        cfg.use_graphs = 1 if use_graphs else 0
        cfg.l2_persist = 1 if l2_persist else 0
        cfg.load_chunk_entries = int(load_chunk_entries)
        cfg.coarsen_mode = int(coarsen_mode)
        self._L = L
        h = ctypes.c_void_p()
        _lib.check(None, L.lvg_create(ctypes.byref(cfg), ctypes.byref(h)))
        self._h = h
        self.n_vertices = 0

    def close(self):
        if getattr(self, "_h", None):
            self._L.lvg_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, status):
        _lib.check(self._h, status)

    # ------------------------------------------------------------------ load
    def load_edges(self, src, dst, w, n_vertices):
        src = np.ascontiguousarray(src, dtype=np.int32)
        dst = np.ascontiguousarray(dst, dtype=np.int32)
        w = np.ascontiguousarray(w, dtype=np.float32)
        if not (len(src) == len(dst) == len(w)):
            raise ValueError("src, dst and w must have the same length")
        self._check(self._L.lvg_load_edges(self._h, _p(src), _p(dst), _p(w), len(src), int(n_vertices)))
        self.n_vertices = int(n_vertices)

    def load_edges_ptr(self, src_ptr, dst_ptr, w_ptr, n_entries, n_vertices):
        """Edge list in host memory given by raw pointers (e.g. pinned torch tensors)."""
        self._check(self._L.lvg_load_edges(self._h, ctypes.c_void_p(src_ptr), ctypes.c_void_p(dst_ptr),
                                            ctypes.c_void_p(w_ptr), int(n_entries), int(n_vertices)))
        self.n_vertices = int(n_vertices)

    def load_edges_device(self, src_ptr, dst_ptr, w_ptr, n_entries, n_vertices):
        """Edge list already on the device (raw pointers, e.g. torch .data_ptr())."""
        self._check(self._L.lvg_load_edges_device(self._h, ctypes.c_void_p(src_ptr), ctypes.c_void_p(dst_ptr),
                                                   ctypes.c_void_p(w_ptr), int(n_entries), int(n_vertices)))
        self.n_vertices = int(n_vertices)

    def set_stream(self, stream_handle):
        self._check(self._L.lvg_set_stream(self._h, ctypes.c_void_p(stream_handle or 0)))

    # ------------------------------------------------------------------ phases
    def modularity(self):
        q = ctypes.c_double()
        self._check(self._L.lvg_modularity(self._h, ctypes.byref(q)))
        return q.value

    def one_level(self, lower):
        q, p = ctypes.c_double(), ctypes.c_int32()
        self._check(self._L.lvg_one_level(self._h, float(lower), ctypes.byref(q), ctypes.byref(p)))
        return q.value, p.value

    def renumber(self):
        V = self.csr_shape()[0]
        out = np.zeros(V, np.int32)
        c = ctypes.c_int32()
        self._check(self._L.lvg_renumber(self._h, _p(out), ctypes.byref(c)))
        return out, c.value

    def induce(self):
        self._check(self._L.lvg_induce(self._h))

    def run(self):
        r = _lib.LvgResult()
        self._check(self._L.lvg_run(self._h, ctypes.byref(r)))
        return RunResult(r.n_levels, r.n_comms, r.q_final, r.pass_entries, r.status)

    def run_batch(self, graphs=None, packed=None):
        """Whole dendrograms of many independent graphs in shared launches
        (lvg_batch_run).  `graphs`: [(n, src, dst, w), ...] with ids local to
        each graph, or `packed` = (src, dst, w, entry_off, vertex_off) as
        pack_graphs returns it.  Each graph's result equals its own run()."""
        src, dst, w, eoff, voff = packed if packed is not None else pack_graphs(graphs)
        src = np.ascontiguousarray(src, np.int32)
        dst = np.ascontiguousarray(dst, np.int32)
        w = np.ascontiguousarray(w, np.float32)
        eoff = np.ascontiguousarray(eoff, np.int64)
        voff = np.ascontiguousarray(voff, np.int32)
        G = len(voff) - 1
        part = np.zeros(int(voff[-1]), np.int32)
        q = np.zeros(G, np.float64)
        levels, comms, status = (np.zeros(G, np.int32) for _ in range(3))
        self._check(self._L.lvg_batch_run(self._h, _p(src), _p(dst), _p(w), _p(eoff), _p(voff), G, _p(part),
                                          _p(q), _p(levels), _p(comms), _p(status)))
        self.n_vertices = 0
        return BatchResult(part, voff, q, levels, comms, status)

    def run_batch_device(self, src_ptr, dst_ptr, w_ptr, entry_off, vertex_off):
        """run_batch over a packed list already in device memory (device
        pointers; e.g. graphgen.DeviceGraphs.src/dst/w and its offsets)."""
        eoff = np.ascontiguousarray(entry_off, np.int64)
        voff = np.ascontiguousarray(vertex_off, np.int32)
        G = len(voff) - 1
        part = np.zeros(int(voff[-1]), np.int32)
        q = np.zeros(G, np.float64)
        levels, comms, status = (np.zeros(G, np.int32) for _ in range(3))
        self._check(self._L.lvg_batch_run_device(self._h, ctypes.c_void_p(src_ptr), ctypes.c_void_p(dst_ptr),
                                                 ctypes.c_void_p(w_ptr), _p(eoff), _p(voff), G, _p(part), _p(q),
                                                 _p(levels), _p(comms), _p(status)))
        self.n_vertices = 0
        return BatchResult(part, voff, q, levels, comms, status)

    # ------------------------------------------------------------------ results
    @property
    def n_levels(self):
        n = ctypes.c_int32()
        self._check(self._L.lvg_num_levels(self._h, ctypes.byref(n)))
        return n.value

    def level_info(self, level):
        i = _lib.LvgLevelInfo()
        self._check(self._L.lvg_get_level_info(self._h, int(level), ctypes.byref(i)))
        return LevelInfo(i.n_vertices, i.n_entries, i.nnz, i.n_comms, i.passes, i.q_start, i.q_level, i.ms_passes,
                         i.ms_build, i.ms_renumber, i.ms_induce)

    def level_partition(self, level):
        out = np.zeros(self.level_info(level).n_vertices, np.int32)
        self._check(self._L.lvg_get_level_partition(self._h, int(level), _p(out)))
        return out

    def level_labels(self, level):
        out = np.zeros(self.level_info(level).n_vertices, np.int32)
        self._check(self._L.lvg_get_level_labels(self._h, int(level), _p(out)))
        return out

    def partition(self, level=-1, out=None):
        """Community of every input vertex at `level` (default: the last).
        `out`: optional destination -- an int32 numpy array of n_vertices, or
        a host tensor (e.g. pinned torch memory, for a fast copy) exposing
        data_ptr() and numel(); it is filled and returned."""
        if level < 0:
            level = self.n_levels - 1
        if out is None:
            out = np.zeros(self.n_vertices, np.int32)
        if hasattr(out, "data_ptr"):
            if out.numel() != self.n_vertices or out.element_size() != 4:
                raise ValueError("out must hold n_vertices int32 values")
            ptr = ctypes.c_void_p(out.data_ptr())
        else:
            if out.dtype != np.int32 or out.size != self.n_vertices or not out.flags.c_contiguous:
                raise ValueError("out must be a contiguous int32 array of n_vertices")
            ptr = _p(out)
        self._check(self._L.lvg_get_partition(self._h, int(level), ptr))
        return out

    def modularity_fp64(self, part):
        part = np.ascontiguousarray(part, np.int32)
        q = ctypes.c_double()
        self._check(self._L.lvg_modularity_fp64(self._h, _p(part), ctypes.byref(q)))
        return q.value

    def csr_shape(self):
        V, nnz, m = ctypes.c_int32(), ctypes.c_int64(), ctypes.c_double()
        self._check(self._L.lvg_get_csr(self._h, ctypes.byref(V), ctypes.byref(nnz), ctypes.byref(m),
                                        None, None, None, None, None, None))
        return V.value, nnz.value, m.value

    def csr(self):
        V, nnz, m = self.csr_shape()
        off = np.zeros(V + 1, np.int64)
        col = np.zeros(nnz, np.int32)
        w = np.zeros(nnz, np.float32)
        k = np.zeros(V, np.float64)
        loopw = np.zeros(V, np.float32)
        hl = np.zeros(V, np.uint8)
        Vc, nc, mc = ctypes.c_int32(), ctypes.c_int64(), ctypes.c_double()
        self._check(self._L.lvg_get_csr(self._h, ctypes.byref(Vc), ctypes.byref(nc), ctypes.byref(mc), _p(off),
                                        _p(col), _p(w), _p(k), _p(loopw), _p(hl)))
        return dict(V=V, nnz=nnz, m=m, off=off, col=col, w=w, k=k, loopw=loopw, has_loop=hl)

    def level_edges(self):
        """The current level's input list (src, dst, w); after induce() the
        coarse list of inducedGraphCUDA (InducedGraphKernel.cu:84-113)."""
        n = ctypes.c_int64()
        self._check(self._L.lvg_get_level_edges(self._h, ctypes.byref(n), None, None, None))
        src, dst = np.zeros(n.value, np.int32), np.zeros(n.value, np.int32)
        w = np.zeros(n.value, np.float32)
        self._check(self._L.lvg_get_level_edges(self._h, ctypes.byref(n), _p(src), _p(dst), _p(w)))
        return src, dst, w

    def set_communities(self, comm):
        comm = np.ascontiguousarray(comm, np.int32)
        self._check(self._L.lvg_set_communities(self._h, _p(comm)))

    def move_decide(self):
        V = self.csr_shape()[0]
        nxt = np.zeros(V, np.int32)
        cand = np.zeros(V, np.int32)
        self._check(self._L.lvg_move_decide(self._h, _p(nxt), _p(cand)))
        return nxt, cand

    def pass_times(self):
        n = ctypes.c_int32()
        self._check(self._L.lvg_last_pass_times(self._h, None, 0, ctypes.byref(n)))
        out = np.zeros(max(n.value, 1), np.float32)
        self._check(self._L.lvg_last_pass_times(self._h, _p(out), n.value, ctypes.byref(n)))
        return out[:n.value]

    def move_pass_times(self):
        """Device ms of the move kernels of each pass of the last one-level phase."""
        n = ctypes.c_int32()
        self._check(self._L.lvg_move_pass_times(self._h, None, 0, ctypes.byref(n)))
        out = np.zeros(max(n.value, 1), np.float32)
        self._check(self._L.lvg_move_pass_times(self._h, _p(out), n.value, ctypes.byref(n)))
        return out[:n.value]

    def move_stats(self):
        """(device ms of the move kernels, passes) of the last one-level phase(s)."""
        ms, n = ctypes.c_double(), ctypes.c_int64()
        self._check(self._L.lvg_move_stats(self._h, ctypes.byref(ms), ctypes.byref(n)))
        return ms.value, n.value

    # ------------------------------------------------------------------ autotuner
    def autotune(self, tile_max_degrees=None, block_max_degrees=None, reps=3, use_cache=False):
        """Time every (tile, block) degree-threshold pair on the loaded
        level-0 graph and keep the fastest (lvg_autotune).  Returns (best,
        points): best = (tile, block, move_ms, build_ms), points = every
        measured pair in that form (empty on a cache hit).  Results of the
        run do not depend on the pair."""
        sp = _lib.LvgTuneSpace()
        keep = []
        if tile_max_degrees is not None:
            t = np.ascontiguousarray(tile_max_degrees, np.int32)
            keep.append(t)
            sp.tile_max_degrees = t.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
            sp.n_tile = len(t)
        if block_max_degrees is not None:
            b = np.ascontiguousarray(block_max_degrees, np.int32)
            keep.append(b)
            sp.block_max_degrees = b.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
            sp.n_block = len(b)
        sp.reps = int(reps)
        sp.use_cache = 1 if use_cache else 0
        cap = 64
        pts = (_lib.LvgTunePoint * cap)()
        n = ctypes.c_int32()
        best = _lib.LvgTunePoint()
        self._check(self._L.lvg_autotune(self._h, ctypes.byref(sp), pts, cap, ctypes.byref(n), ctypes.byref(best)))
        row = lambda p: (p.tile_max_degree, p.block_max_degree, p.move_ms, p.build_ms)
        return row(best), [row(pts[i]) for i in range(min(n.value, cap))]

    def thresholds(self):
        """(tile_max_degree, block_max_degree) the context builds levels with."""
        t, b = ctypes.c_int32(), ctypes.c_int32()
        self._check(self._L.lvg_get_thresholds(self._h, ctypes.byref(t), ctypes.byref(b)))
        return t.value, b.value

    def memory(self):
        cap, peak = ctypes.c_int64(), ctypes.c_int64()
        self._check(self._L.lvg_memory(self._h, ctypes.byref(cap), ctypes.byref(peak)))
        return cap.value, peak.value


def kernel_launches():
    """CUDA kernels launched by liblvg in this process."""
    n = ctypes.c_int64()
    _lib.check(None, _lib.load().lvg_kernel_launches(ctypes.byref(n)))
    return n.value


def tune_pick(points, pref=(512, 4096)):
    """Index of the point the autotuner keeps among (tile, block, move_ms,
    build_ms) rows (lvg_tune_pick; host only): the fastest, or the preferred
    pair when within 2 % of it; -1 when no point was measured."""
    n = len(points)
    arr = (_lib.LvgTunePoint * max(n, 1))()
    for i, p in enumerate(points):
        arr[i].tile_max_degree, arr[i].block_max_degree = int(p[0]), int(p[1])
        arr[i].move_ms, arr[i].build_ms = float(p[2]), float(p[3]) if len(p) > 3 else 0.0
    b = ctypes.c_int32()
    _lib.check(None, _lib.load().lvg_tune_pick(arr, n, int(pref[0]), int(pref[1]), ctypes.byref(b)))
    return b.value


def count_partitions(part):
    """countPartitions (LouvainCPP.cpp:116-127): 1 + max community id."""
    part = np.ascontiguousarray(part, np.int32)
    c = ctypes.c_int32()
    _lib.check(None, _lib.load().lvg_count_partitions(_p(part), len(part), ctypes.byref(c)))
    return c.value
