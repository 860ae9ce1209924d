"""Request server over device-resident graphs (lvg_server_* in include/lvg.h).

    srv = Server(n_slots=4, hbm_budget=150e9)
    rid = srv.submit(src_ptr, dst_ptr, w_ptr, n_entries, n_vertices, part_out=np.empty(n, np.int32))
    srv.drain()
    for r in srv.poll(): ...       # ServeResult with the request's partition in part_out

Slots are worker contexts on their own threads and streams; a free slot takes
the queued requests in arrival order as one batched run (continuous
batching), so every result equals the graph's own run.
"""
import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib


@dataclass
class ServeResult:
    id: int
    tag: int
    status: int
    n_levels: int
    n_comms: int
    batch_graphs: int
    q_final: float
    t_submit: float     # seconds since the server started
    t_start: float
    t_done: float
    part: np.ndarray = None

    @property
    def latency(self):
        return self.t_done - self.t_submit


class Server:
    def __init__(self, n_slots=4, hbm_budget=150e9, max_batch_entries=2.5e8, max_batch_graphs=4096, device=0,
                 pass_min_gain=1e-7, level_min_gain=1e-7, tile_max_degree=0, block_max_degree=0):
        """tile_max_degree / block_max_degree: the slots' degree thresholds
        (0: the defaults), e.g. a pair Louvain.autotune picked on a
        representative graph."""
        self._L = _lib.load()
        cfg = _lib.LvgConfig()
        _lib.check(None, self._L.lvg_config_default(ctypes.byref(cfg)))
        cfg.device = int(device)
        cfg.pass_min_gain = float(pass_min_gain)
        cfg.level_min_gain = float(level_min_gain)
        if tile_max_degree:
            cfg.tile_max_degree = int(tile_max_degree)
        if block_max_degree:
            cfg.block_max_degree = int(block_max_degree)
        h = ctypes.c_void_p()
        st = self._L.lvg_server_create(ctypes.byref(cfg), int(n_slots), int(hbm_budget), int(max_batch_entries),
                                       int(max_batch_graphs), ctypes.byref(h))
        if st != 0:
            raise _lib.LvgError(st, "lvg_server_create failed")
        self._h = h
        self._parts = {}

    def _check(self, st):
        if st != 0:
            raise _lib.LvgError(st, self._L.lvg_server_last_error(self._h).decode())

    def submit(self, src_ptr, dst_ptr, w_ptr, n_entries, n_vertices, part_out=None, tag=0):
        """Queue a graph whose device arrays are complete (synchronise the
        producing stream first) and stay alive until its result is polled."""
        if part_out is not None:
            if part_out.dtype != np.int32 or len(part_out) < n_vertices or not part_out.flags.c_contiguous:
                raise ValueError("part_out must be a contiguous int32 array of n_vertices")
            pp = part_out.ctypes.data_as(ctypes.c_void_p)
        else:
            pp = None
        rid = ctypes.c_int64()
        self._check(self._L.lvg_server_submit(self._h, ctypes.c_void_p(src_ptr), ctypes.c_void_p(dst_ptr),
                                              ctypes.c_void_p(w_ptr), int(n_entries), int(n_vertices), pp,
                                              int(tag), ctypes.byref(rid)))
        self._parts[rid.value] = part_out
        return rid.value

    def poll(self, max_results=4096):
        buf = (_lib.LvgServeResult * max_results)()
        n = ctypes.c_int32()
        self._check(self._L.lvg_server_poll(self._h, buf, int(max_results), ctypes.byref(n)))
        out = []
        for r in buf[:n.value]:
            out.append(ServeResult(r.id, r.tag, r.status, r.n_levels, r.n_comms, r.batch_graphs, r.q_final,
                                   r.t_submit_ns * 1e-9, r.t_start_ns * 1e-9, r.t_done_ns * 1e-9,
                                   self._parts.pop(r.id, None)))
        return out

    def drain(self, timeout_ms=-1):
        self._check(self._L.lvg_server_drain(self._h, int(timeout_ms)))

    def stats(self):
        v = [ctypes.c_int64() for _ in range(4)]
        self._check(self._L.lvg_server_stats(self._h, *[ctypes.byref(x) for x in v]))
        return dict(zip(("submitted", "completed", "batches", "reserved_bytes"), (x.value for x in v)))

    def close(self):
        if getattr(self, "_h", None):
            self._L.lvg_server_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        self.close()
