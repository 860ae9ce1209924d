"""B200-native (sm_100a) Louvain hot path of LouvainGPU behind its phase API.

The compute runs in liblvg.so (hand-written CUDA for sm_100a, C ABI in
include/lvg.h); this package is the Python side of that ABI.
"""
from .louvain import (BatchResult, Louvain, LevelInfo, RunResult, count_partitions, kernel_launches,  # noqa: F401
                      pack_graphs, tune_pick)
from ._lib import LvgError  # noqa: F401
from .compat import start  # noqa: F401

__all__ = ["Louvain", "LevelInfo", "RunResult", "BatchResult", "pack_graphs", "count_partitions", "kernel_launches",
           "tune_pick", "LvgError", "start"]
