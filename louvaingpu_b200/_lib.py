"""ctypes binding of liblvg.so (the C ABI declared in include/lvg.h).

There is no fallback: if the CUDA library is missing or cannot be loaded the
import of the product path raises.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liblvg.so")
GEN_PATH = os.path.join(HERE, "liblvggen.so")

LVG_OK = 0
STATUS_NAMES = {
    0: "LVG_OK", 1: "LVG_ERR_INVALID_ARG", 2: "LVG_ERR_OOM", 3: "LVG_ERR_CAPACITY",
    4: "LVG_ERR_NOT_CONVERGED", 5: "LVG_ERR_CUDA", 6: "LVG_ERR_STATE",
}


class LvgError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


class LvgConfig(ctypes.Structure):
    _fields_ = [
        ("device", ctypes.c_int32),
        ("pass_min_gain", ctypes.c_double),
        ("level_min_gain", ctypes.c_double),
        ("max_passes", ctypes.c_int32),
        ("max_levels", ctypes.c_int32),
        ("arena_bytes", ctypes.c_int64),
        ("tile_max_degree", ctypes.c_int32),
        ("block_max_degree", ctypes.c_int32),
        ("passes_per_sync", ctypes.c_int32),
        ("use_graphs", ctypes.c_int32),
        ("l2_persist", ctypes.c_int32),
        ("load_chunk_entries", ctypes.c_int64),
        ("coarsen_mode", ctypes.c_int32),
    ]


class LvgLevelInfo(ctypes.Structure):
    _fields_ = [
        ("n_vertices", ctypes.c_int32),
        ("n_entries", ctypes.c_int64),
        ("nnz", ctypes.c_int64),
        ("n_comms", ctypes.c_int32),
        ("passes", ctypes.c_int32),
        ("q_start", ctypes.c_double),
        ("q_level", ctypes.c_double),
        ("ms_build", ctypes.c_double),
        ("ms_passes", ctypes.c_double),
        ("ms_renumber", ctypes.c_double),
        ("ms_induce", ctypes.c_double),
    ]


class LvgResult(ctypes.Structure):
    _fields_ = [
        ("n_levels", ctypes.c_int32),
        ("n_comms", ctypes.c_int32),
        ("q_final", ctypes.c_double),
        ("pass_entries", ctypes.c_int64),
        ("status", ctypes.c_int32),
    ]


class LvgServeResult(ctypes.Structure):
    _fields_ = [
        ("id", ctypes.c_int64),
        ("tag", ctypes.c_int64),
        ("status", ctypes.c_int32),
        ("n_levels", ctypes.c_int32),
        ("n_comms", ctypes.c_int32),
        ("batch_graphs", ctypes.c_int32),
        ("q_final", ctypes.c_double),
        ("t_submit_ns", ctypes.c_int64),
        ("t_start_ns", ctypes.c_int64),
        ("t_done_ns", ctypes.c_int64),
    ]


class LvgTunePoint(ctypes.Structure):
    _fields_ = [
        ("tile_max_degree", ctypes.c_int32),
        ("block_max_degree", ctypes.c_int32),
        ("move_ms", ctypes.c_float),
        ("build_ms", ctypes.c_float),
    ]


class LvgTuneSpace(ctypes.Structure):
    _fields_ = [
        ("tile_max_degrees", ctypes.POINTER(ctypes.c_int32)),
        ("n_tile", ctypes.c_int32),
        ("block_max_degrees", ctypes.POINTER(ctypes.c_int32)),
        ("n_block", ctypes.c_int32),
        ("reps", ctypes.c_int32),
        ("use_cache", ctypes.c_int32),
    ]


# Every entry point declared in include/lvg.h, with its ctypes signature.
P = ctypes.c_void_p
i32, i64, dbl = ctypes.c_int32, ctypes.c_int64, ctypes.c_double
SIGNATURES = {
    "lvg_config_default": (i32, [ctypes.POINTER(LvgConfig)]),
    "lvg_create": (i32, [ctypes.POINTER(LvgConfig), ctypes.POINTER(P)]),
    "lvg_destroy": (i32, [P]),
    "lvg_last_error": (ctypes.c_char_p, [P]),
    "lvg_status_string": (ctypes.c_char_p, [i32]),
    "lvg_set_stream": (i32, [P, P]),
    "lvg_load_edges": (i32, [P, P, P, P, i64, i32]),
    "lvg_load_edges_device": (i32, [P, P, P, P, i64, i32]),
    "lvg_modularity": (i32, [P, ctypes.POINTER(dbl)]),
    "lvg_one_level": (i32, [P, dbl, ctypes.POINTER(dbl), ctypes.POINTER(i32)]),
    "lvg_renumber": (i32, [P, P, ctypes.POINTER(i32)]),
    "lvg_induce": (i32, [P]),
    "lvg_run": (i32, [P, ctypes.POINTER(LvgResult)]),
    "lvg_num_levels": (i32, [P, ctypes.POINTER(i32)]),
    "lvg_get_level_info": (i32, [P, i32, ctypes.POINTER(LvgLevelInfo)]),
    "lvg_get_level_partition": (i32, [P, i32, P]),
    "lvg_get_level_labels": (i32, [P, i32, P]),
    "lvg_get_partition": (i32, [P, i32, P]),
    "lvg_count_partitions": (i32, [P, i64, ctypes.POINTER(i32)]),
    "lvg_modularity_fp64": (i32, [P, P, ctypes.POINTER(dbl)]),
    "lvg_get_csr": (i32, [P, ctypes.POINTER(i32), ctypes.POINTER(i64), ctypes.POINTER(dbl), P, P, P, P, P, P]),
    "lvg_get_level_edges": (i32, [P, ctypes.POINTER(i64), P, P, P]),
    "lvg_debug_radix_hold": (i32, [i32, i64]),
    "lvg_set_communities": (i32, [P, P]),
    "lvg_move_decide": (i32, [P, P, P]),
    "lvg_last_pass_times": (i32, [P, P, i32, ctypes.POINTER(i32)]),
    "lvg_move_stats": (i32, [P, ctypes.POINTER(dbl), ctypes.POINTER(i64)]),
    "lvg_move_pass_times": (i32, [P, P, i32, ctypes.POINTER(i32)]),
    "lvg_kernel_launches": (i32, [ctypes.POINTER(i64)]),
    "lvg_memory": (i32, [P, ctypes.POINTER(i64), ctypes.POINTER(i64)]),
    "lvg_batch_run": (i32, [P, P, P, P, P, P, i32, P, P, P, P, P]),
    "lvg_batch_run_device": (i32, [P, P, P, P, P, P, i32, P, P, P, P, P]),
    "lvg_batch_run_graphs": (i32, [P, i32, P, P, P, P, P, P, P, P, P, P]),
    "lvg_batch_footprint": (i32, [i64, i64, i32, ctypes.POINTER(i64)]),
    "lvg_reserve": (i32, [P, i64]),
    "lvg_server_create": (i32, [ctypes.POINTER(LvgConfig), i32, i64, i64, i32, ctypes.POINTER(P)]),
    "lvg_server_submit": (i32, [P, P, P, P, i64, i32, P, i64, ctypes.POINTER(i64)]),
    "lvg_server_poll": (i32, [P, ctypes.POINTER(LvgServeResult), i32, ctypes.POINTER(i32)]),
    "lvg_server_drain": (i32, [P, i64]),
    "lvg_server_stats": (i32, [P, ctypes.POINTER(i64), ctypes.POINTER(i64), ctypes.POINTER(i64),
                               ctypes.POINTER(i64)]),
    "lvg_server_last_error": (ctypes.c_char_p, [P]),
    "lvg_server_destroy": (i32, [P]),
    "lvg_modularity_fp64_noalloc": (i32, [P, P, P, i64, P, i32, P, ctypes.POINTER(dbl)]),
    "lvg_autotune": (i32, [P, ctypes.POINTER(LvgTuneSpace), ctypes.POINTER(LvgTunePoint), i32,
                           ctypes.POINTER(i32), ctypes.POINTER(LvgTunePoint)]),
    "lvg_get_thresholds": (i32, [P, ctypes.POINTER(i32), ctypes.POINTER(i32)]),
    "lvg_tune_pick": (i32, [ctypes.POINTER(LvgTunePoint), i32, i32, i32, ctypes.POINTER(i32)]),
    "lvg_tune_cache_clear": (i32, []),
}

# Device generators declared in include/lvg_gen.h (same library).
GEN_SIGNATURES = {
    "lvg_gen_rmat": (i32, [i32, P, i32, i32, dbl, dbl, dbl, i32, i32, ctypes.c_uint64, ctypes.POINTER(P)]),
    "lvg_gen_sbm_batch": (i32, [i32, P, i32, P, P, P, P, i32, i32, P, ctypes.POINTER(P)]),
    "lvg_dgraph_info": (i32, [P, ctypes.POINTER(i32), ctypes.POINTER(i64), ctypes.POINTER(i64)]),
    "lvg_dgraph_arrays": (i32, [P, ctypes.POINTER(P), ctypes.POINTER(P), ctypes.POINTER(P)]),
    "lvg_dgraph_offsets": (i32, [P, P, P]),
    "lvg_dgraph_copy_to_host": (i32, [P, P, P, P]),
    "lvg_dgraph_free": (None, [P]),
    "lvg_gen_last_error": (ctypes.c_char_p, []),
}

_lib = None


def load():
    """Load liblvg.so and declare its signatures; raises if it is missing."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m louvaingpu_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in list(SIGNATURES.items()) + list(GEN_SIGNATURES.items()):
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(ctx, status):
    if status != LVG_OK:
        msg = load().lvg_last_error(ctx).decode() if ctx else ""
        raise LvgError(status, msg)
