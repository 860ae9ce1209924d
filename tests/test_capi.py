"""CPU checks of the drop-in boundary: liblvg.so loads and exports exactly the
entry points include/lvg.h declares; argument errors are reported as status
codes without touching a GPU."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(lvg_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    from louvaingpu_b200 import build, _lib
    build.build_lvg()
    return _lib.load()


def test_header_declares_entry_points():
    names = declared("lvg.h")
    for must in ["lvg_create", "lvg_destroy", "lvg_load_edges", "lvg_modularity", "lvg_one_level",
                 "lvg_renumber", "lvg_induce", "lvg_run", "lvg_get_partition", "lvg_last_error"]:
        assert must in names


def test_library_exports_every_declared_symbol(lib):
    for header in ("lvg.h", "lvg_gen.h"):
        for name in declared(header):
            assert hasattr(lib, name), name


def test_python_binding_covers_every_symbol():
    from louvaingpu_b200 import _lib
    assert sorted(_lib.SIGNATURES) == declared("lvg.h")
    assert sorted(_lib.GEN_SIGNATURES) == declared("lvg_gen.h")


def test_generator_argument_errors_without_device(lib):
    out = ctypes.c_void_p()
    assert lib.lvg_gen_rmat(0, None, 0, 16, 0.57, 0.19, 0.19, 1, 16, 1, ctypes.byref(out)) == 1
    assert lib.lvg_gen_rmat(0, None, 10, 16, 0.57, 0.19, 0.19, 1, 16, 1, None) == 1
    assert lib.lvg_gen_sbm_batch(0, None, 0, None, None, None, None, 1, 4, None, ctypes.byref(out)) == 1
    assert lib.lvg_dgraph_info(None, None, None, None) == 1


def test_status_strings_and_config_defaults(lib):
    from louvaingpu_b200 import _lib
    assert lib.lvg_status_string(0) == b"ok"
    assert lib.lvg_status_string(4) == b"not converged"
    cfg = _lib.LvgConfig()
    assert lib.lvg_config_default(ctypes.byref(cfg)) == 0
    assert cfg.pass_min_gain == 1e-7 and cfg.level_min_gain == 1e-7
    assert cfg.max_passes == -1 and cfg.tile_max_degree == 512 and cfg.block_max_degree == 4096


def test_null_arguments_rejected_without_device(lib):
    assert lib.lvg_create(None, None) == 1
    assert lib.lvg_config_default(None) == 1
    assert lib.lvg_num_levels(None, None) == 1
    n = ctypes.c_int32()
    assert lib.lvg_count_partitions(None, -1, ctypes.byref(n)) == 1
    a = (ctypes.c_int32 * 4)(0, 3, 1, 3)
    assert lib.lvg_count_partitions(ctypes.cast(a, ctypes.c_void_p), 4, ctypes.byref(n)) == 0
    assert n.value == 4
