"""CPU checks of the autotuner's host logic: the pick rule over measured
points (lvg_tune_pick) and argument errors, with no device call."""
import ctypes
import math

import pytest


@pytest.fixture(scope="module")
def lib():
    from louvaingpu_b200 import build, _lib
    build.build_lvg()
    return _lib.load()


def test_pick_fastest():
    from louvaingpu_b200 import tune_pick
    pts = [(64, 1024, 5.0, 1.0), (128, 2048, 3.0, 1.0), (512, 4096, 4.0, 1.0)]
    assert tune_pick(pts) == 1


def test_pick_prefers_configured_pair_within_two_percent():
    from louvaingpu_b200 import tune_pick
    pts = [(64, 1024, 3.00, 1.0), (512, 4096, 3.05, 1.0)]
    assert tune_pick(pts, pref=(512, 4096)) == 1
    pts = [(64, 1024, 3.00, 1.0), (512, 4096, 3.10, 1.0)]
    assert tune_pick(pts, pref=(512, 4096)) == 0
    assert tune_pick(pts, pref=(256, 4096)) == 0


def test_pick_skips_unmeasured_and_keeps_earliest_tie():
    from louvaingpu_b200 import tune_pick
    pts = [(64, 1024, -1.0, -1.0), (128, 1024, float("nan"), 1.0), (256, 1024, 2.0, 1.0), (512, 1024, 2.0, 1.0)]
    assert tune_pick(pts, pref=(0, 0)) == 2
    assert tune_pick([(64, 1024, -1.0, -1.0)]) == -1
    assert tune_pick([]) == -1


def test_pick_zero_times_fall_to_preferred():
    # a graph whose level stops after the singleton pass has no hashing pass:
    # every pair measures 0 ms and the configured pair stays
    from louvaingpu_b200 import tune_pick
    pts = [(64, 1024, 0.0, 1.0), (512, 4096, 0.0, 1.0)]
    assert tune_pick(pts, pref=(512, 4096)) == 1


def test_autotune_arguments_rejected_without_device(lib):
    from louvaingpu_b200 import _lib
    b = ctypes.c_int32()
    assert lib.lvg_tune_pick(None, 1, 512, 4096, ctypes.byref(b)) == 1
    assert lib.lvg_tune_pick(None, 0, 512, 4096, None) == 1
    n = ctypes.c_int32()
    best = _lib.LvgTunePoint()
    assert lib.lvg_autotune(None, None, None, 0, ctypes.byref(n), ctypes.byref(best)) == 1
    assert lib.lvg_get_thresholds(None, None, None) == 1
    assert lib.lvg_tune_cache_clear() == 0
    assert not math.isnan(best.move_ms)
