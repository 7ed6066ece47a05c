"""Per-shape autotuner (bmmpy_b200.autotune): candidate settings, the JSON
cache and the library's shape tables (CPU), and tuning on the GPU, where
every candidate must reproduce the default setting's exact result."""

import json

import numpy as np
import pytest

from bmmpy_b200 import _native as N
from bmmpy_b200 import autotune as A


def test_candidates_cover_the_shape_classes():
    c64 = A.gray_candidates(64, 24)
    assert (4, -1, 1) in c64 and (2, 10, 2) in c64
    assert all(hs <= 4 for hs, _, lanes in c64 if lanes == 2)
    assert {hs for hs, _, _ in A.gray_candidates(24, 16)} == {0, 2, 3, 4}
    assert {hs for hs, _, _ in A.gray_candidates(4, 16)} == {-1}
    assert all(c <= 9 for _, c, _ in A.gray_candidates(4, 9))


def test_shape_table_arguments_are_checked():
    L = N.lib()
    try:
        N.check(L.bmm_gray_tune_shape(64, 24, 4, 10, 1))
        N.check(L.bmm_spectrum_tune_shape(32, 30))
        for bad in ((0, 24, 4, 10, 1), (64, 41, 4, 10, 1), (64, 24, 7, 10, 1),
                    (64, 24, 5, 10, 2), (64, 24, 4, 40, 1)):
            with pytest.raises(ValueError):
                N.check(L.bmm_gray_tune_shape(*bad))
        with pytest.raises(ValueError):
            N.check(L.bmm_spectrum_tune_shape(32, 34))
        assert L.bmm_spectrum_low_bits(32) == 30
        assert L.bmm_spectrum_low_bits(28) == 28
    finally:
        N.check(L.bmm_tune_reset())
    assert L.bmm_spectrum_low_bits(32) == 32


def test_cache_round_trip(tmp_path, monkeypatch):
    monkeypatch.setenv("BMMPY_B200_CACHE", str(tmp_path))
    monkeypatch.setattr(A, "_device_key", lambda: "dev|v")
    entry = {"gray": {"40x4096k24": {"words_per_row": 64, "k": 24, "setting": [4, 10, 1]}},
             "spectrum": {"32": {"t": 32, "low_bits": 31}}}
    A._store({"dev|v": entry})
    assert json.load(open(tmp_path / "autotune_shapes.json"))["dev|v"] == entry
    try:
        assert A.apply_cached() == entry
        assert N.lib().bmm_spectrum_low_bits(32) == 31
    finally:
        A.reset()


@pytest.mark.gpu
def test_tuning_keeps_results(tmp_path, monkeypatch):
    from bmmpy_b200 import targets as T
    from bmmpy_b200.workloads import gen_instance

    monkeypatch.setenv("BMMPY_B200_CACHE", str(tmp_path))
    m, _ = gen_instance(24, 3000, 0.3, 5)
    t, o = T.cyclic_others(24, 14)
    want = T.gray_targets(m, t, o)
    try:
        entry = A.tune(gray_shapes=[(24, 3000, 14)], spectrum_t=[20], batch=False)
        g = entry["gray"]["24x3000k14"]
        assert g["ms"] <= g["default_ms"]
        got = T.gray_targets(m, t, o)
        assert all(np.array_equal(a, b) for a, b in zip(got, want))
        A.reset()
        assert A.apply_cached()["gray"]["24x3000k14"]["setting"] == g["setting"]
    finally:
        A.reset()


def test_pass_knobs_are_checked():
    """bmm_spectrum_tune_passes / _last_pass accept their documented values only
    (host-side settings; nothing runs on the device)."""
    L = N.lib()
    try:
        for v in (0, 1, 2):
            N.check(L.bmm_spectrum_tune_passes(v))
        for bad in (-1, 3, 7):
            with pytest.raises(ValueError):
                N.check(L.bmm_spectrum_tune_passes(bad))
        for v in (0, 1):
            N.check(L.bmm_spectrum_tune_last_pass(v))
        with pytest.raises(ValueError):
            N.check(L.bmm_spectrum_tune_last_pass(2))
    finally:
        N.check(L.bmm_spectrum_tune_passes(2))
        N.check(L.bmm_spectrum_tune_last_pass(1))


def test_split_window_c_abi_checks_before_device_work():
    """bmm_split_window_dev: the reference's argument checks, in its order, and
    the empty cases, all answered on the host."""
    import ctypes as C

    L = N.lib()
    n = C.c_size_t(7)
    tw = C.c_int32(7)
    with pytest.raises(ValueError, match="low_bits must be <= number of rows"):
        N.check(L.bmm_split_window_dev(None, 2, 1, 10, 3, None, None, None, 0, C.byref(n),
                                       C.byref(tw), None))
    with pytest.raises(ValueError, match="row count must be <= 64"):
        N.check(L.bmm_split_window_dev(None, 65, 1, 10, 2, None, None, None, 0, C.byref(n),
                                       C.byref(tw), None))
    N.check(L.bmm_split_window_dev(None, 0, 0, 10, 0, None, None, None, 0, C.byref(n),
                                   C.byref(tw), None))
    assert (n.value, tw.value) == (0, 0)
    N.check(L.bmm_split_window_dev(None, 3, 1, 0, 1, None, None, None, 0, C.byref(n),
                                   C.byref(tw), None))
    assert (n.value, tw.value) == (0, 0)
