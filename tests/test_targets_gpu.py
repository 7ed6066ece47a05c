"""GPU parity of the per-target searches (the C1 / C2 / C4 workloads) against
the golden vectors the reference produced, and against the oracle."""

import os
import random

import numpy as np
import pytest

from bmmpy_b200 import targets as T
from bmmpy_b200.matrix import BitMatrix
from bmmpy_b200.workloads import C1, C2, batch_instance, gen_instance
from oracle.oracle import port
from tests.golden.fixtures import checksum_pairs

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def wl():
    return np.load(os.path.join(GOLDEN, "workloads.npz"))


def test_c1_fwht_and_gray_targets(wl):
    m, _ = gen_instance(C1["rows"], C1["cols"], C1["p"], C1["seed"])
    t, o = T.cyclic_others(C1["rows"], C1["k"])
    fm, fw = T.fwht_targets(m, t, o)
    gm, gw = T.gray_targets(m, t, o)
    assert np.array_equal(fm, wl["c1_mask"]) and np.array_equal(fw, wl["c1_weight"])
    assert np.array_equal(gm, wl["c1_mask"]) and np.array_equal(gw, wl["c1_weight"])


def test_c2_gray_targets_k16(wl):
    m, _ = gen_instance(C2["rows"], C2["cols"], C2["p"], C2["seed"])
    t, o = T.cyclic_others(C2["rows"], 16)
    gm, gw = T.gray_targets(m, t, o)
    assert np.array_equal(gm, wl["c2k16_mask"]) and np.array_equal(gw, wl["c2k16_weight"])
    fm, fw = T.fwht_targets(m, t, o)
    assert np.array_equal(fm, wl["c2k16_mask"]) and np.array_equal(fw, wl["c2k16_weight"])


def test_c2_gray_targets_full_size(wl):
    """The full 40 x 2^24 workload, bit-exact against the reference."""
    m, _ = gen_instance(C2["rows"], C2["cols"], C2["p"], C2["seed"])
    t, o = T.cyclic_others(C2["rows"], C2["k"])
    gm, gw = T.gray_targets(m, t, o)
    assert np.array_equal(gm, wl["c2_mask"]) and np.array_equal(gw, wl["c2_weight"])


@pytest.mark.parametrize("tiebreak", ["mask", "gray"])
def test_gray_targets_ties_match_oracle(tiebreak):
    """Narrow rows make many subsets share the best weight."""
    P = port()
    rng = random.Random(5)
    for trial in range(6):
        rows = rng.randint(12, 30)
        cols = rng.choice([3, 8, 40, 64, 100])
        words, _ = P.gen_instance(rows, cols, rng.choice([0.2, 0.5]), 1000 + trial)
        k = rng.randint(1, min(rows - 1, 14))
        m = BitMatrix.from_words(words, cols)
        t, o = T.cyclic_others(rows, k, offset=rng.randint(1, rows - k))
        gm, gw = T.gray_targets(m, t, o, tiebreak=tiebreak)
        for i in range(rows):
            exp = P.target_best_gray(words, cols, int(t[i]), o[i].tolist(),
                                     1 if tiebreak == "gray" else 0)
            assert (int(gm[i]), int(gw[i])) == exp, (trial, i)


def test_fwht_targets_small_k_and_wide_rows():
    P = port()
    rng = random.Random(9)
    for trial in range(6):
        rows = rng.randint(3, 40)
        cols = rng.choice([1, 64, 500, 2048, 20000, 32767])
        words, _ = P.gen_instance(rows, cols, rng.choice([0.05, 0.5]), 50 + trial, rows)
        k = rng.choice([1, 2, 9, 15, 16]) if rows > 16 else rng.randint(1, rows - 1)
        m = BitMatrix.from_words(words, cols)
        t, o = T.cyclic_others(rows, k)
        fm, fw = T.fwht_targets(m, t, o)
        for i in range(0, rows, 3):
            assert (int(fm[i]), int(fw[i])) == P.target_best_fwht(words, cols, i, o[i].tolist())


def test_c4_first_instances(wl):
    first = wl["c4_first32"]
    row = 0
    for idx in range(32):
        m, k, _ = batch_instance(idx)
        t, o = T.cyclic_others(m.rows, k)
        fm, fw = T.fwht_targets(m, t, o)
        got = np.stack([fm.astype(np.uint64), fw.astype(np.uint64)], 1)
        assert np.array_equal(got, first[row:row + m.rows])
        assert checksum_pairs(fm, fw) == int(wl["c4_checksums"][idx])
        row += m.rows


@pytest.mark.parametrize("lanes", [1, 2])
@pytest.mark.parametrize("tiebreak", ["mask", "gray"])
def test_gray_targets_lane_shapes_match_oracle(lanes, tiebreak):
    """Rows of 33-64 words on one lane or a lane pair, and wider rows split
    over 2-8 lanes (padded shared-memory slices), with carry-save variants."""
    from bmmpy_b200 import _native as N

    P = port()
    rng = random.Random(17 + lanes)
    L = N.lib()
    try:
        N.check(L.bmm_gray_tune_lanes(lanes))
        for trial, cols in enumerate([2049, 3000, 4096, 4100, 9000, 20000]):
            rows = rng.randint(14, 24)
            words, _ = P.gen_instance(rows, cols, rng.choice([0.01, 0.3, 0.5]), 300 + trial)
            k = rng.randint(6, min(rows - 1, 11))
            m = BitMatrix.from_words(words, cols)
            t, o = T.cyclic_others(rows, k, offset=rng.randint(1, rows - k))
            for hs in ([-1, 0, 2, 4] if 2048 < cols <= 4096 else [-1]):
                N.check(L.bmm_gray_tune(hs, rng.choice([-1, 3, 5])))
                gm, gw = T.gray_targets(m, t, o, tiebreak=tiebreak)
                for i in range(rows):
                    exp = P.target_best_gray(words, cols, int(t[i]), o[i].tolist(),
                                             1 if tiebreak == "gray" else 0)
                    assert (int(gm[i]), int(gw[i])) == exp, (cols, hs, i)
    finally:
        N.check(L.bmm_gray_tune(-1, -1))
        N.check(L.bmm_gray_tune_lanes(-1))


def test_c2_full_size_lane_pairs(wl):
    """The full C2 workload with 32-word lane pairs, bit-exact."""
    from bmmpy_b200 import _native as N

    L = N.lib()
    m, _ = gen_instance(C2["rows"], C2["cols"], C2["p"], C2["seed"])
    t, o = T.cyclic_others(C2["rows"], C2["k"])
    try:
        N.check(L.bmm_gray_tune_lanes(2))
        gm, gw = T.gray_targets(m, t, o)
    finally:
        N.check(L.bmm_gray_tune_lanes(-1))
    assert np.array_equal(gm, wl["c2_mask"]) and np.array_equal(gw, wl["c2_weight"])
