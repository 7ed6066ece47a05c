"""GPU parity of MitmFwhtSearch / CudaMitmFwhtSearch (and of the HBM spectrum
pipeline shared with FwhtSearch) against the reference's golden vectors and
the oracle.  Bit-exact."""

import json
import os
import random

import numpy as np
import pytest

import bmmpy_b200 as bmm
from bmmpy_b200.workloads import C3, gen_instance
from oracle.oracle import port
from tests.golden.fixtures import cuda_equivalence_matrix

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")

SIX = ["110010101001", "101100101100", "011010011001", "111000010111", "000111100011",
       "101011110000"]


@pytest.fixture(scope="module")
def ka():
    with open(os.path.join(GOLDEN, "known_answers.json")) as f:
        return json.load(f)


def as_pairs(cands):
    return [(c.mask_u64(), c.weight) for c in cands]


def weights_recomputed(matrix, rows, cands):
    """Independent check: popcount of the XOR of the selected rows."""
    out = []
    for c in cands:
        acc = np.zeros(matrix.stride_words, np.uint64)
        for j in c.selected_rows():
            acc ^= matrix.words[rows[j]]
        out.append(int(np.unpackbits(acc.view(np.uint8)).sum()))
    return out


def test_mitm_wrapper_matches_fwht(ka):
    m = bmm.matrix_from_rows(SIX)
    w = m.row_window(list(range(6)))
    s = bmm.MitmFwhtSearch(max_candidates=8)
    assert s.name() == "mitm_fwht"
    assert as_pairs(s.search(w)) == [tuple(p) for p in ka["mitm_6x12_k8"]]
    assert as_pairs(s.search(w)) == as_pairs(bmm.FwhtSearch(max_candidates=8).search(w))


@pytest.mark.parametrize("k", [8, 128])
def test_cuda_mitm_equivalence_fixture(ka, k):
    words, cols = cuda_equivalence_matrix(28, 96)
    m = bmm.BitMatrix.from_words(words, cols)
    got = bmm.CudaMitmFwhtSearch(max_candidates=k).search(m.row_window(list(range(28))))
    assert as_pairs(got) == [tuple(p) for p in ka[f"mitm_28x96_k{k}"]]
    got = bmm.MitmFwhtSearch(max_candidates=k).search(m.row_window(list(range(28))))
    assert as_pairs(got) == [tuple(p) for p in ka[f"mitm_28x96_k{k}"]]


@pytest.mark.parametrize("seed", range(3))
def test_mitm_random_vs_oracle(seed):
    P = port()
    rng = random.Random(300 + seed)
    for _ in range(6):
        rows = rng.randint(2, 22)
        cols = rng.choice([3, 64, 100, 777, 5000, 20000])
        words, _ = P.gen_instance(rows, cols, rng.choice([0.05, 0.3, 0.5]), rng.randint(0, 999),
                                  rng.randint(0, 9))
        t = rng.randint(1, rows)
        win = rng.sample(range(rows), t)
        k = rng.choice([1, 5, 64, 129, 1000])
        exp = P.mitm_search(words, cols, win, k)
        got = bmm.MitmFwhtSearch(max_candidates=k).search(
            bmm.BitMatrix.from_words(words, cols).row_window(win))
        assert as_pairs(got) == exp, (rows, cols, t, k)


def test_c3_windows_full_size():
    """Two 32-row windows of the planted 512 x 65536 instance: reference golden."""
    wl = np.load(os.path.join(GOLDEN, "workloads.npz"))
    m, planted = gen_instance(C3["rows"], C3["cols"], C3["p"], C3["seed"], C3["scrambles"])
    assert planted == int(wl["c3_planted"][0])
    s = bmm.MitmFwhtSearch(max_candidates=64)
    for j in range(wl["c3_top64"].shape[0]):
        rows = list(range(32 * j, 32 * j + 32))
        got = s.search(m.row_window(rows))
        assert as_pairs(got) == [tuple(map(int, p)) for p in wl["c3_top64"][j]]
        assert [c.weight for c in got[:8]] == weights_recomputed(m, rows, got[:8])


def test_mitm_sliced_beyond_33_bits_matches_gray():
    """t = 34: the top bit is enumerated (two 2^33 slices); cross-check with the
    Gray-code enumeration of all 2^34 subsets."""
    m, _ = gen_instance(34, 100, 0.3, 77, 5)
    rows = list(range(34))
    w = m.row_window(rows)
    mitm = bmm.MitmFwhtSearch(max_candidates=16).search(w)
    gray = bmm.BruteforceSearch(max_candidates=16).search(w)
    assert as_pairs(mitm) == as_pairs(gray)
    assert [c.weight for c in mitm] == weights_recomputed(m, rows, mitm)


def test_fwht_search_33_bits():
    m, _ = gen_instance(33, 300, 0.3, 91, 7)
    rows = list(range(33))
    got = bmm.FwhtSearch(max_rows=33, max_candidates=32).search(m.row_window(rows))
    assert [c.weight for c in got] == weights_recomputed(m, rows, got)
    assert got == sorted(got, key=lambda c: c.key())
    gray = bmm.BruteforceSearch(max_candidates=32).search(m.row_window(rows))
    assert as_pairs(got) == as_pairs(gray)


@pytest.mark.parametrize("t,k,cols,density", [
    (20, 64, 5000, 0.3), (21, 1, 777, 0.5), (23, 128, 20000, 0.05), (24, 64, 3000, 0.3),
    (26, 5, 60000, 0.02), (29, 129, 4000, 0.4), (31, 64, 65536, 0.02),
])
def test_register_passes_match_tile_passes(t, k, cols, density):
    """The register-resident transform passes (6..9 bits, k <= 128) against the
    cp.async tile passes and, up to t = 26, the oracle: bit-exact top-k lists.
    Windows with a sparse pattern set also exercise the empty-tile bits of the
    first pass."""
    from bmmpy_b200 import _native as N

    P = port()
    words, _ = P.gen_instance(t + 2, cols, density, 1000 + t, 3)
    win = list(range(1, t + 1))
    w = bmm.BitMatrix.from_words(words, cols).row_window(win)
    s = bmm.MitmFwhtSearch(max_candidates=k)
    lib = N.lib()
    try:
        N.check(lib.bmm_spectrum_tune_passes(0), "bmm_spectrum_tune_passes")
        tiles = as_pairs(s.search(w))
        N.check(lib.bmm_spectrum_tune_passes(1), "bmm_spectrum_tune_passes")
        prefetch = as_pairs(s.search(w))
    finally:
        N.check(lib.bmm_spectrum_tune_passes(2), "bmm_spectrum_tune_passes")
    regs = as_pairs(s.search(w))
    assert regs == tiles
    assert prefetch == tiles
    if t <= 26:
        assert regs == P.mitm_search(words, cols, win, k)
    assert len(regs) == k
