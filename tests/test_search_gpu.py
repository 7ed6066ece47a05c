"""GPU parity of the window searches and the transform against the oracle and
the reference's golden vectors.  Bit-exact: weights, masks and order."""

import json
import os
import random

import numpy as np
import pytest

import bmmpy_b200 as bmm
from oracle.oracle import port
from tests.golden.fixtures import cuda_equivalence_matrix, python_random_matrix

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def ka():
    with open(os.path.join(GOLDEN, "known_answers.json")) as f:
        return json.load(f)


def as_pairs(cands):
    return [(c.mask_u64(), c.weight) for c in cands]


def to_bmm(words, cols):
    return bmm.BitMatrix.from_words(words, cols)


# ---- the reference's own API tests (tests/python/test_search_api.py,
# tests/cpp/search_cpu_tests.cpp) against this implementation -------------

def make_search_matrix():
    m = bmm.BitMatrix(2, 5)
    for col in (0, 2, 4):
        m[0, col] = True
        m[1, col] = True
    return m


SIX = ["110010101001", "101100101100", "011010011001", "111000010111", "000111100011",
       "101011110000"]


def test_fwht_search_wrapper(ka):
    m = make_search_matrix()
    s = bmm.FwhtSearch(max_rows=16, max_candidates=1)
    c = s.search(m.row_window([0, 1]))
    assert s.name() == "fwht" and len(c) == 1
    assert (c[0].mask_u64(), c[0].weight) == (0x3, 0)
    full = bmm.FwhtSearch().search(m.row_window([0, 1]))
    assert as_pairs(full) == [tuple(p) for p in ka["fwht_2x5_k64"]]


def test_bruteforce_matches_fwht(ka):
    m = bmm.matrix_from_rows(SIX)
    w = m.row_window(list(range(6)))
    fw = bmm.FwhtSearch(max_rows=16, max_candidates=8).search(w)
    br = bmm.BruteforceSearch(max_candidates=8, chunk_bits=0).search(w)
    assert as_pairs(fw) == as_pairs(br) == [tuple(p) for p in ka["fwht_6x12_k8"]]
    assert as_pairs(bmm.FwhtSearch(max_candidates=63).search(w)) == [
        tuple(p) for p in ka["fwht_6x12_all"]]
    m3 = bmm.matrix_from_rows(["10101", "11100", "00111"])
    assert as_pairs(bmm.BruteforceSearch(max_candidates=4).search(m3.row_window([0, 1, 2]))) == [
        tuple(p) for p in ka["fwht_3x5_k4"]]
    assert as_pairs(bmm.BruteforceSearch(max_candidates=1).search(make_search_matrix().row_window(
        [0, 1]))) == [tuple(p) for p in ka["brute_2x5_k1"]]


@pytest.mark.parametrize("cols,k", [(512, 8), (1024, 128), (4096, 8)])
def test_cuda_bruteforce_equivalence_fixtures(ka, cols, k):
    words, c = cuda_equivalence_matrix(16, cols)
    m = to_bmm(words, c)
    got = bmm.CudaBruteforceSearch(max_candidates=k).search(m.row_window(list(range(16))))
    assert as_pairs(got) == [tuple(p) for p in ka[f"brute_16x{cols}_k{k}"]]


def test_cuda_bruteforce_python_random_fixture(ka):
    words, c = python_random_matrix(16, 512, 42)
    m = to_bmm(words, c)
    got = bmm.CudaBruteforceSearch(max_candidates=8).search(m.row_window(list(range(16))))
    assert as_pairs(got) == [tuple(p) for p in ka["brute_pyrand_16x512_k8"]]


# ---- randomized parity against the oracle ----------------------------------

@pytest.mark.parametrize("seed", range(6))
def test_gray_window_random(seed):
    P = port()
    rng = random.Random(100 + seed)
    for _ in range(8):
        rows = rng.randint(1, 22)
        cols = rng.choice([1, 63, 64, 130, 256, 700, 4096, 4100, 9000])
        words, _ = P.gen_instance(rows, cols, rng.choice([0.05, 0.3, 0.5]), rng.randint(0, 9999),
                                  rng.randint(0, 6))
        t = rng.randint(1, min(rows, 16 if cols > 4096 else 20))
        win = rng.sample(range(rows), t)
        k = rng.choice([1, 2, 31, 32, 33, 64, 128, 129, 500])
        cb = rng.choice([0, 0, 1, t])
        exp = P.bruteforce_search(words, cols, win, k, cb)
        got = bmm.BruteforceSearch(max_candidates=k, chunk_bits=cb).search(
            to_bmm(words, cols).row_window(win))
        assert as_pairs(got) == exp, (rows, cols, t, k, cb)


@pytest.mark.parametrize("seed", range(4))
def test_fwht_window_random(seed):
    P = port()
    rng = random.Random(200 + seed)
    for _ in range(8):
        rows = rng.randint(1, 20)
        cols = rng.choice([1, 5, 64, 65, 256, 1000, 5000])
        words, _ = P.gen_instance(rows, cols, rng.choice([0.02, 0.3, 0.5]), rng.randint(0, 9999),
                                  rng.randint(0, 6))
        t = rng.randint(1, rows)
        win = rng.sample(range(rows), t)
        k = rng.choice([1, 7, 32, 64, 128, 1000])
        exp = P.fwht_search(words, cols, win, 20, k)
        got = bmm.FwhtSearch(max_rows=20, max_candidates=k).search(
            to_bmm(words, cols).row_window(win))
        assert as_pairs(got) == exp, (rows, cols, t, k)


@pytest.mark.parametrize("t", [21, 23])
def test_fwht_window_multipass(t):
    """Spectra of 2^21..2^23 buckets go through the HBM passes."""
    P = port()
    words, _ = P.gen_instance(t, 3000, 0.3, 31 + t, 5)
    win = list(range(t))
    exp = P.fwht_search(words, 3000, win, 30, 64)
    got = bmm.FwhtSearch(max_rows=30, max_candidates=64).search(to_bmm(words, 3000).row_window(win))
    assert as_pairs(got) == exp


def test_search_edge_cases():
    m = bmm.BitMatrix(3, 0)
    assert bmm.FwhtSearch().search(m.row_window([0, 1])) == []
    assert bmm.BruteforceSearch().search(m.row_window([0, 1])) == []
    m = bmm.BitMatrix(4, 100)
    assert bmm.BruteforceSearch().search(m.row_window([])) == []
    # all-zero rows: every mask has weight 0, ordered by mask
    got = bmm.BruteforceSearch(max_candidates=5).search(m.row_window([0, 1, 2]))
    assert as_pairs(got) == [(1, 0), (2, 0), (3, 0), (4, 0), (5, 0)]
    got = bmm.FwhtSearch(max_candidates=5).search(m.row_window([0, 1, 2]))
    assert as_pairs(got) == [(1, 0), (2, 0), (3, 0), (4, 0), (5, 0)]
    with pytest.raises(ValueError):
        bmm.BruteforceSearch(max_candidates=4, chunk_bits=4).search(m.row_window([0, 1, 2]))


# ---- transform --------------------------------------------------------------

@pytest.mark.parametrize("logn", [0, 1, 2, 5, 10, 13, 14, 15, 17, 20, 24])
def test_fwht_i32_matches_oracle(logn):
    rng = np.random.default_rng(logn)
    a = rng.integers(-1000, 1000, size=1 << logn, dtype=np.int32)
    exp = port().fwht_i32(a)
    got = bmm.fwht_i32(a.copy())
    assert np.array_equal(got, exp)


def test_fwht_wrapping_and_errors():
    assert bmm.fwht_i32(np.array([1, 2, 3, 4], np.int32)).tolist() == [10, -2, -4, 0]
    assert bmm.fwht_i16(np.array([32767, 1], np.int16)).tolist() == [-32768, 32766]
    big = np.full(1 << 18, 2 ** 30, np.int32)
    assert np.array_equal(bmm.fwht_i32(big.copy()), port().fwht_i32(big))
    rng = np.random.default_rng(5)
    a16 = rng.integers(-30000, 30000, size=1 << 16, dtype=np.int16)
    assert np.array_equal(bmm.fwht_i16(a16.copy()), port().fwht_i16(a16))
    with pytest.raises(ValueError):
        bmm.fwht_i32(np.zeros(3, np.int32))
