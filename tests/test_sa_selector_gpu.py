"""SASelector with the pairwise score on the GPU: the device synergy table
(2 * popc(r_i & r_j), src/search/sa_selector_pairwise.cpp:21-52) against a
numpy Gram matrix, and whole selections against the reference library and
the oracle, including the reference's own tests
(tests/cpp/sa_selector_tests.cpp, tests/python/test_search_api.py:94-121)."""

import random

import numpy as np
import pytest

import bmmpy_b200 as bmm
from bmmpy_b200 import _native as N
from oracle.oracle import port, ref

pytestmark = pytest.mark.gpu

FIELDS = ("rows", "score", "accepted_moves", "iterations_run", "best_iteration",
          "restart_index", "seed")


def _cluster():
    return bmm.matrix_from_rows(["111111000000"] * 4 + ["000000000000"] * 4)


def _bits(m):
    b = np.unpackbits(np.ascontiguousarray(m.words).view(np.uint8).reshape(m.rows, -1), axis=1,
                      bitorder="little")[:, : m.cols]
    return b.astype(np.int64)


@pytest.mark.parametrize("rows,cols,p", [(1, 5, 0.5), (8, 12, 0.5), (63, 64, 0.3), (65, 65, 0.3),
                                         (130, 700, 0.1), (200, 4100, 0.02)])
def test_pairwise_table_matches_gram(rows, cols, p):
    words, _ = port().gen_instance(rows, cols, p, rows + cols, 0)
    m = bmm.BitMatrix(rows, cols)
    m.words[:] = words[:, : m.stride_words]
    table = np.zeros(rows * rows, np.uint32)
    N.check(N.lib().bmm_sa_pairwise_table(N.u64p(m.words), m.stride_words, rows, cols,
                                          N.u32p(table)))
    b = _bits(m)
    want = 2 * (b @ b.T)
    np.fill_diagonal(want, 0)
    assert np.array_equal(table.reshape(rows, rows), want.astype(np.uint32))


def test_reference_tests():
    m = _cluster()
    # tests/python/test_search_api.py:94-121
    selector = bmm.SASelector(iterations=256, restarts=8, seed=7)
    result = selector.select(m, 4)
    assert result.rows == [0, 1, 2, 3]
    assert result.score == 72
    window = selector.select_window(m, 4)
    assert window.rows == [0, 1, 2, 3]
    assert window.materialize().to_rows() == ["111111000000"] * 4
    # tests/cpp/sa_selector_tests.cpp:10-38: deterministic for a seed
    s = bmm.SASelector(iterations=256, restarts=8, seed=12345, temperature_probe_samples=32)
    a, b = s.select(m, 4), s.select(m, 4)
    assert {k: getattr(a, k) for k in FIELDS} == {k: getattr(b, k) for k in FIELDS}


@pytest.mark.skipif(ref() is None, reason="reference not built (make -C oracle ref)")
def test_pairwise_matches_reference_random():
    rng = random.Random(8)
    for trial in range(40):
        rows = rng.randint(2, 90)
        cols = rng.choice([12, 64, 65, 200, 700, 3000])
        t = rng.randint(0, rows)
        words, _ = port().gen_instance(rows, cols, rng.choice([0.05, 0.2, 0.5]), trial, 0)
        m = bmm.BitMatrix(rows, cols)
        m.words[:] = words[:, : m.stride_words]
        kw = dict(iterations=rng.choice([0, 1, 50, 500]), restarts=rng.randint(1, 4),
                  seed=rng.choice([0, 1, 99]), temperature_probe_samples=rng.choice([0, 1, 16]),
                  initial_acceptance_probability=rng.choice([0.5, 0.8, 0.99]),
                  cooling_rate=rng.choice([0.9, 0.99, 1.0]),
                  min_temperature=rng.choice([1e-6, 1.0, 50.0]))
        r = bmm.SASelector(**kw).select(m, t)
        want = ref().sa_select(np.ascontiguousarray(m.words), cols, t, score_policy=0, **kw)
        assert {k: getattr(r, k) for k in FIELDS} == want, (trial, kw)


def test_planted_instance_matches_oracle():
    # the C3 planted matrix, default iterations, two restarts, 32-row windows
    words, _ = port().gen_instance(512, 65536, 0.02, 2, 2000)
    m = bmm.BitMatrix(512, 65536)
    m.words[:] = words[:, : m.stride_words]
    r = bmm.SASelector(restarts=2, seed=3).select(m, 32)
    want = port().sa_select(np.ascontiguousarray(m.words), 65536, 32, restarts=2, seed=3)
    assert {k: getattr(r, k) for k in FIELDS} == want
