"""search -> apply on the GPU searchers (bmmpy/workflows.py:45-90): the
reference's documented example, and windows of a planted matrix where the
GPU search followed by GreedyApplier / GlobalGreedyApplier leaves exactly the
matrix that the oracle's search followed by the same applier leaves."""

import random

import numpy as np
import pytest

import bmmpy_b200 as bmm
from bmmpy_b200.candidate import Candidate
from bmmpy_b200.matrix import BitMatrix
from oracle.oracle import port

pytestmark = pytest.mark.gpu


def test_reference_example():
    matrix = BitMatrix(2, 5)
    for col in (0, 2, 4):
        matrix[0, col] = True
        matrix[1, col] = True
    window = matrix.row_window([0, 1])
    result = bmm.search_apply(window, searcher=bmm.FwhtSearch(max_rows=16, max_candidates=1),
                              applier=bmm.GreedyApplier(min_gain=1))
    assert result.applied_count >= 1 and result.weight_improvement > 0


@pytest.mark.parametrize("kind", ["greedy", "global"])
def test_search_apply_matches_oracle(kind):
    rng = random.Random(9 if kind == "greedy" else 10)
    for trial in range(12):
        rows, cols = rng.randint(20, 60), rng.choice([200, 1000, 4096])
        words, _ = port().gen_instance(rows, cols, 0.05, rng.randint(0, 99), 3 * rows)
        a = BitMatrix(rows, cols)
        a.words[:] = words[:, : a.stride_words]
        b = BitMatrix(rows, cols)
        b.words[:] = words[:, : b.stride_words]
        for sweep in range(3):
            for j in range(0, rows - 15, 8):
                win_rows = list(range(j, j + 16))
                applier = (bmm.GreedyApplier(1) if kind == "greedy"
                           else bmm.GlobalGreedyApplier())
                got = bmm.search_apply(a.row_window(win_rows),
                                       searcher=bmm.FwhtSearch(max_candidates=64), applier=applier)
                cands = [Candidate.from_u64(mk, w) for mk, w in
                         port().fwht_search(np.ascontiguousarray(b.words), cols, win_rows, 16, 64)]
                want = applier.apply(b.row_window(win_rows), cands)
                assert (got.applied_count, got.weight_improvement) == (
                    want.applied_count, want.weight_improvement)
                assert np.array_equal(a.words, b.words)
