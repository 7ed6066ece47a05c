"""ExactBasisSolver without a GPU: the oracle pinned to the reference's
goldens and to the reference itself, and the solver's argument checks and
degenerate windows, which return before any device work
(src/solver/exact_basis_solver.cpp:58-100)."""

import os
import random

import numpy as np
import pytest

import bmmpy_b200 as bmm
from oracle.oracle import port, ref_scalar
from tests.golden.fixtures import BASIS_CASES

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "workloads.npz"))


def _matrix(rows):
    m = bmm.matrix_from_rows(rows)
    return m, np.ascontiguousarray(m.words)


def test_oracle_reference_example():
    # tests/python/test_matrix_api.py:45-64
    m, words = _matrix(["111", "110", "001"])
    masks, weights, total = port().exact_basis(words, 3, [0, 1, 2])
    assert total == 3 and sorted(weights) == [1, 2] and len(masks) == 2


@pytest.mark.parametrize("case", range(len(BASIS_CASES)))
def test_oracle_matches_reference_goldens(case):
    rows, cols, p, iseed, scr, win = BASIS_CASES[case]
    m, _ = port().gen_instance(rows, cols, p, iseed, scr)
    masks, weights, total = port().exact_basis(m, cols, win)
    assert masks == GOLD[f"basis{case}_masks"].tolist()
    assert weights == GOLD[f"basis{case}_weights"].tolist()
    assert total == int(GOLD[f"basis{case}_scalars"][4])
    counts = port().basis_weight_counts(m, cols, win)
    assert int(counts.sum()) == (1 << len(win)) - 1


@pytest.mark.skipif(ref_scalar() is None, reason="reference not built (make -C oracle ref)")
def test_oracle_matches_reference_random():
    rng = random.Random(5)
    R, P = ref_scalar(), port()
    for trial in range(120):
        t = rng.randint(1, 12)
        cols = rng.choice([1, 5, 63, 64, 65, 130, 257, 700])
        rows = t + rng.randint(0, 4)
        m, _ = P.gen_instance(rows, cols, rng.choice([0.02, 0.1, 0.3, 0.5]), trial, rng.randint(0, 30))
        if trial % 5 == 0 and rows > 2:
            m[2] = m[0] ^ m[1]  # a dependent row
        if trial % 7 == 0:
            m[rows - 1] = 0  # a zero row
        win = rng.sample(range(rows), t)
        want = R.exact_basis(m, cols, win, max_rows=32)
        masks, weights, total = P.exact_basis(m, cols, win)
        assert (masks, weights, total) == (want["basis_masks"], want["basis_weights"],
                                           want["total_weight"]), trial


def _window(rows, cols, t, seed=0, p=0.3):
    m = bmm.BitMatrix(rows, cols)
    words, _ = port().gen_instance(rows, cols, p, seed, 0)
    m.words[:] = words[:, : m.stride_words]
    return m.row_window(list(range(t)))


def test_empty_window():
    m = bmm.BitMatrix(4, 10)
    r = bmm.solver.ExactBasisSolver().solve(m.row_window([]))
    assert (r.input_rows, r.cols, r.rank, r.enumerated_states, r.total_weight) == (0, 10, 0, 0, 0)
    assert r.transform_matrix.shape == (0, 0) and r.basis_matrix.shape == (0, 10)
    assert r.basis_masks == [] and r.basis_weights == []


def test_zero_rank_window():
    m = bmm.BitMatrix(5, 70)
    r = bmm.solver.ExactBasisSolver().solve(m.row_window([0, 2, 4]))
    assert (r.input_rows, r.cols, r.rank, r.enumerated_states, r.total_weight) == (3, 70, 0, 7, 0)
    assert r.transform_matrix.shape == (0, 3) and r.basis_matrix.shape == (0, 70)


def test_argument_errors_match_reference():
    w = _window(40, 64, 25)
    with pytest.raises(ValueError, match="^ExactBasisSolver: window has more rows than the "
                                         "configured max_rows cap$"):
        bmm.solver.ExactBasisSolver().solve(w)
    w33 = _window(40, 64, 33)
    with pytest.raises(ValueError, match="^ExactBasisSolver: this implementation supports at "
                                         "most 32 rows$"):
        bmm.solver.ExactBasisSolver(max_rows=40).solve(w33)
    w10 = _window(40, 64, 10)
    with pytest.raises(ValueError, match="^ExactBasisSolver: state count exceeds the configured "
                                         "max_states cap$"):
        bmm.solver.ExactBasisSolver(max_states=1022).solve(w10)
    with pytest.raises(ValueError, match="^ExactBasisSolver: required packed-mask storage "
                                         "exceeds max_storage_bytes$"):
        bmm.solver.ExactBasisSolver(max_storage_bytes=4091).solve(w10)


def test_config_object_and_repr():
    cfg = bmm.solver.ExactBasisSolverConfig()
    assert (cfg.max_rows, cfg.max_states, cfg.max_storage_bytes) == (24, (1 << 24) - 1,
                                                                     128 * 1024 * 1024)
    cfg.max_rows = 30
    s = bmm.solver.ExactBasisSolver(cfg)
    assert s.max_rows == 30 and s.name() == "exact_basis"
    assert repr(bmm.solver.ExactBasisSolver()) == (
        "ExactBasisSolver(max_rows=24, max_states=16777215, max_storage_bytes=134217728)")


def test_bitmatrix_rank_and_mul():
    m = bmm.matrix_from_rows(["110", "011", "101", "000"])
    assert m.rank() == 2
    t = bmm.matrix_from_rows(["1100", "0011"])
    assert t.mul(m).to_rows() == ["101", "101"]
    assert (t @ m).to_rows() == ["101", "101"]
    assert m.add(m).weight() == 0
    with pytest.raises(bmm.MatrixError, match="Matrix dimensions mismatch"):
        m.mul(m)
    assert bmm.BitMatrix.identity(3).mul(bmm.matrix_from_rows(["1", "0", "1"])).to_rows() == [
        "1", "0", "1"]
