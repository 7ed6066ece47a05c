"""build_compact_split_window on the device (bmm_split_window_dev) against the
oracle's restatement of src/search/split_window_prep.cpp:42-137 and the
reference's own known answer (tests/cpp/search_cpu_tests.cpp, the 4 x 5
window with low_bits = 2)."""

import json
import os

import numpy as np
import pytest

from bmmpy_b200.matrix import BitMatrix
from bmmpy_b200.split_prep import build_compact_split_window, build_compact_split_window_dev
from oracle.oracle import port
from tests.golden.fixtures import matrix_from_rows

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _matrix(dense: np.ndarray) -> BitMatrix:
    """BitMatrix from a (rows, cols) boolean array, bit c of a row = column c."""
    rows, cols = dense.shape
    padded = np.zeros((rows, (cols + 63) // 64 * 64), np.uint8)
    padded[:, :cols] = dense
    words = np.packbits(padded, axis=1, bitorder="little").view("<u8")
    return BitMatrix.from_words(words, cols)


def _oracle(words, cols, win, low_bits):
    q, r, mult, tw = port().split_window(words, cols, win, low_bits)
    return [int(v) for v in q], [int(v) for v in r], [int(v) for v in mult], int(tw)


def _device(words, cols, win, low_bits):
    m = BitMatrix.from_words(np.ascontiguousarray(words), cols)
    out = build_compact_split_window(m.row_window(win), low_bits)
    return out.q, out.r, out.multiplicity, out.total_weight


def test_split_window_argument_checks_cpu():
    """The reference's checks run before any device work."""
    m = BitMatrix(65, 70)
    with pytest.raises(ValueError, match="low_bits must be <= number of rows"):
        build_compact_split_window(m.row_window([0, 1]), 3)
    with pytest.raises(ValueError, match="row count must be <= 64"):
        build_compact_split_window(m.row_window(list(range(65))), 2)
    empty = build_compact_split_window(m.row_window([]), 0)
    assert (empty.t, empty.q, empty.total_weight) == (0, [], 0)


@pytest.mark.gpu
def test_split_window_known_answer_gpu():
    with open(os.path.join(GOLDEN, "known_answers.json")) as f:
        exp = json.load(f)["split_4x5_low2"]
    words, cols = matrix_from_rows(["11001", "00100", "01101", "01001"])
    got = _device(words, cols, [0, 1, 2, 3], 2)
    assert got == (exp["q"], exp["r"], exp["mult"], exp["total_weight"])
    assert got == ([0, 1, 3], [1, 2, 1], [1, 1, 2], 4)


@pytest.mark.gpu
@pytest.mark.parametrize("t,cols,density,low_bits", [
    (1, 1, 0.5, 0), (1, 1, 0.5, 1), (3, 200, 0.3, 0), (5, 64, 0.4, 5), (8, 1000, 0.2, 3),
    (16, 4096, 0.05, 8), (24, 10000, 0.1, 14), (32, 65536, 0.02, 16), (40, 3000, 0.5, 20),
    (63, 777, 0.5, 33), (64, 5000, 0.5, 64), (64, 129, 0.5, 0),
])
def test_split_window_matches_oracle(t, cols, density, low_bits):
    rng = np.random.default_rng(t * 7919 + cols)
    rows = t + 3
    dense = rng.random((rows, cols)) < density
    dense[rows - 1, :] = False  # an all-zero row inside the window
    m = _matrix(dense)
    win = [int(v) for v in rng.permutation(rows - 1)[:t]]
    if t > 2:
        win[1] = rows - 1  # the all-zero row, at window position 1
    assert _device(m.words, cols, win, low_bits) == _oracle(m.words, cols, win, low_bits)


@pytest.mark.gpu
def test_split_window_multiplicity_and_duplicates():
    """Few distinct patterns over many columns: counts, ascending order and
    total weight; an all-zero window gives nothing."""
    cols = 100_000
    t = 6
    pats = np.array([0, 0b101, 0b111111, 0b000001, 0b100000])
    col_pat = pats[(np.arange(cols) * 7) % len(pats)]
    dense = np.zeros((t + 1, cols), bool)
    for i in range(t):
        dense[i] = (col_pat >> i) & 1
    m = _matrix(dense)
    win = list(range(t))
    got = _device(m.words, cols, win, 2)
    assert got == _oracle(m.words, cols, win, 2)
    assert got[3] == int(np.count_nonzero(col_pat))
    assert got[2] == [int(np.count_nonzero(col_pat == p)) for p in sorted(pats[1:])]
    assert _device(m.words, cols, [t], 1) == ([], [], [], 0)


@pytest.mark.gpu
def test_split_window_dev_tensors_and_capacity():
    import torch

    words, cols = matrix_from_rows(["11001", "00100", "01101", "01001"])
    d = torch.from_numpy(np.ascontiguousarray(words).view(np.int64)).cuda()
    q, r, mult, tw = build_compact_split_window_dev(d, cols, 2)
    assert q.is_cuda and mult.dtype == torch.int32
    assert (q.tolist(), r.tolist(), mult.tolist(), tw) == ([0, 1, 3], [1, 2, 1], [1, 1, 2], 4)
    # a wider W than the row width: bits past cols are ignored
    wide = torch.zeros((4, 3), dtype=torch.int64, device="cuda")
    wide[:, :1] = d[:, :1]
    wide[:, 2] = -1
    q2, r2, m2, tw2 = build_compact_split_window_dev(wide, cols, 2)
    assert (q2.tolist(), r2.tolist(), m2.tolist(), tw2) == ([0, 1, 3], [1, 2, 1], [1, 1, 2], 4)
