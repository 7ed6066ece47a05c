"""ExactBasisSolver on the GPU against the reference's goldens and the oracle
(src/solver/exact_basis_solver.cpp:58-157): bit-exact basis masks, weights,
total weight, transform and basis matrices; the weight histogram of the
device enumeration (shared-memory bins, global bins, and the slab-by-slab
path for rows wider than one shared-memory slab); the reference's default
24-row cap and a 26-row window against the oracle; and at 32 rows, where the
oracle would take minutes, the MacWilliams identity between the histogram
of all 2^32 - 1 combinations and the dual code enumerated on the CPU."""

import math
import os
import random

import numpy as np
import pytest

import bmmpy_b200 as bmm
from bmmpy_b200 import _native as N
from oracle.oracle import port
from tests.golden.fixtures import BASIS_CASES

pytestmark = pytest.mark.gpu

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "workloads.npz"))
BIG = dict(max_rows=32, max_states=(1 << 32) - 1, max_storage_bytes=1 << 40)


def _bitmatrix(words, rows, cols):
    m = bmm.BitMatrix(rows, cols)
    m.words[:] = words[:rows, : m.stride_words]
    return m


def _device_counts(m, win):
    counts = np.zeros(m.cols + 1, np.uint64)
    w = np.asarray(win, np.uint32)
    N.check(N.lib().bmm_basis_weight_counts(N.u64p(m.words), m.stride_words, m.cols, N.u32p(w),
                                            len(w), N.u64p(counts)))
    return counts


def _check_consistent(r, window):
    assert r.transform_matrix.shape == (r.rank, window.size)
    assert r.basis_matrix == r.transform_matrix.mul(window.materialize())
    assert r.basis_matrix.rank() == r.rank == window.materialize().rank()
    assert [r.basis_matrix.row_popcount(i) for i in range(r.rank)] == r.basis_weights
    assert r.total_weight == sum(r.basis_weights)
    assert r.basis_weights == sorted(r.basis_weights)


def test_reference_example():
    # tests/python/test_matrix_api.py:45-64
    matrix = bmm.matrix_from_rows(["111", "110", "001"])
    window = matrix.row_window([0, 1, 2])
    result = bmm.solver.ExactBasisSolver().solve(window)
    assert result.input_rows == 3
    assert result.cols == 3
    assert result.rank == 2
    assert result.enumerated_states == 7
    assert result.total_weight == 3
    assert sorted(result.basis_weights) == [1, 2]
    assert result.transform_matrix.shape == (2, 3)
    assert result.basis_matrix.shape == (2, 3)
    assert result.basis_matrix.rank() == 2
    assert result.basis_matrix.weight() == 3


@pytest.mark.parametrize("case", range(len(BASIS_CASES)))
def test_matches_reference_goldens(case):
    rows, cols, p, iseed, scr, win = BASIS_CASES[case]
    words, _ = port().gen_instance(rows, cols, p, iseed, scr)
    m = _bitmatrix(words, rows, cols)
    window = m.row_window(win)
    r = bmm.solver.ExactBasisSolver().solve(window)
    sc = GOLD[f"basis{case}_scalars"].tolist()
    assert [r.input_rows, r.cols, r.rank, r.enumerated_states, r.total_weight] == sc
    assert r.basis_masks == GOLD[f"basis{case}_masks"].tolist()
    assert r.basis_weights == GOLD[f"basis{case}_weights"].tolist()
    assert r.transform_matrix.words[:, 0].tolist() == GOLD[f"basis{case}_transform"].tolist()
    if f"basis{case}_words" in GOLD:
        gw = GOLD[f"basis{case}_words"]
        assert np.array_equal(r.basis_matrix.words[:, : gw.shape[1]], gw[:, : r.basis_matrix.stride_words])
    _check_consistent(r, window)


def test_matches_oracle_random():
    rng = random.Random(21)
    P = port()
    for trial in range(60):
        t = rng.randint(1, 20)
        cols = rng.choice([1, 3, 63, 64, 65, 200, 256, 511, 1000, 5000])
        rows = t + rng.randint(0, 5)
        words, _ = P.gen_instance(rows, cols, rng.choice([0.01, 0.05, 0.2, 0.5]), 100 + trial,
                                  rng.randint(0, 40))
        if trial % 4 == 0 and rows > 3:
            words[3] = words[0] ^ words[1]
        if trial % 6 == 0:
            words[0] = 0
        if trial % 9 == 0 and rows > 1:
            words[1] = words[rows - 1]
        win = rng.sample(range(rows), t)
        m = _bitmatrix(words, rows, cols)
        r = bmm.solver.ExactBasisSolver(**BIG).solve(m.row_window(win))
        masks, weights, total = P.exact_basis(np.ascontiguousarray(m.words), cols, win)
        assert (r.basis_masks, r.basis_weights, r.total_weight) == (masks, weights, total), trial
        assert r.rank == len(masks)


@pytest.mark.parametrize("t,cols,p", [
    (16, 300, 0.3),      # bins in shared memory
    (10, 20000, 0.05),   # bins in global memory
    (12, 140000, 0.01),  # rows wider than one shared-memory slab
    (20, 70000, 0.003),  # 20 rows: slab of 1024 words, rows of 1094
    (5, 64, 0.5),        # fewer states than one sweep
    (1, 7, 0.5),
])
def test_weight_counts_match_oracle(t, cols, p):
    words, _ = port().gen_instance(t + 2, cols, p, 7 * t + cols, 0)
    m = _bitmatrix(words, t + 2, cols)
    win = list(range(2, t + 2))
    got = _device_counts(m, win)
    want = port().basis_weight_counts(np.ascontiguousarray(m.words), cols, win)
    assert np.array_equal(got, want)


def test_wide_rows_solve_matches_oracle():
    words, _ = port().gen_instance(14, 140000, 0.01, 16, 20)
    m = _bitmatrix(words, 14, 140000)
    r = bmm.solver.ExactBasisSolver().solve(m.row_window(list(range(14))))
    masks, weights, total = port().exact_basis(np.ascontiguousarray(m.words), 140000,
                                               list(range(14)))
    assert (r.basis_masks, r.basis_weights, r.total_weight) == (masks, weights, total)


@pytest.mark.parametrize("t,cols,p,caps", [
    (24, 256, 0.5, {}),          # the reference's default max_rows cap
    (24, 4096, 0.02, {}),
    (26, 320, 0.1, BIG),
])
def test_full_size_matches_oracle(t, cols, p, caps):
    words, _ = port().gen_instance(t, cols, p, 1000 + t, 3 * t)
    m = _bitmatrix(words, t, cols)
    window = m.row_window(list(range(t)))
    r = bmm.solver.ExactBasisSolver(**caps).solve(window)
    masks, weights, total = port().exact_basis(np.ascontiguousarray(m.words), cols,
                                               list(range(t)))
    assert (r.basis_masks, r.basis_weights, r.total_weight) == (masks, weights, total)
    _check_consistent(r, window)


def _dual_distribution(rows_bits, n):
    """Weight distribution of the dual code of the row space (null space)."""
    G = [int(r) for r in rows_bits]
    piv = []
    basis = []
    for v in G:
        for b, pc in zip(basis, piv):
            if (v >> pc) & 1:
                v ^= b
        if v:
            pc = v.bit_length() - 1
            for i in range(len(basis)):
                if (basis[i] >> pc) & 1:
                    basis[i] ^= v
            basis.append(v)
            piv.append(pc)
    free = [c for c in range(n) if c not in piv]
    null = []
    for f in free:
        x = 1 << f
        for b, pc in zip(basis, piv):
            if (b >> f) & 1:
                x |= 1 << pc
        null.append(x)
    dist = [0] * (n + 1)
    for s in range(1 << len(null)):
        x = 0
        for i in range(len(null)):
            if (s >> i) & 1:
                x ^= null[i]
        dist[bin(x).count("1")] += 1
    return dist


def _krawtchouk(j, i, n):
    return sum((-1) ** s * math.comb(i, s) * math.comb(n - i, j - s) for s in range(j + 1))


def test_macwilliams_identity_at_32_rows():
    t, n = 32, 40
    rng = np.random.default_rng(32)
    while True:
        bits = rng.random((t, n)) < 0.5
        m = bmm.BitMatrix(t, n)
        for r in range(t):
            for c in np.nonzero(bits[r])[0]:
                m[r, int(c)] = True
        if m.rank() == t:
            break
    counts = _device_counts(m, list(range(t)))
    assert int(counts.sum()) == (1 << t) - 1 and counts[0] == 0
    A = [int(x) for x in counts]
    A[0] += 1  # the zero codeword
    B = [sum(A[i] * _krawtchouk(j, i, n) for i in range(n + 1)) for j in range(n + 1)]
    assert all(b % (1 << t) == 0 for b in B)
    rows_bits = [int(m.words[r, 0]) for r in range(t)]
    assert [b >> t for b in B] == _dual_distribution(rows_bits, n)
    # and the solver at 32 rows: a consistent basis whose lightest vector is
    # the lightest nonzero combination
    r = bmm.solver.ExactBasisSolver(**BIG).solve(m.row_window(list(range(t))))
    _check_consistent(r, m.row_window(list(range(t))))
    assert r.basis_weights[0] == min(w for w in range(1, n + 1) if counts[w])
