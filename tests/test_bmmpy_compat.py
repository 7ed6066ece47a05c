"""The reference's module names on the B200 build: ``import bmmpy`` through
bmmpy_b200/compat, and the native ``_bmmpy`` module (pybind11 over
include/bmmpy/).  CPU tests check names, argument errors and exception types;
GPU tests check the native searchers against the package's and the launch
seam against the window search."""

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
COMPAT = os.path.join(ROOT, "bmmpy_b200", "compat")


@pytest.fixture(scope="module")
def bmm():
    if COMPAT not in sys.path:
        sys.path.insert(0, COMPAT)
    import bmmpy

    return bmmpy


@pytest.fixture(scope="module")
def nb(bmm):
    from bmmpy import _bmmpy

    return _bmmpy


def test_module_names(bmm, nb):
    for name in ("BitMatrix", "RowWindow", "Candidate", "FwhtSearch", "MitmFwhtSearch",
                 "BruteforceSearch", "CudaMitmFwhtSearch", "CudaBruteforceSearch",
                 "GreedyApplier", "GlobalGreedyApplier", "search_apply", "SASelector",
                 "GeneticAlgorithm", "IslandModel", "get_runtime_features"):
        assert hasattr(bmm, name), name
    import bmmpy.ga
    import bmmpy.solver  # noqa: F401

    assert bmmpy.ga.GeneticAlgorithmConfig is not None
    for name in ("BitMatrix", "RowWindow", "Candidate", "FwhtSearch", "MitmFwhtSearch",
                 "BruteforceSearch", "CudaMitmFwhtSearch", "CudaBruteforceSearch",
                 "ExactBasisSolver", "fwht_inplace", "build_compact_split_window",
                 "run_cuda_mitm_fwht_search", "get_runtime_features", "MatrixError"):
        assert hasattr(nb, name), name
    assert nb.FwhtSearch().name() == "fwht"
    assert nb.CudaMitmFwhtSearch(max_candidates=8, low_bits=0).name() == "cuda_mitm_fwht"
    assert nb.CudaBruteforceSearch(max_candidates=8).name() == "cuda_bruteforce"
    assert nb.get_runtime_features().cuda_compiled


def test_native_matrix_and_errors(nb):
    m = nb.BitMatrix(4, 130)
    m[1, 129] = True
    assert m[1, 129] and not m[1, 128] and m.weight() == 1
    assert (m.stride_words, m.words_per_row) == (4, 3)
    with pytest.raises(IndexError):
        m[4, 0]
    with pytest.raises(IndexError):
        m.row_window([0, 9])
    w = nb.BitMatrix.from_rows(["1101", "0111", "1001"]).row_window([0, 1, 2])
    prep = nb.build_compact_split_window(w, 1)
    assert (prep.q, prep.r, prep.multiplicity, prep.total_weight) == (
        [1, 1, 2, 3], [0, 1, 1, 1], [1, 1, 1, 1], 4)
    assert nb.FwhtSearch(max_rows=2).search(w) == []  # t > max_rows: empty, as the reference
    with pytest.raises(ValueError):
        nb.CudaBruteforceSearch().search(w)  # fewer than 16 rows
    big = nb.BitMatrix(20, 40000)
    for c in range(40000):  # every column active in the 16-row window
        big[c % 16, c] = True
    with pytest.raises(ValueError, match="int16-safe"):
        nb.CudaMitmFwhtSearch().search(big.row_window(list(range(16))))
    with pytest.raises(ValueError):
        nb.fwht_inplace(np.zeros(3, np.int32))
    for c in (nb.Candidate.from_u64(0b1011, 7), bmm_candidate(0b1011, 7)):
        assert (len(c), c.rows, c.has_row(3), c.has_row(2)) == (3, [0, 1, 3], True, False)
        assert list(c) == [0, 1, 3] and 3 in c and 2 not in c


def bmm_candidate(mask, weight):
    import bmmpy

    return bmmpy.Candidate.from_u64(mask, weight)


@pytest.mark.gpu
def test_native_searchers_match_the_package(bmm, nb):
    rng = np.random.default_rng(3)
    bits = rng.random((30, 512)) < 0.3
    m = nb.BitMatrix(30, 512)
    pm = bmm.BitMatrix(30, 512)
    for r, c in zip(*np.nonzero(bits)):
        m[int(r), int(c)] = True
        pm[int(r), int(c)] = True
    win = list(range(2, 20))
    want = [(c.mask_u64(), c.weight) for c in
            bmm.BruteforceSearch(max_candidates=32).search(pm.row_window(win))]
    for s in (nb.FwhtSearch(max_rows=18, max_candidates=32), nb.MitmFwhtSearch(max_candidates=32),
              nb.BruteforceSearch(max_candidates=32),
              nb.CudaMitmFwhtSearch(max_candidates=32),
              nb.CudaBruteforceSearch(max_candidates=32)):
        assert [(c.mask_u64(), c.weight) for c in s.search(m.row_window(win))] == want, s.name()
    prep = nb.build_compact_split_window(m.row_window(win), 9)
    assert nb.run_cuda_mitm_fwht_search(prep, 32) == want
    x = np.arange(8, dtype=np.int32)
    nb.fwht_inplace(x)
    assert x.tolist() == [28, -4, -8, 0, -16, 0, 0, 0]
    r = nb.ExactBasisSolver().solve(nb.BitMatrix.identity(5).row_window(list(range(5))))
    assert (r.rank, r.total_weight, r.basis_matrix.weight()) == (5, 5, 5)
