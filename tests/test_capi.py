"""CPU suite: the C ABI library loads and exports every declared entry point;
the host-only parts (generator, argument checks that need no device) work."""

import ctypes
import os
import re

import numpy as np
import pytest

import bmmpy_b200 as bmm
from bmmpy_b200 import _native as N
from bmmpy_b200.workloads import batch_shape, gen_instance
from oracle.oracle import port
from tests.golden.fixtures import batch_shape as fixture_batch_shape

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            with open(os.path.join(ROOT, "include", fn)) as f:
                names |= set(re.findall(r"BMM_API\s+[\w\s\*]+?\b(bmm_\w+)\s*\(", f.read()))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    lib = N.lib()
    names = declared_symbols()
    assert len(names) >= 12
    for name in names:
        assert hasattr(lib, name), name
    # and the binding table covers them
    for name in names:
        assert name in N.SIGNATURES, name


def test_generator_matches_oracle():
    for args in [(40, 4096, 0.3, 1, 0), (64, 256, 0.5, 0, 0), (33, 1000, 0.05, 17, 132)]:
        m, planted = gen_instance(*args)
        m2, planted2 = port().gen_instance(*args)
        assert planted == planted2
        assert np.array_equal(m.words, m2)


def test_batch_shapes_match_fixture_rule():
    for idx in (0, 1, 77, 4095):
        n, m = batch_shape(idx)
        assert (n, m) == fixture_batch_shape(idx)
        assert 16 <= n <= 128 and 64 <= m <= 2048


def test_matrix_layout_and_window():
    m = bmm.matrix_from_rows(["10101", "10101"])
    assert m.shape == (2, 5) and m.stride_words == 4 and m.weight() == 6
    assert m.to_rows() == ["10101", "10101"]
    w = m.row_window([1, 0])
    assert w.rows == [1, 0] and w.total_weight == 3
    with pytest.raises(ValueError):
        m.row_window([0, 0])
    with pytest.raises(IndexError):
        m.row_window([2])


def test_candidate_api():
    c = bmm.Candidate.from_u64(0b1011, 7)
    assert c.rows == [0, 1, 3] and len(c) == 3 and 3 in c and 2 not in c
    assert c.mask_u64() == 11
    with pytest.raises(RuntimeError):
        bmm.Candidate([1, 1], 0).mask_u64()


def test_fwht_search_rejects_oversized_window_on_host():
    m = bmm.BitMatrix(20, 8)
    with pytest.raises(ValueError):
        bmm.FwhtSearch(max_rows=16).search(m.row_window(list(range(17))))


def test_cuda_searchers_validate_like_reference():
    # src/search/cuda_*_search.cpp argument checks, before any device work
    m = bmm.matrix_from_rows(["10101", "11100", "00111"])
    with pytest.raises(ValueError):
        bmm.CudaMitmFwhtSearch().search(m.row_window([0, 1, 2]))
    with pytest.raises(ValueError):
        bmm.CudaBruteforceSearch().search(m.row_window([0, 1, 2]))
    m = bmm.BitMatrix(16, 256)
    with pytest.raises(ValueError):
        bmm.CudaBruteforceSearch().search(m.row_window(list(range(16))))
    m = bmm.BitMatrix(28, 4)
    m[0, 0] = True
    with pytest.raises(ValueError):
        bmm.CudaMitmFwhtSearch(max_candidates=64, low_bits=28).search(m.row_window(list(range(28))))
    m = bmm.BitMatrix(28, 32768)
    for c in range(32768):
        m[0, c] = True
    with pytest.raises(ValueError):
        bmm.CudaMitmFwhtSearch().search(m.row_window(list(range(28))))
    assert bmm.CudaMitmFwhtSearch(max_candidates=8).name() == "cuda_mitm_fwht"
    assert bmm.CudaBruteforceSearch(max_candidates=8).name() == "cuda_bruteforce"
