"""The reference's own GPU searchers (CudaBruteforceSearch, CudaMitmFwhtSearch,
built unmodified for sm_100a into oracle/_ref/cuda) against this library's
classes of the same names on the same windows: identical candidate lists.
Skipped where the reference CUDA build is absent."""

import random

import pytest

import bmmpy_b200 as bmm
from bmmpy_b200.matrix import BitMatrix
from oracle.oracle import port, ref_cuda

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rc():
    R = ref_cuda()
    if R is None:
        pytest.skip("reference CUDA build (make -C oracle ref-cuda) is absent")
    return R


@pytest.mark.parametrize("cols", [512, 1024, 4096])
def test_cuda_bruteforce_matches_reference_gpu(rc, cols):
    P = port()
    rng = random.Random(cols)
    for trial in range(3):
        rows = rng.randint(20, 30)
        words, _ = P.gen_instance(rows, cols, rng.choice([0.1, 0.3, 0.5]), 40 + trial, rows)
        m = BitMatrix.from_words(words, cols)
        t = rng.randint(16, min(rows, 20))
        win = sorted(rng.sample(range(rows), t))
        k = rng.choice([1, 16, 128])
        chunk = rng.choice([0, 5, t - 1])
        want = rc.cuda_bruteforce_search(words, cols, win, k, chunk)
        got = bmm.CudaBruteforceSearch(max_candidates=k, chunk_bits=chunk).search(
            m.row_window(win))
        assert [(c.mask_u64(), c.weight) for c in got] == want, (cols, trial)


def test_cuda_mitm_matches_reference_gpu(rc):
    P = port()
    rng = random.Random(3)
    for trial in range(4):
        rows = rng.randint(20, 26)
        cols = rng.choice([300, 1000, 2048])
        words, _ = P.gen_instance(rows, cols, rng.choice([0.05, 0.2, 0.4]), 70 + trial, rows)
        m = BitMatrix.from_words(words, cols)
        t = rng.randint(16, min(rows, 22))
        win = sorted(rng.sample(range(rows), t))
        k = rng.choice([8, 64, 128])
        low = rng.choice([0, 8, 12])
        want = rc.cuda_mitm_search(words, cols, win, k, low)
        got = bmm.CudaMitmFwhtSearch(max_candidates=k, low_bits=low).search(m.row_window(win))
        assert [(c.mask_u64(), c.weight) for c in got] == want, trial
