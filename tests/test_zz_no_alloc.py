"""The allocation-free per-target entry point (bmm_gray_targets_noalloc).

It exists for callers that may not allocate device memory -- a host
framework's pool or arena that must account for every byte, plug-ins whose
host forbids cudaMalloc/cudaFree, latency-critical loops.  Its scratch is a
fixed 128 KiB device array inside the library, shared by every call.

This file is named so that pytest collects it last.  Each test below calls
the new entry point through the C ABI twice in a row (different inputs, so a
stale key left by the first call would show up in the second) and compares
both results with the existing allocating entry point, bmm_gray_targets_dev.
Results are integers: the comparison is exact.
"""

import ctypes

import numpy as np
import pytest

from bmmpy_b200 import _native as N
from bmmpy_b200.targets import cyclic_others
from bmmpy_b200.workloads import gen_instance

MAX_TARGETS = 16384


def _device_inputs(torch, rows, cols, k, seed):
    m, _ = gen_instance(rows, cols, 0.3, seed, rows)
    t, o = cyclic_others(rows, k)
    dev = torch.device("cuda", 0)
    d_words = torch.from_numpy(m.words.view(np.int64).copy()).to(dev)
    d_t = torch.from_numpy(t.view(np.int32).copy()).to(dev)
    d_o = torch.from_numpy(o.view(np.int32).copy()).to(dev)
    return m, d_words, d_t, d_o


def _call(fn, torch, m, d_words, d_t, d_o, k, tiebreak):
    rows = d_t.numel()
    masks = torch.full((rows,), -1, dtype=torch.int64, device=d_words.device)
    weights = torch.full((rows,), -1, dtype=torch.int32, device=d_words.device)
    stream = torch.cuda.current_stream().cuda_stream
    rc = fn(d_words.data_ptr(), m.rows, m.stride_words, m.cols, d_t.data_ptr(), d_o.data_ptr(),
            rows, k, tiebreak, masks.data_ptr(), weights.data_ptr(), stream)
    N.check(rc)
    torch.cuda.synchronize()
    return masks.cpu().numpy(), weights.cpu().numpy()


@pytest.mark.gpu
@pytest.mark.parametrize("tiebreak", [0, 1])
def test_noalloc_matches_allocating_entry_point_twice(tiebreak):
    import torch

    lib = N.lib()
    cases = [(40, 4096, 14, 3), (64, 256, 16, 4)]  # two calls in a row, different inputs
    for rows, cols, k, seed in cases:
        m, d_words, d_t, d_o = _device_inputs(torch, rows, cols, k, seed)
        want = _call(lib.bmm_gray_targets_dev, torch, m, d_words, d_t, d_o, k, tiebreak)
        got = _call(lib.bmm_gray_targets_noalloc, torch, m, d_words, d_t, d_o, k, tiebreak)
        assert np.array_equal(got[0], want[0])
        assert np.array_equal(got[1], want[1])
        assert (got[1] >= 0).all()


@pytest.mark.gpu
def test_noalloc_rejects_more_targets_than_its_scratch():
    import torch

    lib = N.lib()
    dev = torch.device("cuda", 0)
    n = MAX_TARGETS + 1
    words = torch.zeros((2, 4), dtype=torch.int64, device=dev)
    idx = torch.zeros(n, dtype=torch.int32, device=dev)
    out = torch.zeros(n, dtype=torch.int64, device=dev)
    rc = lib.bmm_gray_targets_noalloc(words.data_ptr(), 2, 4, 64, idx.data_ptr(), idx.data_ptr(),
                                      n, 1, 0, out.data_ptr(), out.data_ptr(),
                                      torch.cuda.current_stream().cuda_stream)
    assert rc == N.EINVAL
    assert "16384" in N.last_error()
