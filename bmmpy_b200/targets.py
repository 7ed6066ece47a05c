"""Per-target searches: for each target row, the best XOR of k other rows.

This is the reference's window search over the (k+1)-row window
[target, o_1..o_k] restricted to masks with bit 0 set: its best mask there is
(S << 1) | 1, with S the bitmask over the others returned here, and the
weight is popcount(row[target] ^ XOR_{j in S} row[o_j]) (S = 0 included).

Host entry points take numpy arrays (the library stages them to the device);
the ``*_dev`` variants take CUDA tensors that are already resident (anything
exposing ``data_ptr()``) and run asynchronously on ``stream`` (an int handle).
"""

from __future__ import annotations

import numpy as np

from . import _native as N
from .matrix import BitMatrix


def cyclic_others(rows: int, k: int, offset: int = 1) -> tuple[np.ndarray, np.ndarray]:
    """targets 0..rows-1 with others (i + offset + j) mod rows, j < k."""
    t = np.arange(rows, dtype=np.uint32)
    o = ((t[:, None] + offset + np.arange(k, dtype=np.uint32)[None, :]) % rows).astype(np.uint32)
    return t, np.ascontiguousarray(o)


def _host_call(fn, matrix: BitMatrix, targets, others, extra):
    words = np.ascontiguousarray(matrix.words)
    targets = np.ascontiguousarray(targets, dtype=np.uint32)
    others = np.ascontiguousarray(others, dtype=np.uint32)
    n = targets.size
    k = others.shape[1] if others.ndim == 2 else (others.size // max(n, 1))
    masks = np.zeros(n, np.uint64)
    weights = np.zeros(n, np.uint32)
    rc = fn(N.u64p(words), matrix.rows, matrix.stride_words, matrix.cols, N.u32p(targets),
            N.u32p(others), n, k, *extra, N.u64p(masks), N.u32p(weights))
    N.check(rc)
    return masks, weights


def gray_targets(matrix: BitMatrix, targets, others, tiebreak: str = "mask"):
    """Exhaustive reflected-Gray enumeration of all 2^k subsets per target.
    tiebreak: "mask" (smallest S, the reference order) or "gray" (smallest
    Gray index)."""
    tb = {"mask": 0, "gray": 1}[tiebreak]
    return _host_call(N.lib().bmm_gray_targets, matrix, targets, others, (tb,))


def fwht_targets(matrix: BitMatrix, targets, others):
    """Signed column histogram + Walsh-Hadamard spectrum per target (k <= 16)."""
    return _host_call(N.lib().bmm_fwht_targets, matrix, targets, others, ())


def gray_targets_dev(words, rows, stride, cols, targets, others, k, masks_out, weights_out,
                     tiebreak: int = 0, stream: int = 0) -> None:
    rc = N.lib().bmm_gray_targets_dev(words.data_ptr(), rows, stride, cols, targets.data_ptr(),
                                      others.data_ptr(), targets.numel(), k, tiebreak,
                                      masks_out.data_ptr(), weights_out.data_ptr(), stream)
    N.check(rc)


def fwht_targets_dev(words, rows, stride, cols, targets, others, k, masks_out, weights_out,
                     stream: int = 0) -> None:
    rc = N.lib().bmm_fwht_targets_dev(words.data_ptr(), rows, stride, cols, targets.data_ptr(),
                                      others.data_ptr(), targets.numel(), k, masks_out.data_ptr(),
                                      weights_out.data_ptr(), stream)
    N.check(rc)
