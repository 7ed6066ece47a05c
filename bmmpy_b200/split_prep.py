"""CompactSplitWindow / build_compact_split_window, built on the device.

Reference: include/bmmpy/search/split_window_prep.hpp:10-26 and
src/search/split_window_prep.cpp:42-137 (the CUDA MITM searcher's host-side
preparation, src/search/cuda_mitm_fwht_search.cpp:155).  The window's
distinct column patterns (bit i = row i of the window), ascending, with
their multiplicities, each split into q = pattern >> low_bits and
r = pattern & (2^low_bits - 1); total_weight = the number of active columns.
Same argument checks and messages as the reference.

``build_compact_split_window_dev`` keeps everything in device memory (the
form a device-side consumer wants); ``build_compact_split_window`` takes a
RowWindow like the reference's overload and returns host lists.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _native as N
from .matrix import RowWindow


@dataclass
class CompactSplitWindow:
    t: int = 0
    low_bits: int = 0
    high_bits: int = 0
    total_weight: int = 0
    q: list = field(default_factory=list)
    r: list = field(default_factory=list)
    multiplicity: list = field(default_factory=list)


def _check_args(t: int, low_bits: int) -> None:
    if low_bits > t:
        raise ValueError("build_compact_split_window: low_bits must be <= number of rows")
    if t > 64:
        raise ValueError("build_compact_split_window: row count must be <= 64")


def build_compact_split_window_dev(d_rows, cols: int, low_bits: int, stream=None):
    """Device build over ``d_rows`` (a CUDA int64/uint64 tensor, t x W words,
    W >= ceil(cols / 64); bits past ``cols`` are ignored).

    Returns ``(q, r, multiplicity, total_weight)``: q, r int64 tensors and
    multiplicity an int32 tensor on the same device, one entry per distinct
    nonzero pattern in ascending pattern order, and total_weight an int.
    """
    import torch

    t = int(d_rows.shape[0]) if d_rows.dim() == 2 else 0
    W = int(d_rows.shape[1]) if d_rows.dim() == 2 else 0
    _check_args(t, int(low_bits))
    dev = d_rows.device
    cap = max(1, int(cols))
    q = torch.empty(cap, dtype=torch.int64, device=dev)
    r = torch.empty(cap, dtype=torch.int64, device=dev)
    mult = torch.empty(cap, dtype=torch.int32, device=dev)
    if t and W and cols:
        d_rows = d_rows.contiguous()
    n_unique = C.c_size_t(0)
    tw = C.c_int32(0)
    if stream is None:
        stream = torch.cuda.current_stream(dev).cuda_stream if dev.type == "cuda" else None
    N.check(N.lib().bmm_split_window_dev(d_rows.data_ptr() if t and W else None, t, W, int(cols),
                                         int(low_bits), q.data_ptr(), r.data_ptr(),
                                         mult.data_ptr(), cap, C.byref(n_unique),
                                         C.byref(tw), stream),
            "build_compact_split_window")
    n = int(n_unique.value)
    return q[:n], r[:n], mult[:n], int(tw.value)


def build_compact_split_window(window: RowWindow, low_bits: int) -> CompactSplitWindow:
    """The reference's ``build_compact_split_window(const RowWindow&, low_bits)``,
    computed on the current CUDA device."""
    t = len(window)
    low_bits = int(low_bits)
    _check_args(t, low_bits)
    out = CompactSplitWindow(t=t, low_bits=low_bits, high_bits=t - low_bits)
    m = window.matrix
    W = m.words_per_row
    if t == 0 or W == 0 or m.cols == 0:
        return out
    import torch

    dev = torch.device("cuda", torch.cuda.current_device())
    rows = np.ascontiguousarray(m.words[window.index_array(), :W]).view(np.int64)
    d_rows = torch.from_numpy(rows).to(dev)
    q, r, mult, tw = build_compact_split_window_dev(d_rows, m.cols, low_bits)
    out.total_weight = tw
    out.q = [int(v) for v in q.cpu().numpy().view(np.uint64)]
    out.r = [int(v) for v in r.cpu().numpy().view(np.uint64)]
    out.multiplicity = [int(v) for v in mult.cpu().numpy()]
    return out


__all__ = ["CompactSplitWindow", "build_compact_split_window", "build_compact_split_window_dev"]
