"""Searchers with the reference's names, arguments and error behaviour.

Each class mirrors its bmmpy counterpart (bmmpy/search.py, python/bindings/
search.cpp, include/bmmpy/search/*.hpp) and runs on the B200 through the
C ABI (include/bmm_b200.h).  ``search(window)`` returns candidates ordered by
(weight, mask); masks are over the window's local rows.

The classes named after the reference's CPU searchers (FwhtSearch,
MitmFwhtSearch, BruteforceSearch) accept what the CPU versions accept.  The
Cuda* classes keep the reference CUDA searchers' stricter argument checks
(window of 16..64 rows, at most 128 candidates, brute-force widths of 512,
1024 or 4096 columns, the int16-safe total weight for MITM) so that code and
tests written against them behave identically.
"""

from __future__ import annotations

import numpy as np

from . import _native as N
from .candidate import Candidate
from .matrix import RowWindow


def _window_args(window: RowWindow):
    m = window.matrix
    words = np.ascontiguousarray(m.words)
    win = np.ascontiguousarray(window.index_array())
    return words, m.stride_words, m.cols, win


def _candidates(buf: np.ndarray, count: int) -> list[Candidate]:
    return [Candidate.from_u64(int(buf["mask"][i]), int(buf["weight"][i])) for i in range(count)]


def _run_window_search(fn, window: RowWindow, k: int, *extra) -> list[Candidate]:
    words, stride, cols, win = _window_args(window)
    t = len(win)
    kk = max(1, min(int(k), (1 << min(t, 40)) - 1 if t else 1))
    out = np.zeros(kk, dtype=N.CAND_DTYPE)
    count = N.C.c_size_t(0)
    rc = fn(N.u64p(words), stride, cols, N.u32p(win), t, *extra, N.candp(out), N.C.byref(count))
    N.check(rc)
    return _candidates(out, count.value)


class FwhtSearch:
    """Column-pattern histogram + Walsh-Hadamard spectrum (src/search/fwht_search.cpp)."""

    __slots__ = ("max_rows", "max_candidates")

    def __init__(self, *, max_rows: int = 16, max_candidates: int = 64) -> None:
        self.max_rows = max_rows
        self.max_candidates = max_candidates

    def __repr__(self) -> str:
        return f"FwhtSearch(max_rows={self.max_rows}, max_candidates={self.max_candidates})"

    def name(self) -> str:
        return "fwht"

    def search(self, window: RowWindow) -> list[Candidate]:
        if len(window) > self.max_rows:  # bmmpy/search.py:202-207
            raise ValueError(
                f"Window has {len(window)} rows, which exceeds the configured "
                f"max_rows={self.max_rows} limit for this searcher.")
        if self.max_candidates == 0 or len(window) == 0:
            return []
        return _run_window_search(N.lib().bmm_fwht_search, window, self.max_candidates,
                                  self.max_rows, self.max_candidates)


class MitmFwhtSearch:
    """Meet-in-the-middle FWHT (src/search/mitm_fwht_search.cpp); exact in int32."""

    __slots__ = ("max_candidates", "low_bits")

    def __init__(self, *, max_candidates: int = 64, low_bits: int = 0) -> None:
        self.max_candidates = max_candidates
        self.low_bits = low_bits

    def __repr__(self) -> str:
        return f"MitmFwhtSearch(max_candidates={self.max_candidates})"

    def name(self) -> str:
        return "mitm_fwht"

    def search(self, window: RowWindow) -> list[Candidate]:
        if self.max_candidates == 0 or len(window) == 0:
            return []
        if len(window) > 64:
            raise ValueError("MitmFwhtSearch: window_rows size must be <= 64")
        return _run_window_search(N.lib().bmm_mitm_search, window, self.max_candidates,
                                  self.max_candidates, self.low_bits)


class BruteforceSearch:
    """Exact Gray-code enumeration (src/search/bruteforce_search.cpp)."""

    __slots__ = ("max_candidates", "chunk_bits")

    def __init__(self, *, max_candidates: int = 64, chunk_bits: int = 0) -> None:
        self.max_candidates = max_candidates
        self.chunk_bits = chunk_bits

    def __repr__(self) -> str:
        return (f"BruteforceSearch(max_candidates={self.max_candidates}, "
                f"chunk_bits={self.chunk_bits})")

    def name(self) -> str:
        return "bruteforce"

    def search(self, window: RowWindow) -> list[Candidate]:
        if self.max_candidates == 0 or len(window) == 0:
            return []
        return _run_window_search(N.lib().bmm_gray_search, window, self.max_candidates,
                                  self.max_candidates, self.chunk_bits)


class CudaMitmFwhtSearch:
    """Same interface and checks as the reference CudaMitmFwhtSearch
    (src/search/cuda_mitm_fwht_search.cpp:123-180)."""

    __slots__ = ("max_candidates", "low_bits")
    k_min_rows, k_max_rows, k_max_low_bits = 16, 64, 15

    def __init__(self, *, max_candidates: int = 64, low_bits: int = 0) -> None:
        self.max_candidates = max_candidates
        self.low_bits = low_bits

    def __repr__(self) -> str:
        return f"CudaMitmFwhtSearch(max_candidates={self.max_candidates}, low_bits={self.low_bits})"

    def name(self) -> str:
        return "cuda_mitm_fwht"

    def search(self, window: RowWindow) -> list[Candidate]:
        if self.max_candidates == 0:
            return []
        t = len(window)
        if t == 0:
            return []
        if t > 64:
            raise ValueError("CudaMitmFwhtSearch: too many rows in the window (must be <= 64)")
        if t < self.k_min_rows or t > self.k_max_rows:
            raise ValueError(
                "CudaMitmFwhtSearch: window_rows size is outside the supported GPU range")
        if self.low_bits != 0 and self.low_bits >= t:
            raise ValueError("CudaMitmFwhtSearch: low_bits must be in [1, t - 1] or 0 for auto")
        if self.low_bits > self.k_max_low_bits:
            raise ValueError(
                "CudaMitmFwhtSearch: low_bits exceeds the specialized CUDA template range")
        if window.cols == 0:
            return []
        if window.total_weight > 32767:
            raise ValueError(
                "CudaMitmFwhtSearch: total_weight must be <= 32767 for int16-safe GPU mode")
        if self.max_candidates > 128:
            raise ValueError("run_cuda_mitm_fwht_search: max_candidates must be <= 128")
        return _run_window_search(N.lib().bmm_mitm_search, window, self.max_candidates,
                                  self.max_candidates, self.low_bits)


class CudaBruteforceSearch:
    """Same interface and checks as the reference CudaBruteforceSearch
    (src/search/cuda_bruteforce_search.cpp:38-103)."""

    __slots__ = ("max_candidates", "chunk_bits")
    k_min_rows, k_max_rows = 16, 64

    def __init__(self, *, max_candidates: int = 64, chunk_bits: int = 0) -> None:
        self.max_candidates = max_candidates
        self.chunk_bits = chunk_bits

    def __repr__(self) -> str:
        return (f"CudaBruteforceSearch(max_candidates={self.max_candidates}, "
                f"chunk_bits={self.chunk_bits})")

    def name(self) -> str:
        return "cuda_bruteforce"

    def search(self, window: RowWindow) -> list[Candidate]:
        if self.max_candidates == 0:
            return []
        t = len(window)
        if t == 0:
            return []
        if t > 64:
            raise ValueError("CudaBruteforceSearch: too many rows in the window (must be <= 64)")
        if t < self.k_min_rows or t > self.k_max_rows:
            raise ValueError(
                "CudaBruteforceSearch: window_rows size is outside the supported GPU range")
        if self.max_candidates > 128:
            raise ValueError("CudaBruteforceSearch: max_candidates must be <= 128")
        wpr = window.matrix.words_per_row
        if wpr == 0:
            return []
        if wpr not in (8, 16, 64):
            raise ValueError("CudaBruteforceSearch: only widths 512, 1024, and 4096 are "
                             "supported in the current GPU path")
        if self.chunk_bits != 0 and self.chunk_bits >= t:
            raise ValueError(
                "CudaBruteforceSearch: chunk_bits must be in [1, t - 1] or 0 for auto")
        return _run_window_search(N.lib().bmm_gray_search, window, self.max_candidates,
                                  self.max_candidates, self.chunk_bits)
