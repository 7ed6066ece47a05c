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

``SASelector`` (window selection by simulated annealing) mirrors the
reference's selector of the same name.
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


_SCORE_POLICIES = {"pairwise_synergy": 0, "higher_order_synergy": 1}
_COOLING_POLICIES = {"adaptive_geometric": 0}


def _resolve_score_policy(name: str) -> int:
    if name in _SCORE_POLICIES:
        return _SCORE_POLICIES[name]
    raise ValueError(f"Unsupported score_policy: {name!r}")


def _resolve_cooling_policy(name: str) -> int:
    if name in _COOLING_POLICIES:
        return _COOLING_POLICIES[name]
    raise ValueError(f"Unsupported cooling_policy: {name!r}")


class SASelectionResult:
    """SASelectionResult (include/bmmpy/search/sa_selector.hpp:37-45)."""

    __slots__ = ("rows", "score", "accepted_moves", "iterations_run", "best_iteration",
                 "restart_index", "seed")

    def __init__(self) -> None:
        self.rows: list[int] = []
        self.score = 0
        self.accepted_moves = 0
        self.iterations_run = 0
        self.best_iteration = 0
        self.restart_index = 0
        self.seed = 0

    def __repr__(self) -> str:
        return (f"SASelectionResult(rows={self.rows}, score={self.score}, "
                f"restart_index={self.restart_index})")


class SASelector:
    """Simulated-annealing window selection (bmmpy/search.py:416-537).

    Same keyword arguments, checks, results and seed semantics as the reference:
    the pairwise synergy table is built on the GPU and the annealing chain
    (bmm_sa_select) replays the reference's generator stream exactly.
    """

    __slots__ = ("iterations", "restarts", "seed", "score_policy", "cooling_policy",
                 "temperature_probe_samples", "initial_acceptance_probability", "cooling_rate",
                 "min_temperature", "_cfg")

    def __init__(self, *, iterations: int = 10000, restarts: int = 8, seed: int = 0,
                 score_policy: str = "pairwise_synergy",
                 cooling_policy: str = "adaptive_geometric",
                 temperature_probe_samples: int = 64,
                 initial_acceptance_probability: float = 0.8, cooling_rate: float = 0.99,
                 min_temperature: float = 1e-6) -> None:
        self._cfg = N.SaConfig_t(iterations, restarts, seed, _resolve_score_policy(score_policy),
                                 _resolve_cooling_policy(cooling_policy),
                                 temperature_probe_samples, initial_acceptance_probability,
                                 cooling_rate, min_temperature)
        self.iterations = iterations
        self.restarts = restarts
        self.seed = seed
        self.score_policy = score_policy
        self.cooling_policy = cooling_policy
        self.temperature_probe_samples = temperature_probe_samples
        self.initial_acceptance_probability = initial_acceptance_probability
        self.cooling_rate = cooling_rate
        self.min_temperature = min_temperature

    def __repr__(self) -> str:
        return ("SASelector("
                f"iterations={self.iterations}, "
                f"restarts={self.restarts}, "
                f"seed={self.seed}, "
                f"score_policy={self.score_policy!r}, "
                f"cooling_policy={self.cooling_policy!r}, "
                f"temperature_probe_samples={self.temperature_probe_samples}, "
                f"initial_acceptance_probability={self.initial_acceptance_probability}, "
                f"cooling_rate={self.cooling_rate}, "
                f"min_temperature={self.min_temperature})")

    def name(self) -> str:
        return "sa"

    def select(self, matrix, window_size: int) -> SASelectionResult:
        """src/search/sa_selector.cpp:10-75."""
        if window_size < 0:
            raise ValueError("window_size must be non-negative")
        res = N.SaResult_t()
        rows = np.zeros(max(1, window_size), dtype=np.uintp)
        words = np.ascontiguousarray(matrix.words)
        N.check(N.lib().bmm_sa_select(N.u64p(words), matrix.stride_words, matrix.rows,
                                      matrix.cols, window_size, self._cfg, res,
                                      rows.ctypes.data_as(N._szp)), "bmm_sa_select")
        out = SASelectionResult()
        out.rows = [int(r) for r in rows[: res.n_rows]]
        out.score = int(res.score)
        out.accepted_moves = int(res.accepted_moves)
        out.iterations_run = int(res.iterations_run)
        out.best_iteration = int(res.best_iteration)
        out.restart_index = int(res.restart_index)
        out.seed = int(res.seed)
        return out

    def select_window(self, matrix, window_size: int) -> RowWindow:
        return matrix.row_window(self.select(matrix, window_size).rows)
