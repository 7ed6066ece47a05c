"""Search-then-apply workflow (bmmpy/workflows.py:45-90), per window on host
matrices, or as device-resident sweeps over many windows (``DeviceMatrix``)."""

from __future__ import annotations

from collections.abc import Iterable
from typing import Protocol

from .apply import ApplyResult
from .candidate import Candidate
from .matrix import RowWindow

__all__ = ["DeviceMatrix", "search_apply"]


class SupportsSearch(Protocol):
    def search(self, window: RowWindow) -> list[Candidate]: ...


class SupportsApply(Protocol):
    def apply(self, window: RowWindow, candidates: Iterable[Candidate]) -> ApplyResult: ...


def search_apply(window: RowWindow, *, searcher: SupportsSearch,
                 applier: SupportsApply) -> ApplyResult:
    """Run ``searcher.search(window)`` and apply its candidates to the same
    window (the underlying matrix is mutated in place)."""
    candidates = searcher.search(window)
    return applier.apply(window, candidates)


class DeviceMatrix:
    """A BitMatrix kept in device memory for search -> apply sweeps.

    ``search_apply(windows, searcher=..., applier=...)`` runs
    ``search_apply(matrix.row_window(w), ...)`` for each window ``w`` in order
    (bmmpy/workflows.py:45-90), entirely on the device: the exact top-k
    spectrum search of ``FwhtSearch`` / ``MitmFwhtSearch`` and the
    ``GreedyApplier`` / ``GlobalGreedyApplier`` bookkeeping per window
    (bmm_search_apply_dev), with one synchronisation per call.  The results
    and the matrix afterwards are those of the host loop; a stochastic
    GreedyApplier's generator advances as it would there.
    """

    def __init__(self, matrix, device: int = 0) -> None:
        import numpy as np
        import torch

        self.rows, self.cols, self.stride = matrix.rows, matrix.cols, matrix.stride_words
        self.device = torch.device("cuda", device)
        words = np.ascontiguousarray(matrix.words).view(np.int64)
        self._words = torch.from_numpy(words.copy()).to(self.device)

    def to_matrix(self):
        from .matrix import BitMatrix

        m = BitMatrix(self.rows, self.cols)
        m.words[:] = self._words.cpu().numpy().view(m.words.dtype).reshape(m.words.shape)
        return m

    def weight(self) -> int:
        import torch

        if self.rows == 0 or self.stride == 0:
            return 0
        w = self._words.view(torch.uint8)
        return int(torch.bitwise_and(w.unsqueeze(-1) >> torch.arange(8, device=w.device,
                                                                      dtype=torch.uint8), 1)
                   .sum().item())

    def search_apply(self, windows, *, searcher, applier) -> list[ApplyResult]:
        import ctypes as C

        import numpy as np
        import torch

        from . import _native as N
        from .apply import GlobalGreedyApplier, GreedyApplier
        from .search import FwhtSearch, MitmFwhtSearch

        wins = np.ascontiguousarray(np.asarray(windows, dtype=np.uint32))
        if wins.ndim != 2:
            raise ValueError("windows must be a list of equal-length row lists")
        n, t = wins.shape
        if n and (wins.max() >= self.rows):
            raise IndexError("row window row out of bounds")
        if isinstance(searcher, FwhtSearch):
            if t > searcher.max_rows:  # as FwhtSearch.search (bmmpy/search.py:202-207)
                raise ValueError(
                    f"Window has {t} rows, which exceeds the configured "
                    f"max_rows={searcher.max_rows} limit for this searcher.")
        elif isinstance(searcher, MitmFwhtSearch):
            if searcher.low_bits != 0 and searcher.low_bits >= t:
                raise ValueError(
                    "MitmFwhtSearch: low_bits must be in [1, t - 1] or 0 for auto")
        else:
            raise TypeError("DeviceMatrix.search_apply supports FwhtSearch and MitmFwhtSearch")
        cfg = N.SweepConfig_t()
        cfg.max_candidates = searcher.max_candidates
        if isinstance(applier, GreedyApplier):
            cfg.applier, cfg.min_gain = 0, int(applier.min_gain)
            cfg.stochastic, cfg.seed = int(bool(applier.stochastic)), applier._state
        elif isinstance(applier, GlobalGreedyApplier):
            cfg.applier, cfg.require_improvement = 1, int(bool(applier.require_improvement))
        else:
            raise TypeError("DeviceMatrix.search_apply supports GreedyApplier and "
                            "GlobalGreedyApplier")
        res = (N.ApplyResult_t * max(1, n))()
        state = C.c_uint64(0)
        stream = torch.cuda.current_stream(self.device).cuda_stream
        N.check(N.lib().bmm_search_apply_dev(self._words.data_ptr(), self.rows, self.stride,
                                             self.cols,
                                             N.u32p(wins), t, n, cfg, res, C.byref(state),
                                             stream), "bmm_search_apply_dev")
        if isinstance(applier, GreedyApplier) and applier.stochastic:
            applier._state = state.value
        return [ApplyResult(int(r.applied_count), int(r.weight_improvement)) for r in res[:n]]
