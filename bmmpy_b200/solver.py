"""Exact minimum-weight basis of a window, with the reference's API.

Mirrors bmmpy.solver (bmmpy/solver.py, include/bmmpy/solver/exact_basis_solver.hpp,
python/bindings/solver.cpp): ``ExactBasisSolver(max_rows=24, max_states=2**24 - 1,
max_storage_bytes=128 MiB).solve(window)`` returns an ``ExactBasisResult`` with
the same fields, values and errors as the reference's.  The enumeration of the
2^t - 1 row combinations runs on the GPU (``bmm_exact_basis``); only the two
result matrices are assembled here from the accepted masks.
"""

from __future__ import annotations

import numpy as np

from . import _native as N
from .matrix import BitMatrix, RowWindow


class ExactBasisSolverConfig:
    """ExactBasisSolverConfig (include/bmmpy/solver/exact_basis_solver.hpp:12-16)."""

    __slots__ = ("max_rows", "max_states", "max_storage_bytes")

    def __init__(self) -> None:
        self.max_rows = 24
        self.max_states = (1 << 24) - 1
        self.max_storage_bytes = 128 * 1024 * 1024

    def __repr__(self) -> str:
        return (f"ExactBasisSolverConfig(max_rows={self.max_rows}, "
                f"max_states={self.max_states}, max_storage_bytes={self.max_storage_bytes})")


class ExactBasisResult:
    """ExactBasisResult (include/bmmpy/solver/exact_basis_solver.hpp:18-28)."""

    __slots__ = ("input_rows", "cols", "rank", "enumerated_states", "total_weight",
                 "basis_masks", "basis_weights", "transform_matrix", "basis_matrix")

    def __init__(self) -> None:
        self.input_rows = 0
        self.cols = 0
        self.rank = 0
        self.enumerated_states = 0
        self.total_weight = 0
        self.basis_masks: list[int] = []
        self.basis_weights: list[int] = []
        self.transform_matrix = BitMatrix()
        self.basis_matrix = BitMatrix()

    def __repr__(self) -> str:
        return (f"ExactBasisResult(input_rows={self.input_rows}, cols={self.cols}, "
                f"rank={self.rank}, total_weight={self.total_weight})")


def _transform_matrix(rows: int, masks: list[int]) -> BitMatrix:
    """Row k holds mask k over the window rows (include/bmmpy/core/detail/
    row_combination.hpp:80-88)."""
    m = BitMatrix(len(masks), rows)
    if masks:
        m._words[:, 0] = np.asarray(masks, dtype=np.uint64)
    return m


class ExactBasisSolver:
    """bmmpy.solver.ExactBasisSolver (bmmpy/solver.py:26-58)."""

    __slots__ = ("max_rows", "max_states", "max_storage_bytes")

    def __init__(self, config: ExactBasisSolverConfig | None = None, *,
                 max_rows: int = 24, max_states: int = (1 << 24) - 1,
                 max_storage_bytes: int = 128 * 1024 * 1024) -> None:
        if config is not None:
            max_rows, max_states = config.max_rows, config.max_states
            max_storage_bytes = config.max_storage_bytes
        self.max_rows = max_rows
        self.max_states = max_states
        self.max_storage_bytes = max_storage_bytes

    def __repr__(self) -> str:
        return ("ExactBasisSolver("
                f"max_rows={self.max_rows}, "
                f"max_states={self.max_states}, "
                f"max_storage_bytes={self.max_storage_bytes})")

    def name(self) -> str:
        return "exact_basis"

    def solve(self, window: RowWindow) -> ExactBasisResult:
        """src/solver/exact_basis_solver.cpp:58-157."""
        m = window.matrix
        t = window.size
        cfg = N.ExactBasisConfig_t(self.max_rows, self.max_states, self.max_storage_bytes)
        res = N.ExactBasisResult_t()
        cap = max(1, min(t, m.cols))
        masks = np.zeros(cap, dtype=np.uint32)
        weights = np.zeros(cap, dtype=np.uint32)
        win = window.index_array()
        L = N.lib()
        N.check(L.bmm_exact_basis(N.u64p(m.words), m.stride_words, m.cols, N.u32p(win), t,
                                  cfg, res, N.u32p(masks), N.u32p(weights)), "bmm_exact_basis")
        out = ExactBasisResult()
        out.input_rows = int(res.input_rows)
        out.cols = int(res.cols)
        out.rank = int(res.rank)
        out.enumerated_states = int(res.enumerated_states)
        out.total_weight = int(res.total_weight)
        r = out.rank
        out.basis_masks = [int(x) for x in masks[:r]]
        out.basis_weights = [int(x) for x in weights[:r]]
        if t == 0:
            out.transform_matrix = BitMatrix(0, 0)
        else:
            out.transform_matrix = _transform_matrix(t, out.basis_masks)
        out.basis_matrix = (out.transform_matrix.mul(window.materialize()) if r
                            else BitMatrix(0, m.cols))
        return out


__all__ = ["ExactBasisResult", "ExactBasisSolver", "ExactBasisSolverConfig"]
