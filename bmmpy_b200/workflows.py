"""Search-then-apply workflow (bmmpy/workflows.py:45-90)."""

from __future__ import annotations

from collections.abc import Iterable
from typing import Protocol

from .apply import ApplyResult
from .candidate import Candidate
from .matrix import RowWindow

__all__ = ["search_apply"]


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
