"""Apply strategies: consume search candidates and update a window's rows.

Mirrors bmmpy.apply (bmmpy/apply.py, include/bmmpy/apply/*.hpp,
src/apply/greedy_applier.cpp:13-109, src/apply/global_greedy_applier.cpp:17-105)
with the same names, arguments, results and errors.  Appliers mutate the
underlying BitMatrix in place through the RowWindow; they are window-sized
bookkeeping (at most 64 rows for GreedyApplier) around row XORs.
"""

from __future__ import annotations

from collections.abc import Iterable

import numpy as np

from .candidate import Candidate
from .matrix import RowWindow, _popcount_words

__all__ = ["ApplyResult", "GreedyApplier", "GlobalGreedyApplier"]

_M64 = (1 << 64) - 1


class ApplyResult:
    """Summary of a candidate-application step (include/bmmpy/apply/apply_result.hpp)."""

    __slots__ = ("applied_count", "weight_improvement")

    def __init__(self, applied_count: int = 0, weight_improvement: int = 0) -> None:
        self.applied_count = applied_count
        self.weight_improvement = weight_improvement

    def __repr__(self) -> str:
        return (f"ApplyResult(applied_count={self.applied_count}, "
                f"weight_improvement={self.weight_improvement})")


class GreedyApplier:
    """Apply candidates greedily to reduce row weights in a window
    (src/apply/greedy_applier.cpp:13-109).

    Candidates are taken lightest first (stable; shuffled first when
    ``stochastic``).  A candidate's mask, over the window's ORIGINAL rows, is
    re-expressed over the current rows; among the rows it involves, the one
    whose weight drops most (by at least ``min_gain``) becomes the candidate
    (first such row, or a random one when ``stochastic``)."""

    __slots__ = ("min_gain", "stochastic", "seed", "_state")

    def __init__(self, min_gain: int, *, stochastic: bool = False, seed: int = 0) -> None:
        self.min_gain = min_gain
        self.stochastic = stochastic
        self.seed = seed
        self._state = (seed if seed != 0 else 0xDEADB) & _M64

    def __repr__(self) -> str:
        return (f"GreedyApplier(min_gain={self.min_gain}, stochastic={self.stochastic}, "
                f"seed={self.seed})")

    def _next(self) -> int:
        x = self._state
        x ^= (x << 13) & _M64
        x ^= x >> 7
        x ^= (x << 17) & _M64
        self._state = x
        return x

    def apply(self, window: RowWindow, candidates: Iterable[Candidate]) -> ApplyResult:
        n = len(window)
        if n > 64:
            raise ValueError("row window size must be <= 64")
        c = [1 << i for i in range(n)]
        cur = [window.row_popcount(i) for i in range(n)]
        cands = list(candidates)
        if self.stochastic:
            for i in range(len(cands), 1, -1):
                j = self._next() % i
                cands[i - 1], cands[j] = cands[j], cands[i - 1]
        cands.sort(key=lambda cand: cand.weight)  # stable
        result = ApplyResult()
        min_gain = int(self.min_gain)
        for cand in cands:
            m = cand.mask_u64()
            a = 0
            for i in range(n):
                if bin(m & c[i]).count("1") & 1:
                    a |= 1 << i
            if a == 0:
                continue
            best_rows: list[int] = []
            best_gain = 0
            cw = int(cand.weight)
            for r in range(n):
                if not (a >> r) & 1:
                    continue
                old = cur[r]
                if old <= cw:
                    continue
                gain = old - cw
                if gain < min_gain:
                    continue
                if gain > best_gain:
                    best_gain = gain
                    best_rows = [r]
                elif gain == best_gain:
                    best_rows.append(r)
            if not best_rows:
                continue
            chosen = best_rows[self._next() % len(best_rows)] if self.stochastic else best_rows[0]
            for i in range(n):
                if i != chosen and (a >> i) & 1:
                    window.row_xor(chosen, i)
            cur[chosen] = cw
            for j in range(n):
                if j != chosen and (a >> j) & 1:
                    c[j] ^= c[chosen]
            result.applied_count += 1
            result.weight_improvement += best_gain
        return result


def _mask_int(cand: Candidate, n: int) -> int:
    """normalize_mask_words (include/bmmpy/core/detail/xor_basis.hpp:93-105)."""
    v = 0
    for w, word in enumerate(cand.mask):
        v |= (int(word) & _M64) << (64 * w)
    if v >> n:
        raise ValueError("mask contains bits outside the supported row range")
    return v


class GlobalGreedyApplier:
    """Greedily assemble one full invertible transform from a candidate pool
    (src/apply/global_greedy_applier.cpp:17-105): the candidates plus the
    identity rows, stable-sorted by weight, inserted into a GF(2) basis until
    it has full rank; the transform replaces the window's rows when it does
    not increase (with ``require_improvement``: strictly lowers) the weight."""

    __slots__ = ("require_improvement",)

    def __init__(self, *, require_improvement: bool = True) -> None:
        self.require_improvement = require_improvement

    def __repr__(self) -> str:
        return f"GlobalGreedyApplier(require_improvement={self.require_improvement})"

    def name(self) -> str:
        return "global_greedy"

    def apply(self, window: RowWindow, candidates: Iterable[Candidate]) -> ApplyResult:
        n = len(window)
        if n == 0:
            return ApplyResult()
        m = window.matrix
        rows = window.rows
        before = m.words[rows].copy()
        old_weight = int(sum(_popcount_words(before[r]) for r in range(n)))
        pool = []
        for cand in candidates:
            pool.append((_mask_int(cand, n), int(cand.weight)))
        for r in range(n):
            w = window.row_popcount(r)
            if w > 0xFFFFFFFF:
                raise ValueError(
                    "GlobalGreedyApplier: row weight exceeds supported u32 candidate range")
            pool.append((1 << r, w))
        pool.sort(key=lambda e: e[1])  # stable
        basis: dict[int, int] = {}
        chosen: list[int] = []
        for mask, _ in pool:
            v = mask
            while v:
                hb = v.bit_length() - 1
                if hb not in basis:
                    basis[hb] = v
                    break
                v ^= basis[hb]
            if v:
                chosen.append(mask)
                if len(chosen) == n:
                    break
        if len(chosen) != n:
            raise RuntimeError("GlobalGreedyApplier: failed to assemble a full invertible transform")
        after = np.zeros_like(before)
        for r, mask in enumerate(chosen):
            acc = np.zeros(before.shape[1], dtype=np.uint64)
            v = mask
            while v:
                b = (v & -v).bit_length() - 1
                acc ^= before[b]
                v &= v - 1
            after[r] = acc
        new_weight = int(sum(_popcount_words(after[r]) for r in range(n)))
        if new_weight > old_weight:
            return ApplyResult()
        if self.require_improvement and new_weight == old_weight:
            return ApplyResult()
        m.words[rows] = after
        return ApplyResult(1, old_weight - new_weight)
