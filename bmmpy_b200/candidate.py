"""Candidate: a row combination (mask over window rows) and its weight.

Mirrors bmmpy.Candidate (include/bmmpy/types/candidate.hpp:19-168,
python/bindings/candidate.cpp:36-61): ``mask`` is a list of 64-bit words,
bit j selecting window row j; ordering everywhere is (weight, mask).
"""

from __future__ import annotations

from collections.abc import Sequence


class Candidate:
    __slots__ = ("mask", "weight")

    def __init__(self, mask: Sequence[int] | None = None, weight: int = 0) -> None:
        self.mask = [int(w) for w in (mask or [])]
        self.weight = int(weight)

    @classmethod
    def from_u64(cls, mask: int, weight: int) -> "Candidate":
        return cls([int(mask)], weight)

    @classmethod
    def make_unit(cls, row_count: int, row: int, weight: int) -> "Candidate":
        words = [0] * ((row_count + 63) // 64)
        words[row // 64] |= 1 << (row % 64)
        return cls(words, weight)

    def has_row(self, i: int) -> bool:
        w = i // 64
        return w < len(self.mask) and bool((self.mask[w] >> (i % 64)) & 1)

    __contains__ = has_row

    def mask_popcount(self) -> int:
        return sum(bin(w).count("1") for w in self.mask)

    __len__ = mask_popcount

    def mask_u64(self) -> int:
        if any(self.mask[1:]):
            raise RuntimeError("Candidate::mask_u64: mask does not fit in u64")
        return self.mask[0] if self.mask else 0

    def selected_rows(self) -> list[int]:
        out = []
        for wi, w in enumerate(self.mask):
            while w:
                b = (w & -w).bit_length() - 1
                out.append(wi * 64 + b)
                w &= w - 1
        return out

    def __iter__(self):
        return iter(self.selected_rows())

    @property
    def rows(self) -> list[int]:
        return self.selected_rows()

    def key(self) -> tuple[int, int]:
        return (self.weight, self.mask[0] if self.mask else 0)

    def __eq__(self, other) -> bool:
        return isinstance(other, Candidate) and self.mask == other.mask and self.weight == other.weight

    def __repr__(self) -> str:
        return f"Candidate(rows={self.selected_rows()}, weight={self.weight})"
