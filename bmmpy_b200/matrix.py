"""Bit-packed matrices and row windows with the reference's layout and names.

``BitMatrix`` mirrors bmmpy.BitMatrix (include/bmmpy/core/bit_matrix.hpp:27-127,
python/bindings/bit_matrix.cpp:100-191): row-major uint64 words, bit c of a row
in word c // 64 at bit c % 64, row stride padded to a multiple of 4 words
(src/core/bit_matrix.cpp:67-72), bits past ``cols`` always zero.  The words live
in a numpy array (host memory) that the search entry points hand to the
device library.

Text and binary IO and ``hash()`` follow src/core/bit_matrix_io.cpp and
src/core/bit_matrix_hash.cpp (formats, messages); text is parsed and
formatted on the device.

``RowWindow`` mirrors bmmpy.RowWindow (include/bmmpy/core/row_window.hpp):
an ordered list of unique rows of one matrix; it borrows the matrix, so
applying a candidate through the window changes the matrix.
"""

from __future__ import annotations

import ctypes as C
import os
from collections.abc import Sequence

import numpy as np

WORD_BITS = 64


def _stride_for(cols: int) -> int:
    words = (cols + WORD_BITS - 1) // WORD_BITS
    return (words + 3) // 4 * 4


def _popcount_words(a: np.ndarray) -> int:
    return int(np.unpackbits(np.ascontiguousarray(a).view(np.uint8)).sum())


class MatrixError(RuntimeError):
    """bmmpy.MatrixError (include/bmmpy/core/bit_matrix.hpp:14, src/core/bit_matrix.cpp:10-20)."""


def _dimension_mismatch() -> MatrixError:
    return MatrixError("Matrix dimensions mismatch")


def gf2_rank_words(words: np.ndarray, cols: int) -> int:
    """Rank over GF(2) of packed rows (src/core/bit_matrix_algebra.cpp:76-99)."""
    a = np.array(words, dtype=np.uint64, copy=True)
    rows = a.shape[0]
    rank = 0
    for c in range(cols):
        if rank == rows:
            break
        w, b = divmod(c, WORD_BITS)
        bit = np.uint64(1 << b)
        hits = np.nonzero(a[rank:, w] & bit)[0]
        if hits.size == 0:
            continue
        piv = rank + int(hits[0])
        if piv != rank:
            a[[rank, piv]] = a[[piv, rank]]
        below = rank + 1 + np.nonzero(a[rank + 1:, w] & bit)[0]
        if below.size:
            a[below] ^= a[rank]
        rank += 1
    return rank


class BitMatrix:
    __slots__ = ("_rows", "_cols", "_words")

    def __init__(self, rows: int = 0, cols: int = 0) -> None:
        if rows < 0 or cols < 0:
            raise ValueError("rows and cols must be non-negative")
        self._rows = int(rows)
        self._cols = int(cols)
        self._words = np.zeros((self._rows, _stride_for(self._cols)), dtype=np.uint64)

    # -- construction --------------------------------------------------------
    @classmethod
    def from_words(cls, words: np.ndarray, cols: int) -> "BitMatrix":
        """Wrap a (rows, stride) uint64 array (copied; padding bits cleared)."""
        words = np.asarray(words, dtype=np.uint64)
        m = cls(words.shape[0], cols)
        wpr = m.words_per_row
        m._words[:, :wpr] = words[:, :wpr]
        m._clear_tail()
        return m

    def _clear_tail(self) -> None:
        tail = self._cols % WORD_BITS
        wpr = self.words_per_row
        if wpr:
            if tail:
                self._words[:, wpr - 1] &= np.uint64((1 << tail) - 1)
            self._words[:, wpr:] = 0

    def copy(self) -> "BitMatrix":
        m = BitMatrix(self._rows, self._cols)
        m._words[...] = self._words
        return m

    # -- shape ---------------------------------------------------------------
    @property
    def rows(self) -> int:
        return self._rows

    @property
    def cols(self) -> int:
        return self._cols

    @property
    def shape(self) -> tuple[int, int]:
        return (self._rows, self._cols)

    @property
    def stride_words(self) -> int:
        return self._words.shape[1]

    @property
    def words_per_row(self) -> int:
        return (self._cols + WORD_BITS - 1) // WORD_BITS

    @property
    def total_words(self) -> int:
        return self._words.size

    @property
    def total_bytes(self) -> int:
        return self._words.nbytes

    @property
    def words(self) -> np.ndarray:
        """The packed (rows, stride_words) uint64 storage (a view)."""
        return self._words

    def __len__(self) -> int:
        return self._rows

    # -- element access ------------------------------------------------------
    def _check(self, row: int, col: int) -> None:
        if not (0 <= row < self._rows and 0 <= col < self._cols):
            raise IndexError("matrix index out of range")

    def get(self, row: int, col: int) -> bool:
        self._check(row, col)
        return bool((int(self._words[row, col // 64]) >> (col % 64)) & 1)

    def set(self, row: int, col: int, value: bool) -> None:
        self._check(row, col)
        bit = np.uint64(1 << (col % 64))
        if value:
            self._words[row, col // 64] |= bit
        else:
            self._words[row, col // 64] &= ~bit

    def __getitem__(self, idx):
        r, c = idx
        return self.get(r, c)

    def __setitem__(self, idx, value) -> None:
        r, c = idx
        self.set(r, c, bool(value))

    # -- row operations ------------------------------------------------------
    def row_xor(self, target_row: int, source_row: int) -> None:
        if not (0 <= target_row < self._rows and 0 <= source_row < self._rows):
            raise IndexError("row index out of range")
        self._words[target_row] ^= self._words[source_row]

    def row_popcount(self, row: int) -> int:
        if not 0 <= row < self._rows:
            raise IndexError("row index out of range")
        return _popcount_words(self._words[row])

    def weight(self) -> int:
        return _popcount_words(self._words)

    def swap_rows(self, r1: int, r2: int) -> None:
        self._words[[r1, r2]] = self._words[[r2, r1]]

    # -- GF(2) algebra (src/core/bit_matrix_algebra.cpp) -----------------------
    @classmethod
    def identity(cls, n: int) -> "BitMatrix":
        m = cls(n, n)
        for i in range(n):
            m.set(i, i, True)
        return m

    def rank(self) -> int:
        return gf2_rank_words(self._words, self._cols)

    def add(self, other: "BitMatrix") -> "BitMatrix":
        if self.shape != other.shape:
            raise _dimension_mismatch()
        m = self.copy()
        m._words ^= other._words
        return m

    def mul(self, other: "BitMatrix") -> "BitMatrix":
        """Product over GF(2): row i of the result XORs the rows k of ``other``
        with bit k set in row i of ``self``."""
        if self._cols != other.rows:
            raise _dimension_mismatch()
        m = BitMatrix(self._rows, other.cols)
        if self._rows == 0 or self._cols == 0:
            return m
        bits = np.unpackbits(self._words.view(np.uint8).reshape(self._rows, -1), axis=1,
                             bitorder="little")[:, : self._cols]
        for i in range(self._rows):
            ks = np.nonzero(bits[i])[0]
            if ks.size:
                m._words[i] = np.bitwise_xor.reduce(other._words[ks], axis=0)
        return m

    __matmul__ = mul

    def row_window(self, rows: Sequence[int]) -> "RowWindow":
        return RowWindow(self, rows)

    def extract_rows_by_indices(self, indices: Sequence[int]) -> "BitMatrix":
        m = BitMatrix(len(indices), self._cols)
        for i, r in enumerate(indices):
            if not 0 <= r < self._rows:
                raise IndexError("row index out of range")
            m._words[i] = self._words[r]
        return m

    def insert_rows_by_indices(self, source: "BitMatrix", indices: Sequence[int]) -> None:
        if source.rows != len(indices) or source.cols != self._cols:
            raise ValueError("dimension mismatch")
        for i, r in enumerate(indices):
            self._words[r] = source._words[i]

    def to_rows(self) -> list[str]:
        if self._rows == 0 or self._cols == 0:
            return [""] * self._rows
        bits = np.unpackbits(self._words.view(np.uint8).reshape(self._rows, -1), axis=1,
                             bitorder="little")
        return ["".join("1" if b else "0" for b in row[: self._cols]) for row in bits]

    # -- text / binary IO and hash (src/core/bit_matrix_io.cpp,
    #    src/core/bit_matrix_hash.cpp; formatted and parsed on the device) --------
    def to_text(self) -> str:
        """save_text: "rows cols\\n" then one '0'/'1' line per row."""
        from . import _native as N

        n = C.c_size_t(0)
        N.check(N.lib().bmm_matrix_text_size(self._rows, self._cols, C.byref(n)))
        buf = C.create_string_buffer(max(1, n.value))
        N.check(N.lib().bmm_matrix_to_text(N.u64p(self._words), self.stride_words, self._rows,
                                           self._cols, buf, n.value, None))
        return buf.raw[: n.value].decode("ascii")

    __str__ = to_text

    @classmethod
    def from_text(cls, text) -> "BitMatrix":
        """load_text over a string: whitespace between bits is ignored."""
        from . import _native as N

        data = text.encode("ascii", "replace") if isinstance(text, str) else bytes(text)
        rows, cols = C.c_uint64(0), C.c_uint64(0)
        N.check(N.lib().bmm_matrix_text_header(data, len(data), C.byref(rows), C.byref(cols)))
        m = cls(rows.value, cols.value)
        N.check(N.lib().bmm_matrix_from_text(data, len(data), N.u64p(m._words), m.stride_words,
                                             m._rows, m._cols))
        return m

    @classmethod
    def load_text_file(cls, path) -> "BitMatrix":
        try:
            with open(os.fspath(path), "rb") as f:
                data = f.read()
        except OSError:
            raise RuntimeError("failed to open matrix text file for reading") from None
        return cls.from_text(data)

    def save_text_file(self, path) -> None:
        text = self.to_text()
        try:
            with open(os.fspath(path), "w", newline="") as f:
                f.write(text)
        except OSError:
            raise RuntimeError("failed to open matrix text file for writing") from None

    def save_binary_file(self, path) -> None:
        from . import _native as N

        N.check(N.lib().bmm_matrix_save_binary(os.fsencode(path), N.u64p(self._words),
                                               self.stride_words, self._rows, self._cols))

    @classmethod
    def load_binary_file(cls, path) -> "BitMatrix":
        from . import _native as N

        p = os.fsencode(path)
        rows, cols = C.c_uint64(0), C.c_uint64(0)
        N.check(N.lib().bmm_matrix_binary_header(p, C.byref(rows), C.byref(cols)))
        m = cls(rows.value, cols.value)
        N.check(N.lib().bmm_matrix_load_binary(p, N.u64p(m._words), m.stride_words, m._rows,
                                               m._cols))
        return m

    def hash(self) -> str:
        """SHA-256 hex of rows, cols and the row words (bits past cols cleared)."""
        from . import _native as N

        out = C.create_string_buffer(65)
        N.check(N.lib().bmm_matrix_hash(N.u64p(self._words), self.stride_words, self._rows,
                                        self._cols, out))
        return out.value.decode("ascii")

    def __eq__(self, other) -> bool:
        return (isinstance(other, BitMatrix) and self.shape == other.shape
                and bool(np.array_equal(self._words, other._words)))

    def __repr__(self) -> str:
        return f"BitMatrix(rows={self._rows}, cols={self._cols}, weight={self.weight()})"


def matrix_from_rows(rows: Sequence[str]) -> BitMatrix:
    """Build a matrix from '0'/'1' strings (bmmpy/matrix.py:72)."""
    rows = list(rows)
    cols = len(rows[0]) if rows else 0
    m = BitMatrix(len(rows), cols)
    for r, s in enumerate(rows):
        if len(s) != cols:
            raise ValueError("row width mismatch")
        for c, ch in enumerate(s):
            if ch == "1":
                m.set(r, c, True)
            elif ch != "0":
                raise ValueError("rows must contain only '0' or '1'")
    return m


class RowWindow:
    __slots__ = ("_matrix", "_rows")

    def __init__(self, matrix: BitMatrix, rows: Sequence[int]) -> None:
        rows = [int(r) for r in rows]
        if len(set(rows)) != len(rows):
            raise ValueError("RowWindow rows must be unique")
        for r in rows:
            if not 0 <= r < matrix.rows:
                raise IndexError("row window row out of bounds")
        self._matrix = matrix
        self._rows = rows

    @property
    def matrix(self) -> BitMatrix:
        return self._matrix

    @property
    def rows(self) -> list[int]:
        return list(self._rows)

    @property
    def size(self) -> int:
        return len(self._rows)

    @property
    def cols(self) -> int:
        return self._matrix.cols

    @property
    def shape(self) -> tuple[int, int]:
        return (len(self._rows), self._matrix.cols)

    def __len__(self) -> int:
        return len(self._rows)

    def global_row(self, local_row: int) -> int:
        return self._rows[local_row]

    def row_popcount(self, local_row: int) -> int:
        return self._matrix.row_popcount(self._rows[local_row])

    def row_xor(self, target_local_row: int, source_local_row: int) -> None:
        self._matrix.row_xor(self._rows[target_local_row], self._rows[source_local_row])

    def weight(self) -> int:
        return sum(self.row_popcount(i) for i in range(len(self._rows)))

    @property
    def total_weight(self) -> int:
        """Columns active in any window row (src/core/row_window.cpp:67-88)."""
        if not self._rows:
            return 0
        acc = np.bitwise_or.reduce(self._matrix.words[self._rows], axis=0)
        return _popcount_words(acc)

    def materialize(self) -> BitMatrix:
        return self._matrix.extract_rows_by_indices(self._rows)

    def assign_materialized(self, rows: BitMatrix) -> None:
        self._matrix.insert_rows_by_indices(rows, self._rows)

    def index_array(self) -> np.ndarray:
        return np.asarray(self._rows, dtype=np.uint32)

    def __repr__(self) -> str:
        return f"RowWindow(rows={self._rows}, cols={self.cols})"
