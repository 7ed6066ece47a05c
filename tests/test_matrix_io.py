"""Matrix IO without a GPU: the text/hash restatements pinned to the reference
library, and the product's host-side parts -- binary save/load and hash() --
against the reference (src/core/bit_matrix_io.cpp:49-67,136-161,
src/core/bit_matrix_hash.cpp:30-58), including its error messages."""

import os
import random

import numpy as np
import pytest

import bmmpy_b200 as bmm
from oracle import oracle as O

R = O.ref()
needs_ref = pytest.mark.skipif(R is None, reason="reference not built (make -C oracle ref)")

SHAPES = [(0, 0), (0, 5), (3, 0), (1, 1), (2, 63), (3, 64), (5, 65), (7, 200), (4, 1000)]


def _matrix(rows, cols, seed, p=0.4):
    m = bmm.BitMatrix(rows, cols)
    if rows and cols:
        words, _ = O.port().gen_instance(rows, cols, p, seed, 0)
        m.words[:] = words[:, : m.stride_words]
    return m


@needs_ref
@pytest.mark.parametrize("rows,cols", SHAPES)
def test_hash_matches_reference_and_hashlib(rows, cols):
    m = _matrix(rows, cols, rows * 7 + cols)
    w = np.ascontiguousarray(m.words)
    want = R.matrix_hash(w, cols)
    assert m.hash() == want == O.matrix_hash(w, rows, cols)


@needs_ref
def test_hash_masks_bits_past_cols():
    m = _matrix(3, 70, 1)
    dirty = m.copy()
    dirty.words[:, 1] |= np.uint64(1 << 63)  # a bit past column 69
    assert dirty.hash() == m.hash()


@needs_ref
@pytest.mark.parametrize("rows,cols", SHAPES)
def test_binary_round_trips_with_reference(tmp_path, rows, cols):
    m = _matrix(rows, cols, 3 * rows + cols)
    ours, theirs = tmp_path / "ours.bin", tmp_path / "theirs.bin"
    m.save_binary_file(ours)
    R.matrix_save_binary(str(theirs), np.ascontiguousarray(m.words), cols)
    assert ours.read_bytes() == theirs.read_bytes()
    back = bmm.BitMatrix.load_binary_file(theirs)
    assert back == m
    w, r, c = R.matrix_load_binary(str(ours))
    assert (r, c) == (rows, cols)
    assert np.array_equal(w[:, : m.stride_words], m.words)


@needs_ref
def test_binary_errors_match_reference(tmp_path):
    good = tmp_path / "good.bin"
    _matrix(4, 100, 9).save_binary_file(good)
    data = good.read_bytes()
    cases = {
        "short_magic": data[:5],
        "bad_magic": b"BMMPYB2\0" + data[8:],
        "short_dims": data[:12],
        "short_payload": data[:-3],
    }
    for name, blob in cases.items():
        p = tmp_path / f"{name}.bin"
        p.write_bytes(blob)
        with pytest.raises(RuntimeError) as theirs:
            R.matrix_load_binary(str(p))
        with pytest.raises(RuntimeError) as ours:
            bmm.BitMatrix.load_binary_file(p)
        assert str(ours.value) == str(theirs.value), name
    with pytest.raises(RuntimeError, match="failed to open matrix binary file for reading"):
        bmm.BitMatrix.load_binary_file(tmp_path / "missing.bin")
    with pytest.raises(RuntimeError, match="failed to open matrix binary file for writing"):
        _matrix(1, 1, 0).save_binary_file(tmp_path / "no_dir" / "x.bin")
    # trailing bytes after the payload are ignored, as in the reference
    p = tmp_path / "extra.bin"
    p.write_bytes(data + b"extra")
    assert bmm.BitMatrix.load_binary_file(p) == _matrix(4, 100, 9)


def _texts(rng):
    out = []
    for rows, cols in SHAPES + [(9, 130)]:
        m = _matrix(rows, cols, rng.randint(0, 99))
        out.append(O.text_format(m.words, rows, cols))
        # the same bits with arbitrary whitespace between them
        bits = "".join(m.to_rows())
        ws = [" ", "\n", "\r", "\t", "\f", "\v", "  \n"]
        body = "".join(b + (rng.choice(ws) if rng.random() < 0.3 else "") for b in bits)
        out.append(f"{rng.choice(['', ' ', chr(10)])}{rows}{rng.choice([' ', chr(9), chr(10)])}"
                   f"{cols}{rng.choice([' ', chr(10)])}{body}{rng.choice(['', chr(10), ' '])}"
                   .encode())
    out += [b"2 3\n10x\n010", b"2 3\n101\n01", b"2 3\n101\n010 1", b"x", b"2", b"", b"  ",
            b"0 0\n 1", b"0 0\n \n", b"2 3 101010", b"+2 3\n101010", b"2 3\n101010\n0",
            b"1 3\n1 0\t1\n\n", b"3 1\n1\n0\n", b"2 2\n1021", b"2 2\n10\n1\x001"]
    return out


@needs_ref
def test_text_restatement_matches_reference():
    for text in _texts(random.Random(5)):
        try:
            w, r, c = R.matrix_from_text(text)
            want = ("ok", r, c, [[int((int(w[i][j // 64]) >> (j % 64)) & 1) for j in range(c)]
                                 for i in range(r)])
        except RuntimeError as e:
            want = ("error", str(e))
        try:
            r, c, bits = O.text_parse(text)
            got = ("ok", r, c, bits)
        except RuntimeError as e:
            got = ("error", str(e))
        assert got == want, text
        if want[0] == "ok":
            m = _matrix(want[1], want[2], 0)
            m.words[:] = 0
            for i, row in enumerate(want[3]):
                for j, b in enumerate(row):
                    if b:
                        m[i, j] = True
            assert O.text_format(m.words, m.rows, m.cols) == R.matrix_to_text(
                np.ascontiguousarray(m.words), m.cols)
