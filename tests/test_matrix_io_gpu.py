"""Matrix text IO on the device against the reference library
(src/core/bit_matrix_io.cpp:34-132): parsing with arbitrary whitespace and
every failure mode (same messages), formatting byte for byte, the full-size
planted 512 x 65536 matrix round trip, and binary loads straight into device
memory."""

import random

import numpy as np
import pytest

import bmmpy_b200 as bmm
from bmmpy_b200 import _native as N
from oracle import oracle as O
from tests.test_matrix_io import SHAPES, _matrix, _texts

pytestmark = pytest.mark.gpu
R = O.ref()
needs_ref = pytest.mark.skipif(R is None, reason="reference not built (make -C oracle ref)")


@needs_ref
def test_from_text_matches_reference():
    for text in _texts(random.Random(6)):
        try:
            w, r, c = R.matrix_from_text(text)
            want = ("ok", r, c, w[:, : max(4, ((c + 63) // 64 + 3) // 4 * 4) if c else 0])
        except RuntimeError as e:
            want = ("error", str(e))
        try:
            m = bmm.BitMatrix.from_text(text)
            got = ("ok", m.rows, m.cols, m.words)
        except RuntimeError as e:
            got = ("error", str(e))
        assert got[0] == want[0] and got[1:3] == want[1:3], (text, got, want)
        if got[0] == "ok" and got[1] and got[2]:
            assert np.array_equal(got[3], want[3][:, : got[3].shape[1]]), text


@needs_ref
@pytest.mark.parametrize("rows,cols", SHAPES)
def test_to_text_matches_reference(rows, cols):
    m = _matrix(rows, cols, rows + 3 * cols)
    want = R.matrix_to_text(np.ascontiguousarray(m.words), cols).decode()
    assert m.to_text() == want == str(m)


def test_text_file_round_trip(tmp_path):
    m = _matrix(9, 300, 4)
    m.save_text_file(tmp_path / "m.txt")
    assert bmm.BitMatrix.load_text_file(tmp_path / "m.txt") == m
    with pytest.raises(RuntimeError, match="failed to open matrix text file for reading"):
        bmm.BitMatrix.load_text_file(tmp_path / "missing.txt")


@needs_ref
def test_planted_full_size_round_trip():
    words, _ = O.port().gen_instance(512, 65536, 0.02, 2, 2000)
    m = bmm.BitMatrix(512, 65536)
    m.words[:] = words[:, : m.stride_words]
    text = m.to_text()
    assert len(text) == len("512 65536\n") + 512 * 65537
    assert text.encode() == R.matrix_to_text(np.ascontiguousarray(m.words), 65536)
    back = bmm.BitMatrix.from_text(text)
    assert back == m and back.hash() == m.hash()
    # the same bits with every row on two lines and tabs between bytes
    rows = m.to_rows()
    alt = "512\t65536\n" + "".join(r[:30000] + "\n\t" + r[30000:] + " \r\n" for r in rows)
    assert bmm.BitMatrix.from_text(alt) == m


def test_binary_load_to_device(tmp_path):
    import torch

    m = _matrix(300, 1000, 12)
    path = tmp_path / "m.bin"
    m.save_binary_file(path)
    stride = m.stride_words + 4  # a wider pitch than the file's rows
    d = torch.full((m.rows * stride,), -1, dtype=torch.int64, device="cuda")
    N.check(N.lib().bmm_matrix_load_binary_dev(str(path).encode(), d.data_ptr(), stride, m.rows,
                                               m.cols, torch.cuda.current_stream().cuda_stream))
    got = d.cpu().numpy().view(np.uint64).reshape(m.rows, stride)
    assert np.array_equal(got[:, : m.stride_words], m.words)
    assert not got[:, m.stride_words:].any()
