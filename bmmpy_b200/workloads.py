"""Seeded synthetic instances standing in for the reference's benchmark shapes.

No dataset is involved: every matrix is regenerated from its seed by the
library's xorshift64 generator (``bmm_gen_instance``).

* ``c1``: 64x256 Bernoulli(0.5), seed 0; target i searches rows i+1..i+16.
* ``c2``: 40x4096 Bernoulli(0.3), seed 1; target i searches rows i+1..i+24.
* ``c3``: 512x65536 Bernoulli(0.02), seed 2, 2000 row-XOR scrambles; windows
  of 32 consecutive rows.
* ``c4``: batch instance idx in [0, 4096): n x m with n, m log-uniform in
  [16, 128] x [64, 2048] (xorshift64 seeded 1000+idx+0x10000, 8 draws
  discarded, then two unit draws), Bernoulli(0.05) seeded 1000+idx, 4n scrambles; k = min(n-1, 16).
"""

from __future__ import annotations

import math

from . import _native as N
from .matrix import BitMatrix

M64 = (1 << 64) - 1

C1 = dict(rows=64, cols=256, p=0.5, seed=0, k=16)
C2 = dict(rows=40, cols=4096, p=0.3, seed=1, k=24)
C3 = dict(rows=512, cols=65536, p=0.02, seed=2, scrambles=2000, window=32)
C4 = dict(count=4096, seed0=1000, p=0.05)


def gen_instance(rows: int, cols: int, p: float, seed: int, scrambles: int = 0):
    """Returns (BitMatrix, planted weight)."""
    m = BitMatrix(rows, cols)
    planted = N.lib().bmm_gen_instance(N.u64p(m.words), rows, cols, m.stride_words, float(p),
                                       int(seed), int(scrambles))
    return m, int(planted)


def _xs(x: int) -> int:
    x ^= (x << 13) & M64
    x ^= x >> 7
    x ^= (x << 17) & M64
    return x


def batch_shape(idx: int) -> tuple[int, int]:
    st = C4["seed0"] + idx + 0x10000
    for _ in range(8):  # small seeds leave the first draws tiny: discard them
        st = _xs(st)
    st = _xs(st)
    u1 = (st >> 11) / 9007199254740992.0
    st = _xs(st)
    u2 = (st >> 11) / 9007199254740992.0
    n = min(128, int(math.floor(math.exp(math.log(16) + u1 * (math.log(128) - math.log(16))))))
    m = min(2048, int(math.floor(math.exp(math.log(64) + u2 * (math.log(2048) - math.log(64))))))
    return n, m


def batch_instance(idx: int):
    """Returns (BitMatrix, k, planted weight) of batch instance idx."""
    n, m = batch_shape(idx)
    mat, planted = gen_instance(n, m, C4["p"], C4["seed0"] + idx, 4 * n)
    return mat, min(n - 1, 16), planted
