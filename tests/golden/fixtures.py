"""Fixture matrices shared by the golden generator and the tests.

The workload constants describe the seeded synthetic inputs that stand in
for the reference's benchmark configurations (no public dataset is
involved).  ``matrix_from_rows``, ``cuda_equivalence_matrix`` and
``python_random_matrix`` rebuild the fixture matrices of the reference's own
tests (tests/support/test_common.hpp:31-53,173-190 and
tests/python/test_cuda_api.py:13-22) in the packed layout.
"""

from __future__ import annotations

import math
import random

import numpy as np

M64 = (1 << 64) - 1

# C1: plain FWHT spectral search, 64x256, Bernoulli(0.5), seed 0, k=16 others
C1 = dict(rows=64, cols=256, p=0.5, seed=0, k=16)
# C2: Gray-code brute force, 40x4096, Bernoulli(0.3), seed 1, k=24 others
C2 = dict(rows=40, cols=4096, p=0.3, seed=1, k=24)
# C3: MITM on a planted 512x65536 instance (p=0.02, seed 2, 2000 scrambles)
C3 = dict(rows=512, cols=65536, p=0.02, seed=2, scrambles=2000, window=32, golden_windows=16)
# C4: 4096 uneven planted instances (seeds 1000..5095)
C4 = dict(count=4096, seed0=1000, p=0.05)
# C5: GA on a planted 256x8192 instance (p=0.01, seed 7, 5000 scrambles)
C5 = dict(rows=256, cols=8192, p=0.01, seed=7, scrambles=5000)

# Single-island GeneticAlgorithm runs pinned by the reference:
# (rows, cols, p, instance seed, scrambles, GA keyword arguments, steps, GA seed)
GA_CASES = [
    (16, 200, 0.2, 3, 40, dict(population_size=20, max_generations=30), 30, 14),
    (40, 512, 0.05, 9, 160, dict(population_size=24, num_parents=3, num_offspring=2,
                                  elite_count=2, max_generations=15), 15, 20),
    (20, 100, 0.3, 1, 50, dict(population_size=16, enable_catastrophe=True,
                                catastrophe_threshold=4, catastrophe_survival_rate=0.25,
                                tournament_size=2, max_generations=50), 50, 12),
    (12, 64, 0.4, 2, 30, dict(population_size=10, target_total_weight=150,
                               max_generations=300), 300, 13),
    (C5["rows"], C5["cols"], C5["p"], C5["seed"], C5["scrambles"],
     dict(population_size=12, max_generations=4), 4, 77),
]

# ExactBasisSolver windows pinned by the reference:
# (rows, cols, p, instance seed, scrambles, window rows)
BASIS_CASES = [
    (24, 256, 0.5, 11, 0, list(range(24))),           # the default max_rows cap
    (20, 96, 0.08, 12, 40, list(range(19, -1, -1))),   # sparse, planted, reversed window
    (18, 12, 0.4, 14, 0, list(range(18))),            # rank 12 < rows
    (30, 2000, 0.02, 15, 60, list(range(3, 19))),      # wide sparse rows, 16-row window
    (14, 140000, 0.01, 16, 20, list(range(14))),       # rows wider than one shared-memory slab
    (9, 64, 0.3, 17, 0, [8, 0, 7, 1, 6, 2, 5, 3, 4]),
]


def stride_for(cols: int) -> int:
    words = (cols + 63) // 64
    return max(4, (words + 3) // 4 * 4)


def matrix_from_rows(rows):
    cols = len(rows[0]) if rows else 0
    m = np.zeros((len(rows), stride_for(cols)), np.uint64)
    for r, s in enumerate(rows):
        for c, ch in enumerate(s):
            if ch == "1":
                m[r, c // 64] |= np.uint64(1 << (c % 64))
    return m, cols


def cuda_equivalence_matrix(rows=28, cols=96):
    m = np.zeros((rows, stride_for(cols)), np.uint64)
    for r in range(rows):
        for c in range(cols):
            mix = (((r + 1) * 0x9E3779B185EBCA87) & M64) ^ (((c + 3) * 0xC2B2AE3D27D4EB4F) & M64) ^ (
                ((r + c + 11) * 0x165667B19E3779F9) & M64)
            folded = mix ^ (mix >> 17) ^ (mix >> 33)
            if folded & 1:
                m[r, c // 64] |= np.uint64(1 << (c % 64))
    return m, cols


def python_random_matrix(rows=16, cols=512, seed=42):
    rng = random.Random(seed)
    m = np.zeros((rows, stride_for(cols)), np.uint64)
    for r in range(rows):
        for c in range(cols):
            if rng.getrandbits(1):
                m[r, c // 64] |= np.uint64(1 << (c % 64))
    return m, cols


def _xs(state):
    x = state
    x ^= (x << 13) & M64
    x ^= x >> 7
    x ^= (x << 17) & M64
    return x


def batch_shape(idx: int):
    """(n, m) of batch instance idx: n, m log-uniform in [16,128] x [64,2048],
    drawn with xorshift64 seeded 1000+idx+0x10000 (8 draws discarded, then
    two unit doubles)."""
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


def batch_instance(P, idx: int):
    n, m = batch_shape(idx)
    mat, planted = P.gen_instance(n, m, C4["p"], C4["seed0"] + idx, 4 * n)
    return mat, n, m, min(n - 1, 16), planted


def checksum_pairs(masks, weights) -> int:
    """Order-sensitive 64-bit FNV-1a over (mask, weight) pairs."""
    h = 0xCBF29CE484222325
    for mk, w in zip(np.asarray(masks).tolist(), np.asarray(weights).tolist()):
        for v in (int(mk), int(w)):
            for _ in range(8):
                h ^= v & 0xFF
                h = (h * 0x100000001B3) & M64
                v >>= 8
    return h
