"""Generate the committed golden vectors from the REFERENCE implementation.

Run in a checkout that can build the reference (``make -C oracle ref``):

    python tests/golden/make_golden.py [--skip-slow]

Every expected value written here comes from the unmodified reference C++
library (oracle/_ref/libbmmref.so), called through oracle/ref_harness.cpp:

* ``known_answers.json`` -- the reference's own known-answer tests
  (tests/cpp/fwht_tests.cpp:58-70, tests/cpp/search_cpu_tests.cpp:18-212,
  tests/cpp/search_cuda_tests.cpp:72-197, tests/python/test_cuda_api.py:63-80)
  re-run through the reference, plus the reference's answers on the fixture
  matrices those tests build.
* ``workloads.npz`` -- per-target results for the seeded synthetic workloads
  (the C1 64x256 FWHT case, the C2 40x4096 Gray-code case at full size, the
  C4 batch as per-instance checksums) and MITM top-k lists for windows of the
  C3 planted instance, and single-island GeneticAlgorithm trajectories (best
  score after every step, final best individual) for the GA_CASES of
  fixtures.py, and ExactBasisSolver results (basis masks and weights, total
  weight, rank, transform rows, basis matrix words up to 4096 columns) for
  the BASIS_CASES windows (from oracle/_ref/libbmmref_scalar.so, the
  reference built without its AVX2 backend, which crashes in this solver on
  rows of 4+ words).  Matrices are regenerated from their seeds at test time
  (xorshift64 Bernoulli fill, see oracle/bmm_oracle.c:orc_gen_instance).
"""

from __future__ import annotations

import argparse
import json
import math
import os
import random
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.oracle import port, ref, ref_scalar  # noqa: E402
from oracle.oracle import ga_config  # noqa: E402
from tests.golden.fixtures import (  # noqa: E402
    C1,
    C2,
    C3,
    BASIS_CASES,
    GA_CASES,
    batch_instance,
    cuda_equivalence_matrix,
    matrix_from_rows,
    python_random_matrix,
    checksum_pairs,
)


def known_answers(R):
    out = {}
    out["fwht_i32"] = {"input": [1, 2, 3, 4], "expected": R.fwht_i32([1, 2, 3, 4]).tolist()}
    out["fwht_i16_wrap"] = {"input": [32767, 1], "expected": R.fwht_i16([32767, 1]).tolist()}

    # 2x5 fixture: rows share columns 0, 2, 4 (tests/cpp/search_cpu_tests.cpp:18-52)
    m, cols = matrix_from_rows(["10101", "10101"])
    out["fwht_2x5_k64"] = R.fwht_search(m, cols, [0, 1], 16, 64)
    out["fwht_2x5_k1"] = R.fwht_search(m, cols, [0, 1], 16, 1)
    out["brute_2x5_k1"] = R.bruteforce_search(m, cols, [0, 1], 1, 0)

    six = ["110010101001", "101100101100", "011010011001", "111000010111", "000111100011",
           "101011110000"]
    m, cols = matrix_from_rows(six)
    out["six_rows"] = six
    out["fwht_6x12_k8"] = R.fwht_search(m, cols, list(range(6)), 16, 8)
    out["mitm_6x12_k8"] = R.mitm_search(m, cols, list(range(6)), 8)
    out["brute_6x12_k8"] = R.bruteforce_search(m, cols, list(range(6)), 8, 0)
    out["fwht_6x12_all"] = R.fwht_search(m, cols, list(range(6)), 16, 63)

    m, cols = matrix_from_rows(["10101", "11100", "00111"])
    out["fwht_3x5_k4"] = R.fwht_search(m, cols, [0, 1, 2], 16, 4)

    m, cols = matrix_from_rows(["11001", "00100", "01101", "01001"])
    q, r, mult, tw = R.split_window(m, cols, [0, 1, 2, 3], 2)
    out["split_4x5_low2"] = {"q": q, "r": r, "mult": mult, "total_weight": tw}

    # reference CUDA-equivalence fixtures (tests/support/test_common.hpp:173-190)
    m, cols = cuda_equivalence_matrix(28, 96)
    out["mitm_28x96_k8"] = R.mitm_search(m, cols, list(range(28)), 8)
    out["mitm_28x96_k128"] = R.mitm_search(m, cols, list(range(28)), 128)
    for c, k in ((512, 8), (1024, 128), (4096, 8)):
        m, cols = cuda_equivalence_matrix(16, c)
        out[f"brute_16x{c}_k{k}"] = R.bruteforce_search(m, cols, list(range(16)), k, 0)
    m, cols = python_random_matrix(16, 512, 42)
    out["brute_pyrand_16x512_k8"] = R.bruteforce_search(m, cols, list(range(16)), 8, 0)
    return out


def per_target(R, m, cols, rows, k, offset=1):
    masks, weights = [], []
    for i in range(rows):
        others = [(i + offset + j) % rows for j in range(k)]
        bm, bw = R.target_best_fwht(m, cols, i, others)
        masks.append(bm)
        weights.append(bw)
    return np.array(masks, np.uint64), np.array(weights, np.uint32)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--skip-slow", action="store_true")
    ap.add_argument("--only", default="", help="comma list of c1,c2,c3,c4,ga,basis,ka to regenerate; "
                    "the other entries of workloads.npz are kept")
    args = ap.parse_args()
    only = set(filter(None, args.only.split(",")))
    want = (lambda name: not only or name in only)
    R = ref()
    if R is None:
        raise SystemExit("build the reference first: make -C oracle ref")
    P = port()

    if want("ka"):
        ka = known_answers(R)
        with open(os.path.join(HERE, "known_answers.json"), "w") as f:
            json.dump(ka, f, indent=1)
        print("known_answers.json written")

    arrays = {}
    npz = os.path.join(HERE, "workloads.npz")
    if only and os.path.exists(npz):
        arrays.update(dict(np.load(npz)))
    t0 = time.time()
    if want("c1"):
        c1(R, P, arrays)
    if want("c2"):
        c2(R, P, arrays)
    if want("c4"):
        c4(R, P, arrays)
    if want("c3") and not args.skip_slow:
        c3(R, P, arrays)
    if want("ga"):
        ga(R, P, arrays)
    if want("basis"):
        basis(ref_scalar(), P, arrays)
    np.savez_compressed(npz, **arrays)
    print("workloads.npz written")


def c1(R, P, arrays):
    t0 = time.time()
    m, _ = P.gen_instance(C1["rows"], C1["cols"], C1["p"], C1["seed"])
    arrays["c1_mask"], arrays["c1_weight"] = per_target(R, m, C1["cols"], C1["rows"], C1["k"])
    # the reference's own FwhtSearch on the 17-row window [i, i+1..i+16]:
    # its best mask with bit 0 set must be (S << 1) | 1 of the per-target best
    win = [0] + [1 + j for j in range(16)]
    top = R.fwht_search(m, C1["cols"], win, 17, (1 << 17) - 1)
    best0 = [c for c in top if c[0] & 1][0]
    arrays["c1_row0_window_best"] = np.array(best0, np.uint64)
    print("C1 done", time.time() - t0)


def c2(R, P, arrays):
    t0 = time.time()
    m, _ = P.gen_instance(C2["rows"], C2["cols"], C2["p"], C2["seed"])
    arrays["c2_mask"], arrays["c2_weight"] = per_target(R, m, C2["cols"], C2["rows"], C2["k"])
    # reduced C2 (k=16) for the exhaustive Gray-code checks
    arrays["c2k16_mask"], arrays["c2k16_weight"] = per_target(R, m, C2["cols"], C2["rows"], 16)
    print("C2 done", time.time() - t0)


def c4(R, P, arrays):
    t0 = time.time()
    sums = []
    first = []
    n_inst = 4096
    for idx in range(n_inst):
        mm, n, cols, k, planted = batch_instance(P, idx)
        ms, ws = per_target(R, mm, cols, n, k)
        sums.append(checksum_pairs(ms, ws))
        if idx < 32:
            first.append(np.stack([ms.astype(np.uint64), ws.astype(np.uint64)], 1))
    arrays["c4_checksums"] = np.array(sums, np.uint64)
    arrays["c4_first32"] = np.concatenate(first, 0)
    print("C4 done", time.time() - t0)


def _c3_window(j):
    # one reference MitmFwhtSearch(k=64) on rows 32j..32j+31 (its search is
    # single-threaded; windows run in parallel worker processes)
    R, P = ref(), port()
    m, _ = P.gen_instance(C3["rows"], C3["cols"], C3["p"], C3["seed"], C3["scrambles"])
    return np.array(R.mitm_search(m, C3["cols"], list(range(32 * j, 32 * j + 32)), 64), np.uint64)


def c3(R, P, arrays):
    import multiprocessing as mp
    from concurrent.futures import ProcessPoolExecutor

    t0 = time.time()
    m, planted = P.gen_instance(C3["rows"], C3["cols"], C3["p"], C3["seed"], C3["scrambles"])
    arrays["c3_planted"] = np.array([planted], np.uint64)
    n = C3["golden_windows"]
    with ProcessPoolExecutor(max_workers=min(n, os.cpu_count() or 1),
                             mp_context=mp.get_context("spawn")) as pool:
        tops = list(pool.map(_c3_window, range(n)))
    arrays["c3_top64"] = np.stack(tops, 0)
    print("C3 done", n, "windows", time.time() - t0)


def ga(R, P, arrays):
    t0 = time.time()
    for i, (rows, cols, p, iseed, scr, kw, steps, gseed) in enumerate(GA_CASES):
        m, _ = P.gen_instance(rows, cols, p, iseed, scr)
        scores, bm, bw, secs = R.ga_run(m, cols, list(range(rows)), ga_config(**kw), gseed, steps)
        arrays[f"ga{i}_scores"] = np.array(scores, np.uint64)
        arrays[f"ga{i}_masks"] = bm
        arrays[f"ga{i}_weights"] = bw
        print(f"  GA case {i}: {len(scores) - 1} steps, best {scores[-1]}, {secs:.2f}s")
    print("GA done", time.time() - t0)


def basis(R, P, arrays):
    t0 = time.time()
    for i, (rows, cols, p, iseed, scr, win) in enumerate(BASIS_CASES):
        m, _ = P.gen_instance(rows, cols, p, iseed, scr)
        r = R.exact_basis(m, cols, win)
        arrays[f"basis{i}_masks"] = np.array(r["basis_masks"], np.uint32)
        arrays[f"basis{i}_weights"] = np.array(r["basis_weights"], np.uint32)
        arrays[f"basis{i}_transform"] = np.array(r["transform"], np.uint64)
        arrays[f"basis{i}_scalars"] = np.array(
            [r["input_rows"], r["cols"], r["rank"], r["enumerated_states"], r["total_weight"]],
            np.uint64)
        if cols <= 4096:
            arrays[f"basis{i}_words"] = r["basis_words"]
        print(f"  basis case {i}: rank {r['rank']}, total {r['total_weight']}")
    print("basis done", time.time() - t0)


if __name__ == "__main__":
    main()
