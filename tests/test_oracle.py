"""CPU suite: the oracle (C restatement) is pinned to the reference.

* against the reference's own known-answer tests and the golden vectors the
  reference produced (tests/golden/, made by tests/golden/make_golden.py);
* against the reference library itself (oracle/_ref) on random windows when
  that library was built in this checkout.
"""

import json
import os
import random

import numpy as np
import pytest

from oracle.oracle import ga_config, port, ref
from tests.golden.fixtures import (
    C1,
    C2,
    GA_CASES,
    batch_instance,
    checksum_pairs,
    cuda_equivalence_matrix,
    matrix_from_rows,
    python_random_matrix,
)

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def ka():
    with open(os.path.join(GOLDEN, "known_answers.json")) as f:
        return json.load(f)


@pytest.fixture(scope="module")
def wl():
    return np.load(os.path.join(GOLDEN, "workloads.npz"))


def pairs(x):
    return [tuple(map(int, p)) for p in x]


def test_fwht_known_answers(ka):
    P = port()
    assert P.fwht_i32([1, 2, 3, 4]).tolist() == [10, -2, -4, 0] == ka["fwht_i32"]["expected"]
    assert P.fwht_i16([32767, 1]).tolist() == [-32768, 32766] == ka["fwht_i16_wrap"]["expected"]
    with pytest.raises(ValueError):
        P.fwht_i32([1, 2, 3])


def test_search_known_answers(ka):
    P = port()
    m, cols = matrix_from_rows(["10101", "10101"])
    got = P.fwht_search(m, cols, [0, 1], 16, 64)
    assert pairs(got) == pairs(ka["fwht_2x5_k64"])
    assert got[0] == (3, 0) and len(got) == 3
    assert pairs(P.fwht_search(m, cols, [0, 1], 16, 1)) == pairs(ka["fwht_2x5_k1"])
    assert pairs(P.bruteforce_search(m, cols, [0, 1], 1, 0)) == pairs(ka["brute_2x5_k1"])
    m, cols = matrix_from_rows(ka["six_rows"])
    six = list(range(6))
    assert pairs(P.fwht_search(m, cols, six, 16, 8)) == pairs(ka["fwht_6x12_k8"])
    assert pairs(P.mitm_search(m, cols, six, 8)) == pairs(ka["mitm_6x12_k8"])
    assert pairs(P.bruteforce_search(m, cols, six, 8, 0)) == pairs(ka["brute_6x12_k8"])
    assert pairs(P.fwht_search(m, cols, six, 16, 63)) == pairs(ka["fwht_6x12_all"])
    m, cols = matrix_from_rows(["10101", "11100", "00111"])
    assert pairs(P.fwht_search(m, cols, [0, 1, 2], 16, 4)) == pairs(ka["fwht_3x5_k4"])


def test_split_window_known_answer(ka):
    m, cols = matrix_from_rows(["11001", "00100", "01101", "01001"])
    q, r, mult, tw = port().split_window(m, cols, [0, 1, 2, 3], 2)
    exp = ka["split_4x5_low2"]
    assert (q, r, mult, tw) == (exp["q"], exp["r"], exp["mult"], exp["total_weight"])
    assert (q, r, mult, tw) == ([0, 1, 3], [1, 2, 1], [1, 1, 2], 4)


def test_cuda_equivalence_fixtures(ka):
    P = port()
    m, cols = cuda_equivalence_matrix(28, 96)
    assert pairs(P.mitm_search(m, cols, list(range(28)), 8)) == pairs(ka["mitm_28x96_k8"])
    for c, k in ((512, 8), (1024, 128)):
        m, cols = cuda_equivalence_matrix(16, c)
        got = P.bruteforce_search(m, cols, list(range(16)), k, 0)
        assert pairs(got) == pairs(ka[f"brute_16x{c}_k{k}"])
    m, cols = python_random_matrix(16, 512, 42)
    assert pairs(P.bruteforce_search(m, cols, list(range(16)), 8, 0)) == pairs(
        ka["brute_pyrand_16x512_k8"])


def test_c1_golden(wl):
    P = port()
    m, _ = P.gen_instance(C1["rows"], C1["cols"], C1["p"], C1["seed"])
    for i in range(C1["rows"]):
        others = [(i + 1 + j) % C1["rows"] for j in range(C1["k"])]
        f = P.target_best_fwht(m, C1["cols"], i, others)
        assert f == (int(wl["c1_mask"][i]), int(wl["c1_weight"][i]))
        if i < 4:
            assert P.target_best_gray(m, C1["cols"], i, others) == f
    # the per-target best is the reference window search's best mask with bit 0
    mask, weight = (int(v) for v in wl["c1_row0_window_best"])
    assert (mask, weight) == ((int(wl["c1_mask"][0]) << 1) | 1, int(wl["c1_weight"][0]))


def test_c2_reduced_golden(wl):
    P = port()
    m, _ = P.gen_instance(C2["rows"], C2["cols"], C2["p"], C2["seed"])
    for i in range(0, C2["rows"], 7):
        others = [(i + 1 + j) % C2["rows"] for j in range(16)]
        g = P.target_best_gray(m, C2["cols"], i, others)
        assert g == (int(wl["c2k16_mask"][i]), int(wl["c2k16_weight"][i]))


def test_c4_first_instances_golden(wl):
    P = port()
    first = wl["c4_first32"]
    row = 0
    for idx in range(8):
        mm, n, cols, k, _ = batch_instance(P, idx)
        ms, ws = [], []
        for i in range(n):
            others = [(i + 1 + j) % n for j in range(k)]
            bm, bw = P.target_best_fwht(mm, cols, i, others)
            ms.append(bm)
            ws.append(bw)
            assert (bm, bw) == (int(first[row][0]), int(first[row][1]))
            row += 1
        assert checksum_pairs(ms, ws) == int(wl["c4_checksums"][idx])


def test_ga_kernels_small():
    """mutate / local_improvement restatements keep their invariants."""
    P = port()
    m, _ = P.gen_instance(20, 150, 0.3, 9, 10)
    win = list(range(20))
    n, mw = 20, 1
    masks = np.array([[1 << i] for i in range(n)], np.uint64)
    weights = np.array([P.eval_cand_weight(m, 150, win, masks[i]) for i in range(n)], np.uint32)
    st = P.mutate(m, 150, win, masks, weights, 0.3, 12345)
    assert st != 12345
    for i in range(n):
        assert weights[i] == P.eval_cand_weight(m, 150, win, masks[i])
    P.local_improvement(m, 150, win, masks, weights)
    for i in range(n):
        assert weights[i] == P.eval_cand_weight(m, 150, win, masks[i])


@pytest.mark.parametrize("case", range(len(GA_CASES)))
def test_ga_port_matches_reference_golden(wl, case):
    """The C GeneticAlgorithm restatement reproduces the reference's
    trajectories (best score after every step) and best individuals."""
    rows, cols, p, iseed, scr, kw, steps, gseed = GA_CASES[case]
    m, _ = port().gen_instance(rows, cols, p, iseed, scr)
    scores, bm, bw = port().ga_run(m, cols, list(range(rows)), ga_config(**kw), gseed, steps)
    assert scores == wl[f"ga{case}_scores"].tolist()
    assert np.array_equal(bm, wl[f"ga{case}_masks"])
    assert np.array_equal(bw, wl[f"ga{case}_weights"])


def test_ga_crossover_port_pads_with_unit_weight_one():
    """crossover (operators.cpp:58-98): pool sorted by (weight, mask
    popcount), stable; dependent candidates skipped; unit padding weighs 1."""
    pm = np.array([[[0b011], [0b011], [0b000]], [[0b010], [0b110], [0b011]]], np.uint64)
    pw = np.array([[5, 2, 0], [2, 9, 2]], np.uint32)
    cm, cw = port().crossover(pm, pw)
    # pool order: (0,w0 pc0) idx2, (2,pc1) idx3, (2,pc2) idx1, (2,pc2) idx5, (5) idx0, (9) idx4
    # zero mask rejected; 0b010 -> pivot 1; 0b011 -> reduced 0b001 -> pivot 0; 0b011 (idx5)
    # dependent; 0b011 (idx0) dependent; 0b110 -> reduced 0b100 -> pivot 2: full rank
    assert cm[:, 0].tolist() == [0b010, 0b011, 0b110]
    assert cw.tolist() == [2, 2, 9]
    pm2 = np.array([[[0b001], [0b001], [0b000]]], np.uint64)
    cm2, cw2 = port().crossover(pm2, np.array([[4, 3, 1]], np.uint32))
    assert cm2[:, 0].tolist() == [0b001, 0b010, 0b100]
    assert cw2.tolist() == [3, 1, 1]


@pytest.mark.skipif(ref() is None, reason="reference library not built (make -C oracle ref)")
def test_ga_port_matches_reference_random():
    P, R = port(), ref()
    rng = random.Random(11)
    for trial in range(12):
        rows = rng.randint(1, 40)
        cols = rng.choice([1, 63, 64, 130, 300])
        m, _ = P.gen_instance(rows, cols, rng.choice([0.05, 0.3]), rng.randint(0, 99),
                              rng.randint(0, 3 * rows))
        kw = dict(population_size=rng.randint(1, 20), elite_count=rng.randint(0, 4),
                  tournament_size=rng.randint(0, 4), num_parents=rng.randint(1, 3),
                  num_offspring=rng.randint(1, 3), mutation_rate=rng.choice([0.1, 0.3, 1.2]),
                  enable_catastrophe=rng.random() < 0.3, catastrophe_threshold=rng.randint(0, 5),
                  max_generations=rng.randint(0, 25))
        if rng.random() < 0.3:
            kw["max_stale_generations"] = rng.randint(1, 6)
        win = rng.sample(range(rows), rng.randint(1, rows))
        seed = rng.randint(0, 2**64 - 1)
        a = P.ga_run(m, cols, win, ga_config(**kw), seed, 25)
        b = R.ga_run(m, cols, win, ga_config(**kw), seed, 25)
        assert a[0] == b[0]
        assert np.array_equal(a[1], b[1]) and np.array_equal(a[2], b[2])


@pytest.mark.skipif(ref() is None, reason="reference library not built (make -C oracle ref)")
def test_port_matches_reference_random():
    P, R = port(), ref()
    rng = random.Random(7)
    for trial in range(40):
        rows = rng.randint(1, 18)
        cols = rng.choice([1, 7, 64, 65, 200, 513])
        m, _ = P.gen_instance(rows, cols, rng.choice([0.1, 0.5]), rng.randint(0, 1000),
                              rng.randint(0, 5))
        t = rng.randint(1, rows)
        win = rng.sample(range(rows), t)
        k = rng.choice([1, 3, 64, 500])
        assert P.fwht_search(m, cols, win, 16, k) == R.fwht_search(m, cols, win, 16, k)
        assert P.mitm_search(m, cols, win, k) == R.mitm_search(m, cols, win, k)
        cb = rng.choice([0, 1, t])
        assert P.bruteforce_search(m, cols, win, k, cb) == R.bruteforce_search(m, cols, win, k, cb)
        lb = rng.randint(0, t)
        assert P.split_window(m, cols, win, lb) == R.split_window(m, cols, win, lb)


@pytest.mark.skipif(ref() is None, reason="reference library not built (make -C oracle ref)")
def test_port_error_classes_match_reference():
    P, R = port(), ref()
    m, cols = matrix_from_rows(["101"] * 3)
    with pytest.raises(ValueError):
        R.bruteforce_search(m, cols, [0, 1, 2], 4, 5)
    with pytest.raises(ValueError):
        P.bruteforce_search(m, cols, [0, 1, 2], 4, 5)


def test_mlp_oracle_gradients_match_finite_differences():
    """The network oracle's analytic backward pass (float64, no rounding)
    against central differences on a sample of every parameter block."""
    from oracle import mlp_oracle as M

    rng = np.random.default_rng(3)
    p = (rng.standard_normal(M.N_PARAMS) * 0.05).astype(np.float64)
    X = rng.standard_normal((3, M.K_IN))
    T = rng.random((3, M.K_OUT))
    T /= T.sum(axis=1, keepdims=True)
    _, g = M.loss_and_grads(p, X, T, round_bf16=False)
    idx = np.concatenate([rng.integers(a, b, 6) for a, b in
                          [(M.W1, M.B1), (M.B1, M.W2), (M.W2, M.B2), (M.B2, M.W3),
                           (M.W3, M.B3), (M.B3, M.N_PARAMS)]])
    h = 1e-6
    for i in idx:
        q = p.copy()
        q[i] += h
        lp, _ = M.loss_and_grads(q, X, T, round_bf16=False)
        q[i] -= 2 * h
        lm, _ = M.loss_and_grads(q, X, T, round_bf16=False)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-4 * abs(fd), (i, fd, g[i])


def test_bf16_rounding_is_nearest_even():
    from oracle import mlp_oracle as M

    x = np.array([1.0, 1.00390625, 1.01171875, -2.5, 3.0e-3], np.float32)
    # 1 + 2^-8 is a tie -> even (1.0); 1 + 3*2^-8 is a tie -> even (1 + 2^-6)
    assert M.bf16(x).tolist() == [1.0, 1.0, 1.015625, -2.5, np.float32(0.0030059814453125)]


def _apply_case(rng, rows, cols, t, n_cand, multiword=False):
    from bmmpy_b200.candidate import Candidate
    from bmmpy_b200.matrix import BitMatrix

    P = port()
    words, _ = P.gen_instance(rows, cols, rng.choice([0.1, 0.3, 0.5]), rng.randint(0, 999),
                              rng.randint(0, rows))
    m = BitMatrix(rows, cols)
    m.words[:] = words[:, : m.stride_words]
    win = rng.sample(range(rows), t)
    mw = (t + 63) // 64 if multiword else 1
    masks = np.zeros((n_cand, mw), np.uint64)
    weights = np.zeros(n_cand, np.uint32)
    cands = []
    for c in range(n_cand):
        v = rng.getrandbits(t) or 1
        for q in range(mw):
            masks[c, q] = np.uint64((v >> (64 * q)) & ((1 << 64) - 1))
        # weights: the true weight of the combination, sometimes perturbed (stale)
        acc = np.zeros(m.stride_words, np.uint64)
        for b in range(t):
            if (v >> b) & 1:
                acc ^= m.words[win[b]]
        wt = int(sum(bin(int(x)).count("1") for x in acc))
        if rng.random() < 0.2:
            wt = max(0, wt + rng.randint(-5, 5))
        weights[c] = wt
        cands.append(Candidate([int(x) for x in masks[c]], wt))
    return words, m, win, masks, weights, cands


@pytest.mark.skipif(ref() is None, reason="reference library not built (make -C oracle ref)")
def test_greedy_applier_matches_reference():
    from bmmpy_b200.apply import GreedyApplier

    R = ref()
    rng = random.Random(5)
    for trial in range(60):
        rows = rng.randint(1, 70)
        t = rng.randint(1, min(rows, 64))
        cols = rng.choice([5, 64, 130, 700])
        words, m, win, masks, weights, cands = _apply_case(rng, rows, cols, t, rng.randint(0, 40))
        stochastic = rng.random() < 0.4
        seed = rng.choice([0, 7, 2**63 + 5])
        min_gain = rng.choice([0, 1, 3])
        want, a, imp = R.apply(words, cols, win, masks, weights, False, min_gain, stochastic, seed)
        got = GreedyApplier(min_gain, stochastic=stochastic, seed=seed).apply(
            m.row_window(win), cands)
        assert (got.applied_count, got.weight_improvement) == (a, imp)
        assert np.array_equal(m.words, want[:, : m.stride_words])


@pytest.mark.skipif(ref() is None, reason="reference library not built (make -C oracle ref)")
def test_global_greedy_applier_matches_reference():
    from bmmpy_b200.apply import GlobalGreedyApplier

    R = ref()
    rng = random.Random(6)
    for trial in range(60):
        rows = rng.randint(1, 90)
        t = rng.randint(1, min(rows, 80))
        cols = rng.choice([5, 64, 200])
        words, m, win, masks, weights, cands = _apply_case(rng, rows, cols, t,
                                                           rng.randint(0, 30), multiword=True)
        req = rng.random() < 0.5
        want, a, imp = R.apply(words, cols, win, masks, weights, True, require_improvement=req)
        got = GlobalGreedyApplier(require_improvement=req).apply(m.row_window(win), cands)
        assert (got.applied_count, got.weight_improvement) == (a, imp)
        assert np.array_equal(m.words, want[:, : m.stride_words])


def test_apply_errors_match_reference_classes():
    from bmmpy_b200.apply import GlobalGreedyApplier, GreedyApplier
    from bmmpy_b200.candidate import Candidate
    from bmmpy_b200.matrix import BitMatrix

    m = BitMatrix(70, 8)
    with pytest.raises(ValueError):
        GreedyApplier(1).apply(m.row_window(list(range(65))), [])
    with pytest.raises(RuntimeError):  # mask_u64 of a two-word mask
        GreedyApplier(1).apply(m.row_window([0, 1]), [Candidate([1, 1], 0)])
    with pytest.raises(ValueError):  # bits outside the window
        GlobalGreedyApplier().apply(m.row_window([0, 1]), [Candidate([4], 0)])
