"""SASelector without a GPU: the oracle restatement against the reference
library (both score policies), the product's higher-order chain (it builds no
device table) against the reference, and the argument checks, which run before
any device work (src/search/sa_selector.cpp:10-75)."""

import random

import numpy as np
import pytest

import bmmpy_b200 as bmm
from oracle.oracle import port, ref

FIELDS = ("rows", "score", "accepted_moves", "iterations_run", "best_iteration",
          "restart_index", "seed")


def _cluster():
    # tests/cpp/sa_selector_tests.cpp / tests/support/test_common.hpp:160-171
    return bmm.matrix_from_rows(["111111000000"] * 4 + ["000000000000"] * 4)


def _random_case(rng, trial):
    rows = rng.randint(2, 40)
    cols = rng.choice([12, 64, 65, 200, 700])
    t = rng.randint(0, rows)
    words, _ = port().gen_instance(rows, cols, rng.choice([0.05, 0.2, 0.5]), trial, 0)
    kw = dict(iterations=rng.choice([0, 1, 50, 300]), restarts=rng.randint(1, 4),
              seed=rng.choice([0, 1, 99]), temperature_probe_samples=rng.choice([0, 1, 16]),
              initial_acceptance_probability=rng.choice([0.5, 0.8, 0.99]),
              cooling_rate=rng.choice([0.9, 0.99, 1.0]),
              min_temperature=rng.choice([1e-6, 1.0, 50.0]))
    return rows, cols, t, words, kw


def test_oracle_reference_cluster_example():
    w = np.ascontiguousarray(_cluster().words)
    r = port().sa_select(w, 12, 4, iterations=256, restarts=8, seed=7)
    assert r["rows"] == [0, 1, 2, 3] and r["score"] == 72


@pytest.mark.skipif(ref() is None, reason="reference not built (make -C oracle ref)")
@pytest.mark.parametrize("policy", [0, 1])
def test_oracle_matches_reference(policy):
    rng = random.Random(11 + policy)
    for trial in range(40):
        rows, cols, t, words, kw = _random_case(rng, trial)
        a = port().sa_select(words, cols, t, score_policy=policy, **kw)
        b = ref().sa_select(words, cols, t, score_policy=policy, **kw)
        assert a == b, (trial, kw)


@pytest.mark.skipif(ref() is None, reason="reference not built (make -C oracle ref)")
def test_higher_order_chain_matches_reference():
    rng = random.Random(4)
    for trial in range(40):
        rows, cols, t, words, kw = _random_case(rng, trial)
        m = bmm.BitMatrix(rows, cols)
        m.words[:] = words[:, : m.stride_words]
        r = bmm.SASelector(score_policy="higher_order_synergy", **kw).select(m, t)
        want = ref().sa_select(np.ascontiguousarray(m.words), cols, t, score_policy=1, **kw)
        assert {k: getattr(r, k) for k in FIELDS} == want, (trial, kw)


def test_higher_order_reference_cluster():
    m = _cluster()
    r = bmm.SASelector(iterations=256, restarts=8, seed=7,
                       score_policy="higher_order_synergy").select(m, 4)
    want = port().sa_select(np.ascontiguousarray(m.words), 12, 4, iterations=256, restarts=8,
                            seed=7, score_policy=1)
    assert {k: getattr(r, k) for k in FIELDS} == want
    assert r.rows == [0, 1, 2, 3]


def test_argument_errors_match_reference():
    m = _cluster()
    cases = [
        (dict(restarts=0), "SASelector: restarts must be >= 1"),
        (dict(initial_acceptance_probability=1.0),
         r"SASelector: initial_acceptance_probability must be in \(0, 1\)"),
        (dict(initial_acceptance_probability=0.0),
         r"SASelector: initial_acceptance_probability must be in \(0, 1\)"),
        (dict(cooling_rate=0.0), r"SASelector: cooling_rate must be in \(0, 1\]"),
        (dict(cooling_rate=1.5), r"SASelector: cooling_rate must be in \(0, 1\]"),
        (dict(min_temperature=0.0), "SASelector: min_temperature must be > 0"),
    ]
    for kw, msg in cases:
        with pytest.raises(ValueError, match=msg):
            bmm.SASelector(**kw).select(m, 4)
    with pytest.raises(ValueError, match="SASelector: window_size exceeds matrix row count"):
        bmm.SASelector().select(m, 9)
    with pytest.raises(ValueError, match="Unsupported score_policy: 'nope'"):
        bmm.SASelector(score_policy="nope")
    with pytest.raises(ValueError, match="Unsupported cooling_policy: 'linear'"):
        bmm.SASelector(cooling_policy="linear")


def test_empty_window_and_names():
    r = bmm.SASelector(seed=0).select(_cluster(), 0)
    assert r.rows == [] and r.score == 0 and r.seed == 0x9E3779B97F4A7C15
    s = bmm.SASelector(iterations=256, restarts=4, seed=7)
    assert s.name() == "sa"
    assert repr(s).startswith("SASelector(iterations=256, restarts=4, seed=7, "
                              "score_policy='pairwise_synergy'")
