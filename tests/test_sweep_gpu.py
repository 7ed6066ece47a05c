"""Device-resident search -> apply sweeps (DeviceMatrix.search_apply,
bmm_search_apply_dev) against the host loop of search_apply over the same
windows (bmmpy/workflows.py:45-90), whose searchers and appliers are
parity-tested against the reference: same ApplyResults per window and the
same matrix afterwards, for GreedyApplier (deterministic and stochastic, the
generator carried across windows and calls) and GlobalGreedyApplier."""

import random

import numpy as np
import pytest

import bmmpy_b200 as bmm
from oracle.oracle import port

pytestmark = pytest.mark.gpu


def _instance(rows, cols, p, seed, scrambles):
    words, _ = port().gen_instance(rows, cols, p, seed, scrambles)
    m = bmm.BitMatrix(rows, cols)
    m.words[:] = words[:, : m.stride_words]
    return m


def _windows(rng, rows, t, n):
    return [sorted(rng.sample(range(rows), t)) for _ in range(n)]


APPLIERS = [
    lambda: bmm.GreedyApplier(1),
    lambda: bmm.GreedyApplier(3),
    lambda: bmm.GreedyApplier(1, stochastic=True, seed=11),
    lambda: bmm.GlobalGreedyApplier(),
    lambda: bmm.GlobalGreedyApplier(require_improvement=False),
]


@pytest.mark.parametrize("make_applier", APPLIERS)
@pytest.mark.parametrize("searcher", [bmm.MitmFwhtSearch(max_candidates=64),
                                      bmm.FwhtSearch(max_rows=20, max_candidates=16)])
def test_sweep_matches_host_loop(make_applier, searcher):
    rng = random.Random(7)
    host = _instance(96, 3000, 0.05, 21, 300)
    dev = bmm.DeviceMatrix(host)
    wins = _windows(rng, 96, 18, 24)
    a_host, a_dev = make_applier(), make_applier()
    want = [bmm.search_apply(host.row_window(w), searcher=searcher, applier=a_host)
            for w in wins]
    got = dev.search_apply(wins, searcher=searcher, applier=a_dev)
    assert [(r.applied_count, r.weight_improvement) for r in got] == [
        (r.applied_count, r.weight_improvement) for r in want]
    assert dev.to_matrix() == host
    assert dev.weight() == host.weight()
    # a second call continues from the matrix (and generator) state
    wins2 = _windows(rng, 96, 18, 8)
    want2 = [bmm.search_apply(host.row_window(w), searcher=searcher, applier=a_host)
             for w in wins2]
    got2 = dev.search_apply(wins2, searcher=searcher, applier=a_dev)
    assert [(r.applied_count, r.weight_improvement) for r in got2] == [
        (r.applied_count, r.weight_improvement) for r in want2]
    assert dev.to_matrix() == host


def test_sweep_planted_c3_windows():
    # 32-row windows of the planted 512 x 65536 matrix, one sweep of 16
    host = _instance(512, 65536, 0.02, 2, 2000)
    dev = bmm.DeviceMatrix(host)
    perm = np.random.default_rng(2).permutation(512)
    wins = [sorted(int(r) for r in perm[32 * j: 32 * (j + 1)]) for j in range(16)]
    searcher, a_host, a_dev = bmm.MitmFwhtSearch(max_candidates=64), bmm.GreedyApplier(1), \
        bmm.GreedyApplier(1)
    want = [bmm.search_apply(host.row_window(w), searcher=searcher, applier=a_host)
            for w in wins]
    got = dev.search_apply(wins, searcher=searcher, applier=a_dev)
    assert [(r.applied_count, r.weight_improvement) for r in got] == [
        (r.applied_count, r.weight_improvement) for r in want]
    assert dev.to_matrix() == host


def test_sweep_argument_errors():
    m = _instance(20, 100, 0.2, 1, 0)
    dev = bmm.DeviceMatrix(m)
    with pytest.raises(ValueError, match="exceeds the configured max_rows=16"):
        dev.search_apply([list(range(17))], searcher=bmm.FwhtSearch(), applier=bmm.GreedyApplier(1))
    with pytest.raises(ValueError, match="low_bits must be in"):
        dev.search_apply([list(range(8))], searcher=bmm.MitmFwhtSearch(low_bits=8),
                         applier=bmm.GreedyApplier(1))
    with pytest.raises(ValueError, match="window rows must be unique"):
        dev.search_apply([[1, 1, 2]], searcher=bmm.MitmFwhtSearch(),
                         applier=bmm.GreedyApplier(1))
    with pytest.raises(IndexError):
        dev.search_apply([[1, 2, 20]], searcher=bmm.MitmFwhtSearch(),
                         applier=bmm.GreedyApplier(1))
    assert dev.search_apply(np.zeros((0, 4), np.uint32), searcher=bmm.MitmFwhtSearch(),
                            applier=bmm.GreedyApplier(1)) == []
    assert dev.to_matrix() == m


def test_sweep_c_abi_rejects_out_of_range_rows():
    # a C caller that skips the Python wrapper's IndexError check gets
    # BMM_EINVAL from the library before anything is launched, and the
    # matrix is untouched
    import ctypes as C

    from bmmpy_b200 import _native as N

    m = _instance(20, 100, 0.2, 1, 0)
    dev = bmm.DeviceMatrix(m)
    wins = np.ascontiguousarray(np.array([[1, 2, 3], [4, 5, 20]], dtype=np.uint32))
    cfg = N.SweepConfig_t()
    cfg.max_candidates = 8
    res = (N.ApplyResult_t * 2)()
    state = C.c_uint64(0)
    rc = N.lib().bmm_search_apply_dev(dev._words.data_ptr(), dev.rows, dev.stride, dev.cols,
                                      N.u32p(wins), 3, 2, cfg, res, C.byref(state), 0)
    assert rc == N.EINVAL
    assert b"out of range" in N.lib().bmm_last_error()
    assert dev.to_matrix() == m
