"""Partitioned searches on the CUDA library, one GPU: every rank's share of a
window's spectrum slices is computed in turn with the real kernels
(bmm_spectrum_topk_slices_dev) and the (weight, mask) merge of the shares must
equal the single-call MitmFwhtSearch result; shares never wait on one
another, so running them one after another on one device is exact."""

import os

import numpy as np
import pytest

import bmmpy_b200 as bmm
from bmmpy_b200 import shard
from bmmpy_b200 import targets as T
from bmmpy_b200.matrix import BitMatrix
from bmmpy_b200.workloads import gen_instance
from oracle.oracle import port

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _shares(window, k, world, low_bits=None):
    m = window.matrix
    rows = np.ascontiguousarray(m.words[window.index_array(), :m.words_per_row])
    t = len(window)
    lb, slices = shard.slice_plan(t, world, low_bits)
    lists = []
    for r in range(world):
        b, e = shard.shard_range(slices, r, world)
        if e > b:
            lists.append(shard.device_slices_search(rows, t, m.cols, k, lb, b, e))
    return shard.merge_topk(lists, k)


@pytest.mark.parametrize("t,world,low_bits", [(16, 2, None), (20, 4, None), (22, 3, 14),
                                              (24, 8, None), (26, 1, 18)])
def test_slice_shares_merge_to_the_window_result(t, world, low_bits):
    P = port()
    words, _ = P.gen_instance(40, 3000, 0.2, 100 + t, 80)
    m = BitMatrix.from_words(words, 3000)
    win = list(range(3, 3 + t))
    want = [(c.mask_u64(), c.weight) for c in
            bmm.MitmFwhtSearch(max_candidates=48).search(m.row_window(win))]
    assert _shares(m.row_window(win), 48, world, low_bits) == want


def test_c3_window_over_eight_shares(tmp_path):
    """A full-size 32-row window of the planted 512 x 65536 matrix split over 8
    shares (2^29 spectrum each) equals the reference's MITM answer."""
    wl = np.load(os.path.join(GOLDEN, "workloads.npz"))
    m, _ = gen_instance(512, 65536, 0.02, 2, 2000)
    got = _shares(m.row_window(list(range(32))), 64, 8)
    assert [tuple(int(v) for v in c) for c in wl["c3_top64"][0]] == got


def test_default_low_bits_tuning_keeps_results():
    P = port()
    words, _ = P.gen_instance(40, 3000, 0.2, 9, 80)
    m = BitMatrix.from_words(words, 3000)
    w = m.row_window(list(range(24)))
    want = [(c.mask_u64(), c.weight) for c in bmm.MitmFwhtSearch(max_candidates=64).search(w)]
    L = bmm._native.lib()
    try:
        for lb in (14, 17, 20):
            bmm._native.check(L.bmm_spectrum_tune(lb))
            got = [(c.mask_u64(), c.weight) for c in
                   bmm.MitmFwhtSearch(max_candidates=64).search(w)]
            assert got == want, lb
    finally:
        bmm._native.check(L.bmm_spectrum_tune(-1))


def test_targets_sharded_without_a_group_is_the_plain_call():
    m, _ = gen_instance(30, 2000, 0.3, 5)
    t, o = T.cyclic_others(30, 12)
    assert all(np.array_equal(a, b) for a, b in
               zip(shard.gray_targets_sharded(m, t, o), T.gray_targets(m, t, o)))
    assert all(np.array_equal(a, b) for a, b in
               zip(shard.fwht_targets_sharded(m, t, o), T.fwht_targets(m, t, o)))
