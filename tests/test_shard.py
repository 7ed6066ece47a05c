"""Partitioned searches (bmmpy_b200.shard) on CPU with two and three gloo
ranks: the partition, the all-gather and the (weight, mask) merge.  Each
rank's own share is computed by the oracle (compute=), so these run without a
GPU; tests/test_shard_gpu.py runs the shares on the CUDA library."""

import os
import random
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from bmmpy_b200 import shard
from bmmpy_b200.matrix import BitMatrix
from bmmpy_b200 import targets as T
from oracle.oracle import port


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_shard_range_partitions():
    for n in (0, 1, 5, 40, 97):
        for world in (1, 2, 3, 8):
            parts = [shard.shard_range(n, r, world) for r in range(world)]
            assert parts[0][0] == 0 and parts[-1][1] == n
            assert all(parts[i][1] == parts[i + 1][0] for i in range(world - 1))
            sizes = [e - b for b, e in parts]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard.shard_range(4, 2, 2)


def test_merge_topk_is_the_sorted_union():
    rng = random.Random(1)
    lists, union = [], []
    for _ in range(4):
        lst = [(rng.randrange(1, 1 << 40), rng.randrange(0, 50)) for _ in range(30)]
        lists.append(lst + [(0, 3), (5, 0xFFFFFFFF)])  # empty entries are dropped
        union += lst
    want = sorted(union, key=lambda c: (c[1], c[0]))[:25]
    assert shard.merge_topk(lists, 25) == want


def test_slice_plan_gives_every_rank_a_slice():
    assert shard.slice_plan(16, 2) == (15, 2)
    assert shard.slice_plan(32, 8) == (29, 8)
    assert shard.slice_plan(32, 1, 24) == (24, 256)
    assert shard.slice_plan(12, 4) == (12, 1)
    with pytest.raises(ValueError):
        shard.slice_plan(20, 2, 13)


def _oracle_slices(words, win):
    """compute= for window_search_sharded: every candidate of the window from
    the oracle, restricted to the rank's slices."""
    P = port()

    def run(rows, t, cols, k, low_bits, begin, end):
        allc = P.bruteforce_search(words, cols, win, (1 << t) - 1, 0)
        mine = [(m, w) for m, w in allc if begin <= (m >> low_bits) < end]
        mine.sort(key=lambda c: (c[1], c[0]))
        return mine[:k]
    return run


def _rank(rank, world, port_, out, case):
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port_}", rank=rank,
                            world_size=world)
    try:
        P = port()
        words, _ = P.gen_instance(18, 300, 0.3, 7 + case, 0)
        m = BitMatrix.from_words(words, 300)
        t, o = T.cyclic_others(18, 6)
        gm, gw = shard.gray_targets_sharded(
            m, t, o, compute=lambda mm, tt, oo: (
                np.array([P.target_best_gray(words, 300, int(a), list(map(int, b)))[0]
                          for a, b in zip(tt, oo)], np.uint64),
                np.array([P.target_best_gray(words, 300, int(a), list(map(int, b)))[1]
                          for a, b in zip(tt, oo)], np.uint32)))
        win = list(range(1, 17))
        cands = shard.window_search_sharded(m.row_window(win), 20, compute=_oracle_slices(words, win))
        out[rank] = (gm.tolist(), gw.tolist(), [(c.mask_u64(), c.weight) for c in cands])
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_searches_match_single_process(world):
    port_ = _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(_rank, args=(world, port_, out, world), nprocs=world, join=True,
                           start_method="spawn")
        got = dict(out)
    P = port()
    words, _ = P.gen_instance(18, 300, 0.3, 7 + world, 0)
    t, o = T.cyclic_others(18, 6)
    want_m, want_w = zip(*[P.target_best_gray(words, 300, int(a), list(map(int, b)))
                           for a, b in zip(t, o)])
    want_c = P.bruteforce_search(words, 300, list(range(1, 17)), 20, 0)
    for r in range(world):
        assert got[r][0] == list(want_m) and got[r][1] == list(want_w)
        assert got[r][2] == want_c
