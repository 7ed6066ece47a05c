"""Searches partitioned across ranks: one process per GPU, torch.distributed.

The reference searches on one device; these entry points split one search's
independent units over the ranks of a process group and give every rank the
same result the single-device search gives:

* :func:`gray_targets_sharded` / :func:`fwht_targets_sharded` -- the
  per-target searches: rank r takes a contiguous share of the targets, and one
  all-gather of the (mask, weight) records assembles the full arrays.
* :func:`window_search_sharded` -- one window's exact top-k (the
  MitmFwhtSearch / FwhtSearch result): the masks split into low bits (one
  materialised spectrum per slice) and high bits (the slice index); rank r
  takes a contiguous range of slices, one all-gather exchanges the k-entry
  lists (16 bytes per entry) and every rank merges them by (weight, mask).

Nothing else crosses ranks: no data-path collective inside the searches, one
gather at the end.  The collectives are torch.distributed's (NCCL between
GPUs, gloo on CPU), so the same code runs under torchrun on a GPU node and in
CPU tests.  ``compute=`` replaces the per-rank device call (tests substitute a
CPU checker there; the product passes nothing and runs the CUDA library).
"""

from __future__ import annotations

from typing import Callable, Optional

import numpy as np

from . import _native as N
from .candidate import Candidate
from .matrix import BitMatrix, RowWindow

EMPTY_WEIGHT = 0xFFFFFFFF


def shard_range(n: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous balanced share [begin, end) of n units for `rank`: the first
    n % world ranks take one unit more."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must be in [0, world)")
    base, extra = divmod(int(n), world)
    begin = rank * base + min(rank, extra)
    return begin, begin + base + (1 if rank < extra else 0)


def merge_topk(lists, k: int) -> list[tuple[int, int]]:
    """Exact merge of candidate lists: the k smallest (weight, mask) over all
    of them (mask compared as an unsigned 64-bit value), empty entries
    (weight 0xffffffff or mask 0) dropped.  Each input is an iterable of
    (mask, weight) pairs."""
    pool = [(int(w), int(m)) for lst in lists for (m, w) in lst
            if int(w) != EMPTY_WEIGHT and int(m) != 0]
    pool.sort()
    out, seen = [], set()
    for w, m in pool:
        if m in seen:  # a mask belongs to one slice only; kept for robustness
            continue
        seen.add(m)
        out.append((m, w))
        if len(out) == k:
            break
    return out


def _group_info(group):
    import torch.distributed as dist

    if not dist.is_available() or not dist.is_initialized():
        return None, 0, 1
    return dist, dist.get_rank(group), dist.get_world_size(group)


def _gather_rows(dist, group, local: np.ndarray, width: int, counts: list[int], device):
    """all-gather of per-rank int64 record arrays [count_r, width] (padded to
    the largest count) and their concatenation in rank order."""
    import torch

    world = len(counts)
    cap = max(max(counts), 1)
    buf = np.zeros((cap, width), np.int64)
    buf[: local.shape[0]] = local
    t = torch.from_numpy(buf).to(device)
    parts = [torch.empty_like(t) for _ in range(world)]
    dist.all_gather(parts, t, group=group)
    return np.concatenate([p.cpu().numpy()[: counts[r]] for r, p in enumerate(parts)], axis=0)


def _comm_device(dist, group):
    import torch

    backend = dist.get_backend(group)
    if backend == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def _targets_sharded(kind: str, matrix: BitMatrix, targets, others, group, compute, extra):
    targets = np.ascontiguousarray(targets, dtype=np.uint32).ravel()
    others = np.ascontiguousarray(others, dtype=np.uint32).reshape(targets.size, -1)
    dist, rank, world = _group_info(group)
    b, e = shard_range(targets.size, rank, world)
    if compute is None:
        from . import targets as T

        fn = T.gray_targets if kind == "gray" else T.fwht_targets
        compute = lambda m, t, o: fn(m, t, o, *extra)  # noqa: E731
    if e > b:
        masks, weights = compute(matrix, targets[b:e], others[b:e])
    else:
        masks, weights = np.zeros(0, np.uint64), np.zeros(0, np.uint32)
    if dist is None:
        return np.asarray(masks, np.uint64), np.asarray(weights, np.uint32)
    local = np.stack([np.asarray(masks, np.uint64).view(np.int64),
                      np.asarray(weights, np.uint32).astype(np.int64)], axis=1)
    counts = [shard_range(targets.size, r, world) for r in range(world)]
    counts = [hi - lo for lo, hi in counts]
    rows = _gather_rows(dist, group, local, 2, counts, _comm_device(dist, group))
    return rows[:, 0].view(np.uint64).copy(), rows[:, 1].astype(np.uint32)


def gray_targets_sharded(matrix: BitMatrix, targets, others, *, tiebreak: str = "mask",
                         group=None, compute: Optional[Callable] = None):
    """bmmpy_b200.targets.gray_targets with the targets split across the
    ranks of `group` (default: the default process group; none initialised:
    this process does everything).  Every rank returns the full
    (best_mask, best_weight) arrays."""
    return _targets_sharded("gray", matrix, targets, others, group, compute, (tiebreak,))


def fwht_targets_sharded(matrix: BitMatrix, targets, others, *, group=None,
                         compute: Optional[Callable] = None):
    """bmmpy_b200.targets.fwht_targets with the targets split across ranks."""
    return _targets_sharded("fwht", matrix, targets, others, group, compute, ())


def slice_plan(t: int, world: int, low_bits: Optional[int] = None) -> tuple[int, int]:
    """(low_bits, slices) for splitting a t-row window's masks over `world`
    ranks: the library's default split, lowered (not below 14) until there
    are at least `world` slices, so every rank gets work when it can."""
    if low_bits is None:
        low_bits = int(N.lib().bmm_spectrum_low_bits(t)) if t <= 40 else -1
        if low_bits < 0:
            raise ValueError("window search: t must be in [1, 40]")
        while low_bits > 14 and (1 << (t - low_bits)) < world:
            low_bits -= 1
    if t > 14 and not 14 <= low_bits <= min(t, 33):
        raise ValueError("low_bits must be in [14, min(t, 33)]")
    if t <= 14:
        low_bits = t
    return low_bits, 1 << (t - low_bits)


def device_slices_search(rows: np.ndarray, t: int, cols: int, k: int, low_bits: int,
                         begin: int, end: int) -> list[tuple[int, int]]:
    """Top-k (mask, weight) of the window rows (t x W host words) over the
    masks in slices [begin, end), on this process's current CUDA device."""
    import torch

    dev = torch.device("cuda", torch.cuda.current_device())
    d_rows = torch.from_numpy(np.ascontiguousarray(rows).view(np.int64)).to(dev)
    kk = max(1, min(int(k), (1 << t) - 1))
    d_out = torch.empty(kk * 2, dtype=torch.int64, device=dev)  # 16-byte records
    stream = torch.cuda.current_stream(dev).cuda_stream
    N.check(N.lib().bmm_spectrum_topk_slices_dev(d_rows.data_ptr(), t, rows.shape[1], cols, kk,
                                                 low_bits, begin, end, d_out.data_ptr(), stream),
            "bmm_spectrum_topk_slices_dev")
    rec = d_out.cpu().numpy().view(N.CAND_DTYPE)
    return [(int(r["mask"]), int(r["weight"])) for r in rec if int(r["weight"]) != EMPTY_WEIGHT]


def window_search_sharded(window: RowWindow, k: int = 64, *, low_bits: Optional[int] = None,
                          group=None, compute: Optional[Callable] = None) -> list[Candidate]:
    """The exact top-k of one window (MitmFwhtSearch(max_candidates=k)'s
    result) with its masks' slices split across the ranks of `group`; every
    rank returns the same list."""
    t = len(window)
    if k == 0 or t == 0:
        return []
    if t > 40:
        raise ValueError(f"MitmFwhtSearch: 2^{t} combinations cannot be enumerated")
    m = window.matrix
    W = m.words_per_row
    rows = np.ascontiguousarray(m.words[window.index_array(), :W]) if W else None
    if W == 0:
        return []
    dist, rank, world = _group_info(group)
    lb, slices = slice_plan(t, world, low_bits)
    b, e = shard_range(slices, rank, world)
    compute = compute or device_slices_search
    local = compute(rows, t, m.cols, k, lb, b, e) if e > b else []
    if dist is None:
        merged = merge_topk([local], k)
    else:
        kk = max(1, min(int(k), (1 << t) - 1))
        rec = np.zeros((len(local), 2), np.int64)
        for i, (mask, w) in enumerate(local):
            rec[i] = (np.uint64(mask).view(np.int64), w)
        counts = [kk] * world
        pad = np.zeros((kk, 2), np.int64)
        pad[:, 1] = EMPTY_WEIGHT
        pad[: len(local)] = rec
        rows_all = _gather_rows(dist, group, pad, 2, counts, _comm_device(dist, group))
        lists = [[(int(np.int64(r[0]).view(np.uint64)), int(r[1])) for r in
                  rows_all[q * kk:(q + 1) * kk]] for q in range(world)]
        merged = merge_topk(lists, k)
    return [Candidate.from_u64(mask, w) for mask, w in merged]


__all__ = ["shard_range", "merge_topk", "slice_plan", "gray_targets_sharded",
           "fwht_targets_sharded", "window_search_sharded", "device_slices_search"]
