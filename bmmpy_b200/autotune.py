"""Autotuner: per-shape launch settings, timed on this GPU, cached as JSON.

For the per-target Gray-code search it picks, per (words per row, k), the
carry-save blocks per step (the ALU/XU split of the popcount), the Gray-swept
chunk bits per prefix and the lanes per prefix (one lane or a 32-word lane
pair); for the spectrum search it picks, per window size t, the low bits
materialised per slice; for batches it picks the Gray/transform crossover
(:func:`bmmpy_b200.batch.autotune`).  Every candidate setting is checked to
give the default setting's exact result before it can win.  Winners go into
the library's shape tables (bmm_gray_tune_shape, bmm_spectrum_tune_shape) and
into a JSON cache keyed by device name and library version, so a later
process applies them without timing (:func:`apply_cached`).
"""

from __future__ import annotations

import json
import os
from collections.abc import Iterable

import numpy as np

from . import _native as N

# (rows, cols, k): the per-target Gray workloads measured in this project --
# 64 x 256 with 16 others, 40 x 4096 with 24 others -- and a mid-width shape.
DEFAULT_GRAY_SHAPES = ((64, 256, 16), (40, 4096, 24), (40, 2048, 20))
# window rows of the spectrum search tuned by default
DEFAULT_SPECTRUM_T = (24, 28, 32)


def _cache_path() -> str:
    root = os.environ.get("BMMPY_B200_CACHE") or os.path.join(
        os.path.expanduser("~"), ".cache", "bmmpy_b200")
    return os.path.join(root, "autotune_shapes.json")


def _device_key() -> str:
    from .runtime import get_runtime_features, get_version

    return f"{get_runtime_features().device_name}|{get_version()}"


def _load() -> dict:
    try:
        with open(_cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store(data: dict) -> None:
    path = _cache_path()
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        with open(path + ".tmp", "w") as f:
            json.dump(data, f, indent=1, sort_keys=True)
        os.replace(path + ".tmp", path)
    except OSError:
        pass


def gray_candidates(words_per_row: int, k: int) -> list[tuple[int, int, int]]:
    """(hs_blocks, chunk_bits, lanes) settings worth timing for a shape; -1
    keeps the built-in choice."""
    chunks = sorted({-1, *[c for c in range(8, 14) if c <= k]})
    if 32 < words_per_row <= 64:
        lanes1 = [(hs, c, 1) for hs in (3, 4, 5, 6) for c in chunks]
        lanes2 = [(hs, c, 2) for hs in (2, 3) for c in chunks]
        return lanes1 + lanes2
    if 16 < words_per_row <= 32:
        return [(hs, c, -1) for hs in (0, 2, 3, 4) for c in chunks]
    return [(-1, c, -1) for c in chunks]


def _time(fn, reps: int) -> float:
    import torch

    for _ in range(2):
        fn()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(reps):
        fn()
    b.record()
    torch.cuda.synchronize()
    return a.elapsed_time(b) / reps


def tune_gray_shape(rows: int, cols: int, k: int, reps: int = 3, seed: int = 1) -> dict:
    """Times the candidate settings of one per-target shape on a seeded
    Bernoulli(0.3) instance (targets i against rows i+1..i+k) and registers
    the fastest; returns {"setting": (hs, chunk, lanes), "ms": ..., "default_ms": ...}."""
    import torch

    from . import targets as T
    from .workloads import gen_instance

    L = N.lib()
    dev = torch.device("cuda", torch.cuda.current_device())
    m, _ = gen_instance(rows, cols, 0.3, seed)
    W = m.words_per_row
    t_idx, o_idx = T.cyclic_others(rows, k)
    d_words = torch.from_numpy(m.words.view(np.int64).copy()).to(dev)
    d_t = torch.from_numpy(t_idx.view(np.int32).copy()).to(dev)
    d_o = torch.from_numpy(o_idx.view(np.int32).copy()).to(dev)
    d_mask = torch.empty(rows, dtype=torch.int64, device=dev)
    d_w = torch.empty(rows, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream

    def run():
        T.gray_targets_dev(d_words, rows, m.stride_words, cols, d_t, d_o, k, d_mask, d_w, 0,
                           stream)

    N.check(L.bmm_gray_tune_shape(W, k, -1, -1, -1))
    default_ms = _time(run, reps)
    want = (d_mask.cpu().numpy().copy(), d_w.cpu().numpy().copy())
    best, best_ms = (-1, -1, -1), default_ms
    for hs, chunk, lanes in gray_candidates(W, k):
        N.check(L.bmm_gray_tune_shape(W, k, hs, chunk, lanes))
        ms = _time(run, reps)
        if not (np.array_equal(d_mask.cpu().numpy(), want[0]) and
                np.array_equal(d_w.cpu().numpy(), want[1])):
            raise RuntimeError(f"gray setting {(hs, chunk, lanes)} changed the result")
        if ms < best_ms:
            best, best_ms = (hs, chunk, lanes), ms
    N.check(L.bmm_gray_tune_shape(W, k, *best))
    return {"words_per_row": W, "k": k, "setting": list(best), "ms": best_ms,
            "default_ms": default_ms, "shape": [rows, cols, k]}


def tune_spectrum_t(t: int, cols: int = 65536, reps: int = 2, seed: int = 2) -> dict:
    """Times the spectrum split (low bits per slice) for t-row windows on a
    seeded Bernoulli(0.3) window and registers the fastest."""
    import torch

    from .workloads import gen_instance

    L = N.lib()
    dev = torch.device("cuda", torch.cuda.current_device())
    m, _ = gen_instance(t, cols, 0.3, seed)
    W = m.words_per_row
    rows = torch.from_numpy(np.ascontiguousarray(m.words[:, :W]).view(np.int64)).to(dev)
    out = torch.empty(64 * 2, dtype=torch.int64, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    top = min(t, 33)
    results, want, best, best_ms = {}, None, top, None
    for lb in range(top, max(14, top - 4) - 1, -1):
        def run():
            N.check(L.bmm_spectrum_topk_slices_dev(rows.data_ptr(), t, W, cols, 64, lb, 0,
                                                   1 << (t - lb), out.data_ptr(), stream))
        ms = _time(run, reps)
        got = out.cpu().numpy().copy()
        if want is None:
            want = got
        elif not np.array_equal(got, want):
            raise RuntimeError(f"spectrum split {lb} changed the result")
        results[lb] = ms
        if best_ms is None or ms < best_ms:
            best, best_ms = lb, ms
    N.check(L.bmm_spectrum_tune_shape(t, best))
    return {"t": t, "low_bits": best, "ms": best_ms, "per_low_bits_ms": results}


def tune(gray_shapes: Iterable[tuple[int, int, int]] = DEFAULT_GRAY_SHAPES,
         spectrum_t: Iterable[int] = DEFAULT_SPECTRUM_T, batch: bool = True,
         use_cache: bool = True) -> dict:
    """Tunes every shape not yet in the cache for this device (all of them
    when use_cache is False), applies every entry, and stores the cache."""
    from . import batch as B

    data = _load() if use_cache else {}
    key = _device_key()
    entry = data.setdefault(key, {"gray": {}, "spectrum": {}})
    for rows, cols, k in gray_shapes:
        name = f"{rows}x{cols}k{k}"
        if name not in entry["gray"]:
            entry["gray"][name] = tune_gray_shape(rows, cols, k)
    for t in spectrum_t:
        if str(t) not in entry["spectrum"]:
            entry["spectrum"][str(t)] = tune_spectrum_t(t)
    if batch:
        entry["batch"] = B.autotune(use_cache=use_cache)
    _store(data)
    apply(entry)
    return entry


def apply(entry: dict) -> None:
    """Registers a cache entry's settings in the library."""
    L = N.lib()
    for g in entry.get("gray", {}).values():
        N.check(L.bmm_gray_tune_shape(g["words_per_row"], g["k"], *g["setting"]))
    for s in entry.get("spectrum", {}).values():
        N.check(L.bmm_spectrum_tune_shape(s["t"], s["low_bits"]))
    if "batch" in entry:
        from . import batch as B

        B.set_policy(entry["batch"]["gray_max_words"])


def apply_cached() -> dict | None:
    """Applies this device's cached settings, if any; returns the entry."""
    entry = _load().get(_device_key())
    if entry:
        apply(entry)
    return entry


def reset() -> None:
    """Drops every tuned setting (the built-in policies apply again)."""
    N.check(N.lib().bmm_tune_reset())
