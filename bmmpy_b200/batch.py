"""Batched per-target searches over many uneven instances (one persistent launch).

Every row r of an n-row instance is searched against the k rows
(r + 1 + j) mod n, j < k: the best subset S of those rows to XOR into row r
(weight = popcount of the result; ties to the smallest S).  The device plan
runs all rows of all instances from one work queue, choosing per shape between
the packed Walsh-Hadamard transform and a direct Gray enumeration; the choice
comes from :func:`autotune`, which times both methods on this GPU and keeps the
crossover in a JSON cache.
"""

from __future__ import annotations

import ctypes as C
import json
import os
import time
from collections.abc import Sequence

import numpy as np

from . import _native as N
from .matrix import BitMatrix


class Batch:
    """Instances packed into one word buffer plus a descriptor table."""

    def __init__(self, instances: Sequence[tuple[BitMatrix, int]]):
        desc = np.zeros(len(instances), dtype=N.INSTANCE_DTYPE)
        chunks, off, out = [], 0, 0
        for i, (m, k) in enumerate(instances):
            desc[i] = (off, m.rows, m.cols, m.stride_words, int(k), out)
            chunks.append(np.ascontiguousarray(m.words).ravel())
            off += m.words.size
            out += m.rows
        self.words = np.concatenate(chunks) if chunks else np.zeros(1, np.uint64)
        self.desc = desc
        self.n_out = out
        self.rows = [m.rows for m, _ in instances]
        self._plan = None

    # -- host path -----------------------------------------------------------
    def run(self):
        """Returns (masks, weights) arrays over all rows of all instances."""
        masks = np.zeros(max(self.n_out, 1), np.uint64)
        weights = np.zeros(max(self.n_out, 1), np.uint32)
        rc = N.lib().bmm_batch_targets(N.u64p(self.words), self.words.size,
                                       self.desc.ctypes.data, len(self.desc), N.u64p(masks),
                                       N.u32p(weights))
        N.check(rc)
        return masks[: self.n_out], weights[: self.n_out]

    def split(self, arr):
        """Per-instance views of a flat per-row array."""
        out, o = [], 0
        for n in self.rows:
            out.append(arr[o:o + n])
            o += n
        return out

    # -- device path (plan + CUDA graph replay) --------------------------------
    def plan(self):
        if self._plan is None:
            h = C.c_void_p()
            N.check(N.lib().bmm_batch_create(self.desc.ctypes.data, len(self.desc), C.byref(h)))
            self._plan = h
        return self._plan

    def info(self):
        n_items, n_out = C.c_longlong(), C.c_size_t()
        methods = (C.c_int * 3)()
        N.check(N.lib().bmm_batch_info(self.plan(), C.byref(n_items), C.byref(n_out), methods))
        return {"items": n_items.value, "outputs": n_out.value,
                "fwht16": methods[0], "fwht_small": methods[1], "gray": methods[2]}

    def run_dev(self, d_words, d_mask, d_weight, stream: int = 0) -> None:
        """d_words / d_mask / d_weight: CUDA tensors (anything with data_ptr())."""
        N.check(N.lib().bmm_batch_run(self.plan(), d_words.data_ptr(), d_mask.data_ptr(),
                                      d_weight.data_ptr(), stream))

    def close(self) -> None:
        if self._plan is not None:
            N.lib().bmm_batch_destroy(self._plan)
            self._plan = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def set_policy(gray_max_words: int, force_method: int = -1) -> None:
    N.check(N.lib().bmm_batch_policy(int(gray_max_words), int(force_method)))


# ---------------------------------------------------------------------------
def _cache_path() -> str:
    root = os.environ.get("BMMPY_B200_CACHE") or os.path.join(
        os.path.expanduser("~"), ".cache", "bmmpy_b200")
    return os.path.join(root, "autotune.json")


def autotune(use_cache: bool = True, reps: int = 3) -> dict:
    """Pick, for 16-other searches, the widest row (in 64-bit words, <= 8) for
    which the Gray enumeration beats the transform on this GPU; apply it and
    cache it (JSON, keyed by device name and library version)."""
    import torch

    from .runtime import get_runtime_features, get_version
    from .workloads import gen_instance

    feats = get_runtime_features()
    key = f"{feats.device_name}|{get_version()}"
    path = _cache_path()
    if use_cache and os.path.exists(path):
        try:
            with open(path) as f:
                cached = json.load(f).get(key)
            if cached:
                set_policy(cached["gray_max_words"])
                return cached
        except (OSError, ValueError):
            pass
    dev = torch.device("cuda", torch.cuda.current_device())
    stream = torch.cuda.current_stream()
    timings = {}
    best = 0
    for W in range(1, 9):
        insts = [gen_instance(17, 64 * W, 0.3, 7000 + W * 1000 + i)[0] for i in range(256)]
        b = Batch([(m, 16) for m in insts])
        dw = torch.from_numpy(b.words.view(np.int64)).to(dev)
        dm = torch.empty(b.n_out, dtype=torch.int64, device=dev)
        dwt = torch.empty(b.n_out, dtype=torch.int32, device=dev)
        res = {}
        for name, force in (("fwht", 0), ("gray", 2)):
            set_policy(8, force)
            b.close()
            for _ in range(2):
                b.run_dev(dw, dm, dwt, stream.cuda_stream)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for _ in range(reps):
                b.run_dev(dw, dm, dwt, stream.cuda_stream)
            torch.cuda.synchronize()
            res[name] = (time.perf_counter() - t0) / reps / b.n_out
        b.close()
        timings[W] = res
        if res["gray"] < res["fwht"]:
            best = W
    set_policy(best, -1)
    out = {"gray_max_words": best,
           "per_item_seconds": {str(w): v for w, v in timings.items()}}
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        data = {}
        if os.path.exists(path):
            with open(path) as f:
                data = json.load(f)
        data[key] = out
        with open(path, "w") as f:
            json.dump(data, f, indent=1)
    except (OSError, ValueError):
        pass
    return out
