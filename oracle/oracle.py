"""ctypes front-end for the two CPU checkers (test infrastructure only).

* :data:`port` -- the plain-C restatement in ``oracle/bmm_oracle.c``
  (``oracle/liboracle.so``), always available once ``make -C oracle`` ran.
* :func:`ref` -- the unmodified reference C++ library compiled from its own
  sources by ``make -C oracle ref`` (``oracle/_ref/libbmmref.so``); ``None``
  where it was not built.
* :func:`ref_cuda` -- the same with the reference's CUDA backend
  (``make -C oracle ref-cuda``): CudaBruteforceSearch and CudaMitmFwhtSearch
  running the reference's own kernels; ``None`` where it was not built.

Only the tests, ``__graft_entry__.smoke()`` and the CPU legs of ``bench.py``
import this module; the product never does.  Matrices are numpy ``uint64``
arrays of shape ``(rows, stride)`` in the reference's packed layout.
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libbmmref.so")
# the reference built without its AVX2 backend (used for ExactBasisSolver,
# which the AVX2 build crashes on for rows of 4+ words: aligned loads in
# src/core/bit_ops_avx2.cpp:21-24 on an unaligned std::vector)
REF_SCALAR_SO = os.path.join(HERE, "_ref", "libbmmref_scalar.so")
# the reference with its CUDA backend (its own GPU kernels, built for sm_100a
# by ``make -C oracle ref-cuda``): the GPU bar bench.py's reference-gpu arm
# times on the same B200
REF_CUDA_SO = os.path.join(HERE, "_ref", "cuda", "libbmmref_cuda.so")

_u64p = C.POINTER(C.c_uint64)
_u32p = C.POINTER(C.c_uint32)
_i32p = C.POINTER(C.c_int32)
_i16p = C.POINTER(C.c_int16)
_szp = C.POINTER(C.c_size_t)
_sz = C.c_size_t


class OracleError(RuntimeError):
    pass


class MatrixErrorRef(RuntimeError):
    """The reference's MatrixError, as raised through the harness."""


# ---- matrix IO restated (src/core/bit_matrix_io.cpp:34-175,
#      src/core/bit_matrix_hash.cpp:30-58); plain Python for small matrices ----
_WS = b" \n\r\t\f\v"


def text_format(words, rows, cols) -> bytes:
    """save_text: header line, then one '0'/'1' line per row."""
    out = [f"{rows} {cols}\n".encode()]
    for r in range(rows):
        line = bytearray(b"0" * cols)
        for c in range(cols):
            if (int(words[r][c // 64]) >> (c % 64)) & 1:
                line[c] = ord("1")
        out.append(bytes(line) + b"\n")
    return b"".join(out)


def text_parse(text: bytes):
    """load_text: (rows, cols, list of row bit lists) or raises RuntimeError
    with the reference's message."""
    p, n, dims = 0, len(text), []
    for _ in range(2):
        while p < n and text[p:p + 1] in [bytes([b]) for b in _WS]:
            p += 1
        neg = False
        if p < n and text[p:p + 1] in (b"+", b"-"):
            neg = text[p:p + 1] == b"-"
            p += 1
        q = p
        while p < n and 48 <= text[p] <= 57:
            p += 1
        if q == p or int(text[q:p]) >= 1 << 64:
            raise RuntimeError("failed to read matrix text header")
        v = int(text[q:p])
        dims.append((-v) % (1 << 64) if neg else v)
    rows, cols = dims
    total = rows * cols
    bits = []
    while len(bits) < total and p < n:
        ch = text[p]
        p += 1
        if ch in (48, 49):
            bits.append(ch - 48)
        elif ch not in _WS:
            raise RuntimeError("matrix text contains invalid character")
    if len(bits) != total:
        raise RuntimeError("failed to read matrix text payload")
    while p < n:
        if text[p] not in _WS:
            raise RuntimeError("matrix text contains trailing data")
        p += 1
    return rows, cols, [bits[r * cols:(r + 1) * cols] for r in range(rows)]


def matrix_hash(words, rows, cols) -> str:
    """SHA-256 (hashlib) over little-endian u64 rows, cols, tail-masked words."""
    import hashlib

    h = hashlib.sha256()
    h.update(int(rows).to_bytes(8, "little") + int(cols).to_bytes(8, "little"))
    W = (cols + 63) // 64
    tail = (1 << (cols % 64)) - 1 if cols % 64 else (1 << 64) - 1
    for r in range(rows):
        for w in range(W):
            v = int(words[r][w]) & (tail if w == W - 1 else (1 << 64) - 1)
            h.update(v.to_bytes(8, "little"))
    return h.hexdigest()


class GaConfig(C.Structure):
    """GeneticAlgorithmConfig as orc_ga_config / refh_ga_config (flags: 1
    max_generations, 2 max_stale_generations, 4 target_total_weight)."""

    _fields_ = [("population_size", C.c_size_t), ("elite_count", C.c_size_t),
                ("num_parents", C.c_size_t), ("num_offspring", C.c_size_t),
                ("tournament_size", C.c_size_t), ("enable_catastrophe", C.c_int),
                ("catastrophe_threshold", C.c_size_t),
                ("catastrophe_survival_rate", C.c_double), ("mutation_rate", C.c_double),
                ("flags", C.c_uint), ("max_generations", C.c_uint64),
                ("max_stale_generations", C.c_uint64), ("target_total_weight", C.c_uint64)]


def ga_config(population_size=300, elite_count=3, num_parents=2, num_offspring=1,
              tournament_size=3, enable_catastrophe=False, catastrophe_threshold=30,
              catastrophe_survival_rate=0.2, mutation_rate=0.3, max_generations=None,
              max_stale_generations=None, target_total_weight=None) -> GaConfig:
    """Defaults of include/bmmpy/ga/genetic_algorithm.hpp:17-29."""
    flags = ((1 if max_generations is not None else 0)
             | (2 if max_stale_generations is not None else 0)
             | (4 if target_total_weight is not None else 0))
    return GaConfig(population_size, elite_count, num_parents, num_offspring, tournament_size,
                    int(bool(enable_catastrophe)), catastrophe_threshold,
                    catastrophe_survival_rate, mutation_rate, flags, max_generations or 0,
                    max_stale_generations or 0, target_total_weight or 0)


ERRORS = {-1: ValueError, -2: OverflowError, -3: IndexError, -4: RuntimeError, -5: RuntimeError}


def _ptr(a, typ):
    return a.ctypes.data_as(typ)


def _build_port():
    if not os.path.exists(PORT_SO):
        subprocess.run(["make", "-s", "-C", HERE, "liboracle.so"], check=True)


def _load_port():
    _build_port()
    lib = C.CDLL(PORT_SO)
    lib.orc_gen_instance.restype = C.c_uint64
    lib.orc_gen_instance.argtypes = [_u64p, _sz, _sz, _sz, C.c_double, C.c_uint64, _sz]
    lib.orc_fwht_i32.argtypes = [_i32p, _sz]
    lib.orc_fwht_i16.argtypes = [_i16p, _sz]
    for name in ("orc_fwht_search",):
        getattr(lib, name).restype = C.c_long
        getattr(lib, name).argtypes = [_u64p, _sz, _sz, _szp, _sz, _sz, _sz, _u64p, _u32p, _sz]
    lib.orc_mitm_search.restype = C.c_long
    lib.orc_mitm_search.argtypes = [_u64p, _sz, _sz, _szp, _sz, _sz, _u64p, _u32p, _sz]
    lib.orc_bruteforce_search.restype = C.c_long
    lib.orc_bruteforce_search.argtypes = [_u64p, _sz, _sz, _szp, _sz, _sz, _sz, _u64p, _u32p, _sz]
    lib.orc_split_window.restype = C.c_long
    lib.orc_split_window.argtypes = [_u64p, _sz, _sz, _szp, _sz, _sz, _u64p, _u64p, _i32p, _sz, _i32p]
    lib.orc_target_best_gray.argtypes = [_u64p, _sz, _sz, _sz, _szp, _sz, C.c_int, _u64p, _u32p]
    lib.orc_target_best_fwht.argtypes = [_u64p, _sz, _sz, _sz, _szp, _sz, _u64p, _u32p]
    lib.orc_eval_cand_weight.restype = C.c_uint32
    lib.orc_eval_cand_weight.argtypes = [_u64p, _sz, _sz, _szp, _sz, _u64p, _sz]
    lib.orc_mutate.argtypes = [_u64p, _sz, _sz, _szp, _sz, _u64p, _u32p, _sz, C.c_double, _u64p]
    lib.orc_local_improvement.argtypes = [_u64p, _sz, _sz, _szp, _sz, _u64p, _u32p, _sz]
    lib.orc_crossover.argtypes = [_sz, _sz, _u64p, _u32p, _u64p, _u32p]
    lib.orc_ga_run.restype = C.c_long
    lib.orc_ga_run.argtypes = [_u64p, _sz, _sz, _szp, _sz, C.POINTER(GaConfig), C.c_uint64,
                               C.c_uint64, _u64p, _u64p, _u32p]
    lib.orc_exact_basis.restype = C.c_long
    lib.orc_exact_basis.argtypes = [_u64p, _sz, _sz, _szp, _sz, _u32p, _u32p, _u64p]
    lib.orc_basis_weight_counts.argtypes = [_u64p, _sz, _sz, _szp, _sz, _u64p]
    lib.orc_sa_select.restype = C.c_long
    lib.orc_sa_select.argtypes = [_u64p, _sz, _sz, _sz, _sz, C.c_uint64, C.c_uint64, C.c_uint64,
                                  C.c_int, C.c_uint64, C.c_double, C.c_double, C.c_double,
                                  C.POINTER(C.c_int64), _szp]
    return lib


class _Searches:
    """Common window-search calls over either checker library."""

    prefix = ""

    def __init__(self, lib):
        self.lib = lib

    def _win(self, win):
        return np.ascontiguousarray(np.asarray(win, dtype=np.uintp))

    def sa_select(self, m, cols, window_size, iterations=10000, restarts=8, seed=0,
                  score_policy=0, temperature_probe_samples=64,
                  initial_acceptance_probability=0.8, cooling_rate=0.99,
                  min_temperature=1e-6):
        """SASelector.select: dict of the SASelectionResult fields."""
        m = np.ascontiguousarray(m, dtype=np.uint64)
        sc = np.zeros(6, np.int64)
        rows = np.zeros(max(window_size, 1), np.uintp)
        args = (window_size, iterations, restarts, seed, score_policy, temperature_probe_samples,
                initial_acceptance_probability, cooling_rate, min_temperature,
                _ptr(sc, C.POINTER(C.c_int64)), _ptr(rows, _szp))
        if self.prefix == "refh":
            n = self.lib.refh_sa_select(_ptr(m, _u64p), m.shape[0], cols, m.shape[1], *args)
        else:
            n = self.lib.orc_sa_select(_ptr(m, _u64p), m.shape[1], m.shape[0], cols, *args)
        if n < 0:
            raise ERRORS.get(n, OracleError)(f"checker error {n}")
        return {"rows": [int(r) for r in rows[:n]], "score": int(sc[0]),
                "accepted_moves": int(sc[1]), "iterations_run": int(sc[2]),
                "best_iteration": int(sc[3]), "restart_index": int(sc[4]),
                "seed": int(np.uint64(sc[5]))}

    def _result(self, count, masks, weights):
        if count < 0:
            raise ERRORS.get(count, OracleError)(f"checker error {count}")
        n = min(count, len(masks))
        return [(int(masks[i]), int(weights[i])) for i in range(n)]


class Port(_Searches):
    def __init__(self):
        super().__init__(_load_port())

    def gen_instance(self, rows, cols, p, seed, scrambles=0, stride=None):
        stride = stride or max(4, ((cols + 63) // 64 + 3) // 4 * 4)
        m = np.zeros((rows, stride), dtype=np.uint64)
        planted = self.lib.orc_gen_instance(_ptr(m, _u64p), rows, cols, stride, p, seed, scrambles)
        return m, int(planted)

    def fwht_i32(self, a):
        a = np.ascontiguousarray(a, dtype=np.int32).copy()
        rc = self.lib.orc_fwht_i32(_ptr(a, _i32p), a.size)
        if rc:
            raise ValueError("size must be a power of two")
        return a

    def fwht_i16(self, a):
        a = np.ascontiguousarray(a, dtype=np.int16).copy()
        rc = self.lib.orc_fwht_i16(_ptr(a, _i16p), a.size)
        if rc:
            raise ValueError("size must be a power of two")
        return a

    def fwht_search(self, m, cols, win, max_rows=16, k=64):
        win = self._win(win)
        cap = max(1, min(k, 1 << min(len(win), 24)))
        masks = np.zeros(cap, np.uint64)
        ws = np.zeros(cap, np.uint32)
        c = self.lib.orc_fwht_search(_ptr(m, _u64p), m.shape[1], cols, _ptr(win, _szp), len(win),
                                     max_rows, k, _ptr(masks, _u64p), _ptr(ws, _u32p), cap)
        return self._result(c, masks, ws)

    def mitm_search(self, m, cols, win, k=64):
        win = self._win(win)
        cap = max(1, min(k, 1 << min(len(win), 24)))
        masks = np.zeros(cap, np.uint64)
        ws = np.zeros(cap, np.uint32)
        c = self.lib.orc_mitm_search(_ptr(m, _u64p), m.shape[1], cols, _ptr(win, _szp), len(win),
                                     k, _ptr(masks, _u64p), _ptr(ws, _u32p), cap)
        return self._result(c, masks, ws)

    def bruteforce_search(self, m, cols, win, k=128, chunk_bits=0):
        win = self._win(win)
        cap = max(1, min(k, 1 << min(len(win), 24)))
        masks = np.zeros(cap, np.uint64)
        ws = np.zeros(cap, np.uint32)
        c = self.lib.orc_bruteforce_search(_ptr(m, _u64p), m.shape[1], cols, _ptr(win, _szp),
                                           len(win), k, chunk_bits, _ptr(masks, _u64p),
                                           _ptr(ws, _u32p), cap)
        return self._result(c, masks, ws)

    def split_window(self, m, cols, win, low_bits):
        win = self._win(win)
        cap = max(1, cols)
        q = np.zeros(cap, np.uint64)
        r = np.zeros(cap, np.uint64)
        mult = np.zeros(cap, np.int32)
        tw = C.c_int32(0)
        u = self.lib.orc_split_window(_ptr(m, _u64p), m.shape[1], cols, _ptr(win, _szp), len(win),
                                      low_bits, _ptr(q, _u64p), _ptr(r, _u64p), _ptr(mult, _i32p),
                                      cap, C.byref(tw))
        if u < 0:
            raise ERRORS.get(u, OracleError)(f"checker error {u}")
        return q[:u].tolist(), r[:u].tolist(), mult[:u].tolist(), tw.value

    def target_best_gray(self, m, cols, target, others, tiebreak=0):
        others = self._win(others)
        bm = C.c_uint64(0)
        bw = C.c_uint32(0)
        rc = self.lib.orc_target_best_gray(_ptr(m, _u64p), m.shape[1], cols, target,
                                           _ptr(others, _szp), len(others), tiebreak,
                                           C.byref(bm), C.byref(bw))
        if rc:
            raise ValueError("k too large")
        return int(bm.value), int(bw.value)

    def target_best_fwht(self, m, cols, target, others):
        others = self._win(others)
        bm = C.c_uint64(0)
        bw = C.c_uint32(0)
        rc = self.lib.orc_target_best_fwht(_ptr(m, _u64p), m.shape[1], cols, target,
                                           _ptr(others, _szp), len(others), C.byref(bm), C.byref(bw))
        if rc:
            raise ValueError("k too large")
        return int(bm.value), int(bw.value)

    def eval_cand_weight(self, m, cols, win, mask_words):
        win = self._win(win)
        mk = np.ascontiguousarray(mask_words, dtype=np.uint64)
        return int(self.lib.orc_eval_cand_weight(_ptr(m, _u64p), m.shape[1], cols, _ptr(win, _szp),
                                                 len(win), _ptr(mk, _u64p), mk.size))

    def mutate(self, m, cols, win, masks, weights, rate, rng_state):
        """masks: (n, mw) uint64 (modified in place); returns new rng state."""
        win = self._win(win)
        st = C.c_uint64(rng_state)
        self.lib.orc_mutate(_ptr(m, _u64p), m.shape[1], cols, _ptr(win, _szp), len(win),
                            _ptr(masks, _u64p), _ptr(weights, _u32p), masks.shape[1], rate,
                            C.byref(st))
        return int(st.value)

    def local_improvement(self, m, cols, win, masks, weights):
        win = self._win(win)
        self.lib.orc_local_improvement(_ptr(m, _u64p), m.shape[1], cols, _ptr(win, _szp),
                                       len(win), _ptr(masks, _u64p), _ptr(weights, _u32p),
                                       masks.shape[1])

    def crossover(self, parent_masks, parent_weights):
        """parent_masks: (parents, n, mw) uint64; parent_weights: (parents, n)."""
        pm = np.ascontiguousarray(parent_masks, dtype=np.uint64)
        pw = np.ascontiguousarray(parent_weights, dtype=np.uint32)
        np_, n, mw = pm.shape
        cm = np.zeros((n, mw), np.uint64)
        cw = np.zeros(n, np.uint32)
        self.lib.orc_crossover(n, np_, _ptr(pm, _u64p), _ptr(pw, _u32p), _ptr(cm, _u64p),
                               _ptr(cw, _u32p))
        return cm, cw

    def exact_basis(self, m, cols, win):
        """ExactBasisSolver without caps: (masks, weights, total_weight)."""
        win = self._win(win)
        t = len(win)
        masks = np.zeros(max(t, 1), np.uint32)
        ws = np.zeros(max(t, 1), np.uint32)
        total = C.c_uint64(0)
        r = self.lib.orc_exact_basis(_ptr(m, _u64p), m.shape[1], cols, _ptr(win, _szp), t,
                                     _ptr(masks, _u32p), _ptr(ws, _u32p), C.byref(total))
        if r < 0:
            raise ERRORS.get(r, OracleError)(f"oracle error {r}")
        return [int(x) for x in masks[:r]], [int(x) for x in ws[:r]], int(total.value)

    def basis_weight_counts(self, m, cols, win):
        win = self._win(win)
        counts = np.zeros(cols + 1, np.uint64)
        rc = self.lib.orc_basis_weight_counts(_ptr(m, _u64p), m.shape[1], cols, _ptr(win, _szp),
                                              len(win), _ptr(counts, _u64p))
        if rc < 0:
            raise ERRORS.get(rc, OracleError)(f"oracle error {rc}")
        return counts

    def ga_run(self, m, cols, win, cfg: GaConfig, seed, max_steps):
        """initialize() + step()s: (scores per step, best masks (n, mw), best weights)."""
        win = self._win(win)
        n = len(win)
        mw = (n + 63) // 64
        scores = np.zeros(max_steps + 1, np.uint64)
        bm = np.zeros((n, mw), np.uint64)
        bw = np.zeros(n, np.uint32)
        g = self.lib.orc_ga_run(_ptr(m, _u64p), m.shape[1], cols, _ptr(win, _szp), n,
                                C.byref(cfg), seed, max_steps, _ptr(scores, _u64p),
                                _ptr(bm, _u64p), _ptr(bw, _u32p))
        if g < 0:
            raise ERRORS.get(g, OracleError)("oracle error")
        return scores[: g + 1].tolist(), bm, bw


class Ref(_Searches):
    """The reference library itself (oracle/_ref/libbmmref.so)."""

    prefix = "refh"

    def __init__(self, lib):
        super().__init__(lib)
        L = lib
        L.refh_fwht_i32.restype = C.c_long
        L.refh_fwht_i32.argtypes = [_i32p, _sz]
        L.refh_fwht_i16.restype = C.c_long
        L.refh_fwht_i16.argtypes = [_i16p, _sz]
        L.refh_fwht_search.restype = C.c_long
        L.refh_fwht_search.argtypes = [_u64p, _sz, _sz, _sz, _szp, _sz, _sz, _sz, _u64p, _u32p, _sz]
        L.refh_mitm_search.restype = C.c_long
        L.refh_mitm_search.argtypes = [_u64p, _sz, _sz, _sz, _szp, _sz, _sz, _u64p, _u32p, _sz]
        L.refh_bruteforce_search.restype = C.c_long
        L.refh_bruteforce_search.argtypes = [_u64p, _sz, _sz, _sz, _szp, _sz, _sz, _sz, _u64p,
                                             _u32p, _sz]
        L.refh_split_window.restype = C.c_long
        L.refh_split_window.argtypes = [_u64p, _sz, _sz, _sz, _szp, _sz, _sz, _u64p, _u64p, _i32p,
                                        _sz, _i32p]
        L.refh_target_best_fwht.restype = C.c_long
        L.refh_target_best_fwht.argtypes = [_u64p, _sz, _sz, _sz, _sz, _szp, _sz, _u64p, _u32p]
        L.refh_ga_run.restype = C.c_long
        L.refh_ga_run.argtypes = [_u64p, _sz, _sz, _sz, _szp, _sz, C.POINTER(GaConfig),
                                  C.c_uint64, _sz, _u64p, _u64p, _u32p, C.POINTER(C.c_double)]
        L.refh_apply.restype = C.c_long
        L.refh_apply.argtypes = [_u64p, _sz, _sz, _sz, _szp, _sz, _u64p, _sz, _u32p, _sz, C.c_int,
                                 C.c_uint64, C.c_int, C.c_uint64, C.c_int, _u64p, _u64p, _u64p]
        L.refh_exact_basis.restype = C.c_long
        L.refh_exact_basis.argtypes = [_u64p, _sz, _sz, _sz, _szp, _sz, _sz, C.c_uint64, _sz,
                                       _u64p, _u32p, _u32p, _u64p, _u64p]
        L.refh_sa_select.restype = C.c_long
        L.refh_sa_select.argtypes = [_u64p, _sz, _sz, _sz, _sz, _sz, _sz, C.c_uint64, C.c_int,
                                     _sz, C.c_double, C.c_double, C.c_double,
                                     C.POINTER(C.c_int64), _szp]
        L.refh_last_error.restype = C.c_char_p
        L.refh_last_error.argtypes = []
        L.refh_matrix_from_text.restype = C.c_long
        L.refh_matrix_from_text.argtypes = [C.c_char_p, _sz, _u64p, _u64p, _sz, _sz]
        L.refh_matrix_to_text.restype = C.c_long
        L.refh_matrix_to_text.argtypes = [_u64p, _sz, _sz, _sz, C.c_char_p, _sz]
        L.refh_matrix_hash.restype = C.c_long
        L.refh_matrix_hash.argtypes = [_u64p, _sz, _sz, _sz, C.c_char_p]
        L.refh_matrix_save_binary.restype = C.c_long
        L.refh_matrix_save_binary.argtypes = [C.c_char_p, _u64p, _sz, _sz, _sz]
        L.refh_matrix_load_binary.restype = C.c_long
        L.refh_matrix_load_binary.argtypes = [C.c_char_p, _u64p, _u64p, _sz, _sz]
        L.refh_island_run.restype = C.c_long
        L.refh_island_run.argtypes = [_u64p, _sz, _sz, _sz, _szp, _sz, _sz, _sz, _sz, C.c_uint64,
                                      _sz, C.c_uint64, C.c_double, _u64p, C.POINTER(C.c_double)]

    def fwht_i32(self, a):
        a = np.ascontiguousarray(a, dtype=np.int32).copy()
        rc = self.lib.refh_fwht_i32(_ptr(a, _i32p), a.size)
        if rc:
            raise ERRORS.get(rc, OracleError)("reference error")
        return a

    def fwht_i16(self, a):
        a = np.ascontiguousarray(a, dtype=np.int16).copy()
        rc = self.lib.refh_fwht_i16(_ptr(a, _i16p), a.size)
        if rc:
            raise ERRORS.get(rc, OracleError)("reference error")
        return a

    def _call(self, fn, m, cols, win, k, *extra):
        win = self._win(win)
        cap = max(1, min(k, 1 << min(len(win), 24)))
        masks = np.zeros(cap, np.uint64)
        ws = np.zeros(cap, np.uint32)
        c = fn(_ptr(m, _u64p), m.shape[0], cols, m.shape[1], _ptr(win, _szp), len(win), *extra,
               _ptr(masks, _u64p), _ptr(ws, _u32p), cap)
        return self._result(c, masks, ws)

    def fwht_search(self, m, cols, win, max_rows=16, k=64):
        return self._call(self.lib.refh_fwht_search, m, cols, win, k, max_rows, k)

    def mitm_search(self, m, cols, win, k=64):
        return self._call(self.lib.refh_mitm_search, m, cols, win, k, k)

    def bruteforce_search(self, m, cols, win, k=128, chunk_bits=0):
        return self._call(self.lib.refh_bruteforce_search, m, cols, win, k, k, chunk_bits)

    def split_window(self, m, cols, win, low_bits):
        win = self._win(win)
        cap = max(1, cols)
        q = np.zeros(cap, np.uint64)
        r = np.zeros(cap, np.uint64)
        mult = np.zeros(cap, np.int32)
        tw = C.c_int32(0)
        u = self.lib.refh_split_window(_ptr(m, _u64p), m.shape[0], cols, m.shape[1],
                                       _ptr(win, _szp), len(win), low_bits, _ptr(q, _u64p),
                                       _ptr(r, _u64p), _ptr(mult, _i32p), cap, C.byref(tw))
        if u < 0:
            raise ERRORS.get(u, OracleError)(f"reference error {u}")
        return q[:u].tolist(), r[:u].tolist(), mult[:u].tolist(), tw.value

    def target_best_fwht(self, m, cols, target, others):
        others = self._win(others)
        bm = C.c_uint64(0)
        bw = C.c_uint32(0)
        rc = self.lib.refh_target_best_fwht(_ptr(m, _u64p), m.shape[0], cols, m.shape[1], target,
                                            _ptr(others, _szp), len(others), C.byref(bm),
                                            C.byref(bw))
        if rc < 0:
            raise ERRORS.get(rc, OracleError)("reference error")
        return int(bm.value), int(bw.value)

    def ga_run(self, m, cols, win, cfg: GaConfig, seed, max_steps):
        """GeneticAlgorithm: (scores per step, best masks (n, mw), best weights, seconds)."""
        win = self._win(win)
        n = len(win)
        mw = (n + 63) // 64
        scores = np.zeros(max_steps + 1, np.uint64)
        bm = np.zeros((n, mw), np.uint64)
        bw = np.zeros(n, np.uint32)
        secs = C.c_double(0)
        g = self.lib.refh_ga_run(_ptr(m, _u64p), m.shape[0], cols, m.shape[1], _ptr(win, _szp),
                                 n, C.byref(cfg), seed, max_steps, _ptr(scores, _u64p),
                                 _ptr(bm, _u64p), _ptr(bw, _u32p), C.byref(secs))
        if g < 0:
            raise ERRORS.get(g, OracleError)("reference error")
        return scores[: g + 1].tolist(), bm, bw, secs.value

    def apply(self, m, cols, win, masks, weights, global_=False, min_gain=1, stochastic=False,
              seed=0, require_improvement=True):
        """The reference applier on a copy of m: (new words, applied, improvement).
        masks: (n_cand, mw) uint64."""
        win = self._win(win)
        masks = np.ascontiguousarray(masks, dtype=np.uint64)
        masks = masks.reshape(len(weights), -1) if len(weights) else np.zeros((0, 1), np.uint64)
        if masks.shape[1] == 0:
            masks = np.zeros((len(weights), 1), np.uint64)
        ws = np.ascontiguousarray(weights, dtype=np.uint32)
        out = np.zeros_like(m)
        a = C.c_uint64(0)
        imp = C.c_uint64(0)
        rc = self.lib.refh_apply(_ptr(m, _u64p), m.shape[0], cols, m.shape[1], _ptr(win, _szp),
                                 len(win), _ptr(masks, _u64p), masks.shape[1], _ptr(ws, _u32p),
                                 len(ws), int(global_), min_gain, int(stochastic), seed,
                                 int(require_improvement), _ptr(out, _u64p), C.byref(a),
                                 C.byref(imp))
        if rc < 0:
            raise ERRORS.get(rc, OracleError)(f"reference error {rc}")
        return out, int(a.value), int(imp.value)

    def exact_basis(self, m, cols, win, max_rows=24, max_states=(1 << 24) - 1,
                    max_storage_bytes=128 * 1024 * 1024):
        """The reference ExactBasisSolver: dict of the ExactBasisResult fields
        (transform rows as ints, basis_matrix as (rank, stride) words)."""
        win = self._win(win)
        t = len(win)
        sc = np.zeros(5, np.uint64)
        masks = np.zeros(max(t, 1), np.uint32)
        ws = np.zeros(max(t, 1), np.uint32)
        tr = np.zeros(max(t, 1), np.uint64)
        bw = np.zeros((max(t, 1), m.shape[1]), np.uint64)
        r = self.lib.refh_exact_basis(_ptr(m, _u64p), m.shape[0], cols, m.shape[1],
                                      _ptr(win, _szp), t, max_rows, max_states, max_storage_bytes,
                                      _ptr(sc, _u64p), _ptr(masks, _u32p), _ptr(ws, _u32p),
                                      _ptr(tr, _u64p), _ptr(bw, _u64p))
        if r < 0:
            raise ERRORS.get(r, OracleError)(f"reference error {r}")
        return {"input_rows": int(sc[0]), "cols": int(sc[1]), "rank": int(sc[2]),
                "enumerated_states": int(sc[3]), "total_weight": int(sc[4]),
                "basis_masks": [int(x) for x in masks[:r]],
                "basis_weights": [int(x) for x in ws[:r]],
                "transform": [int(x) for x in tr[:r]], "basis_words": bw[:r].copy()}

    def _raise(self, rc):
        msg = self.lib.refh_last_error().decode()
        raise {-5: RuntimeError, -6: MatrixErrorRef}.get(rc, ERRORS.get(rc, OracleError))(msg)

    def matrix_from_text(self, text: bytes):
        """BitMatrix::load_text: (words (rows, stride), rows, cols); raises with
        the reference's message (RuntimeError, or MatrixErrorRef)."""
        dims = np.zeros(2, np.uint64)
        rc = self.lib.refh_matrix_from_text(text, len(text), _ptr(dims, _u64p),
                                            _ptr(np.zeros(1, np.uint64), _u64p), 1, 0)
        if rc < 0:
            self._raise(rc)
        rows, cols = int(dims[0]), int(dims[1])
        stride = max(4, ((cols + 63) // 64 + 3) // 4 * 4)
        out = np.zeros((max(rows, 1), stride), np.uint64)
        rc = self.lib.refh_matrix_from_text(text, len(text), _ptr(dims, _u64p), _ptr(out, _u64p),
                                            stride, out.size)
        return out[:rows], rows, cols

    def matrix_to_text(self, m, cols) -> bytes:
        m = np.ascontiguousarray(m, dtype=np.uint64)
        n = self.lib.refh_matrix_to_text(_ptr(m, _u64p), m.shape[0], cols, m.shape[1], None, 0)
        buf = C.create_string_buffer(max(n, 1))
        self.lib.refh_matrix_to_text(_ptr(m, _u64p), m.shape[0], cols, m.shape[1], buf, n)
        return buf.raw[:n]

    def matrix_hash(self, m, cols) -> str:
        m = np.ascontiguousarray(m, dtype=np.uint64)
        out = C.create_string_buffer(65)
        rc = self.lib.refh_matrix_hash(_ptr(m, _u64p), m.shape[0], cols, m.shape[1], out)
        if rc < 0:
            self._raise(rc)
        return out.value.decode()

    def matrix_save_binary(self, path, m, cols):
        m = np.ascontiguousarray(m, dtype=np.uint64)
        rc = self.lib.refh_matrix_save_binary(os.fsencode(path), _ptr(m, _u64p), m.shape[0], cols,
                                              m.shape[1])
        if rc < 0:
            self._raise(rc)

    def matrix_load_binary(self, path):
        p = os.fsencode(path)
        dims = np.zeros(2, np.uint64)
        rc = self.lib.refh_matrix_load_binary(p, _ptr(dims, _u64p),
                                              _ptr(np.zeros(1, np.uint64), _u64p), 1, 0)
        if rc < 0:
            self._raise(rc)
        rows, cols = int(dims[0]), int(dims[1])
        stride = max(4, ((cols + 63) // 64 + 3) // 4 * 4)
        out = np.zeros((max(rows, 1), stride), np.uint64)
        self.lib.refh_matrix_load_binary(p, _ptr(dims, _u64p), _ptr(out, _u64p), stride, out.size)
        return out[:rows], rows, cols

    def island_run(self, m, cols, win, islands, population, interval, seed, max_gens, target,
                   cap_seconds):
        win = self._win(win)
        best = C.c_uint64(0)
        secs = C.c_double(0)
        rc = self.lib.refh_island_run(_ptr(m, _u64p), m.shape[0], cols, m.shape[1],
                                      _ptr(win, _szp), len(win), islands, population, interval,
                                      seed, max_gens, target, cap_seconds, C.byref(best),
                                      C.byref(secs))
        if rc < 0:
            raise ERRORS.get(rc, OracleError)("reference error")
        return int(best.value), secs.value


_port = None


def port() -> Port:
    global _port
    if _port is None:
        _port = Port()
    return _port


_ref = None


def ref():
    """The reference library, or None where oracle/_ref was not built."""
    global _ref
    if _ref is None and os.path.exists(REF_SO):
        _ref = Ref(C.CDLL(REF_SO))
    return _ref


_ref_scalar = None


def ref_scalar():
    """The reference built without its AVX2 backend, or None."""
    global _ref_scalar
    if _ref_scalar is None and os.path.exists(REF_SCALAR_SO):
        _ref_scalar = Ref(C.CDLL(REF_SCALAR_SO))
    return _ref_scalar


class RefCuda:
    """The reference's GPU searchers (oracle/_ref/cuda/libbmmref_cuda.so):
    CudaBruteforceSearch / CudaMitmFwhtSearch on a window of a packed
    matrix, through the reference's own classes and kernels."""

    def __init__(self, lib):
        self.lib = lib
        for name in ("refc_cuda_bruteforce_search", "refc_cuda_mitm_search"):
            fn = getattr(lib, name)
            fn.restype = C.c_long
            fn.argtypes = [_u64p, _sz, _sz, _sz, _szp, _sz, _sz, _sz, _u64p, _u32p, _sz]
        lib.refc_last_error.restype = C.c_char_p

    def _call(self, fn, m, cols, win, k, extra):
        m = np.ascontiguousarray(m, dtype=np.uint64)
        win = np.ascontiguousarray(win, dtype=np.uintp)
        cap = max(int(k), 1)
        masks = np.zeros(cap, np.uint64)
        weights = np.zeros(cap, np.uint32)
        n = fn(_ptr(m, _u64p), m.shape[0], cols, m.shape[1], _ptr(win, _szp), len(win), k, extra,
               _ptr(masks, _u64p), _ptr(weights, _u32p), cap)
        if n < 0:
            raise ERRORS.get(n, OracleError)(self.lib.refc_last_error().decode())
        n = min(n, cap)
        return list(zip(masks[:n].tolist(), weights[:n].tolist()))

    def cuda_bruteforce_search(self, m, cols, win, k=128, chunk_bits=0):
        return self._call(self.lib.refc_cuda_bruteforce_search, m, cols, win, k, chunk_bits)

    def cuda_mitm_search(self, m, cols, win, k=64, low_bits=0):
        return self._call(self.lib.refc_cuda_mitm_search, m, cols, win, k, low_bits)


_ref_cuda = None


def ref_cuda():
    """The reference's CUDA searchers, or None where they were not built."""
    global _ref_cuda
    if _ref_cuda is None and os.path.exists(REF_CUDA_SO):
        _ref_cuda = RefCuda(C.CDLL(REF_CUDA_SO))
    return _ref_cuda
