"""ctypes binding of the in-tree CUDA library ``libbmm_b200.so``.

There is no CPU fallback: if the library is missing, every call raises.  Status
codes map to the exception classes the reference's bindings raise for the
corresponding C++ exceptions (std::invalid_argument -> ValueError,
std::overflow_error -> OverflowError, std::runtime_error -> RuntimeError).
"""

from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libbmm_b200.so")

OK, EINVAL, EOVERFLOW, ECUDA, ENODEV, ETIMEOUT, ENOMEM, ERUNTIME, EMATRIX = (
    0, -1, -2, -3, -4, -5, -6, -7, -8)


class Candidate_t(C.Structure):
    _fields_ = [("mask", C.c_uint64), ("weight", C.c_uint32), ("reserved", C.c_uint32)]


class Features_t(C.Structure):
    _fields_ = [("cuda_compiled", C.c_int), ("cuda_available", C.c_int),
                ("device_count", C.c_int), ("sm_count", C.c_int), ("cc_major", C.c_int),
                ("cc_minor", C.c_int), ("device_name", C.c_char * 64)]


CAND_DTYPE = np.dtype([("mask", np.uint64), ("weight", np.uint32), ("reserved", np.uint32)])

_u64p = C.POINTER(C.c_uint64)
_u32p = C.POINTER(C.c_uint32)
_i32p = C.POINTER(C.c_int32)
_i16p = C.POINTER(C.c_int16)
_sz = C.c_size_t
_szp = C.POINTER(C.c_size_t)
_vp = C.c_void_p
_candp = C.POINTER(Candidate_t)
_f32p = C.POINTER(C.c_float)


class Instance_t(C.Structure):
    _fields_ = [("word_offset", C.c_uint64), ("rows", C.c_uint32), ("cols", C.c_uint32),
                ("stride", C.c_uint32), ("k", C.c_uint32), ("out_offset", C.c_uint64)]


INSTANCE_DTYPE = np.dtype([("word_offset", np.uint64), ("rows", np.uint32), ("cols", np.uint32),
                           ("stride", np.uint32), ("k", np.uint32), ("out_offset", np.uint64)])
_instp = C.POINTER(Instance_t)

GA_STOP_MAX_GENERATIONS, GA_STOP_MAX_STALE, GA_STOP_TARGET = 1, 2, 4


class GaConfig_t(C.Structure):
    """bmm_ga_config (GeneticAlgorithmConfig)."""

    _fields_ = [("population_size", C.c_uint32), ("elite_count", C.c_uint32),
                ("num_parents", C.c_uint32), ("num_offspring", C.c_uint32),
                ("tournament_size", C.c_uint32), ("enable_catastrophe", C.c_uint32),
                ("catastrophe_threshold", C.c_uint32), ("flags", C.c_uint32),
                ("catastrophe_survival_rate", C.c_double), ("mutation_rate", C.c_double),
                ("max_generations", C.c_uint64), ("max_stale_generations", C.c_uint64),
                ("target_total_weight", C.c_uint64), ("seed", C.c_uint64)]


class GaProposal_t(C.Structure):
    """bmm_ga_proposal."""

    _fields_ = [("mode", C.c_uint32), ("queries_per_elite", C.c_uint32),
                ("train_steps", C.c_uint32), ("reserved", C.c_uint32),
                ("learning_rate", C.c_float), ("learned_fraction", C.c_float),
                ("seed", C.c_uint64)]


class GaProposalStats_t(C.Structure):
    """bmm_ga_proposal_stats."""

    _fields_ = [("tried_learned", C.c_uint64), ("improved_learned", C.c_uint64),
                ("tried_uniform", C.c_uint64), ("improved_uniform", C.c_uint64),
                ("examples", C.c_uint64), ("last_loss", C.c_float),
                ("learned_fraction", C.c_float), ("paired_generations", C.c_uint64),
                ("paired_rate_learned", C.c_double), ("paired_rate_uniform", C.c_double)]


class GaMigration_t(C.Structure):
    """bmm_ga_migration (MigrationPolicy subset)."""

    _fields_ = [("interval_generations", C.c_uint32), ("import_count", C.c_uint32)]


class GaStats_t(C.Structure):
    """bmm_ga_island_stats (RunStats plus the island's best score)."""

    _fields_ = [("generations", C.c_uint64), ("evaluations", C.c_uint64),
                ("stale_generations", C.c_uint64), ("seed", C.c_uint64),
                ("best_score", C.c_uint64), ("done", C.c_uint32),
                ("no_improvement", C.c_uint32), ("mutation_rate", C.c_double)]

class ExactBasisConfig_t(C.Structure):
    """bmm_exact_basis_config (ExactBasisSolverConfig)."""

    _fields_ = [("max_rows", C.c_size_t), ("max_states", C.c_uint64),
                ("max_storage_bytes", C.c_size_t)]


class ExactBasisResult_t(C.Structure):
    """bmm_exact_basis_result (ExactBasisResult without its matrices)."""

    _fields_ = [("input_rows", C.c_size_t), ("cols", C.c_size_t), ("rank", C.c_size_t),
                ("enumerated_states", C.c_uint64), ("total_weight", C.c_uint64)]


class SaConfig_t(C.Structure):
    """bmm_sa_config (SASelectorConfig)."""

    _fields_ = [("iterations", C.c_uint64), ("restarts", C.c_uint64), ("seed", C.c_uint64),
                ("score_policy", C.c_uint32), ("cooling_policy", C.c_uint32),
                ("temperature_probe_samples", C.c_uint64),
                ("initial_acceptance_probability", C.c_double), ("cooling_rate", C.c_double),
                ("min_temperature", C.c_double)]


class SaResult_t(C.Structure):
    """bmm_sa_result (SASelectionResult without its rows)."""

    _fields_ = [("score", C.c_int64), ("accepted_moves", C.c_uint64),
                ("iterations_run", C.c_uint64), ("best_iteration", C.c_uint64),
                ("restart_index", C.c_uint64), ("seed", C.c_uint64), ("n_rows", C.c_size_t)]


class SweepConfig_t(C.Structure):
    """bmm_sweep_config."""

    _fields_ = [("max_candidates", C.c_uint64), ("applier", C.c_uint32),
                ("stochastic", C.c_uint32), ("min_gain", C.c_uint64), ("seed", C.c_uint64),
                ("require_improvement", C.c_uint32), ("reserved", C.c_uint32)]


class ApplyResult_t(C.Structure):
    """bmm_apply_result."""

    _fields_ = [("applied_count", C.c_uint64), ("weight_improvement", C.c_uint64)]


# name -> argtypes (all return int unless listed in _RESTYPES)
SIGNATURES = {
    "bmm_gen_instance": [_u64p, _sz, _sz, _sz, C.c_double, C.c_uint64, _sz],
    "bmm_probe_xor_popc": [C.POINTER(C.c_double)],
    "bmm_gray_tune": [C.c_int, C.c_int],
    "bmm_gray_tune_lanes": [C.c_int],
    "bmm_spectrum_tune": [C.c_int],
    "bmm_spectrum_tune_last_pass": [C.c_int],
    "bmm_spectrum_tune_passes": [C.c_int],
    "bmm_gray_tune_shape": [_sz, _sz, C.c_int, C.c_int, C.c_int],
    "bmm_spectrum_tune_shape": [_sz, C.c_int],
    "bmm_tune_reset": [],
    "bmm_spectrum_low_bits": [_sz],
    "bmm_spectrum_topk_slices_dev": [_vp, _sz, _sz, _sz, _sz, C.c_int, C.c_int64, C.c_int64, _vp,
                                     _vp],
    "bmm_split_window_dev": [_vp, _sz, _sz, _sz, _sz, _vp, _vp, _vp, _sz, _szp,
                             C.POINTER(C.c_int32), _vp],
    "bmm_last_error": [],
    "bmm_version": [],
    "bmm_runtime_features": [C.POINTER(Features_t)],
    "bmm_fwht_i32": [_i32p, _sz],
    "bmm_fwht_i16": [_i16p, _sz],
    "bmm_fwht_i32_dev": [_vp, _sz, _vp],
    "bmm_fwht_search": [_u64p, _sz, _sz, _u32p, _sz, _sz, _sz, _candp, _szp],
    "bmm_mitm_search": [_u64p, _sz, _sz, _u32p, _sz, _sz, _sz, _candp, _szp],
    "bmm_gray_search": [_u64p, _sz, _sz, _u32p, _sz, _sz, _sz, _candp, _szp],
    "bmm_gray_targets": [_u64p, _sz, _sz, _sz, _u32p, _u32p, _sz, _sz, C.c_int, _u64p, _u32p],
    "bmm_gray_targets_dev": [_vp, _sz, _sz, _sz, _vp, _vp, _sz, _sz, C.c_int, _vp, _vp, _vp],
    "bmm_gray_targets_noalloc": [_vp, _sz, _sz, _sz, _vp, _vp, _sz, _sz, C.c_int, _vp, _vp, _vp],
    "bmm_batch_create": [_vp, _sz, C.POINTER(_vp)],
    "bmm_batch_info": [_vp, C.POINTER(C.c_longlong), _szp, C.POINTER(C.c_int)],
    "bmm_batch_run": [_vp, _vp, _vp, _vp, _vp],
    "bmm_batch_destroy": [_vp],
    "bmm_batch_targets": [_u64p, _sz, _vp, _sz, _u64p, _u32p],
    "bmm_batch_policy": [C.c_int, C.c_int],
    "bmm_fwht_targets": [_u64p, _sz, _sz, _sz, _u32p, _u32p, _sz, _sz, _u64p, _u32p],
    "bmm_fwht_targets_dev": [_vp, _sz, _sz, _sz, _vp, _vp, _sz, _sz, _vp, _vp, _vp],
    "bmm_ga_create": [_u64p, _sz, _sz, _szp, _sz, C.POINTER(GaConfig_t), _sz,
                      C.POINTER(GaMigration_t), C.POINTER(_vp)],
    "bmm_ga_run": [_vp, C.c_uint64, C.c_uint32, _u64p, C.POINTER(C.c_int)],
    "bmm_ga_stats": [_vp, _sz, C.POINTER(GaStats_t)],
    "bmm_ga_best": [_vp, _sz, _u64p, _u32p, _u64p],
    "bmm_ga_population": [_vp, _sz, _u64p, _u32p, _u64p],
    "bmm_ga_destroy": [_vp],
    "bmm_ga_set_proposal": [_vp, C.POINTER(GaProposal_t)],
    "bmm_ga_get_proposal_stats": [_vp, C.POINTER(GaProposalStats_t)],
    "bmm_ga_eval": [_u64p, _sz, _sz, _szp, _sz, _u64p, _sz, _u32p],
    "bmm_ga_mutate": [_u64p, _sz, _sz, _szp, _sz, _u64p, _u32p, C.c_double, _u64p],
    "bmm_ga_local_improve": [_u64p, _sz, _sz, _szp, _sz, _u64p, _u32p],
    "bmm_ga_crossover": [_sz, _sz, _u64p, _u32p, _u64p, _u32p],
    "bmm_mlp_create": [C.c_uint64, C.c_float, C.POINTER(_vp)],
    "bmm_mlp_destroy": [_vp],
    "bmm_mlp_param_count": [],
    "bmm_mlp_get_params": [_vp, _f32p],
    "bmm_mlp_set_params": [_vp, _f32p],
    "bmm_mlp_forward": [_vp, _f32p, _sz, _f32p],
    "bmm_mlp_grads": [_vp, _f32p, _f32p, _sz, _f32p, _f32p],
    "bmm_mlp_train": [_vp, _f32p, _f32p, _sz, C.c_int, _f32p],
    "bmm_mlp_gemm": [_f32p, _f32p, C.c_int, C.c_int, C.c_int, _f32p],
    "bmm_mlp_create_on_stream": [C.c_uint64, C.c_float, _vp, C.POINTER(_vp)],
    "bmm_mlp_forward_dev": [_vp, _vp, _sz, _vp],
    "bmm_mlp_train_dev": [_vp, _vp, _vp, _sz, C.c_int],
    "bmm_mlp_forward_bf16_dev": [_vp, _vp, _sz, _vp],
    "bmm_mlp_tune": [C.c_int],
    "bmm_exact_basis": [_u64p, _sz, _sz, _u32p, _sz, C.POINTER(ExactBasisConfig_t),
                        C.POINTER(ExactBasisResult_t), _u32p, _u32p],
    "bmm_basis_weight_counts": [_u64p, _sz, _sz, _u32p, _sz, _u64p],
    "bmm_basis_weight_counts_dev": [_vp, _sz, _sz, _vp, _vp],
    "bmm_basis_tune": [C.c_int],
    "bmm_sa_select": [_u64p, _sz, _sz, _sz, _sz, C.POINTER(SaConfig_t), C.POINTER(SaResult_t),
                      _szp],
    "bmm_sa_pairwise_table": [_u64p, _sz, _sz, _sz, _u32p],
    "bmm_matrix_text_header": [C.c_char_p, _sz, _u64p, _u64p],
    "bmm_matrix_from_text": [C.c_char_p, _sz, _u64p, _sz, _sz, _sz],
    "bmm_matrix_from_text_dev": [_vp, _sz, _vp, _sz, _sz, _sz, _vp],
    "bmm_matrix_text_size": [_sz, _sz, _szp],
    "bmm_matrix_to_text": [_u64p, _sz, _sz, _sz, C.c_char_p, _sz, _szp],
    "bmm_matrix_save_binary": [C.c_char_p, _u64p, _sz, _sz, _sz],
    "bmm_matrix_binary_header": [C.c_char_p, _u64p, _u64p],
    "bmm_matrix_load_binary": [C.c_char_p, _u64p, _sz, _sz, _sz],
    "bmm_matrix_load_binary_dev": [C.c_char_p, _vp, _sz, _sz, _sz, _vp],
    "bmm_matrix_hash": [_u64p, _sz, _sz, _sz, C.c_char_p],
    "bmm_search_apply_dev": [_vp, _sz, _sz, _sz, _u32p, _sz, _sz, C.POINTER(SweepConfig_t),
                             C.POINTER(ApplyResult_t), _u64p, _vp],
    "bmm_sa_pairwise_table_dev": [_vp, _sz, _sz, _sz, _vp, _vp],
}
_RESTYPES = {"bmm_last_error": C.c_char_p, "bmm_version": C.c_char_p,
             "bmm_gen_instance": C.c_uint64, "bmm_mlp_param_count": C.c_size_t}

_lib = None


def lib():
    """Load libbmm_b200.so (raises ImportError when it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m bmmpy_b200.build`; "
                "bmmpy_b200 has no CPU fallback")
        L = C.CDLL(LIB_PATH)
        for name, args in SIGNATURES.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = _RESTYPES.get(name, C.c_int)
        _lib = L
    return _lib


def has(name: str) -> bool:
    return hasattr(lib(), name)


def last_error() -> str:
    msg = lib().bmm_last_error()
    return msg.decode() if msg else ""


def check(rc: int, what: str = "") -> None:
    if rc == OK:
        return
    msg = last_error() or what
    if rc == EINVAL:
        raise ValueError(msg)
    if rc == EOVERFLOW:
        raise OverflowError(msg)
    if rc == ENOMEM:
        raise MemoryError(msg)
    if rc == EMATRIX:
        from .matrix import MatrixError

        raise MatrixError(msg)
    if rc == ERUNTIME:
        raise RuntimeError(msg)
    raise RuntimeError(f"{msg} (status {rc})")


def ptr(a: np.ndarray, typ):
    return a.ctypes.data_as(typ)


def u64p(a):
    return ptr(a, _u64p)


def u32p(a):
    return ptr(a, _u32p)


def f32p(a):
    return ptr(a, _f32p)


def szp(a):
    return ptr(a, _szp)


def candp(a):
    return a.ctypes.data_as(_candp)
