"""Runtime queries and the FWHT entry points (python/bindings/runtime.cpp,
python/bindings/math.cpp of the reference)."""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import _native as N


@dataclass
class RuntimeFeatures:
    """bmmpy.RuntimeFeatures (include/bmmpy/stub.hpp:7-17), device side."""

    cuda_compiled: bool = True
    cuda_available: bool = False
    device_count: int = 0
    sm_count: int = 0
    compute_capability: tuple = (0, 0)
    device_name: str = ""
    fwht_backend: str = "cuda-sm100a"
    bit_ops_backend: str = "cuda-sm100a"


def get_runtime_features() -> RuntimeFeatures:
    f = N.Features_t()
    N.check(N.lib().bmm_runtime_features(N.C.byref(f)))
    return RuntimeFeatures(bool(f.cuda_compiled), bool(f.cuda_available), f.device_count,
                           f.sm_count, (f.cc_major, f.cc_minor), f.device_name.decode())


def get_version() -> str:
    return N.lib().bmm_version().decode()


def fwht_i32(data) -> np.ndarray:
    """In-place unnormalised Walsh-Hadamard transform of an int32 array
    (bmmpy.fwht_i32, include/bmmpy/math/fwht.hpp:9); also returns it."""
    a = data if isinstance(data, np.ndarray) and data.dtype == np.int32 and \
        data.flags.c_contiguous else np.ascontiguousarray(data, dtype=np.int32)
    N.check(N.lib().bmm_fwht_i32(N.ptr(a, N._i32p), a.size))
    if a is not data and isinstance(data, np.ndarray) and data.dtype == np.int32:
        data[...] = a
    return a


def fwht_i16(data) -> np.ndarray:
    """int16 variant with wrapping arithmetic (include/bmmpy/math/fwht.hpp:8)."""
    a = data if isinstance(data, np.ndarray) and data.dtype == np.int16 and \
        data.flags.c_contiguous else np.ascontiguousarray(data, dtype=np.int16)
    N.check(N.lib().bmm_fwht_i16(N.ptr(a, N._i16p), a.size))
    if a is not data and isinstance(data, np.ndarray) and data.dtype == np.int16:
        data[...] = a
    return a
