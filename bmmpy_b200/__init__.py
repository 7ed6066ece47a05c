"""bmmpy_b200: B200-native (sm_100a) weight-minimisation hot path of bmmpy.

Same public names as bmmpy for the search / FWHT path: build a BitMatrix,
take a RowWindow, run a searcher, get Candidates ordered by (weight, mask).
Every search runs on the GPU through libbmm_b200.so; there is no CPU
fallback (importing the package works without a GPU, calling a search
does not).
"""

from __future__ import annotations

from .candidate import Candidate
from .matrix import BitMatrix, RowWindow, matrix_from_rows
from .runtime import RuntimeFeatures, fwht_i16, fwht_i32, get_runtime_features, get_version
from .search import (
    BruteforceSearch,
    CudaBruteforceSearch,
    CudaMitmFwhtSearch,
    FwhtSearch,
    MitmFwhtSearch,
)

__all__ = [
    "BitMatrix",
    "BruteforceSearch",
    "Candidate",
    "CudaBruteforceSearch",
    "CudaMitmFwhtSearch",
    "FwhtSearch",
    "MitmFwhtSearch",
    "RowWindow",
    "RuntimeFeatures",
    "fwht_i16",
    "fwht_i32",
    "get_runtime_features",
    "get_version",
    "matrix_from_rows",
]
