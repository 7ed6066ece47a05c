"""bmmpy_b200: B200-native (sm_100a) weight-minimisation hot path of bmmpy.

Same public names as bmmpy for the search / FWHT path: build a BitMatrix,
take a RowWindow, run a searcher, get Candidates ordered by (weight, mask).
The genetic optimizers (GeneticAlgorithm, IslandModel) run whole generations
on the device.  Every search runs on the GPU through libbmm_b200.so; there is no CPU
fallback (importing the package works without a GPU, calling a search
does not).
"""

from __future__ import annotations

from . import ga, solver
from .apply import ApplyResult, GlobalGreedyApplier, GreedyApplier
from .candidate import Candidate
from .ga import (
    GeneticAlgorithm,
    IslandModel,
    IslandModelSnapshot,
    IslandSnapshot,
    IslandSpec,
    MigrationPolicy,
    OverflowPolicy,
    RunStats,
    StopCriteria,
)
from .matrix import BitMatrix, MatrixError, RowWindow, matrix_from_rows
from .runtime import RuntimeFeatures, fwht_i16, fwht_i32, get_runtime_features, get_version
from .search import (
    BruteforceSearch,
    CudaBruteforceSearch,
    CudaMitmFwhtSearch,
    FwhtSearch,
    MitmFwhtSearch,
    SASelectionResult,
    SASelector,
)

from .workflows import DeviceMatrix, search_apply

__all__ = [
    "ApplyResult",
    "BitMatrix",
    "BruteforceSearch",
    "Candidate",
    "CudaBruteforceSearch",
    "CudaMitmFwhtSearch",
    "FwhtSearch",
    "GeneticAlgorithm",
    "GlobalGreedyApplier",
    "GreedyApplier",
    "IslandModel",
    "IslandModelSnapshot",
    "IslandSnapshot",
    "IslandSpec",
    "MigrationPolicy",
    "MitmFwhtSearch",
    "OverflowPolicy",
    "RunStats",
    "StopCriteria",
    "RowWindow",
    "SASelectionResult",
    "SASelector",
    "RuntimeFeatures",
    "fwht_i16",
    "fwht_i32",
    "get_runtime_features",
    "get_version",
    "MatrixError",
    "matrix_from_rows",
    "solver",
    "search_apply",
    "DeviceMatrix",
]
