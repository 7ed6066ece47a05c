"""Genetic-algorithm optimizers over a row window, run on the B200.

Mirrors bmmpy.ga (bmmpy/ga.py, python/bindings/ga.cpp): the same class,
attribute and method names and the same argument checks.  The generations run
on the device (bmm_ga_* in include/bmm_b200.h): every island draws from its
own xorshift64 stream in the reference's order, so a GeneticAlgorithm gives
the same trajectory, best individual and best score as bmmpy's for the same
seed.  The IslandModel runs all islands in one set of kernel launches per
generation and exchanges best individuals along a ring (island i imports
island i-1's best whenever i-1's interval divides its generation count);
bmmpy's threads-and-shared-pool channel has no deterministic counterpart, so
``channel_capacity`` and ``overflow_policy`` are validated and kept for
compatibility only.

Limits of the device implementation: windows of at most 256 rows,
populations of at most 1024, 1..4 parents, and islands of one model share
population_size, elite_count, tournament_size, num_parents, num_offspring
and the catastrophe settings (seeds, mutation rates and stop criteria may
differ).
"""

from __future__ import annotations

import ctypes as C
import enum
import threading
from collections.abc import Sequence

import numpy as np

from . import _native as N
from .candidate import Candidate
from .matrix import RowWindow

__all__ = [
    "StopCriteria", "RunStats", "MigrationPolicy", "IslandSpec", "IslandSnapshot",
    "IslandModelSnapshot", "GeneticAlgorithmConfig", "IslandModelConfig", "OverflowPolicy",
    "GeneticAlgorithm", "IslandModel", "ProposalConfig",
]


class OverflowPolicy(enum.Enum):
    DropOldest = 0
    DropNewest = 1
    RejectPublish = 2


class StopCriteria:
    """Stopping rules for the genetic optimizers (ga/types.hpp:13-18)."""

    __slots__ = ("max_generations", "max_stale_generations", "target_total_weight")

    def __init__(self) -> None:
        self.max_generations: int | None = None
        self.max_stale_generations: int | None = None
        self.target_total_weight: int | None = None


class RunStats:
    """Runtime counters collected during a genetic run (ga/types.hpp:20-25)."""

    __slots__ = ("generations", "evaluations", "stale_generations", "seed")

    def __init__(self) -> None:
        self.generations = 0
        self.evaluations = 0
        self.stale_generations = 0
        self.seed = 0


class MigrationPolicy:
    """Per-island migration settings (ga/types.hpp:28-33)."""

    __slots__ = ("interval_generations", "export_count", "import_count", "shared_pool_capacity")

    def __init__(self) -> None:
        self.interval_generations = 32
        self.export_count = 2
        self.import_count = 2
        self.shared_pool_capacity = 128


class IslandSpec:
    """Static configuration for one island in the island model."""

    __slots__ = ("island_id", "migration")

    def __init__(self) -> None:
        self.island_id = 0
        self.migration = MigrationPolicy()


class IslandSnapshot:
    """Per-island runtime snapshot."""

    __slots__ = ("island_id", "running", "stop_requested", "finished", "stats", "best_score",
                 "best_individual")

    def __init__(self) -> None:
        self.island_id = 0
        self.running = False
        self.stop_requested = False
        self.finished = False
        self.stats = RunStats()
        self.best_score = 0
        self.best_individual: list[Candidate] = []


class IslandModelSnapshot:
    """Whole-model runtime snapshot."""

    __slots__ = ("running", "stop_requested", "island_count", "total_generations", "best_score",
                 "best_individual", "islands")

    def __init__(self) -> None:
        self.running = False
        self.stop_requested = False
        self.island_count = 0
        self.total_generations = 0
        self.best_score = 0
        self.best_individual: list[Candidate] = []
        self.islands: list[IslandSnapshot] = []


class GeneticAlgorithmConfig:
    """Low-level GA configuration (genetic_algorithm.hpp:17-29)."""

    __slots__ = ("population_size", "elite_count", "num_parents", "num_offspring",
                 "tournament_size", "enable_catastrophe", "catastrophe_threshold",
                 "catastrophe_survival_rate", "mutation_rate", "stop", "seed")

    def __init__(self) -> None:
        self.population_size = 300
        self.elite_count = 3
        self.num_parents = 2
        self.num_offspring = 1
        self.tournament_size = 3
        self.enable_catastrophe = False
        self.catastrophe_threshold = 30
        self.catastrophe_survival_rate = 0.2
        self.mutation_rate = 0.3
        self.stop = StopCriteria()
        self.seed = 0


class IslandModelConfig:
    """Low-level island-model configuration."""

    __slots__ = ("islands",)

    def __init__(self) -> None:
        self.islands: list[IslandSpec] = []


# ---------------------------------------------------------------------------
def _build_ga_config(*, population_size, elite_count, tournament_size, num_parents,
                     num_offspring, enable_catastrophe, catastrophe_threshold,
                     catastrophe_survival_rate, mutation_rate, max_generations,
                     max_stale_generations, target_total_weight, seed) -> GeneticAlgorithmConfig:
    c = GeneticAlgorithmConfig()
    c.population_size = population_size
    c.elite_count = elite_count
    c.tournament_size = tournament_size
    c.num_parents = num_parents
    c.num_offspring = num_offspring
    c.enable_catastrophe = enable_catastrophe
    c.catastrophe_threshold = catastrophe_threshold
    c.catastrophe_survival_rate = catastrophe_survival_rate
    c.mutation_rate = mutation_rate
    c.stop.max_generations = max_generations
    c.stop.max_stale_generations = max_stale_generations
    c.stop.target_total_weight = target_total_weight
    c.seed = seed
    return c


def _clone_ga_config(config: GeneticAlgorithmConfig) -> GeneticAlgorithmConfig:
    return _build_ga_config(
        population_size=config.population_size, elite_count=config.elite_count,
        tournament_size=config.tournament_size, num_parents=config.num_parents,
        num_offspring=config.num_offspring, enable_catastrophe=config.enable_catastrophe,
        catastrophe_threshold=config.catastrophe_threshold,
        catastrophe_survival_rate=config.catastrophe_survival_rate,
        mutation_rate=config.mutation_rate, max_generations=config.stop.max_generations,
        max_stale_generations=config.stop.max_stale_generations,
        target_total_weight=config.stop.target_total_weight, seed=config.seed)


def _resolve_overflow_policy(policy) -> OverflowPolicy:
    if isinstance(policy, str):
        normalized = policy.strip().lower()
        table = {"drop_oldest": OverflowPolicy.DropOldest,
                 "drop_newest": OverflowPolicy.DropNewest,
                 "reject_publish": OverflowPolicy.RejectPublish}
        if normalized in table:
            return table[normalized]
        raise ValueError(f"Unsupported overflow_policy: {policy!r}")
    if policy not in (OverflowPolicy.DropOldest, OverflowPolicy.DropNewest,
                      OverflowPolicy.RejectPublish):
        raise ValueError(f"Unsupported overflow_policy: {policy!r}")
    return policy


def _native_config(c: GeneticAlgorithmConfig) -> N.GaConfig_t:
    def u32(v, what):
        v = int(v)
        if v < 0:
            raise OverflowError(f"{what} must be non-negative")
        return min(v, 0xFFFFFFFF)

    stop = c.stop
    flags = ((N.GA_STOP_MAX_GENERATIONS if stop.max_generations is not None else 0)
             | (N.GA_STOP_MAX_STALE if stop.max_stale_generations is not None else 0)
             | (N.GA_STOP_TARGET if stop.target_total_weight is not None else 0))
    return N.GaConfig_t(
        u32(c.population_size, "population_size"), u32(c.elite_count, "elite_count"),
        u32(c.num_parents, "num_parents"), u32(c.num_offspring, "num_offspring"),
        u32(c.tournament_size, "tournament_size"), 1 if c.enable_catastrophe else 0,
        u32(c.catastrophe_threshold, "catastrophe_threshold"), flags,
        float(c.catastrophe_survival_rate), float(c.mutation_rate),
        int(stop.max_generations or 0), int(stop.max_stale_generations or 0),
        int(stop.target_total_weight or 0), int(c.seed) & 0xFFFFFFFFFFFFFFFF)


def _individual(masks: np.ndarray, weights: np.ndarray) -> list[Candidate]:
    return [Candidate([int(w) for w in masks[i]], int(weights[i])) for i in range(len(weights))]


class ProposalConfig:
    """Learned proposal step (no bmmpy counterpart; bmm_ga_proposal).

    mode: "off" (the reference GA), "learned" (windows of 16 rows drawn from
    the proposal network's scores, with uniform exploration, exhaustively
    searched and trained on the improving subsets), "uniform" (uniform
    windows only, the ablation without the network) or "ranked" (the 16
    rows whose XOR alone changes the target row's weight least)."""

    __slots__ = ("mode", "queries_per_elite", "train_steps", "learning_rate",
                 "learned_fraction", "seed")

    def __init__(self, mode: str = "off", queries_per_elite: int = 2, train_steps: int = 2,
                 learning_rate: float = 1e-3, learned_fraction: float = 0.5,
                 seed: int = 1) -> None:
        if mode not in ("off", "learned", "uniform", "ranked"):
            raise ValueError(f"Unsupported proposal mode: {mode!r}")
        self.mode = mode
        self.queries_per_elite = queries_per_elite
        self.train_steps = train_steps
        self.learning_rate = learning_rate
        self.learned_fraction = learned_fraction
        self.seed = seed

    def native(self) -> N.GaProposal_t:
        return N.GaProposal_t({"off": 0, "learned": 1, "uniform": 2, "ranked": 3}[self.mode],
                              int(self.queries_per_elite), int(self.train_steps), 0,
                              float(self.learning_rate), float(self.learned_fraction),
                              int(self.seed) & 0xFFFFFFFFFFFFFFFF)


class _Engine:
    """One device run of `islands` islands (the bmm_ga handle)."""

    def __init__(self, window: RowWindow, configs: Sequence[GeneticAlgorithmConfig],
                 migration: Sequence[MigrationPolicy] | None,
                 proposal: ProposalConfig | None = None) -> None:
        m = window.matrix
        self.words = np.ascontiguousarray(m.words)
        self.win = np.ascontiguousarray(window.index_array(), dtype=np.uintp)
        self.n = len(self.win)
        self.mw = (self.n + 63) // 64
        self.islands = len(configs)
        cfgs = (N.GaConfig_t * self.islands)(*[_native_config(c) for c in configs])
        mig = None
        if migration is not None:
            mig = (N.GaMigration_t * self.islands)(
                *[N.GaMigration_t(min(int(p.interval_generations), 0xFFFFFFFF),
                                  min(int(p.import_count), 0xFFFFFFFF)) for p in migration])
        h = C.c_void_p()
        N.check(N.lib().bmm_ga_create(N.u64p(self.words), m.stride_words, m.cols,
                                      N.szp(self.win), self.n, cfgs, self.islands, mig,
                                      C.byref(h)))
        self.h = h
        self.lock = threading.Lock()
        if proposal is not None and proposal.mode != "off":
            cfg = proposal.native()
            N.check(N.lib().bmm_ga_set_proposal(self.h, C.byref(cfg)))

    def proposal_stats(self) -> dict:
        out = N.GaProposalStats_t()
        with self.lock:
            N.check(N.lib().bmm_ga_get_proposal_stats(self.h, C.byref(out)))
        return {k: getattr(out, k) for k, _ in out._fields_}

    def run(self, generations: int, check_every: int = 1) -> tuple[int, bool]:
        ran = C.c_uint64(0)
        done = C.c_int(0)
        with self.lock:
            N.check(N.lib().bmm_ga_run(self.h, int(generations), int(check_every),
                                       C.byref(ran), C.byref(done)))
        return int(ran.value), bool(done.value)

    def stats(self, island: int) -> N.GaStats_t:
        out = N.GaStats_t()
        with self.lock:
            N.check(N.lib().bmm_ga_stats(self.h, island, C.byref(out)))
        return out

    def best(self, island: int | None = None) -> tuple[list[Candidate], int]:
        masks = np.zeros((self.n, self.mw), np.uint64)
        weights = np.zeros(self.n, np.uint32)
        score = C.c_uint64(0)
        idx = C.c_size_t(-1).value if island is None else island
        with self.lock:
            N.check(N.lib().bmm_ga_best(self.h, idx, N.u64p(masks), N.u32p(weights),
                                        C.byref(score)))
        return _individual(masks, weights), int(score.value)

    def population(self, island: int, population_size: int):
        masks = np.zeros((population_size, self.n, self.mw), np.uint64)
        weights = np.zeros((population_size, self.n), np.uint32)
        fit = np.zeros(population_size, np.uint64)
        with self.lock:
            N.check(N.lib().bmm_ga_population(self.h, island, N.u64p(masks), N.u32p(weights),
                                              N.u64p(fit)))
        return masks, weights, fit

    def close(self) -> None:
        if getattr(self, "h", None) is not None and self.h.value:
            N.lib().bmm_ga_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _check_window(window: RowWindow) -> None:
    if len(window) == 0 or window.cols == 0:
        raise ValueError("GeneticAlgorithm::initialize: empty window is not supported")


# ---------------------------------------------------------------------------
class GeneticAlgorithm:
    """Genetic optimizer over a row window.

    The returned value is a full list of Candidate objects with length equal
    to the window size; each describes one output row of the found transform.
    """

    __slots__ = ("population_size", "elite_count", "tournament_size", "num_parents",
                 "num_offspring", "enable_catastrophe", "catastrophe_threshold",
                 "catastrophe_survival_rate", "mutation_rate", "max_generations",
                 "max_stale_generations", "target_total_weight", "seed", "_engine", "_done",
                 "proposal")

    def __init__(self, *, population_size: int = 300, elite_count: int = 3,
                 tournament_size: int = 3, num_parents: int = 2, num_offspring: int = 1,
                 enable_catastrophe: bool = False, catastrophe_threshold: int = 30,
                 catastrophe_survival_rate: float = 0.2, mutation_rate: float = 0.3,
                 max_generations: int | None = None, max_stale_generations: int | None = None,
                 target_total_weight: int | None = None, seed: int = 0,
                 proposal: ProposalConfig | None = None) -> None:
        self.population_size = population_size
        self.elite_count = elite_count
        self.tournament_size = tournament_size
        self.num_parents = num_parents
        self.num_offspring = num_offspring
        self.enable_catastrophe = enable_catastrophe
        self.catastrophe_threshold = catastrophe_threshold
        self.catastrophe_survival_rate = catastrophe_survival_rate
        self.mutation_rate = mutation_rate
        self.max_generations = max_generations
        self.max_stale_generations = max_stale_generations
        self.target_total_weight = target_total_weight
        self.seed = seed
        self.proposal = proposal
        self._engine: _Engine | None = None
        self._done = False

    def __repr__(self) -> str:
        return (f"GeneticAlgorithm(population_size={self.population_size}, "
                f"elite_count={self.elite_count}, tournament_size={self.tournament_size}, "
                f"num_parents={self.num_parents}, num_offspring={self.num_offspring}, "
                f"enable_catastrophe={self.enable_catastrophe}, "
                f"catastrophe_threshold={self.catastrophe_threshold}, "
                f"catastrophe_survival_rate={self.catastrophe_survival_rate}, "
                f"mutation_rate={self.mutation_rate}, max_generations={self.max_generations}, "
                f"max_stale_generations={self.max_stale_generations}, "
                f"target_total_weight={self.target_total_weight}, seed={self.seed})")

    def _config(self) -> GeneticAlgorithmConfig:
        return _build_ga_config(
            population_size=self.population_size, elite_count=self.elite_count,
            tournament_size=self.tournament_size, num_parents=self.num_parents,
            num_offspring=self.num_offspring, enable_catastrophe=self.enable_catastrophe,
            catastrophe_threshold=self.catastrophe_threshold,
            catastrophe_survival_rate=self.catastrophe_survival_rate,
            mutation_rate=self.mutation_rate, max_generations=self.max_generations,
            max_stale_generations=self.max_stale_generations,
            target_total_weight=self.target_total_weight, seed=self.seed)

    def name(self) -> str:
        return "ga"

    def initialize(self, window: RowWindow) -> None:
        _check_window(window)
        if self.population_size == 0:
            raise ValueError(
                "GeneticAlgorithm::initialize: population_size must be greater than zero")
        if self._engine is not None:
            self._engine.close()
        self._engine = _Engine(window, [self._config()], None, self.proposal)
        self._done = bool(self._engine.stats(0).done)

    def step(self) -> None:
        if self._engine is None or self._done:
            return
        _, self._done = self._engine.run(1)

    def done(self) -> bool:
        return self._done

    def generation(self) -> int:
        return int(self._engine.stats(0).generations) if self._engine else 0

    def best_individual(self) -> list[Candidate]:
        if self._engine is None:
            return []
        return self._engine.best(0)[0]

    def stats(self) -> RunStats:
        out = RunStats()
        out.seed = self.seed
        if self._engine is not None:
            s = self._engine.stats(0)
            out.generations = int(s.generations)
            out.evaluations = int(s.evaluations)
            out.stale_generations = int(s.stale_generations)
        return out

    def best_score(self) -> int:
        return int(self._engine.stats(0).best_score) if self._engine else 0

    def population(self) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
        """The current population in order: masks (P, n, ceil(n/64)), weights
        (P, n), fitness (P,).  No reference counterpart (inspection aid)."""
        return self._engine.population(0, self.population_size)

    def optimize(self, window: RowWindow) -> list[Candidate]:
        self.initialize(window)
        while not self._done:
            _, self._done = self._engine.run(1 << 62, check_every=8)
        return self.best_individual()


class IslandModel:
    """Island-model wrapper around GeneticAlgorithm.

    By default one GA configuration per island is built from the common keyword
    arguments (island i seeded with seed + i * seed_stride); for heterogeneous
    islands pass ga_configs with one GeneticAlgorithmConfig per IslandSpec.
    """

    __slots__ = ("island_count", "channel_capacity", "overflow_policy", "_specs", "_configs",
                 "_engine", "_thread", "_running", "_stop", "_error", "_initialized",
                 "_proposal")

    def __init__(self, *, islands: Sequence[IslandSpec],
                 ga_configs: Sequence[GeneticAlgorithmConfig] | None = None,
                 population_size: int = 300, elite_count: int = 3, tournament_size: int = 3,
                 num_parents: int = 2, num_offspring: int = 1, enable_catastrophe: bool = False,
                 catastrophe_threshold: int = 30, catastrophe_survival_rate: float = 0.2,
                 mutation_rate: float = 0.3, max_generations: int | None = None,
                 max_stale_generations: int | None = None,
                 target_total_weight: int | None = None, seed: int = 0, seed_stride: int = 1,
                 channel_capacity: int = 256, overflow_policy="drop_oldest",
                 proposal: ProposalConfig | None = None) -> None:
        island_list = list(islands)
        if not island_list:
            raise ValueError("IslandModel requires at least one island")
        if channel_capacity <= 0:
            raise ValueError("channel_capacity must be greater than zero")
        if seed_stride < 0:
            raise ValueError("seed_stride must be non-negative")
        ids = [s.island_id for s in island_list]
        if len(set(ids)) != len(ids):
            raise ValueError("IslandModel: island_id values must be unique")
        common = dict(population_size=population_size, elite_count=elite_count,
                      tournament_size=tournament_size, num_parents=num_parents,
                      num_offspring=num_offspring, enable_catastrophe=enable_catastrophe,
                      catastrophe_threshold=catastrophe_threshold,
                      catastrophe_survival_rate=catastrophe_survival_rate,
                      mutation_rate=mutation_rate, max_generations=max_generations,
                      max_stale_generations=max_stale_generations,
                      target_total_weight=target_total_weight)
        if ga_configs is not None:
            if len(ga_configs) != len(island_list):
                raise ValueError("ga_configs length must match the number of islands")
            defaults = dict(population_size=300, elite_count=3, tournament_size=3,
                            num_parents=2, num_offspring=1, enable_catastrophe=False,
                            catastrophe_threshold=30, catastrophe_survival_rate=0.2,
                            mutation_rate=0.3, max_generations=None,
                            max_stale_generations=None, target_total_weight=None)
            if common != defaults or seed != 0 or seed_stride != 1:
                raise ValueError(
                    "Pass either ga_configs or common GA keyword arguments, not both")
            configs = [_clone_ga_config(c) for c in ga_configs]
        else:
            configs = [_build_ga_config(**common, seed=seed + i * seed_stride)
                       for i in range(len(island_list))]
        self.island_count = len(island_list)
        self.channel_capacity = channel_capacity
        self.overflow_policy = _resolve_overflow_policy(overflow_policy)
        self._specs = island_list
        self._configs = configs
        self._engine: _Engine | None = None
        self._thread: threading.Thread | None = None
        self._running = False
        self._stop = threading.Event()
        self._error: BaseException | None = None
        self._initialized = False
        self._proposal = proposal

    def __repr__(self) -> str:
        return (f"IslandModel(island_count={self.island_count}, "
                f"channel_capacity={self.channel_capacity}, "
                f"overflow_policy={self.overflow_policy})")

    def name(self) -> str:
        return "island_model"

    def initialize(self, window: RowWindow) -> None:
        if self._running:
            raise RuntimeError("IslandModel::initialize: model is already running")
        _check_window(window)
        if self._engine is not None:
            self._engine.close()
        self._engine = _Engine(window, self._configs, [s.migration for s in self._specs],
                               self._proposal)
        self._stop.clear()
        self._initialized = True

    def _loop(self) -> None:
        try:
            while not self._stop.is_set():
                _, done = self._engine.run(8, check_every=8)
                if done:
                    break
        except BaseException as e:  # surfaced by wait()
            self._error = e

    def start(self) -> None:
        if not self._initialized:
            raise RuntimeError("IslandModel::start: model must be initialized first")
        if self._running:
            raise RuntimeError("IslandModel::start: model is already running")
        self._stop.clear()
        self._error = None
        self._running = True
        self._thread = threading.Thread(target=self._loop, daemon=True)
        self._thread.start()

    def request_stop(self) -> None:
        self._stop.set()

    def wait(self) -> None:
        if self._thread is not None:
            self._thread.join()
            self._thread = None
        self._running = False
        if self._error is not None:
            err, self._error = self._error, None
            raise err

    def running(self) -> bool:
        return self._running and self._thread is not None and self._thread.is_alive()

    def stop_requested(self) -> bool:
        return self._stop.is_set()

    def best_individual(self) -> list[Candidate]:
        if self._engine is None:
            return []
        return self._engine.best(None)[0]

    def snapshot(self) -> IslandModelSnapshot:
        snap = IslandModelSnapshot()
        snap.running = self.running()
        snap.stop_requested = self.stop_requested()
        snap.island_count = self.island_count
        if self._engine is None:
            return snap
        best = None
        for i, spec in enumerate(self._specs):
            s = self._engine.stats(i)
            isl = IslandSnapshot()
            isl.island_id = spec.island_id
            isl.running = snap.running and not s.done
            isl.stop_requested = snap.stop_requested
            isl.finished = bool(s.done) or (self._initialized and not snap.running
                                            and self._thread is None and snap.stop_requested)
            isl.stats.generations = int(s.generations)
            isl.stats.evaluations = int(s.evaluations)
            isl.stats.stale_generations = int(s.stale_generations)
            isl.stats.seed = int(s.seed)
            isl.best_score = int(s.best_score)
            isl.best_individual = self._engine.best(i)[0]
            snap.total_generations += isl.stats.generations
            if best is None or isl.best_score < best:
                best = isl.best_score
                snap.best_individual = isl.best_individual
            snap.islands.append(isl)
        snap.best_score = best if best is not None else 0
        return snap

    def proposal_stats(self) -> dict:
        """Counters of the learned proposal step (no bmmpy counterpart)."""
        return self._engine.proposal_stats() if self._engine else {}

    def run_to_completion(self, window: RowWindow) -> list[Candidate]:
        self.initialize(window)
        self.start()
        self.wait()
        return self.best_individual()
