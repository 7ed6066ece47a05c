"""Benchmark: Gray-code per-target search, 40 x 4096 matrix, 24 others per target.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Workload (the Gray-code brute-force configuration): a 40 x 4096 Bernoulli(0.3)
matrix (xorshift64 seed 1, packed as 64 uint64 words per row); for every
target row i, all 2^24 XOR combinations of rows i+1..i+24 (mod 40) are
enumerated in reflected-Gray order and the minimum popcount(row_i ^ XOR) and
its subset are returned (ties: smallest subset mask, the reference order).
One step = all 40 targets = 40 * 2^24 = 671,088,640 row-combos.

* ``value``: combos/s with the matrix resident in HBM, CUDA-event timed on the
  launching stream; L2 is flushed (256 MB write) before every timed step.
* ``e2e``: the same metric through the public host API
  (bmmpy_b200.targets.gray_targets) from pinned host buffers: H2D of the
  matrix and index lists and D2H of the results inside the timed region.
* ``roofline``: the dominant kernel (gray_targets_kernel) is bound by the
  ALU and XU integer pipes (LOP3 XOR / carry-save adders and POPC), not by
  HBM (its rows live in shared memory) nor by tensor cores; the peak is the
  pipe bound of its instruction mix (counted by ncu) at the sampled SM clock.
* The timed result is asserted equal to the reference's per-target answers
  (tests/golden/workloads.npz) before the line is printed.
* ``cpu_baseline``: the reference's BruteforceSearch (oracle/_ref, OpenMP on
  all host threads) on the 25-row window [i, others] for a bounded sample of
  targets; falls back to the oracle's C port when oracle/_ref is absent.

Multi-GPU: one process per GPU (torchrun); rank r runs the same workload on
its own instance (seed 1 + r), no collective on the data path ("weak").
``--impl reference`` times the reference CPU implementation instead (rank 0
only).  ``--impl reference-gpu`` times the reference's own CUDA searchers
(CudaBruteforceSearch on the same 25-row windows, CudaMitmFwhtSearch on an
int16-safe 32-row window) built for sm_100a, next to this library's classes of
the same names on the same windows, and checks the results are equal.

``--workload basis`` (1 GPU) measures ExactBasisSolver on ten 24-row windows
of the planted 256 x 8192 matrix: ``value`` from the device histogram pass on
resident rows, ``e2e`` from the public solve() on host windows.

``--workload sa`` (1 GPU) measures SASelector (pairwise synergy, defaults) on
the planted 512 x 65536 matrix: ``value`` from the device synergy table,
``e2e`` from select().

``--workload io`` (1 GPU) measures matrix IO on the same matrix: the text
payload parsed on the device, BitMatrix.from_text and a binary file loaded
into device memory end to end.

``--workload c1`` / ``--workload batch`` (1 GPU) measure the per-target
transform on the 64 x 256 matrix (16 others per target) and on the 4096 uneven
planted instances in one persistent launch, checked against the reference's
answers, with an ALU-pipe roofline.

``--workload mlp`` (1 GPU) measures the proposal network's tcgen05 GEMMs
(forward and training step on 16384 resident rows).

``--workload ga`` (1 GPU) measures the island-model GA instead: the planted
256 x 8192 matrix (density 0.01, 5000 scrambles, seed 7), 64 islands x 256,
ring migration every 20 generations, stop at the planted weight or the
wall-clock cap; the plain GA (the reference's algorithm), the proposal step
with uniform windows, and the learned proposal step, over --seeds seeds.
Reports generations/s and, per seed, the wall-clock each variant needs to
reach the best weight the plain GA reaches within the cap (time-to-threshold;
no variant reaches the planted weight within the cap).  With --impl reference
the reference IslandModel (one thread per island, host cores) runs the same
configuration under the same cap.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

K_OTHERS = 24
ROWS, COLS, P, SEED = 40, 4096, 0.3, 1
COMBOS_PER_TARGET = 1 << K_OTHERS
METRIC = "row-combos evaluated/s"
UNIT = "combos/s"


def workload_config(n):
    return {
        "workload": "gray-code per-target search: 40x4096 Bernoulli(0.3) (seed 1+rank), "
                    "each row vs all 2^24 XORs of the next 24 rows, 64 words/row",
        "targets": ROWS, "others_per_target": K_OTHERS, "cols": COLS,
        "combos_per_step": ROWS * COMBOS_PER_TARGET,
        "tiebreak": "smallest subset mask (reference order)",
        "l2": "flushed before every timed step (256 MB device write)",
        "parallelism": f"independent instances x{n}",
    }


# ---------------------------------------------------------------------------
def max_over_ranks(value, dist=None, device="cpu"):
    """The largest per-rank value over all ranks (a job's time is its slowest
    rank's); with no process group, the value itself."""
    if not dist:
        return float(value)
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def weak_throughput(world, units_per_rank, seconds):
    """Whole-job rate of a weak-scaling run: every rank processed the same
    number of units (its own instance) within the slowest rank's time."""
    return world * units_per_rank / seconds


# ---------------------------------------------------------------------------
def clock_sampler(uuid):
    """Sample SM clocks and throttle reasons while the timed region runs."""
    fields = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    cmd = ["nvidia-smi", f"--query-gpu={fields}", "--format=csv,noheader,nounits", "-lms", "100"]
    if uuid:
        cmd += ["-i", uuid]
    try:
        proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
    except OSError:
        return None
    lines = []
    t = threading.Thread(target=lambda: lines.extend(proc.stdout), daemon=True)
    t.start()
    return proc, lines, t


def clock_summary(sampler):
    if sampler is None:
        return None
    proc, lines, t = sampler
    proc.terminate()
    try:
        proc.wait(timeout=5)
    except subprocess.TimeoutExpired:
        proc.kill()
    t.join(timeout=2)
    sms, maxs, reasons = [], [], set()
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    for ln in lines:
        parts = [x.strip() for x in ln.split(",")]
        if len(parts) < 8:
            continue
        try:
            sms.append(float(parts[0]))
            maxs.append(float(parts[1]))
        except ValueError:
            continue
        for name, val in zip(names, parts[4:8]):
            if val.lower().startswith("active"):
                reasons.add(name)
    if not sms:
        return None
    return {"sm_mhz": statistics.median(sms), "sm_max_mhz": max(maxs),
            "reasons": sorted(reasons), "samples": len(sms)}


# Roofline of gray_targets_kernel<64, 1, 4, 0> (the C2 step).  Its rows live
# in shared memory and registers, so neither HBM nor tensor cores bound it:
# each Gray step is 64 word XORs plus a popcount, split between LOP3 on the
# ALU pipe (16 lanes per SM sub-partition: 2 cycles per warp instruction) and
# POPC on the XU pipe (4 lanes: 8 cycles).  Warp instructions per warp-step
# (32 lanes, one combo each, 64 words each) counted by ncu on this kernel
# (smsp__inst_executed_pipe_{alu,xu}.sum and smsp__inst_executed.sum over one
# C2 launch divided by its 40 * 2^24 / 32 warp-steps):
GRAY_MIX = {"alu": 287.3, "xu": 74.1, "issue": 470.9}
# DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum) from the
# same capture: the rows are read once into shared memory.
GRAY_TRAFFIC = 43520


def gray_pipe_bound(sm_count, mhz, mix=None, words=64):
    """Words/s the SMs can process at the pipe bound of an instruction mix:
    per sub-partition a warp-step takes max(2 * ALU, 8 * XU, issue) cycles."""
    mix = mix or GRAY_MIX
    cycles = max(2 * mix["alu"], 8 * mix["xu"], mix["issue"])
    return sm_count * 4 * mhz * 1e6 * 32 * words / cycles


def gray_best_mix_bound(sm_count, mhz, words=64, overhead_alu=10, overhead_xu=9):
    """The same bound for the best split of a 64-word step between carry-save
    LOP3 (2 per 32-bit word, ALU) and POPC (1 per 32-bit word, XU), with the
    128 XOR LOP3 and the popcount sums on the FMA pipe: min over x of
    max(2 * (128 + 256 x + oa), 8 * (128 (1 - x) + ox))."""
    best = None
    for i in range(0, 1001):
        x = i / 1000
        c = max(2 * (2 * words + 4 * words * x + overhead_alu),
                8 * (2 * words * (1 - x) + overhead_xu))
        best = c if best is None or c < best else best
    return sm_count * 4 * mhz * 1e6 * 32 * words / best


# ---------------------------------------------------------------------------
def cpu_baseline_sample(budget_s=12.0):
    """Reference BruteforceSearch (or the oracle port) on a bounded sample."""
    from oracle.oracle import port, ref
    R = ref()
    P = port()
    words, _ = P.gen_instance(ROWS, COLS, P_DENS, SEED)
    cores = os.cpu_count() or 1
    combos = 0
    t0 = time.perf_counter()
    n = 0
    kind = "reference" if R is not None else "port"
    for i in range(ROWS):
        win = [i] + [(i + 1 + j) % ROWS for j in range(K_OTHERS)]
        if R is not None:
            R.bruteforce_search(words, COLS, win, 128, 0)
            combos += (1 << (K_OTHERS + 1)) - 1
        else:
            P.target_best_gray(words, COLS, i, win[1:])
            combos += COMBOS_PER_TARGET
            cores = 1
        n += 1
        if time.perf_counter() - t0 > budget_s:
            break
    dt = time.perf_counter() - t0
    sample = (f"{n} of {ROWS} targets; reference BruteforceSearch(k=128) on the 25-row window "
              f"[i, i+1..i+24] = 2^25-1 combos each, OpenMP {cores} threads" if kind == "reference"
              else f"{n} of {ROWS} targets; oracle C port Gray sweep, 2^24 combos each, 1 thread")
    return {"value": combos / dt, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample}


P_DENS = P


def run_reference(args, rank, world):
    if rank != 0:
        return 0
    from oracle.oracle import port, ref

    R = ref()
    Pp = port()
    words, _ = Pp.gen_instance(ROWS, COLS, P_DENS, SEED)
    kind = "reference" if R is not None else "port"
    cores = (os.cpu_count() or 1) if R is not None else 1

    def step(i):
        tgt = i % ROWS
        win = [tgt] + [(tgt + 1 + j) % ROWS for j in range(K_OTHERS)]
        if R is not None:
            R.bruteforce_search(words, COLS, win, 128, 0)
            return (1 << (K_OTHERS + 1)) - 1
        Pp.target_best_gray(words, COLS, tgt, win[1:])
        return COMBOS_PER_TARGET

    for i in range(args.warmup):
        step(i)
    combos = 0
    t0 = time.perf_counter()
    for i in range(args.steps):
        combos += step(args.warmup + i)
    dt = time.perf_counter() - t0
    value = combos / dt
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3 / max(args.steps, 1),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
        "data": "synthetic (xorshift64 seed 1)", "config": workload_config(1),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": kind,
                         "sample": "one target per step: reference BruteforceSearch(k=128) on the "
                                   "25-row window [i, i+1..i+24] (2^25-1 combos)"
                                   if kind == "reference" else
                                   "one target per step: oracle C port Gray sweep (2^24 combos)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# The reference's own CUDA searchers on the same B200 (the GPU bar): the
# unmodified reference built with its CUDA backend for sm_100a
# (oracle/_ref/cuda, make -C oracle ref-cuda), called through its public
# classes, next to this library's classes of the same names on the same
# windows, results compared.
MITM16 = dict(rows=32, cols=2048, p=0.2, seed=2)  # total weight ~13k: int16-safe


def run_reference_gpu(args, rank, world):
    if rank != 0:
        return 0
    from oracle.oracle import port, ref_cuda

    RC = ref_cuda()
    if RC is None:
        print(json.dumps({"impl": "reference-gpu",
                          "unavailable": "oracle/_ref/cuda was not built (make -C oracle "
                                         "ref-cuda needs the reference checkout)"}))
        return 0
    import bmmpy_b200 as bmm
    from bmmpy_b200.matrix import BitMatrix

    P = port()
    words, _ = P.gen_instance(ROWS, COLS, P_DENS, SEED)
    m = BitMatrix.from_words(words, COLS)

    def window(i):
        i %= ROWS
        return [i] + [(i + 1 + j) % ROWS for j in range(K_OTHERS)]

    def timed(fn, steps):
        out, per = None, []
        for i in range(steps):
            t0 = time.perf_counter()
            out = fn(i)
            per.append(time.perf_counter() - t0)
        return out, per

    # brute force: CudaBruteforceSearch(k=128) on the 25-row window [i, i+1..i+24]
    ours = bmm.CudaBruteforceSearch(max_candidates=128)
    ref_bf = lambda i: RC.cuda_bruteforce_search(words, COLS, window(i), 128)
    our_bf = lambda i: [(c.mask_u64(), c.weight) for c in ours.search(m.row_window(window(i)))]
    timed(ref_bf, args.warmup)
    timed(our_bf, args.warmup)
    want, ref_per = timed(ref_bf, args.steps)
    got, our_per = timed(our_bf, args.steps)
    assert got == want, "CudaBruteforceSearch results differ from the reference's"
    combos = (1 << (K_OTHERS + 1)) - 1
    ref_v = combos * len(ref_per) / sum(ref_per)
    our_v = combos * len(our_per) / sum(our_per)

    # meet-in-the-middle: CudaMitmFwhtSearch(k=64) on a 32-row window whose
    # total weight fits the reference's int16 guard
    mw, _ = P.gen_instance(MITM16["rows"], MITM16["cols"], MITM16["p"], MITM16["seed"])
    mm = BitMatrix.from_words(mw, MITM16["cols"])
    win = list(range(MITM16["rows"]))
    t0 = time.perf_counter()
    mwant = RC.cuda_mitm_search(mw, MITM16["cols"], win, 64)
    ref_mitm_s = time.perf_counter() - t0
    osearch = bmm.CudaMitmFwhtSearch(max_candidates=64)
    osearch.search(mm.row_window(win))  # warm
    t0 = time.perf_counter()
    mgot = [(c.mask_u64(), c.weight) for c in osearch.search(mm.row_window(win))]
    our_mitm_s = time.perf_counter() - t0
    assert mgot == mwant, "CudaMitmFwhtSearch results differ from the reference's"

    line = {
        "impl": "reference-gpu", "metric": METRIC, "value": ref_v, "unit": UNIT,
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * sum(ref_per) / len(ref_per), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u64",
        "data": "synthetic (xorshift64 seed 1)",
        "config": {"workload": "reference CudaBruteforceSearch(k=128) on the 25-row windows "
                               "[i, i+1..i+24] of the 40x4096 Bernoulli(0.3) matrix (seed 1), "
                               "one window per step, 2^25-1 combos each",
                   "kernel": "bruteforce_persistent_kernel<64> (reference, sm_100a)"},
        "timing": "host wall clock around the synchronous public search() call "
                  "(plan upload, kernels, result copy), both libraries alike",
        "b200_same_call": {"value": our_v, "unit": UNIT,
                           "ms_per_step": 1e3 * sum(our_per) / len(our_per),
                           "ratio": our_v / ref_v, "results_equal": True},
        "mitm": {"workload": f"CudaMitmFwhtSearch(k=64) on a {MITM16['rows']}x{MITM16['cols']} "
                             f"Bernoulli({MITM16['p']}) window (seed {MITM16['seed']}), "
                             "2^32 subsets, total weight within the reference's int16 guard",
                 "reference_s": ref_mitm_s, "b200_s": our_mitm_s,
                 "reference_combos_per_s": float(1 << 32) / ref_mitm_s,
                 "b200_combos_per_s": float(1 << 32) / our_mitm_s,
                 "ratio": ref_mitm_s / our_mitm_s, "results_equal": True},
        "e2e": {"value": ref_v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
GA = dict(rows=256, cols=8192, p=0.01, seed=7, scrambles=5000, interval=20)


def _ga_first_time(trace, threshold):
    for t, g, best in trace:
        if best <= threshold:
            return t, g
    return None, None


def run_ga(args):
    """Time-to-threshold of the plain / uniform-window / learned GA."""
    if args.impl == "reference":
        return run_ga_reference(args)
    import bmmpy_b200 as bmm
    from bmmpy_b200.ga import ProposalConfig
    from bmmpy_b200.workloads import gen_instance

    m, planted = gen_instance(GA["rows"], GA["cols"], GA["p"], GA["seed"], GA["scrambles"])
    win = m.row_window(list(range(GA["rows"])))

    def spec(i):
        sp = bmm.IslandSpec()
        sp.island_id = i
        sp.migration.interval_generations = GA["interval"]
        sp.migration.import_count = 1
        return sp

    runs = {}
    for seed in range(1, args.seeds + 1):
        for mode in ("off", "uniform", "learned"):
            prop = ProposalConfig(mode, queries_per_elite=32, train_steps=1, seed=seed)
            model = bmm.IslandModel(islands=[spec(i) for i in range(args.islands)],
                                    population_size=args.population,
                                    target_total_weight=planted, max_generations=10 ** 9,
                                    seed=1000 * seed, proposal=prop)
            t0 = time.perf_counter()
            model.initialize(win)
            eng = model._engine
            trace = [(time.perf_counter() - t0, 0, min(int(eng.stats(i).best_score)
                                                    for i in range(args.islands)))]
            gens = 0
            while time.perf_counter() - t0 < args.cap:
                ran, done = eng.run(1)
                gens += ran
                best = min(int(eng.stats(i).best_score) for i in range(args.islands))
                trace.append((time.perf_counter() - t0, gens, best))
                if done:
                    break
            elapsed = time.perf_counter() - t0
            runs[(mode, seed)] = {"trace": trace, "gens": gens, "elapsed": elapsed,
                                  "best": trace[-1][2],
                                  "proposal": model.proposal_stats() if mode != "off" else None}
            del model, eng
    seeds_out = []
    for seed in range(1, args.seeds + 1):
        plain = runs[("off", seed)]
        thr = plain["best"]
        entry = {"seed": seed, "threshold_plain_best": thr}
        for mode in ("off", "uniform", "learned"):
            r = runs[(mode, seed)]
            t, g = _ga_first_time(r["trace"], thr)
            entry[mode] = {"best_at_cap": r["best"], "generations": r["gens"],
                           "gens_per_s": r["gens"] / r["elapsed"], "time_to_threshold_s": t,
                           "gens_to_threshold": g, "reached_planted": r["best"] <= planted}
            if r["proposal"]:
                entry[mode]["proposal"] = r["proposal"]
        ulr = runs[("uniform", seed)]["best"]
        tl, _ = _ga_first_time(runs[("learned", seed)]["trace"], ulr)
        tu, _ = _ga_first_time(runs[("uniform", seed)]["trace"], ulr)
        entry["learned_vs_uniform"] = {"threshold_uniform_best": ulr, "uniform_s": tu,
                                       "learned_s": tl}
        seeds_out.append(entry)
    def spread(vals):
        vals = sorted(v for v in vals if v is not None)
        if not vals:
            return None
        q = lambda f: float(np.quantile(vals, f))  # noqa: E731
        return {"median": q(0.5), "q25": q(0.25), "q75": q(0.75), "min": vals[0],
                "max": vals[-1], "n": len(vals)}

    def ratio(a, b):
        return a / b if a is not None and b else None

    speedups = [e["off"]["time_to_threshold_s"] / e["learned"]["time_to_threshold_s"]
                for e in seeds_out if e["learned"]["time_to_threshold_s"]]
    summary = {
        "learned_vs_plain": spread(ratio(e["off"]["time_to_threshold_s"],
                                         e["learned"]["time_to_threshold_s"]) for e in seeds_out),
        "uniform_vs_plain": spread(ratio(e["off"]["time_to_threshold_s"],
                                         e["uniform"]["time_to_threshold_s"]) for e in seeds_out),
        "learned_vs_uniform": spread(ratio(e["learned_vs_uniform"]["uniform_s"],
                                           e["learned_vs_uniform"]["learned_s"])
                                     for e in seeds_out),
        "paired_rate_learned": spread(e["learned"]["proposal"]["paired_rate_learned"]
                                      for e in seeds_out if e["learned"].get("proposal")),
        "paired_rate_uniform_in_learned_runs": spread(
            e["learned"]["proposal"]["paired_rate_uniform"]
            for e in seeds_out if e["learned"].get("proposal")),
        "reached_planted": {m: sum(e[m]["reached_planted"] for e in seeds_out)
                            for m in ("off", "uniform", "learned")},
        "note": "ratios are time-to-threshold quotients (>1: the first variant is faster); "
                "learned_vs_uniform uses the uniform-window run's best at the cap as the "
                "threshold",
    }
    line = {
        "metric": "time-to-threshold speed-up, learned vs plain GA (threshold: the plain GA's "
                  "best weight within the cap)",
        "value": statistics.median(speedups) if speedups else None, "unit": "x",
        "higher_is_better": True, "n_gpus": 1, "dtype": "u64 (+bf16 network)",
        "data": "synthetic planted matrix (xorshift64 seed 7)", "vs_baseline": None,
        "config": {"workload": "GA island model on a planted 256x8192 matrix (density 0.01, "
                               "5000 scrambles, seed 7)", "islands": args.islands,
                   "population": args.population, "migration": "ring, every 20 generations",
                   "cap_s": args.cap, "planted_weight": planted,
                   "proposal": "32 queries per elite, 16-row windows, 1 Adam step/generation"},
        "summary": summary,
        "seeds": seeds_out,
    }
    print(json.dumps(line), flush=True)
    return 0


def run_ga_reference(args):
    from oracle.oracle import port, ref

    R = ref()
    if R is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref was not built"}))
        return 0
    P = port()
    words, planted = P.gen_instance(GA["rows"], GA["cols"], GA["p"], GA["seed"], GA["scrambles"])
    out = []
    for seed in range(1, args.seeds + 1):
        best, secs = R.island_run(words, GA["cols"], list(range(GA["rows"])), args.islands,
                                  args.population, GA["interval"], seed, 10 ** 9, planted,
                                  args.cap)
        out.append({"seed": seed, "best_at_cap": best, "seconds": secs,
                    "reached_planted": best <= planted})
    line = {"impl": "reference", "metric": "GA best weight within the cap (reference IslandModel)",
            "value": statistics.median([o["best_at_cap"] for o in out]), "unit": "weight",
            "higher_is_better": False, "n_gpus": 0,
            "config": {"workload": "GA island model on a planted 256x8192 matrix",
                       "islands": args.islands, "population": args.population,
                       "migration": "shared pool every 20 generations (reference channel)",
                       "cap_s": args.cap, "planted_weight": planted,
                       "cores": os.cpu_count()},
            "seeds": out}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
C3 = dict(rows=512, cols=65536, p=0.02, seed=2, scrambles=2000, window=32)


def run_mitm(args):
    """Search -> apply sweeps over the planted 512 x 65536 matrix: every sweep
    splits the rows into 16 windows of 32 by a seeded random permutation; each
    window is searched exhaustively (all 2^32 subsets, spectrum FWHT, top 64)
    and applied with GreedyApplier(min_gain=1), the whole sweep on the device
    (DeviceMatrix.search_apply); until four sweeps in a row improve nothing,
    or the cap.  combos_per_s and seconds_per_window include the applies."""
    if args.impl == "reference":
        from oracle.oracle import port, ref

        R = ref()
        P = port()
        words, planted = P.gen_instance(C3["rows"], C3["cols"], C3["p"], C3["seed"],
                                        C3["scrambles"])
        if R is None:
            print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref was not built"}))
            return 0
        t0 = time.perf_counter()
        R.mitm_search(words, C3["cols"], list(range(32)), 64)
        dt = time.perf_counter() - t0
        print(json.dumps({"impl": "reference", "metric": "row-combos evaluated/s",
                          "value": float(1 << 32) / dt, "unit": "combos/s",
                          "higher_is_better": True,
                          "config": {"workload": "one 32-row window of the planted 512x65536 "
                                                 "matrix, reference MitmFwhtSearch(k=64)",
                                     "cores": 1},
                          "seconds_per_window": dt}), flush=True)
        return 0
    import bmmpy_b200 as bmm
    from bmmpy_b200.workloads import gen_instance

    m, planted = gen_instance(C3["rows"], C3["cols"], C3["p"], C3["seed"], C3["scrambles"])
    start = m.weight()
    searcher = bmm.MitmFwhtSearch(max_candidates=64)
    applier = bmm.GreedyApplier(1)
    window = args.window or C3["window"]
    nwin = C3["rows"] // window
    sweeps = []
    rng = np.random.default_rng(C3["seed"])
    dev = bmm.DeviceMatrix(m)  # the matrix stays on the device for the whole run
    t0 = time.perf_counter()
    windows = 0
    sweep = 0
    idle = 0
    weight = start
    while time.perf_counter() - t0 < args.cap and idle < 4:
        perm = rng.permutation(C3["rows"])
        wins = [sorted(int(r) for r in perm[window * j: window * (j + 1)])
                for j in range(nwin)]
        res = dev.search_apply(wins, searcher=searcher, applier=applier)
        windows += nwin
        gained = sum(r.weight_improvement for r in res)
        weight -= gained
        sweeps.append({"sweep": sweep, "weight": weight, "gained": gained,
                       "t": round(time.perf_counter() - t0, 3)})
        sweep += 1
        idle = idle + 1 if gained == 0 else 0
    search_s = time.perf_counter() - t0
    m = dev.to_matrix()
    assert m.weight() == weight, "bookkept weight differs from the matrix"
    line = {
        "metric": "recovered weight (search -> apply) vs planted weight",
        "value": m.weight(), "unit": "weight", "higher_is_better": False, "n_gpus": 1,
        "dtype": "int32 spectra", "data": "synthetic planted matrix (xorshift64 seed 2)",
        "vs_baseline": None,
        "config": {"workload": "planted 512x65536 matrix (density 0.02, 2000 scrambles, seed 2), "
                               f"sweeps of {nwin} random {window}-row windows, "
                               "MitmFwhtSearch(k=64) + GreedyApplier(1) as one device-resident "
                               "sweep per call",
                   "cap_s": args.cap, "window": window},
        "planted_weight": planted, "start_weight": start,
        "combos_per_s": windows * float(1 << window) / search_s,
        "seconds_per_window": search_s / windows,
        "sweeps": sweeps,
    }
    print(json.dumps(line), flush=True)
    return 0


BASIS_T, BASIS_WINDOWS = 24, 10
C5 = dict(rows=256, cols=8192, p=0.01, seed=7, scrambles=5000)  # the GA's planted instance


def _basis_windows():
    return [list(range(BASIS_T * j, BASIS_T * (j + 1))) for j in range(BASIS_WINDOWS)]


def _basis_config():
    return {"workload": "ExactBasisSolver on 24-row windows (the reference's default max_rows "
                        "cap) of the planted 256x8192 matrix (density 0.01, 5000 scrambles, "
                        "seed 7): rows 24j..24j+23 for j < 10, 2^24-1 combinations each",
            "windows_per_step": BASIS_WINDOWS, "window_rows": BASIS_T, "cols": C5["cols"],
            "combos_per_step": BASIS_WINDOWS * ((1 << BASIS_T) - 1),
            "l2": "flushed before every timed step (256 MB device write)"}


def run_basis_reference(args):
    """The reference ExactBasisSolver (built without its AVX2 backend, which
    crashes in this solver on rows of 4+ words) on the same windows."""
    from oracle.oracle import port, ref_scalar

    R = ref_scalar()
    if R is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref was not built"}))
        return 0
    words, _ = port().gen_instance(C5["rows"], C5["cols"], C5["p"], C5["seed"], C5["scrambles"])
    wins = _basis_windows()
    for _ in range(1):
        R.exact_basis(words, C5["cols"], wins[0])
    per = []
    for i in range(args.steps):
        t0 = time.perf_counter()
        R.exact_basis(words, C5["cols"], wins[i % len(wins)])
        per.append(time.perf_counter() - t0)
    combos = (1 << BASIS_T) - 1
    v = combos * len(per) / sum(per)
    print(json.dumps({"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT,
                      "higher_is_better": True, "n_gpus": 0, "steps": args.steps,
                      "config": _basis_config(),
                      "cpu_baseline": {"value": v, "unit": UNIT, "cores": 1, "kind": "reference",
                                       "sample": f"{len(per)} windows, one per step, reference "
                                                 "ExactBasisSolver (scalar build, 1 thread)"},
                      "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0,
                              "d2h_bytes_per_step": 0},
                      "seconds_per_window": sum(per) / len(per)}), flush=True)
    return 0


def run_basis(args):
    """ExactBasisSolver windows: the device histogram pass timed with CUDA
    events on resident rows (``value``), the public solve() from host memory
    (``e2e``), parity of every solved window against the reference's answer
    for the first window."""
    if args.impl == "reference":
        return run_basis_reference(args)
    import ctypes

    import torch

    import bmmpy_b200 as bmm
    from bmmpy_b200 import _native as N
    from bmmpy_b200.workloads import gen_instance

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    stream = torch.cuda.current_stream(dev)
    m, _ = gen_instance(C5["rows"], C5["cols"], C5["p"], C5["seed"], C5["scrambles"])
    wins = _basis_windows()
    W = m.words_per_row
    rows = [torch.from_numpy(np.ascontiguousarray(m.words[w, :W]).view(np.int64)).to(dev)
            for w in wins]
    counts = torch.zeros((len(wins), m.cols + 1), dtype=torch.int64, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    L = N.lib()

    def launch():
        for j, r in enumerate(rows):
            N.check(L.bmm_basis_weight_counts_dev(r.data_ptr(), BASIS_T, m.cols,
                                                  counts[j].data_ptr(), stream.cuda_stream))

    for _ in range(args.warmup):
        flush.zero_()
        launch()
    torch.cuda.synchronize()
    sampler = clock_sampler(None)
    time.sleep(0.3)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    for i in range(args.steps):
        flush.zero_()
        evs[i][0].record(stream)
        launch()
        evs[i][1].record(stream)
    torch.cuda.synchronize()
    clocks = clock_summary(sampler)
    total_ms = sum(a.elapsed_time(b) for a, b in evs)
    combos_step = len(wins) * ((1 << BASIS_T) - 1)
    value = combos_step * args.steps / (total_ms / 1e3)
    assert all(int(c.sum()) == (1 << BASIS_T) - 1 for c in counts.cpu())

    # end to end: the public solve() on host windows
    solver = bmm.solver.ExactBasisSolver()
    first = solver.solve(m.row_window(wins[0]))
    e_steps = max(3, args.steps // 2)
    t0 = time.perf_counter()
    for _ in range(e_steps):
        res = [solver.solve(m.row_window(w)) for w in wins]
    e_dt = time.perf_counter() - t0
    e2e_value = combos_step * e_steps / e_dt
    assert res[0].basis_masks == first.basis_masks

    peak = ctypes.c_double(0)
    N.check(L.bmm_probe_xor_popc(ctypes.byref(peak)))
    per_launch_ms = total_ms / (args.steps * len(wins))
    achieved = ((1 << BASIS_T) - 1) * W / (per_launch_ms / 1e3)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u64",
        "data": "synthetic planted matrix (xorshift64 seed 7)",
        "config": _basis_config(),
        "e2e": {"value": e2e_value, "unit": UNIT,
                "h2d_bytes_per_step": int(len(wins) * BASIS_T * W * 8),
                "d2h_bytes_per_step": int(len(wins) * (m.cols + 1) * 8),
                "seconds_per_window": e_dt / (e_steps * len(wins)),
                "note": "solve() = histogram pass + collection pass(es) + host greedy; "
                        "combos counted once per window"},
        "gpu_launches": args.steps * len(wins),
        "roofline": {"bound": "int-popc", "achieved": achieved / 1e9, "peak": peak.value / 1e9,
                     "unit": "G words/s (64-bit XOR+POPC)", "frac": achieved / peak.value,
                     "peak_source": "measured in this run: register-only XOR+POPC probe kernel",
                     "traffic": None},
        "clocks": clocks,
        "total_weight_window0": first.total_weight,
    }
    if not args.no_cpu_baseline:
        from oracle.oracle import port, ref_scalar

        R = ref_scalar()
        if R is not None:
            words, _ = port().gen_instance(C5["rows"], C5["cols"], C5["p"], C5["seed"],
                                           C5["scrambles"])
            t0 = time.perf_counter()
            want = R.exact_basis(words, C5["cols"], wins[0])
            dt = time.perf_counter() - t0
            assert want["basis_masks"] == first.basis_masks, "differs from the reference"
            line["cpu_baseline"] = {"value": ((1 << BASIS_T) - 1) / dt, "unit": UNIT, "cores": 1,
                                    "kind": "reference",
                                    "sample": "window 0, reference ExactBasisSolver (scalar "
                                              "build, 1 thread); basis identical to the GPU's"}
    print(json.dumps(line), flush=True)
    return 0


SA_WINDOW = 32


def _sa_config():
    return {"workload": "SASelector(pairwise_synergy, 10000 iterations, 8 restarts, seed 1) "
                        "choosing a 32-row window of the planted 512x65536 matrix (density 0.02, "
                        "2000 scrambles, seed 2)",
            "rows": C3["rows"], "cols": C3["cols"], "window": SA_WINDOW}


def run_sa(args):
    """SASelector: the device synergy table timed with CUDA events (value =
    row-pair words/s), select() end to end from host memory (e2e), and the
    reference selector on the same matrix as the CPU arm."""
    from oracle.oracle import port, ref

    words, _ = port().gen_instance(C3["rows"], C3["cols"], C3["p"], C3["seed"], C3["scrambles"])
    if args.impl == "reference":
        R = ref()
        if R is None:
            print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref was not built"}))
            return 0
        per = []
        for _ in range(max(1, args.steps)):
            t0 = time.perf_counter()
            R.sa_select(words, C3["cols"], SA_WINDOW, seed=1)
            per.append(time.perf_counter() - t0)
        v = len(per) / sum(per)
        print(json.dumps({"impl": "reference", "metric": "SASelector.select calls/s", "value": v,
                          "unit": "selections/s", "higher_is_better": True, "n_gpus": 0,
                          "steps": len(per), "config": _sa_config(),
                          "cpu_baseline": {"value": v, "unit": "selections/s", "cores": 1,
                                           "kind": "reference",
                                           "sample": f"{len(per)} selections"},
                          "e2e": {"value": v, "unit": "selections/s", "h2d_bytes_per_step": 0,
                                  "d2h_bytes_per_step": 0},
                          "seconds_per_select": sum(per) / len(per)}), flush=True)
        return 0
    import ctypes

    import torch

    import bmmpy_b200 as bmm
    from bmmpy_b200 import _native as N

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    stream = torch.cuda.current_stream(dev)
    m = bmm.BitMatrix(C3["rows"], C3["cols"])
    m.words[:] = words[:, : m.stride_words]
    rows, W = m.rows, m.words_per_row
    d_words = torch.from_numpy(np.ascontiguousarray(m.words).view(np.int64)).to(dev)
    d_table = torch.empty(rows * rows, dtype=torch.int32, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    L = N.lib()

    def launch():
        N.check(L.bmm_sa_pairwise_table_dev(d_words.data_ptr(), m.stride_words, rows, m.cols,
                                            d_table.data_ptr(), stream.cuda_stream))

    for _ in range(args.warmup):
        flush.zero_()
        launch()
    torch.cuda.synchronize()
    sampler = clock_sampler(None)
    time.sleep(0.3)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    for i in range(args.steps):
        flush.zero_()
        evs[i][0].record(stream)
        launch()
        evs[i][1].record(stream)
    torch.cuda.synchronize()
    clocks = clock_summary(sampler)
    ms = sum(a.elapsed_time(b) for a, b in evs) / args.steps
    pair_words = rows * (rows - 1) // 2 * W
    value = pair_words / (ms / 1e3)

    selector = bmm.SASelector(seed=1)
    first = selector.select(m, SA_WINDOW)
    e_steps = max(3, args.steps // 2)
    t0 = time.perf_counter()
    for _ in range(e_steps):
        res = selector.select(m, SA_WINDOW)
    e_dt = (time.perf_counter() - t0) / e_steps
    assert res.rows == first.rows

    peak = ctypes.c_double(0)
    N.check(L.bmm_probe_xor_popc(ctypes.byref(peak)))
    line = {
        "metric": "synergy-table row-pair words/s", "value": value, "unit": "words/s",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
        "data": "synthetic planted matrix (xorshift64 seed 2)", "config": _sa_config(),
        "e2e": {"value": 1.0 / e_dt, "unit": "selections/s",
                "h2d_bytes_per_step": int(m.words.nbytes),
                "d2h_bytes_per_step": int(rows * rows * 4),
                "seconds_per_select": e_dt,
                "note": "select(): device table + its D2H + the 80000-step chain on the host"},
        "gpu_launches": args.steps,
        "roofline": {"bound": "int-popc", "achieved": value / 1e9, "peak": peak.value / 1e9,
                     "unit": "G words/s (64-bit AND+POPC)", "frac": value / peak.value,
                     "peak_source": "measured in this run: register-only XOR+POPC probe kernel",
                     "traffic": None},
        "clocks": clocks,
        "selected_rows": first.rows, "score": first.score,
    }
    if not args.no_cpu_baseline:
        R = ref()
        if R is not None:
            t0 = time.perf_counter()
            want = R.sa_select(words, C3["cols"], SA_WINDOW, seed=1)
            dt = time.perf_counter() - t0
            assert want["rows"] == first.rows and want["score"] == first.score
            line["cpu_baseline"] = {"value": 1.0 / dt, "unit": "selections/s", "cores": 1,
                                    "kind": "reference",
                                    "sample": "one select(), reference SASelector (AVX2 build); "
                                              "same rows and score as the GPU run"}
    print(json.dumps(line), flush=True)
    return 0


def run_io(args):
    """Matrix IO on the planted 512 x 65536 matrix: text payload parsed on the
    device from resident bytes (value, GB/s of text), and end to end through
    the public API: BitMatrix.from_text on host text, and a BMMPYB1 file
    loaded straight into device memory."""
    import tempfile

    import torch

    import bmmpy_b200 as bmm
    from bmmpy_b200 import _native as N
    from oracle.oracle import port, ref

    words, _ = port().gen_instance(C3["rows"], C3["cols"], C3["p"], C3["seed"], C3["scrambles"])
    m = bmm.BitMatrix(C3["rows"], C3["cols"])
    m.words[:] = words[:, : m.stride_words]
    text = m.to_text().encode()
    head = len(f"{m.rows} {m.cols}")
    if args.impl == "reference":
        R = ref()
        t0 = time.perf_counter()
        for _ in range(max(1, args.steps)):
            R.matrix_from_text(text)
        dt = (time.perf_counter() - t0) / max(1, args.steps)
        v = len(text) / dt / 1e9
        print(json.dumps({"impl": "reference", "metric": "text matrix parse GB/s", "value": v,
                          "unit": "GB/s", "higher_is_better": True, "n_gpus": 0,
                          "config": {"workload": "BitMatrix::load_text of the planted 512x65536 "
                                                 "matrix (33.5 MB of text)"},
                          "cpu_baseline": {"value": v, "unit": "GB/s", "cores": 1,
                                           "kind": "reference", "sample": "whole matrix"},
                          "e2e": {"value": v, "unit": "GB/s", "h2d_bytes_per_step": 0,
                                  "d2h_bytes_per_step": 0}}), flush=True)
        return 0
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    stream = torch.cuda.current_stream(dev)
    payload = torch.from_numpy(np.frombuffer(text[head:], dtype=np.uint8).copy()).to(dev)
    d_words = torch.empty(m.rows * m.stride_words, dtype=torch.int64, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    L = N.lib()

    def launch():
        N.check(L.bmm_matrix_from_text_dev(payload.data_ptr(), payload.numel(),
                                           d_words.data_ptr(), m.stride_words, m.rows, m.cols,
                                           stream.cuda_stream))

    for _ in range(args.warmup):
        launch()
    sampler = clock_sampler(None)
    time.sleep(0.3)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    for i in range(args.steps):
        flush.zero_()
        evs[i][0].record(stream)
        launch()
        evs[i][1].record(stream)
    torch.cuda.synchronize()
    time.sleep(0.3)  # the timed region is shorter than one clock sample
    clocks = clock_summary(sampler)
    ms = sum(a.elapsed_time(b) for a, b in evs) / args.steps
    got = d_words.cpu().numpy().view(np.uint64).reshape(m.rows, m.stride_words)
    assert np.array_equal(got, m.words)
    algo = payload.numel() + m.words.nbytes  # text read once, rows written once
    peak = 6650.0
    e_steps = max(3, args.steps // 2)
    t0 = time.perf_counter()
    for _ in range(e_steps):
        back = bmm.BitMatrix.from_text(text)
    e_dt = (time.perf_counter() - t0) / e_steps
    assert back == m
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "m.bin")
        m.save_binary_file(path)
        bin_bytes = os.path.getsize(path)
        t0 = time.perf_counter()
        for _ in range(e_steps):
            N.check(L.bmm_matrix_load_binary_dev(path.encode(), d_words.data_ptr(),
                                                 m.stride_words, m.rows, m.cols,
                                                 stream.cuda_stream))
        b_dt = (time.perf_counter() - t0) / e_steps
    line = {
        "metric": "text matrix parse GB/s", "value": payload.numel() / (ms / 1e3) / 1e9,
        "unit": "GB/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u8", "data": "synthetic planted matrix (xorshift64 seed 2)",
        "config": {"workload": "text payload of the planted 512x65536 matrix (33.5 MB) parsed "
                               "on the device; BMMPYB1 file (4 MB) loaded into device memory",
                   "l2": "flushed before every timed step (256 MB device write)"},
        "e2e": {"value": len(text) / e_dt / 1e9, "unit": "GB/s",
                "h2d_bytes_per_step": len(text), "d2h_bytes_per_step": int(m.words.nbytes),
                "seconds_per_parse": e_dt, "binary_file_to_device_s": b_dt,
                "binary_file_bytes": bin_bytes},
        "gpu_launches": 3 * args.steps,
        "roofline": {"bound": "hbm", "achieved": algo / (ms / 1e3) / 1e9, "peak": peak,
                     "unit": "GB/s", "frac": algo / (ms / 1e3) / 1e9 / peak,
                     "peak_source": "fallback 6.65 TB/s (no measured peaks file)",
                     "traffic": None},
        "clocks": clocks,
    }
    if not args.no_cpu_baseline:
        R = ref()
        if R is not None:
            t0 = time.perf_counter()
            R.matrix_from_text(text)
            dt = time.perf_counter() - t0
            line["cpu_baseline"] = {"value": len(text) / dt / 1e9, "unit": "GB/s", "cores": 1,
                                    "kind": "reference",
                                    "sample": "BitMatrix::load_text of the same 33.5 MB text"}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# Per-target transform workloads: C1 (64 x 256, 16 others per target) and C4
# (4096 uneven planted instances in one persistent launch).  The transform of
# a k = 16 item packs two 16-bit spectrum lanes in one int32 word, so one
# IADD or ISUB performs two butterflies' halves: one butterfly per ALU op.
# Bound: the ALU pipe, 64 int32 ops per clock per SM (the FMA pipe takes no
# part in these adds), i.e. sm_count * 64 * f_SM butterflies/s.


def _butterflies(k):
    return k * (1 << (k - 1)) if k > 0 else 0


def run_transform_targets(args):
    import torch

    from bmmpy_b200 import batch as B
    from bmmpy_b200 import targets as T
    from bmmpy_b200.workloads import C1, C4, batch_instance, gen_instance
    from tests.golden.fixtures import checksum_pairs

    if args.impl == "reference":
        print(json.dumps({"impl": "reference", "unavailable": "the C1/C4 per-target transform "
                          "workloads have no reference entry point beyond FwhtSearch per window "
                          "(bench.py --workload gray --impl reference times the reference "
                          "searcher)"}))
        return 0
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    stream = torch.cuda.current_stream(dev)
    gold = np.load(os.path.join(ROOT, "tests", "golden", "workloads.npz"))
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    if args.workload == "c1":
        m, _ = gen_instance(C1["rows"], C1["cols"], C1["p"], C1["seed"])
        t_idx, o_idx = T.cyclic_others(C1["rows"], C1["k"])
        d_words = torch.from_numpy(m.words.view(np.int64).copy()).to(dev)
        d_t = torch.from_numpy(t_idx.view(np.int32).copy()).to(dev)
        d_o = torch.from_numpy(o_idx.view(np.int32).copy()).to(dev)
        d_m = torch.empty(C1["rows"], dtype=torch.int64, device=dev)
        d_w = torch.empty(C1["rows"], dtype=torch.int32, device=dev)
        items, ks = C1["rows"], [C1["k"]] * C1["rows"]

        def launch():
            T.fwht_targets_dev(d_words, C1["rows"], m.stride_words, C1["cols"], d_t, d_o, C1["k"],
                               d_m, d_w, stream.cuda_stream)

        def check():
            assert np.array_equal(d_m.cpu().numpy().view(np.uint64), gold["c1_mask"])
            assert np.array_equal(d_w.cpu().numpy().view(np.uint32), gold["c1_weight"])

        def e2e():
            return T.fwht_targets(m, t_idx, o_idx)

        h2d, d2h = m.words.nbytes + t_idx.nbytes + o_idx.nbytes, C1["rows"] * 12
        workload = ("C1 per-target transform: 64 x 256 Bernoulli(0.5) (seed 0), each row vs "
                    "all 2^16 XORs of the next 16 rows")
    else:
        insts = [batch_instance(i) for i in range(C4["count"])]
        b = B.Batch([(mm, k) for mm, k, _ in insts])
        ks = [k for mm, k, _ in insts for _ in range(mm.rows)]
        items = b.n_out
        dw = torch.from_numpy(b.words.view(np.int64).copy()).to(dev)
        d_m = torch.empty(b.n_out, dtype=torch.int64, device=dev)
        d_w = torch.empty(b.n_out, dtype=torch.int32, device=dev)

        def launch():
            b.run_dev(dw, d_m, d_w, stream.cuda_stream)

        def check():
            ms = b.split(d_m.cpu().numpy().view(np.uint64))
            ws = b.split(d_w.cpu().numpy().view(np.uint32))
            bad = [i for i, (a, c) in enumerate(zip(ms, ws))
                   if checksum_pairs(a, c) != int(gold["c4_checksums"][i])]
            assert not bad, f"{len(bad)} instances differ from the reference"

        def e2e():
            return b.run()

        h2d, d2h = b.words.nbytes + b.desc.nbytes, b.n_out * 12
        workload = ("C4 batch: 4096 planted instances, n in [16,128], m in [64,2048] "
                    "log-uniform, density 0.05, 4n scrambles, k = min(n-1, 16), one "
                    "persistent launch replayed as a CUDA graph")
    combos = float(sum(1 << k for k in ks))
    bfly = float(sum(_butterflies(k) for k in ks))
    for _ in range(args.warmup):
        flush.zero_()
        launch()
    torch.cuda.synchronize()
    check()
    sampler = clock_sampler(None)
    time.sleep(0.3)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    for i in range(args.steps):
        flush.zero_()
        evs[i][0].record(stream)
        launch()
        evs[i][1].record(stream)
    torch.cuda.synchronize()
    time.sleep(0.3)
    clocks = clock_summary(sampler)
    ms = sum(a.elapsed_time(c) for a, c in evs) / args.steps
    check()
    e_steps = max(3, args.steps // 2)
    e2e()
    t0 = time.perf_counter()
    for _ in range(e_steps):
        e2e()
    e_dt = (time.perf_counter() - t0) / e_steps
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    mhz = (clocks or {}).get("sm_mhz") or 1965.0
    peak = sms * 64 * mhz * 1e6
    achieved = bfly / (ms / 1e3)
    line = {
        "metric": METRIC, "value": combos / (ms / 1e3), "unit": UNIT, "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32 (two int16 lanes packed)",
        "data": "synthetic (xorshift64 seeded instances)",
        "config": {"workload": workload, "items": items, "combos_per_step": combos,
                   "l2": "flushed before every timed step (256 MB device write)"},
        "e2e": {"value": combos / e_dt, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h)},
        "gpu_launches": args.steps,
        "roofline": {"bound": "alu", "achieved": achieved / 1e12, "peak": peak / 1e12,
                     "unit": "T butterflies/s", "frac": achieved / peak,
                     "peak_source": f"ALU pipe: {sms} SMs x 64 int32 ops/clk x {mhz:.0f} MHz "
                                    "sampled; one packed IADD/ISUB = one butterfly",
                     "traffic": None},
        "clocks": clocks,
        "results": "equal to the reference's per-target answers (golden)",
    }
    print(json.dumps(line), flush=True)
    return 0


def run_mlp(args):
    """The proposal network's tcgen05 GEMMs: forward passes and training steps
    (forward, backward, Adam) on 16384 resident query rows, CUDA-event timed
    on the network's stream; TFLOP/s of the GEMM work (forward 2 x rows x
    262144 flops, a training step 3x that)."""
    import ctypes

    import torch

    from bmmpy_b200 import _native as N

    if args.impl == "reference":
        print(json.dumps({"impl": "reference",
                          "unavailable": "the proposal network has no counterpart in the "
                                         "reference (its GA mutates uniformly)"}))
        return 0
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream(device=dev)
    rows = 16384
    g = torch.Generator(device=dev).manual_seed(0)
    x = torch.rand((rows, 512), generator=g, device=dev)
    t = torch.rand((rows, 256), generator=g, device=dev)
    t /= t.sum(1, keepdim=True)
    logits = torch.empty((rows, 256), device=dev)
    torch.cuda.synchronize()
    L = N.lib()
    h = ctypes.c_void_p()
    N.check(L.bmm_mlp_create_on_stream(1, 1e-3, stream.cuda_stream, ctypes.byref(h)))
    flops_fwd = 2.0 * rows * (512 * 256 + 256 * 256 + 256 * 256)
    xb = x.to(torch.bfloat16)
    out = {}

    def timed(fn):
        for _ in range(args.warmup):
            N.check(fn())
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(args.steps):
            N.check(fn())
        b.record(stream)
        torch.cuda.synchronize()
        return a.elapsed_time(b) / args.steps

    for name, fn, flops, tma in (
            ("forward_bf16_tma",
             lambda: L.bmm_mlp_forward_bf16_dev(h, xb.data_ptr(), rows, logits.data_ptr()),
             flops_fwd, 1),
            ("forward_bf16_thread_staged",
             lambda: L.bmm_mlp_forward_bf16_dev(h, xb.data_ptr(), rows, logits.data_ptr()),
             flops_fwd, 0),
            ("forward_fp32_input",
             lambda: L.bmm_mlp_forward_dev(h, x.data_ptr(), rows, logits.data_ptr()),
             flops_fwd, 1),
            ("train_step", lambda: L.bmm_mlp_train_dev(h, x.data_ptr(), t.data_ptr(), rows, 1),
             3 * flops_fwd, 1)):
        N.check(L.bmm_mlp_tune(tma))
        ms = timed(fn)
        out[name] = {"ms": ms, "tflops": flops / (ms / 1e3) / 1e12}
    N.check(L.bmm_mlp_tune(1))
    N.check(L.bmm_mlp_destroy(h))
    peak, src = 1590.0, "fallback 1.59 PFLOP/s dense BF16 (no measured peaks file)"
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peak = float(json.load(f)["bf16_tflops"])
        src = "MEASURED_PEAKS.json bf16_tflops (cuBLAS 8192^3, burst): of measured"
    except (OSError, ValueError, KeyError):
        pass
    v = out["forward_bf16_tma"]["tflops"]
    line = {"metric": "proposal-network GEMM TFLOP/s (BF16 operands, FP32 accumulate, tcgen05)",
            "value": v, "unit": "TFLOP/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": out["forward_bf16_tma"]["ms"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "bf16",
            "data": "synthetic features and targets (torch.rand, seed 0)",
            "config": {"workload": "512-256-256-256 MLP, 16384 query rows resident on the "
                                   "device: forward on BF16 features (the GA's proposal "
                                   "input) with TMA-fed GEMMs; thread-staged GEMMs, FP32 input "
                                   "and the training step (forward, backward, Adam) beside it"},
            **out,
            "roofline": {"bound": "tensor", "achieved": v, "peak": peak, "unit": "TFLOP/s",
                         "frac": v / peak, "peak_source": src, "traffic": None,
                         "note": "three GEMMs of 16384 x 256 x {512, 256, 256} plus a 16 MB "
                                 "logits copy per forward; each GEMM is one wave of 128 CTAs"}}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference", "reference-gpu"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="gray",
                    choices=["gray", "ga", "mitm", "basis", "sa", "io", "mlp", "c1", "batch"])
    ap.add_argument("--cap", type=float, default=60.0, help="GA: wall-clock cap per run (s)")
    ap.add_argument("--window", type=int, default=0,
                    help="mitm: window rows (default 32; one sweep = rows / window windows)")
    ap.add_argument("--seeds", type=int, default=2, help="GA: seeds per variant")
    ap.add_argument("--islands", type=int, default=64)
    ap.add_argument("--population", type=int, default=256)
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.workload == "ga":
        return run_ga(args)
    if args.workload == "mitm":
        return run_mitm(args)
    if args.workload == "basis":
        return run_basis(args)
    if args.workload == "sa":
        return run_sa(args)
    if args.workload == "io":
        return run_io(args)
    if args.workload == "mlp":
        return run_mlp(args)
    if args.workload in ("c1", "batch"):
        return run_transform_targets(args)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.impl == "reference-gpu":
        return run_reference_gpu(args, rank, world)

    import torch

    from bmmpy_b200 import _native as N
    from bmmpy_b200 import targets as T
    from bmmpy_b200.workloads import gen_instance

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)

    m, _ = gen_instance(ROWS, COLS, P_DENS, SEED + rank)
    t_idx, o_idx = T.cyclic_others(ROWS, K_OTHERS)
    d_words = torch.from_numpy(m.words.view(np.int64).copy()).to(dev)
    d_t = torch.from_numpy(t_idx.view(np.int32).copy()).to(dev)
    d_o = torch.from_numpy(o_idx.view(np.int32).copy()).to(dev)
    d_mask = torch.empty(ROWS, dtype=torch.int64, device=dev)
    d_w = torch.empty(ROWS, dtype=torch.int32, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    def launch():
        T.gray_targets_dev(d_words, ROWS, m.stride_words, COLS, d_t, d_o, K_OTHERS, d_mask, d_w,
                           0, stream.cuda_stream)

    for _ in range(args.warmup):
        flush.zero_()
        launch()
    torch.cuda.synchronize()

    uuid = None
    try:
        uuid = str(torch.cuda.get_device_properties(dev).uuid)
        if uuid and not uuid.startswith("GPU-"):
            uuid = "GPU-" + uuid
    except Exception:
        uuid = None
    sampler = clock_sampler(uuid)
    time.sleep(0.3)

    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    for i in range(args.steps):
        flush.zero_()
        evs[i][0].record(stream)
        launch()
        evs[i][1].record(stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = clock_summary(sampler)
    total_ms = sum(a.elapsed_time(b) for a, b in evs)
    max_ms = max_over_ranks(total_ms, dist, dev)
    combos_step = ROWS * COMBOS_PER_TARGET
    value = weak_throughput(world, combos_step * args.steps, max_ms / 1e3)

    # correctness of what was timed: rank 0's instance (seed 1) is the C2
    # workload, whose per-target answers the reference produced
    got_w = d_w.cpu().numpy().view(np.uint32)
    got_m = d_mask.cpu().numpy().view(np.uint64)
    if rank == 0:
        gold = np.load(os.path.join(ROOT, "tests", "golden", "workloads.npz"))
        assert np.array_equal(got_w, gold["c2_weight"]) and np.array_equal(
            got_m, gold["c2_mask"]), "timed result differs from the reference's answer"

    # end to end through the public host API, pinned host inputs
    pinned = torch.empty(m.words.size, dtype=torch.int64, pin_memory=True).numpy()
    pinned[:] = m.words.view(np.int64).ravel()
    from bmmpy_b200.matrix import BitMatrix

    hm = BitMatrix(ROWS, COLS)
    hm._words = pinned.view(np.uint64).reshape(m.words.shape)
    pt = torch.empty(ROWS, dtype=torch.int32, pin_memory=True).numpy().view(np.uint32)
    pt[:] = t_idx
    po = torch.empty(ROWS * K_OTHERS, dtype=torch.int32, pin_memory=True).numpy().view(np.uint32)
    po[:] = o_idx.ravel()
    po = po.reshape(ROWS, K_OTHERS)
    T.gray_targets(hm, pt, po)  # warm
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e_steps = max(3, args.steps // 2)
    t0 = time.perf_counter()
    for _ in range(e_steps):
        em, ew = T.gray_targets(hm, pt, po)
    e_dt = time.perf_counter() - t0
    e2e_value = weak_throughput(world, combos_step * e_steps, max_over_ranks(e_dt, dist, dev))
    assert np.array_equal(ew, got_w), "e2e and resident results differ"

    # roofline: 64-bit words XORed and counted per second by the targets
    # kernel against the ALU/XU pipe bound of its instruction mix at the clock
    # sampled during the timed region
    import ctypes

    per_launch_ms = max_ms / args.steps
    words = m.words_per_row
    achieved = combos_step * words / (per_launch_ms / 1e3)
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    mhz = (clocks or {}).get("sm_mhz") or 1965.0
    peak = gray_pipe_bound(sms, mhz)
    probe = ctypes.c_double(0)
    N.check(N.lib().bmm_probe_xor_popc(ctypes.byref(probe)))
    roofline = {
        "bound": "alu+xu pipes",
        "achieved": achieved / 1e9, "peak": peak / 1e9, "unit": "G words/s (64-bit XOR+popcount)",
        "frac": achieved / peak,
        "peak_source": f"ALU/XU pipe bound of the kernel's instruction mix per warp-step "
                       f"(ncu: {GRAY_MIX['alu']} ALU, {GRAY_MIX['xu']} XU, {GRAY_MIX['issue']} "
                       f"issued) x {sms} SMs x {mhz:.0f} MHz sampled",
        "frac_of_best_mix": achieved / gray_best_mix_bound(sms, mhz),
        "xor_popc_probe": probe.value / 1e9,
        "traffic": GRAY_TRAFFIC,
    }

    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": max_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u64",
        "data": "synthetic (xorshift64 Bernoulli matrix, seed 1+rank)",
        "config": workload_config(world),
        "e2e": {"value": e2e_value, "unit": UNIT,
                "h2d_bytes_per_step": int(pinned.nbytes + pt.nbytes + po.nbytes),
                "d2h_bytes_per_step": int(ROWS * 8 + ROWS * 4)},
        "gpu_launches": 2 * args.steps,
        "roofline": roofline,
        "clocks": clocks,
    }
    if world == 1 and not args.no_cpu_baseline:
        try:
            line["cpu_baseline"] = cpu_baseline_sample()
        except Exception as exc:  # the GPU result stands without it
            line["cpu_baseline"] = {"value": None, "error": str(exc)}
    print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
