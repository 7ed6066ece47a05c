"""The multi-rank bookkeeping of bench.py on CPU, with two gloo ranks: every
rank learns the slowest rank's time (the job's time), and the whole-job rate
counts every rank's units over that time (weak scaling: each rank runs its
own instance, no data-path collective)."""

import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world)
    try:
        local_ms = [12.5, 30.25][rank]
        job_ms = bench.max_over_ranks(local_ms, dist)
        out[rank] = (job_ms, bench.weak_throughput(world, 1000, job_ms / 1e3))
    finally:
        dist.destroy_process_group()


def test_two_rank_timing_takes_the_slowest_rank():
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.start_processes(_rank, args=(2, port, out), nprocs=2, join=True,
                           start_method="spawn")
        got = dict(out)
    assert got[0] == got[1] == (30.25, 2 * 1000 / 0.03025)


def test_single_process_needs_no_group():
    assert bench.max_over_ranks(7.5) == 7.5
    assert bench.weak_throughput(1, 10, 2.0) == 5.0
    assert bench.workload_config(4)["parallelism"] == "independent instances x4"
