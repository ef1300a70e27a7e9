"""The multi-process host logic of bench.py on CPU ranks (gloo, world size 2):
the timed region is the slowest rank's, every rank holds its own maps, the
job's throughput counts the units of all ranks, and under torchrun the
reference arm runs on rank 0 only.  (On GPUs the same helpers run over NCCL;
the engine path itself has no exchange between ranks: replicas only.)"""
import datetime
import os
import socket
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        sys.path.insert(0, str(ROOT))
        import bench
        ms = bench.max_over_ranks(torch, dist, 10.0 + 5.0 * rank, "cpu")
        seeds = [None] * world
        dist.all_gather_object(seeds, bench.rank_seeds(rank, 4))
        out.put((rank, ms, seeds))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    # both ranks see the slowest rank's time
    assert [r[1] for r in res] == [15.0, 15.0]
    seeds = res[0][2]
    assert seeds == res[1][2] == [[0, 1, 2, 3], [4, 5, 6, 7]]  # disjoint maps per rank


def test_job_rate_and_single_process():
    sys.path.insert(0, str(ROOT))
    import bench
    import torch
    assert bench.job_rate(4, 40, 2000.0) == pytest.approx(80.0)
    assert bench.max_over_ranks(torch, None, 3.5, "cpu") == 3.5
    assert bench.rank_seeds(0, 4) == [0, 1, 2, 3]


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    sys.path.insert(0, str(ROOT))
    import bench
    monkeypatch.setenv("RANK", "1")
    import argparse
    ns = argparse.Namespace(steps=1, warmup=0, gpus=2)
    assert bench.run_reference(ns) is None  # returns at once, prints nothing
    assert capsys.readouterr().out == ""
