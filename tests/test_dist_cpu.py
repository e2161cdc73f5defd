"""The multi-process side of bench.py on the host (world size 2, gloo).

With N GPUs the bench runs N independent replicas (no collective on the data
path): every rank takes the same barrier and max-reduction steps, the job's
time is the slowest rank's, each replica draws its own noise seed, and the
reference arm runs on rank 0 alone.
"""
import os
import socket
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, str(ROOT))
    import bench

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        bench.barrier(dist)
        ms = bench.max_over_ranks(dist, 10.0 + rank)   # rank 1 is the slow one
        bench.barrier(dist)
        cfg = dict(bench.CONFIGS["c2"])
        seed = cfg["seed"] + rank                      # make_sim(..., seed_offset=rank)
        out.put((rank, ms, seed))
    finally:
        dist.destroy_process_group()


def test_replicas_take_the_slowest_rank_and_distinct_seeds():
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [11.0, 11.0]
    assert res[0][2] != res[1][2]


def test_reference_arm_runs_on_rank_zero_only(capsys, monkeypatch):
    sys.path.insert(0, str(ROOT))
    import bench

    monkeypatch.setenv("RANK", "1")

    class Args:
        steps, warmup, gpus = 3, 3, 2

    bench.run_reference(Args(), dict(bench.CONFIGS["c2"]))
    assert capsys.readouterr().out == ""
