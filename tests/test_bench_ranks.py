"""The multi-rank timing of bench.py with two gloo ranks on the CPU: every rank
reports its own elapsed time and all agree on the slowest one, and the
aggregate rate counts the work of every replica."""
import os
import socket
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, str(ROOT))
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        local_ms = 100.0 + 50.0 * rank  # rank 1 is the slow one
        out[rank] = bench.max_over_ranks(local_ms, dist, "cpu")
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_with_two_gloo_ranks():
    world = 2
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = _free_port()
        procs = [ctx.Process(target=_worker, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        assert out[0] == out[1] == 150.0


def test_aggregate_rate_counts_every_replica():
    sys.path.insert(0, str(ROOT))
    import bench

    one = bench.aggregate_rate(1000, 1, 10, 100.0)
    assert one == pytest.approx(1000 * 10 / 0.1)
    assert bench.aggregate_rate(1000, 4, 10, 100.0) == pytest.approx(4 * one)


def test_max_over_ranks_without_process_group():
    sys.path.insert(0, str(ROOT))
    import bench

    assert bench.max_over_ranks(12.5, None, "cpu") == 12.5
