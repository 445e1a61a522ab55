"""The multi-rank path of bench.py on CPU: two gloo ranks, each a replica with its
own time and ray count; the whole-job figures are the slowest rank's time and the
rays of both ranks, the same on every rank."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime
    import sys
    from pathlib import Path
    import torch
    import torch.distributed as dist
    sys.path.insert(0, str(Path(__file__).resolve().parent.parent))
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        t, rays = bench.aggregate(10.0 + rank, 1000 * (rank + 1), dist, torch.device("cpu"))
        out[rank] = (t, rays)
    finally:
        dist.destroy_process_group()


def test_two_ranks_aggregate():
    world = 2
    ctx = mp.get_context("spawn")
    manager = ctx.Manager()
    out = manager.dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    assert out[0] == out[1] == (11.0, 3000.0)


def test_one_rank_is_identity():
    import bench
    assert bench.aggregate(2.5, 7, None, None) == (2.5, 7.0)
