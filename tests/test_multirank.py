"""Two ranks over gloo on the CPU: the host side of `bench.py --gpus N`.

Each rank steps its own independent tanks (weak scaling, no exchange on the data
path); the only collective is the max over ranks of the timed duration. These
tests run that reduction and the per-rank batch draw with world size 2.
"""
import os
import socket
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime

    import torch
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "physics-engine_b200"))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        from physics_engine_rs import scenes

        slowest = bench.max_over_ranks(10.0 + rank, torch)
        spec = scenes.batch_spec(6, seed=bench.SEED + rank)
        fluid = sum(s["block"][0] * s["block"][1] * s["block"][2] for s in spec)
        totals = [None] * world
        dist.all_gather_object(totals, fluid)
        out.put((rank, slowest, totals))
    finally:
        dist.destroy_process_group()


def test_two_ranks_time_max_and_own_batches():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    # both ranks report the slowest rank's time
    assert [r[1] for r in res] == [11.0, 11.0]
    # each rank drew its own batch (different seeds), and all ranks see both totals
    assert res[0][2] == res[1][2]
    assert res[0][2][0] != res[0][2][1]


def test_one_rank_reduction_is_identity():
    import torch

    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks(3.25, torch) == 3.25
