"""Two ranks over gloo on the CPU: the host side of `bench.py --gpus N`.

Each rank steps its own independent tanks (weak scaling, no exchange on the data
path); the only collective is the max over ranks of the timed duration. These
tests run, with world size 2, that reduction, the per-rank batch draw, and two
replicas that each step their own tank (the oracle standing in for the device
step) and form the job's throughput as bench.py does.
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


def _replica_main(rank, world, port, out):
    """One rank of `bench.py --gpus N`'s replica scheme: it builds and steps its
    own tank (the oracle stands in for the device step, which needs a GPU),
    times it, and takes part only in the max-over-ranks reduction."""
    import datetime
    import time

    import torch
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        import oracle as O

        w = O.World(O.dam_break_scene(None, nxyz=(8, 6, 5), box=(0.2, 0.1, 0.12), seed=bench.SEED + rank),
                    O.dam_break_params(materialize=False))
        dist.barrier()
        t0 = time.perf_counter()
        w.run(bench.DT, 3)
        ms = (time.perf_counter() - t0) * 1e3
        slowest = bench.max_over_ranks(ms, torch)
        value = bench.job_throughput(8 * 6 * 5, 3, slowest, world)
        out.put((rank, w.hash64(), ms, slowest, value))
    finally:
        dist.destroy_process_group()


def test_two_replicas_step_their_own_tanks():
    """Each rank's tank evolves exactly as it does alone (no exchange on the
    data path), both ranks report the slowest rank's time, and the job value
    counts both ranks' particles over that time."""
    import torch.multiprocessing as mp

    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import bench
    import oracle as O

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_replica_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, h, ms, slowest, value in res:
        alone = O.World(O.dam_break_scene(None, nxyz=(8, 6, 5), box=(0.2, 0.1, 0.12), seed=bench.SEED + rank),
                        O.dam_break_params(materialize=False))
        alone.run(bench.DT, 3)
        assert h == alone.hash64(), rank
        assert slowest == max(r[2] for r in res)
        assert value == 2 * 8 * 6 * 5 * 3 / (slowest / 1e3)
    assert res[0][1] != res[1][1]  # different seeds, different tanks
