"""bench.py's multi-rank logic on CPU: world-size-2 gloo ranks (spawned
processes, rendezvous on 127.0.0.1) combine their timings as the slowest rank
and their work as the sum; under torchrun only rank 0 runs the reference arm."""
import argparse
import datetime
import os
import socket

import pytest


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        seconds, units = bench.combine_ranks(10.0 + rank, 100.0 * (rank + 1), world)
        q.put((rank, seconds, units))
    finally:
        dist.destroy_process_group()


def test_combine_ranks_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    assert got == [(0, 11.0, 300.0), (1, 11.0, 300.0)]


def test_combine_ranks_single_process():
    import bench
    assert bench.combine_ranks(3.5, 7.0, 1) == (3.5, 7.0)


def test_reference_arm_only_on_rank_zero(capsys):
    import bench
    args = argparse.Namespace(warmup=1, steps=1, config="tc_chung_lu_317k")
    assert bench.main_reference(args, rank=1, world=2) == 0
    assert capsys.readouterr().out == ""  # rank 1 does no work and prints nothing
