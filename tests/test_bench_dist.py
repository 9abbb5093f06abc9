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


def test_roofline_line_fields_and_arithmetic():
    """The bench line's roofline object: the dominant class by device time,
    achieved = its algorithmic bytes over its event time, frac against the
    measured peak, traffic from the committed DRAM ratio."""
    import bench
    prof = {"bitmap_expand": {"launches": 46, "timed_launches": 23, "seconds": 0.027, "bytes": 33.26e9},
            "bitmap_extract": {"launches": 3, "timed_launches": 3, "seconds": 0.0107, "bytes": 27.58e9},
            "host_sync": {"launches": 29, "timed_launches": 29, "seconds": 0.02, "bytes": 0.0}}
    roofline, kernels, host, launches = bench.roofline_of(prof, 0.046)
    assert roofline["kernel"] == "bitmap_expand" and roofline["bound"] == "hbm" and roofline["unit"] == "GB/s"
    assert abs(roofline["achieved"] - 33.26e9 / 0.027 / 1e9) < 1e-6
    assert abs(roofline["frac"] - roofline["achieved"] / roofline["peak"]) < 1e-12
    assert roofline["traffic"] is None or roofline["traffic"] > 0
    assert set(kernels) == {"bitmap_expand", "bitmap_extract"} and set(host) == {"host_sync"}
    assert launches == 49


def test_clock_sampler_keeps_only_timed_samples(monkeypatch):
    """Clock samples taken before the timed region (the warm-up) do not count;
    throttle reasons seen inside it are reported."""
    import bench
    c = bench.ClockSampler(0)
    c.proc = type("P", (), {"terminate": lambda self: None, "wait": lambda self, timeout=None: 0})()
    c.thread = type("T", (), {"join": lambda self, timeout=None: None})()
    c.lines = [(1.0, "0, 900, 1965, 500, 0x4, Not Active, Not Active, Active, Not Active"),
               (5.0, "0, 1965, 1965, 700, 0x0, Not Active, Not Active, Not Active, Active")]
    c.t_mark = 2.0
    monkeypatch.setattr(bench.time, "monotonic", lambda: 6.0)
    out = c.stop()
    assert out["sm_mhz"] == 1965.0 and out["samples"] == 1
    assert out["reasons"] == ["sw_power_cap"]
