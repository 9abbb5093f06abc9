"""The partitioned multi-rank fixpoint on the GPU (DeviceOps: every step is a
libmnmgdl call, the send side of every exchange is dl_partition) against the
one-GPU engine: equal iteration counts, per-iteration |delta| and rows.

World size 1 runs over NCCL (the multi-rank exchange itself is covered on
CPU ranks by test_partitioned.py; a machine with several GPUs runs it with
one rank per GPU).
"""
import datetime
import os
import socket

import numpy as np
import pytest

from conftest import load_input

pytestmark = pytest.mark.gpu

CASES = [("tc", "data_7035.bin", {}), ("tc", "data_23874.bin", {}), ("sg", "synth_lattice_small.bin", {}),
         ("sg", "data_7035.bin", {}), ("wcc", "data_23874.bin", {"stop": "reference"}),
         ("wcc", "data_214078.bin", {"stop": "fixpoint"})]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, backend, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch
    import torch.distributed as dist
    torch.cuda.set_device(0)
    dist.init_process_group(backend, rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        from mnmgdatalog_b200 import Engine, partitioned
        out = []
        with Engine(0) as eng:
            ops = partitioned.DeviceOps(eng)
            for prog, fname, kw in CASES:
                res = partitioned.run(prog, load_input(fname), ops, **kw)
                rows = partitioned.gather_rows(ops, res.rows)
                out.append((res.iterations, list(res.deltas), rows))
        if rank == 0:
            q.put(out)
    finally:
        dist.destroy_process_group()


def _run(world, backend):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, backend, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = q.get(timeout=600)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    return out


@pytest.mark.parametrize("world,backend", [(1, "nccl")])
def test_partitioned_equals_engine(engine, world, backend):
    results = _run(world, backend)
    for (prog, fname, kw), (iters, deltas, rows) in zip(CASES, results):
        edges = load_input(fname)
        if prog == "wcc":
            want = engine.run("wcc", edges, wcc_stop=kw["stop"], labels=True)
            assert iters == want.iterations and deltas == want.deltas.tolist(), (prog, fname)
            got = rows[np.argsort(rows[:, 0], kind="stable")]
            assert np.array_equal(got[:, 0], want.node_ids) and np.array_equal(got[:, 1], want.labels)
            continue
        want = engine.run(prog, edges)
        assert iters == want.iterations and deltas == want.deltas.tolist(), (prog, fname)
        got = rows[np.lexsort((rows[:, 1], rows[:, 0]))]
        if prog == "tc":  # (z, x) paths -> file rows (x, z) ordered by (z, x)
            got = np.ascontiguousarray(got[:, ::-1])
        assert np.array_equal(got, want.rows), (prog, fname)


def test_partition_groups_rows_by_owner(engine):
    """dl_partition: a permutation of the rows, grouped by owner, with the
    owner of every row the fmix32 mixer of its key mod ranks."""
    import torch

    from mnmgdatalog_b200 import partitioned
    from test_partitioned import fmix32_owner
    rng = np.random.default_rng(5)
    a = rng.integers(-2**31, 2**31, size=(200_000, 2), dtype=np.int64).astype(np.int32)
    ops = partitioned.DeviceOps(engine)
    for ranks, swap in [(1, False), (3, False), (8, True), (4096, False)]:
        out, counts = ops.partition(torch.from_numpy(a).cuda(), ranks, swap)
        got = out.cpu().numpy()
        src = a[:, ::-1] if swap else a
        assert sum(counts) == len(a)
        assert np.array_equal(np.sort(got.view(np.int64).ravel()), np.sort(np.ascontiguousarray(src).view(np.int64).ravel()))
        own = fmix32_owner(got[:, 0], ranks)
        assert np.array_equal(own, np.repeat(np.arange(ranks), counts))
