"""The partitioned multi-rank fixpoint (mnmgdatalog_b200.partitioned) on CPU
ranks: world sizes 2 and 3 over gloo, with the relational steps done by the
oracle's numpy restatements of the reference's thrust idioms and get_join
(oracle/ops.py), so that what is tested is this module's partitioning,
all-to-all exchange and termination logic. The gathered result, the number
of iterations and every iteration's global |delta| must equal the oracle's
one-rank run of the same program (oracle/cpu.py)."""
import datetime
import os
import socket

import numpy as np
import pytest

from conftest import load_input


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def fmix32_owner(keys: np.ndarray, ranks: int) -> np.ndarray:
    """owner = murmur3 fmix32 of the key's unsigned 32-bit pattern, mod ranks
    (what dl_partition computes on the device)."""
    h = np.asarray(keys, dtype=np.int64).astype(np.uint32).astype(np.uint64)
    m = np.uint64(0xFFFFFFFF)
    h ^= h >> np.uint64(16)
    h = (h * np.uint64(0x85EBCA6B)) & m
    h ^= h >> np.uint64(13)
    h = (h * np.uint64(0xC2B2AE35)) & m
    h ^= h >> np.uint64(16)
    return (h % np.uint64(ranks)).astype(np.int64)


class HostOps:
    """The partitioned driver's relational steps on host arrays (oracle)."""

    def __init__(self):
        from oracle import ops
        self.ops = ops

    def from_host(self, a):
        return np.ascontiguousarray(a, dtype=np.int32).reshape(-1, 2)

    def to_host(self, a):
        return a

    def empty(self, n):
        return np.zeros((n, 2), dtype=np.int32)

    def size(self, a):
        return len(a)

    def partition(self, rel, ranks, swap):
        r = rel[:, ::-1] if swap else rel
        own = fmix32_owner(r[:, 0], ranks)
        order = np.argsort(own, kind="stable")
        return np.ascontiguousarray(r[order]), np.bincount(own, minlength=ranks).tolist()

    def concat(self, parts):
        return np.concatenate(parts) if parts else self.empty(0)

    def index(self, rel):
        return rel

    def join(self, ht, probe):
        return self.ops.join(ht, probe)

    def sort_unique(self, a):
        return self.ops.sort_unique(a)

    def set_difference(self, a, b):
        return self.ops.set_difference(a, b)

    def merge(self, a, b):
        return self.ops.merge(a, b)

    def unique_by_key_min(self, a):
        return self.ops.unique_by_key_min(a)

    def remove_self_pairs(self, a):
        return self.ops.remove_self_pairs(a)

    def key_equal_value(self, a):
        return np.stack([a[:, 0], a[:, 0]], axis=1).astype(np.int32)


CASES = [("tc", "data_10.bin", {}), ("tc", "hipc_2019.bin", {}), ("tc", "synth_dag_c0.bin", {}),
         ("sg", "data_10.bin", {}), ("sg", "hipc_2019.bin", {}), ("sg", "synth_lattice_small.bin", {}),
         ("wcc", "dummy.bin", {"stop": "reference"}), ("wcc", "data_7035.bin", {"stop": "reference"}),
         ("wcc", "data_23874.bin", {"stop": "reference"}), ("wcc", "data_23874.bin", {"stop": "fixpoint"})]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        from mnmgdatalog_b200 import partitioned
        out = []
        for prog, fname, kw in CASES:  # every rank runs every case, in the same order
            res = partitioned.run(prog, load_input(fname), HostOps(), **kw)
            rows = partitioned.gather_rows(HostOps(), res.rows)
            out.append((res.iterations, list(res.deltas), rows))
        if rank == 0:
            q.put(out)
    finally:
        dist.destroy_process_group()


_RESULTS = {}


def _results(world):
    """All CASES on `world` gloo ranks (spawned once per world size)."""
    if world not in _RESULTS:
        import torch.multiprocessing as mp
        ctx = mp.get_context("spawn")
        q = ctx.Queue()
        port = _free_port()
        procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
        for p in procs:
            p.start()
        out = q.get(timeout=600)
        for p in procs:
            p.join(timeout=60)
            assert p.exitcode == 0
        _RESULTS[world] = out
    return _RESULTS[world]


def _case(world, prog, fname, **kw):
    return _results(world)[CASES.index((prog, fname, kw))]


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("fname", ["data_10.bin", "hipc_2019.bin", "synth_dag_c0.bin"])
def test_partitioned_tc(world, fname):
    from oracle import cpu
    iters, deltas, rows = _case(world, "tc", fname)
    want = cpu.tc(load_input(fname))
    assert iters == want.iterations and deltas == want.deltas.tolist()
    # ranks hold (z, x) paths; the reference's file rows are (x, z) ordered by (z, x)
    got = np.ascontiguousarray(rows[np.lexsort((rows[:, 1], rows[:, 0]))][:, ::-1])
    assert np.array_equal(got, want.rows)


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("fname", ["data_10.bin", "hipc_2019.bin", "synth_lattice_small.bin"])
def test_partitioned_sg(world, fname):
    from oracle import cpu
    iters, deltas, rows = _case(world, "sg", fname)
    want = cpu.sg(load_input(fname))
    assert iters == want.iterations and deltas == want.deltas.tolist()
    got = rows[np.lexsort((rows[:, 1], rows[:, 0]))]
    assert np.array_equal(got, want.rows)


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("fname,stop", [("dummy.bin", "reference"), ("data_7035.bin", "reference"),
                                        ("data_23874.bin", "reference"), ("data_23874.bin", "fixpoint")])
def test_partitioned_wcc(world, fname, stop):
    from oracle import cpu
    iters, deltas, rows = _case(world, "wcc", fname, stop=stop)
    want = cpu.wcc(load_input(fname), cpu.STOP_REFERENCE if stop == "reference" else cpu.STOP_FIXPOINT)
    assert iters == want.iterations and deltas == want.deltas.tolist()
    got = rows[np.argsort(rows[:, 0], kind="stable")]
    assert np.array_equal(got[:, 0], want.node_ids) and np.array_equal(got[:, 1], want.labels)


def test_owner_matches_rank_count():
    own = fmix32_owner(np.arange(-1000, 1000), 7)
    assert own.min() >= 0 and own.max() < 7 and len(np.unique(own)) == 7
