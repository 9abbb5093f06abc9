"""Partitioned multi-GPU fixpoint: the reference's multi-node multi-GPU scheme.

One process per GPU over a torch.distributed process group (NCCL between
GPUs; gloo for host-side exchanges). Every relation is hash-partitioned by
its join column -- a row belongs to rank fmix32(key) mod G (dl_partition) --
and each iteration runs, on every rank:

    local join against the rank's edge index        (common/join.cu:51-87)
    one all-to-all-v of the join output, keyed by   (common/comm.cu:3-182,
      the column the next step joins or dedups on     get_split_relation)
    local dedup, set difference and merge           (tc.cu:250-286)
    an all-reduce of |delta| for termination        (tc.cu:294-304)

TC follows tc.cu:100-314, SG sg.cu:100-390 (base join, then two joins and
two exchanges per iteration), WCC wcc.cu:120-387 (both stop rules). The
global delta of every iteration is the disjoint union of the ranks' deltas,
so iteration counts and per-iteration |delta| equal the one-GPU engine's.

The relational steps go through an `ops` object. `DeviceOps` is the product:
every step is a libmnmgdl call on this rank's GPU, with rows held in CUDA
tensors. The exchange uses all_to_all_single on those tensors (NCCL); with a
gloo group the rows are staged through host memory. Tests may pass other ops
with the same methods (host arrays), which exercises the partitioning,
exchange and termination logic of this module on CPU ranks.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass
class PartitionedResult:
    program: str
    iterations: int
    deltas: list                  # global |delta| of every iteration
    rows: object                  # this rank's rows of the result (ops' row type)
    full_rows: list = field(default_factory=list)  # global |full| after every iteration


class DeviceOps:
    """Relational steps on this rank's GPU through libmnmgdl (CUDA tensors
    of shape (n, 2) int32 in the reference's Entity layout)."""

    def __init__(self, engine):
        import torch
        self.eng = engine
        self.torch = torch
        self.device = torch.device("cuda", engine.device)

    def from_host(self, rows: np.ndarray):
        a = np.ascontiguousarray(rows, dtype=np.int32).reshape(-1, 2)
        return self.torch.from_numpy(a).to(self.device)

    def to_host(self, rel) -> np.ndarray:
        return rel.cpu().numpy()

    def empty(self, n: int):
        return self.torch.empty((n, 2), dtype=self.torch.int32, device=self.device)

    def size(self, rel) -> int:
        return int(rel.shape[0])

    def partition(self, rel, ranks: int, swap: bool):
        import ctypes as C

        from .capi import check, lib
        from .engine import _check_rel
        n = self.size(rel)
        out = self.empty(n)
        counts = np.zeros(ranks, dtype=np.int64)
        if n:
            _check_rel(rel)
        check(lib().dl_partition(self.eng.ctx, C.c_void_p(rel.data_ptr() if n else 0), n, ranks, 1 if swap else 0,
                                 C.c_void_p(out.data_ptr() if n else 0), counts.ctypes.data))
        return out, counts.tolist()

    def concat(self, parts):
        return self.torch.cat(parts) if parts else self.empty(0)

    def index(self, rel):
        return self.eng.build_hash_table(rel)

    def join(self, ht, probe):
        return self.eng.join(ht, probe) if self.size(probe) else self.empty(0)

    def sort_unique(self, rel):
        return self.eng.sort_unique(rel).clone() if self.size(rel) else rel

    def set_difference(self, a, b):
        return self.eng.set_difference(a, b) if self.size(a) else a

    def merge(self, a, b):
        if not self.size(b):
            return a
        if not self.size(a):
            return b
        return self.eng.merge(a, b)

    def unique_by_key_min(self, rel):
        return self.eng.unique_by_key_min(rel).clone() if self.size(rel) else rel

    def remove_self_pairs(self, rel):
        return self.eng.remove_self_pairs(rel).clone() if self.size(rel) else rel

    def key_equal_value(self, rel):
        """(key, key) for every row (same_key_value_entity_ar)."""
        out, _ = self.partition(rel, 1, False)
        out[:, 1] = out[:, 0]
        return out


def exchange(ops, rel, swap: bool, group=None):
    """Every row (after the optional column swap) to the rank that owns its
    key: one all-to-all of the per-destination counts, one all-to-all-v of
    the rows (get_split_relation, common/comm.cu:3-182)."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rows, counts = ops.partition(rel, world, swap)
    if world == 1:
        return rows
    backend = dist.get_backend(group)
    on_cuda = isinstance(rows, torch.Tensor) and rows.is_cuda
    dev = rows.device if (on_cuda and backend == "nccl") else torch.device("cpu")
    send_n = torch.tensor(counts, dtype=torch.int64, device=dev)
    recv_n = torch.empty(world, dtype=torch.int64, device=dev)
    dist.all_to_all_single(recv_n, send_n, group=group)
    recv_counts = recv_n.tolist()
    if isinstance(rows, torch.Tensor):
        src = rows if rows.device == dev else rows.cpu()
    else:
        src = torch.from_numpy(np.ascontiguousarray(rows, dtype=np.int32).reshape(-1, 2))
    out = torch.empty((int(sum(recv_counts)), 2), dtype=torch.int32, device=dev)
    dist.all_to_all_single(out, src.contiguous(), recv_counts, counts, group=group)
    if isinstance(rows, torch.Tensor):
        return out if out.device == rows.device else out.to(rows.device)
    return out.numpy()


def _global_sum(n: int, ops, group=None) -> int:
    import torch
    import torch.distributed as dist
    dev = getattr(ops, "device", None)
    if dist.get_backend(group) != "nccl":
        dev = torch.device("cpu")
    t = torch.tensor([n], dtype=torch.int64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return int(t.item())


def _local_slice(edges: np.ndarray, rank: int, world: int) -> np.ndarray:
    """This rank's contiguous share of the input rows (parallel_read,
    common/parallel_io.cu:1-40)."""
    e = np.ascontiguousarray(edges, dtype=np.int32).reshape(-1, 2)
    n = len(e)
    lo, hi = n * rank // world, n * (rank + 1) // world
    return e[lo:hi]


def tc(ops, edges_local, group=None, max_iterations: int = 0) -> PartitionedResult:
    """Transitive closure; this rank's rows are (z, x) paths x -> z with
    owner(z) == rank, set_cmp-sorted (tc.cu:100-314)."""
    e = ops.from_host(edges_local) if isinstance(edges_local, np.ndarray) else edges_local
    edge_idx_rel = exchange(ops, e, swap=False, group=group)     # (x, y) keyed by x
    delta = ops.sort_unique(exchange(ops, e, swap=True, group=group))  # (y, x) keyed by y
    full = delta
    ht = ops.index(edge_idx_rel)
    deltas, fulls = [], []
    total = _global_sum(ops.size(full), ops, group)
    while True:
        j = ops.join(ht, delta)                                   # (z, x)
        j = ops.sort_unique(exchange(ops, j, swap=False, group=group))
        delta = ops.set_difference(j, full)
        full = ops.merge(full, delta)
        nd = _global_sum(ops.size(delta), ops, group)
        total += nd
        deltas.append(nd)
        fulls.append(total)
        if nd == 0 or (max_iterations and len(deltas) >= max_iterations):
            break
    return PartitionedResult("tc", len(deltas), deltas, full, fulls)


def sg(ops, edges_local, group=None, max_iterations: int = 0) -> PartitionedResult:
    """Same generation; this rank's rows are (x, y) with owner(x) == rank,
    set_cmp-sorted (sg.cu:100-390)."""
    e = ops.from_host(edges_local) if isinstance(edges_local, np.ndarray) else edges_local
    edge_rel = ops.sort_unique(exchange(ops, e, swap=False, group=group))  # e(a, x) keyed by a
    ht = ops.index(edge_rel)
    base = ops.remove_self_pairs(ops.join(ht, edge_rel))                  # (x, y), x != y
    delta = ops.sort_unique(exchange(ops, base, swap=False, group=group))
    full = delta
    total = _global_sum(ops.size(full), ops, group)
    deltas, fulls = [], []
    while True:
        j1 = ops.join(ht, delta)                                          # (x, b) from sg(a, b), e(a, x)
        j1 = ops.sort_unique(exchange(ops, j1, swap=True, group=group))   # (b, x) keyed by b
        j2 = ops.join(ht, j1)                                             # (y, x) from e(b, y)
        j2 = ops.sort_unique(exchange(ops, j2, swap=True, group=group))   # (x, y) keyed by x
        delta = ops.set_difference(j2, full)
        full = ops.merge(full, delta)
        nd = _global_sum(ops.size(delta), ops, group)
        total += nd
        deltas.append(nd)
        fulls.append(total)
        if nd == 0 or (max_iterations and len(deltas) >= max_iterations):
            break
    return PartitionedResult("sg", len(deltas), deltas, full, fulls)


def wcc(ops, edges_local, group=None, stop: str = "reference", max_iterations: int = 0) -> PartitionedResult:
    """Weakly connected components by min-label propagation; this rank's
    rows are (node, label) with owner(node) == rank, one per node
    (wcc.cu:120-387). stop="reference" ends when the global |delta| equals
    the previous one (the reference's rule); "fixpoint" when it is zero."""
    e = ops.from_host(edges_local) if isinstance(edges_local, np.ndarray) else edges_local
    both = ops.concat([e, ops.partition(e, 1, True)[0]])             # edges and their reverses
    edge_rel = ops.sort_unique(exchange(ops, both, swap=False, group=group))
    cc = ops.unique_by_key_min(ops.sort_unique(ops.key_equal_value(edge_rel)))  # (node, node)
    delta = cc
    prev = _global_sum(ops.size(delta), ops, group)
    ht = ops.index(edge_rel)
    deltas = []
    while True:
        j = ops.join(ht, delta)                                          # (neighbour, label)
        j = ops.sort_unique(exchange(ops, j, swap=False, group=group))
        new_cc = ops.unique_by_key_min(ops.merge(cc, j))
        delta = ops.set_difference(new_cc, cc)
        cc = new_cc
        nd = _global_sum(ops.size(delta), ops, group)
        deltas.append(nd)
        done = (nd == prev) if stop == "reference" else (nd == 0)
        prev = nd
        if done or (max_iterations and len(deltas) >= max_iterations):
            break
    return PartitionedResult("wcc", len(deltas), deltas, cc)


PROGRAMS = {"tc": tc, "sg": sg, "wcc": wcc}


def run(program: str, edges: np.ndarray, ops, group=None, **kw) -> PartitionedResult:
    """Runs `program` on the whole input `edges`, every rank taking its
    contiguous share of the rows (as each reference rank reads its share of
    the file)."""
    import torch.distributed as dist
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    return PROGRAMS[program](ops, _local_slice(edges, rank, world), group=group, **kw)


def gather_rows(ops, rows, group=None) -> np.ndarray | None:
    """Every rank's result rows on rank 0 (host array, concatenated in rank
    order; None on the other ranks)."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    host = ops.to_host(rows) if not isinstance(rows, np.ndarray) else rows
    if world == 1:
        return host
    parts = [None] * world
    dist.all_gather_object(parts, host, group=group)
    return np.concatenate(parts) if dist.get_rank(group) == 0 else None
