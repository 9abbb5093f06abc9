"""Python host mirror of the engine's C-ABI (libmnmgdl.so).

Programs (the reference drivers tc.cu, sg.cu, wcc.cu, single_join.cu):

    eng = Engine()
    r = eng.tc(edges)            # edges: (n, 2) int32 numpy array or CUDA tensor
    r.rows, r.iterations, r.deltas

Relational operators on CUDA tensors of shape (n, 2) int32 laid out like the
reference's Entity, under the names the reference uses for them:

    get_hash_table(rel)          common/hash_table.cu:24-55
    get_join(ht, probe)          common/join.cu:51-87
    get_join_nl(sorted, probe)   common/join.cu:144-180
    sort_unique / set_difference / merge / unique_by_key_min / remove_self_pairs
                                 the thrust idioms of the drivers (set_cmp order)

Every call goes to the CUDA library; a missing library or device raises
DatalogError. Torch is used for device buffers only.
"""
from __future__ import annotations

import ctypes as C
import weakref
from dataclasses import dataclass, field

import numpy as np

from . import capi
from .capi import DatalogError, check, lib

PROGRAMS = {"tc": capi.PROGRAM_TC, "sg": capi.PROGRAM_SG, "wcc": capi.PROGRAM_WCC,
            "single_join": capi.PROGRAM_SINGLE_JOIN}


def _torch():
    import torch
    return torch


@dataclass
class RunResult:
    program: str
    rows: object                 # (n, 2) int32: numpy (host) or torch tensor (device), reference file order
    iterations: int
    deltas: np.ndarray
    output_tuples: int
    nodes: int
    seconds: float               # device time of the run (input upload through last iteration)
    phases: dict = field(default_factory=dict)
    largest_component: int = 0   # WCC
    join_rows_total: int = 0     # join output rows over all iterations (before dedup)
    join_rows_max: int = 0
    join_rows: np.ndarray | None = None   # per iteration
    full_rows: np.ndarray | None = None   # |full| after each iteration
    node_ids: np.ndarray | None = None
    labels: np.ndarray | None = None


class HashTable:
    """Handle of a dl_build_hash_table index (device memory owned by the library)."""

    def __init__(self, engine: "Engine", handle: C.c_void_p):
        self._engine = engine
        self.handle = handle
        s, d, r = C.c_int64(), C.c_int64(), C.c_int64()
        check(lib().dl_hash_table_info(handle, C.byref(s), C.byref(d), C.byref(r)))
        self.slots, self.distinct_keys, self.rows = s.value, d.value, r.value

    def close(self):
        if self.handle:
            lib().dl_hash_table_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _as_rows_np(edges) -> np.ndarray:
    a = np.ascontiguousarray(np.asarray(edges, dtype=np.int32))
    if a.size == 0:
        return np.zeros((0, 2), dtype=np.int32)
    return a.reshape(-1, 2)


def _check_rel(t):
    torch = _torch()
    if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.int32 and t.is_contiguous()):
        raise DatalogError(1, "relations must be contiguous int32 CUDA tensors of shape (n, 2)")
    if t.numel() and (t.dim() != 2 or t.shape[1] != 2):
        raise DatalogError(1, "relations must have shape (n, 2)")
    # The library works on its own stream: finish torch's pending writes first.
    torch.cuda.current_stream(t.device).synchronize()
    return t


class Engine:
    """One device + stream (a torch stream may be passed; default: the
    library's own non-blocking stream)."""

    def __init__(self, device: int = 0, stream=None):
        self.device = device
        h = C.c_void_p()
        s = None
        if stream is not None:
            s = C.c_void_p(stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream))
        self._stream_obj = stream
        self._sessions = weakref.WeakSet()
        check(lib().dl_context_create(device, s, C.byref(h)))
        self.ctx = h

    def close(self):
        if getattr(self, "ctx", None):
            for sess in list(getattr(self, "_sessions", ())):  # sessions hand their memory back first
                sess.close()
            lib().dl_context_destroy(self.ctx)
            self.ctx = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def synchronize(self):
        check(lib().dl_context_synchronize(self.ctx))

    def release_memory(self):
        """Free the device memory the context keeps between calls (workspace,
        cached buffers, the last TC run's bit matrix); live results stay."""
        check(lib().dl_context_release_memory(self.ctx))

    TUNING_FIELDS = ("sort_algorithm", "sort_ranking", "sort_keys_per_thread", "sort_input_tma", "dense_ratio",
                     "small_ratio", "hash_load_factor", "join_first_pass", "bitmap_max_gib",
                     "bitmap_unit_rows", "cache_max_gib", "bitmap_result")

    def tuning(self) -> dict:
        """The context's engine knobs (dl_tuning)."""
        t = capi.dl_tuning()
        check(lib().dl_context_get_tuning(self.ctx, C.byref(t)))
        return {f: getattr(t, f) for f in self.TUNING_FIELDS}

    def set_tuning(self, tuning: dict | None = None, **kw) -> None:
        """Sets engine knobs (unspecified ones keep their value); results do
        not depend on them. `tuning` may be a dict or a JSON file path."""
        if isinstance(tuning, str):
            import json
            with open(tuning) as f:
                tuning = json.load(f)
            tuning = tuning.get("tuning", tuning)
        cur = self.tuning()
        cur.update({k: v for k, v in (tuning or {}).items() if k in self.TUNING_FIELDS})
        cur.update({k: v for k, v in kw.items() if k in self.TUNING_FIELDS})
        unknown = set(kw) - set(self.TUNING_FIELDS)
        if unknown:
            raise DatalogError(1, f"unknown tuning fields {sorted(unknown)}")
        t = capi.dl_tuning(**cur)
        check(lib().dl_context_set_tuning(self.ctx, C.byref(t)))

    def profile(self, enabled: bool = True) -> None:
        """Reset the live kernel profile; enabled=True times every launch."""
        check(lib().dl_profile_enable(self.ctx, 1 if enabled else 0))

    def profile_read(self) -> dict:
        """{kernel class: {launches, timed_launches, seconds, bytes}}."""
        arr = (capi.dl_kernel_stat * 64)()
        n = C.c_int32()
        check(lib().dl_profile_read(self.ctx, arr, 64, C.byref(n)))
        return {arr[i].name.decode(): {"launches": arr[i].launches, "timed_launches": arr[i].timed_launches,
                                       "seconds": arr[i].seconds, "bytes": arr[i].bytes}
                for i in range(min(n.value, 64))}

    # ---- programs ----------------------------------------------------------
    def run(self, program: str, edges, *, wcc_stop: str = "reference", max_iterations: int = 0,
            phase_timing: bool = False, output: str = "host", labels: bool = False, out=None,
            dedup: str = "auto") -> RunResult:
        """Run one program. `edges` is an (n, 2) int32 host array or a CUDA
        tensor (then the input stays on the device). `output` is "host"
        (numpy), "device" (torch tensor) or "none"; `out` optionally supplies
        the (capacity, 2) int32 destination (e.g. pinned host memory), or a
        callable that returns one for the result's row count."""
        torch = _torch()
        prog = PROGRAMS[program]
        opts = capi.dl_options()
        opts.wcc_stop = {"reference": capi.WCC_STOP_REFERENCE, "fixpoint": capi.WCC_STOP_FIXPOINT}[wcc_stop]
        opts.max_iterations = max_iterations
        opts.phase_timing = 1 if phase_timing else 0
        opts.dedup = {"auto": capi.DEDUP_AUTO, "sort": capi.DEDUP_SORT, "hash": capi.DEDUP_HASH,
                      "bitmap": capi.DEDUP_BITMAP}[dedup]
        keep = None
        if isinstance(edges, torch.Tensor) and edges.is_cuda:
            keep = _check_rel(edges) if edges.numel() else edges
            ptr, n, on_dev = keep.data_ptr(), keep.shape[0] if keep.numel() else 0, 1
        else:
            keep = _as_rows_np(edges)
            ptr, n, on_dev = keep.ctypes.data, keep.shape[0], 0
        run = C.c_void_p()
        check(lib().dl_run_program(self.ctx, prog, C.c_void_p(ptr), n, on_dev, C.byref(opts), C.byref(run)))
        try:
            info = capi.dl_run_info()
            check(lib().dl_run_get_info(run, C.byref(info)))
            deltas = np.zeros(max(info.iterations, 0), dtype=np.int64)
            check(lib().dl_run_copy_deltas(run, deltas.ctypes.data, deltas.size))
            jr = np.zeros(max(info.iterations, 1), dtype=np.int64)
            fr = np.zeros(max(info.iterations, 1), dtype=np.int64)
            check(lib().dl_run_copy_iteration_stats(run, jr.ctypes.data, fr.ctypes.data, jr.size))
            nout = info.output_rows
            rows = None
            if callable(out):
                out = out(nout)  # a buffer of at least nout rows, or None
            if output == "host":
                if out is not None:
                    if len(out) < nout or out.dtype != np.int32 or not out.flags.c_contiguous:
                        raise DatalogError(1, f"out holds {len(out)} rows, the result has {nout}")
                    rows = out[:nout]
                else:
                    rows = np.empty((nout, 2), dtype=np.int32)
                check(lib().dl_run_copy_output(run, rows.ctypes.data if nout else None, nout, 0))
            elif output == "device":
                rows = out[:nout] if out is not None else torch.empty((nout, 2), dtype=torch.int32,
                                                                      device=f"cuda:{self.device}")
                check(lib().dl_run_copy_output(run, C.c_void_p(rows.data_ptr()) if nout else None, nout, 1))
            res = RunResult(program, rows, info.iterations, deltas, info.output_tuples, info.nodes,
                            info.seconds_total, largest_component=info.largest_component,
                            join_rows_total=info.join_rows_total, join_rows_max=info.join_rows_max,
                            join_rows=jr[: len(deltas)], full_rows=fr[: len(deltas)])
            if phase_timing:
                res.phases = {"initialization": info.seconds_init, "join": info.seconds_join,
                              "deduplication": info.seconds_dedup, "merge": info.seconds_merge,
                              "finalization": info.seconds_finalize}
            if labels and prog == capi.PROGRAM_WCC:
                ids = np.empty(info.nodes, dtype=np.int32)
                lab = np.empty(info.nodes, dtype=np.int32)
                check(lib().dl_run_copy_labels(run, ids.ctypes.data, lab.ctypes.data, info.nodes))
                res.node_ids, res.labels = ids, lab
            return res
        finally:
            lib().dl_run_destroy(run)

    def tc(self, edges, **kw) -> RunResult:
        return self.run("tc", edges, **kw)

    def sg(self, edges, **kw) -> RunResult:
        return self.run("sg", edges, **kw)

    def wcc(self, edges, **kw) -> RunResult:
        return self.run("wcc", edges, **kw)

    def single_join(self, rows, **kw) -> RunResult:
        return self.run("single_join", rows, **kw)

    # ---- batched / served forms (mnmgdatalog_b200/session.py) ---------------
    def session(self, program: str, **kw):
        """A union session of one program (dl_session_create)."""
        from .session import Session
        return Session(self, program, **kw)

    def run_batch(self, program: str, edge_sets, **kw) -> list:
        """Every edge set as one instance of one union fixpoint (dl_run_batch)."""
        from .session import run_batch
        return run_batch(self, program, edge_sets, **kw)

    # ---- relational operators (CUDA tensors) -------------------------------
    def sort_unique(self, rel):
        """thrust::sort(set_cmp) + thrust::unique(is_equal), in place; returns
        the deduplicated prefix view."""
        _check_rel(rel)
        n = C.c_int64()
        check(lib().dl_sort_unique(self.ctx, C.c_void_p(rel.data_ptr()), rel.shape[0] if rel.numel() else 0,
                                   C.byref(n)))
        return rel[: n.value]

    def sort(self, rel):
        _check_rel(rel)
        check(lib().dl_sort(self.ctx, C.c_void_p(rel.data_ptr()), rel.shape[0] if rel.numel() else 0))
        return rel

    def set_difference(self, a, b):
        """a \\ b for sorted duplicate-free a, b (thrust::set_difference)."""
        torch = _torch()
        _check_rel(a), _check_rel(b)
        out = torch.empty_like(a)
        n = C.c_int64()
        check(lib().dl_set_difference(self.ctx, C.c_void_p(a.data_ptr()), len(a), C.c_void_p(b.data_ptr()), len(b),
                                      C.c_void_p(out.data_ptr()), C.byref(n)))
        self.synchronize()
        return out[: n.value]

    def merge(self, a, b):
        """thrust::merge(set_cmp): stable, duplicates kept."""
        torch = _torch()
        _check_rel(a), _check_rel(b)
        out = torch.empty((len(a) + len(b), 2), dtype=torch.int32, device=a.device)
        check(lib().dl_merge(self.ctx, C.c_void_p(a.data_ptr()), len(a), C.c_void_p(b.data_ptr()), len(b),
                             C.c_void_p(out.data_ptr())))
        return out

    def diff_merge(self, full, j):
        """(full u j, dedup(j) \\ full) for sorted full (duplicate-free) and j."""
        torch = _torch()
        _check_rel(full), _check_rel(j)
        fo = torch.empty((len(full) + len(j), 2), dtype=torch.int32, device=full.device)
        do = torch.empty((max(len(j), 1), 2), dtype=torch.int32, device=full.device)
        n = C.c_int64()
        check(lib().dl_diff_merge(self.ctx, C.c_void_p(full.data_ptr()), len(full), C.c_void_p(j.data_ptr()),
                                  len(j), C.c_void_p(fo.data_ptr()), C.c_void_p(do.data_ptr()), C.byref(n)))
        self.synchronize()
        return fo[: len(full) + n.value], do[: n.value]

    def unique_by_key_min(self, rel):
        """thrust::unique(is_equal_key) on a set_cmp-sorted relation, in place."""
        _check_rel(rel)
        n = C.c_int64()
        check(lib().dl_unique_by_key_min(self.ctx, C.c_void_p(rel.data_ptr()), len(rel), C.byref(n)))
        return rel[: n.value]

    def remove_self_pairs(self, rel):
        """thrust::remove_if(is_key_equal_value), in place."""
        _check_rel(rel)
        n = C.c_int64()
        check(lib().dl_remove_self_pairs(self.ctx, C.c_void_p(rel.data_ptr()), len(rel), C.byref(n)))
        return rel[: n.value]

    def build_hash_table(self, rel, load_factor: float = 0.0) -> HashTable:
        _check_rel(rel)
        h = C.c_void_p()
        check(lib().dl_build_hash_table(self.ctx, C.c_void_p(rel.data_ptr()), len(rel), load_factor, C.byref(h)))
        return HashTable(self, h)

    def _adopt(self, ptr: C.c_void_p, n: int):
        """Copy a library-allocated join result into a torch tensor, free it."""
        torch = _torch()
        out = torch.empty((n, 2), dtype=torch.int32, device=f"cuda:{self.device}")
        if n:
            try:
                check(lib().dl_memcpy(self.ctx, C.c_void_p(out.data_ptr()), ptr, n * 8))
            finally:
                check(lib().dl_free(self.ctx, ptr))
        return out

    def join(self, ht: HashTable, probe):
        """get_join: for probe (k, v) and indexed (k, w) emit (w, v)."""
        _check_rel(probe)
        out, n = C.c_void_p(), C.c_int64()
        check(lib().dl_join(self.ctx, ht.handle, C.c_void_p(probe.data_ptr()), len(probe), C.byref(out), C.byref(n)))
        return self._adopt(out, n.value)

    def join_sorted(self, rel, probe):
        """get_join_nl: the same join through binary search of a key-sorted relation."""
        _check_rel(rel), _check_rel(probe)
        out, n = C.c_void_p(), C.c_int64()
        check(lib().dl_join_sorted(self.ctx, C.c_void_p(rel.data_ptr()), len(rel), C.c_void_p(probe.data_ptr()),
                                   len(probe), C.byref(out), C.byref(n)))
        return self._adopt(out, n.value)

    # reference names
    get_hash_table = build_hash_table
    get_join = join
    get_join_nl = join_sorted


def generate_rows(rows: int, rand_range: int, seed: int = 1) -> np.ndarray:
    """The reference's synthetic single-join relation (parallel_generate,
    common/parallel_io.cu:79-108): glibc srand(seed), rand() % range + 1."""
    out = np.empty((rows, 2), dtype=np.int32)
    check(lib().dl_generate_rows(rows, rand_range, seed, out.ctypes.data if rows else None))
    return out


def read_edges(path: str) -> np.ndarray:
    """Binary edge file: int32 pairs, row count = file size / 8 (parallel_read)."""
    a = np.fromfile(path, dtype=np.int32)
    return a[: (a.size // 2) * 2].reshape(-1, 2)


def write_rows(path: str, rows: np.ndarray) -> None:
    np.ascontiguousarray(rows, dtype=np.int32).tofile(path)
