"""Batched and served forms: many fixpoint instances in one union session.

A session (dl_session in include/mnmgdl.h) runs every admitted instance of
one program as one union fixpoint: each iteration's launches process all
active instances at once, instances join between any two steps and leave at
their own fixpoint. Every instance's result equals Engine.run on its edges.

    with Engine() as eng:
        s = eng.session("tc")
        a = s.admit(edges_a); b = s.admit(edges_b)
        while s.step():
            for i in s.poll(): print(i, s.result(i).rows.shape)

    results = eng.run_batch("wcc", [edges_a, edges_b, ...])   # dl_run_batch

The reference has no batched or served form: each of its drivers runs one
program on one edge file per process (tc.cu:42-423, sg.cu:40-477,
wcc.cu:58-585).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import capi
from .capi import DatalogError, check, lib


def _options(wcc_stop: str, max_iterations: int) -> capi.dl_options:
    o = capi.dl_options()
    o.wcc_stop = {"reference": capi.WCC_STOP_REFERENCE, "fixpoint": capi.WCC_STOP_FIXPOINT}[wcc_stop]
    o.max_iterations = max_iterations
    return o


def _edge_arg(edges):
    """(pointer, rows, on_device, keep-alive) for a numpy array or CUDA tensor."""
    from .engine import _as_rows_np, _check_rel, _torch
    torch = _torch()
    if isinstance(edges, torch.Tensor) and edges.is_cuda:
        if edges.numel() == 0:
            return None, 0, 1, edges
        t = _check_rel(edges)
        return t.data_ptr(), t.shape[0], 1, t
    a = _as_rows_np(edges)
    return (a.ctypes.data if len(a) else None), a.shape[0], 0, a


class Session:
    """Union fixpoint of one program over many instances (dl_session_*)."""

    def __init__(self, engine, program: str, *, wcc_stop: str = "reference", max_iterations: int = 0,
                 max_nodes: int = 0, _handle=None):
        from .engine import PROGRAMS
        self.engine = engine
        self.program = program
        self._prog = PROGRAMS[program]
        if self._prog == capi.PROGRAM_SINGLE_JOIN:
            raise DatalogError(1, "sessions run tc, sg or wcc")
        if _handle is not None:
            self.handle = _handle
        else:
            h = C.c_void_p()
            opts = _options(wcc_stop, max_iterations)
            check(lib().dl_session_create(engine.ctx, self._prog, C.byref(opts), max_nodes, C.byref(h)))
            self.handle = h
        engine._sessions.add(self)

    def close(self):
        if getattr(self, "handle", None):
            lib().dl_session_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def admit(self, edges) -> int:
        """Adds an instance; returns its id. Its first iteration runs in the next step()."""
        ptr, n, on_dev, _keep = _edge_arg(edges)
        i = C.c_int64()
        check(lib().dl_session_admit(self.handle, C.c_void_p(ptr) if ptr else None, n, on_dev, C.byref(i)))
        return i.value

    def admit_many(self, edge_sets) -> list[int]:
        """Adds several instances with one ranking sort and one edge sort;
        returns their ids (consecutive)."""
        args = [_edge_arg(e) for e in edge_sets]
        if not args:
            return []
        on_dev = {a[2] for a in args if a[1]}
        if len(on_dev) > 1:
            raise DatalogError(1, "edge sets must all be host arrays or all CUDA tensors")
        count = len(args)
        ptrs = (C.c_void_p * count)(*[C.c_void_p(a[0]) if a[0] else None for a in args])
        rows = (C.c_int64 * count)(*[a[1] for a in args])
        first = C.c_int64()
        check(lib().dl_session_admit_many(self.handle, ptrs, rows, count, on_dev.pop() if on_dev else 0,
                                          C.byref(first)))
        return list(range(first.value, first.value + count))

    def step(self) -> int:
        """One iteration of every active instance; returns how many are still active."""
        a = C.c_int64()
        check(lib().dl_session_step(self.handle, C.byref(a)))
        return a.value

    def poll(self, capacity: int = 4096) -> list[int]:
        """Ids of the instances finished since the last poll."""
        out: list[int] = []
        buf = np.empty(capacity, dtype=np.int64)
        while True:
            n = C.c_int64()
            check(lib().dl_session_poll(self.handle, buf.ctypes.data, capacity, C.byref(n)))
            out.extend(int(x) for x in buf[: n.value])
            if n.value < capacity:
                return out

    def memory(self) -> tuple[int, int]:
        """(device bytes held, active instances)."""
        b, a = C.c_int64(), C.c_int64()
        check(lib().dl_session_memory(self.handle, C.byref(b), C.byref(a)))
        return b.value, a.value

    def info(self, instance: int) -> capi.dl_run_info:
        info = capi.dl_run_info()
        check(lib().dl_session_get_info(self.handle, instance, C.byref(info)))
        return info

    def result(self, instance: int, *, output: str = "host", labels: bool = False, out=None):
        """RunResult of a finished instance (rows in the reference's file order).
        `out` optionally supplies the destination rows, or a callable that
        returns one for the result's row count."""
        from .engine import RunResult, _torch
        info = self.info(instance)
        deltas = np.zeros(max(info.iterations, 0), dtype=np.int64)
        check(lib().dl_session_copy_deltas(self.handle, instance, deltas.ctypes.data if deltas.size else None,
                                           deltas.size))
        nout = info.output_rows
        rows = None
        if callable(out):
            out = out(nout)  # a buffer of at least nout rows, or None
        if output not in ("host", "device", "none"):
            raise DatalogError(1, f"output must be host, device or none, not {output!r}")
        if output == "host":
            rows = out[:nout] if out is not None else np.empty((nout, 2), dtype=np.int32)
            check(lib().dl_session_copy_output(self.handle, instance, rows.ctypes.data if nout else None, nout, 0))
        elif output == "device":
            torch = _torch()
            rows = out[:nout] if out is not None else torch.empty((nout, 2), dtype=torch.int32,
                                                                  device=f"cuda:{self.engine.device}")
            check(lib().dl_session_copy_output(self.handle, instance, C.c_void_p(rows.data_ptr()) if nout else None,
                                               nout, 1))
        res = RunResult(self.program, rows, info.iterations, deltas, info.output_tuples, info.nodes, 0.0,
                        largest_component=info.largest_component)
        if labels and self._prog == capi.PROGRAM_WCC:
            ids = np.empty(info.nodes, dtype=np.int32)
            lab = np.empty(info.nodes, dtype=np.int32)
            check(lib().dl_session_copy_labels(self.handle, instance, ids.ctypes.data if info.nodes else None,
                                               lab.ctypes.data if info.nodes else None, info.nodes))
            res.node_ids, res.labels = ids, lab
        return res

    def release(self, instance: int) -> None:
        """Frees a finished instance's result memory."""
        check(lib().dl_session_release(self.handle, instance))

    def run(self) -> None:
        """Steps until no instance is active."""
        while self.step():
            pass


def run_batch(engine, program: str, edge_sets, *, wcc_stop: str = "reference", max_iterations: int = 0,
              output: str = "host", labels: bool = False) -> list:
    """dl_run_batch: every edge set as one instance of one union fixpoint;
    returns one RunResult per edge set, in order."""
    from .engine import PROGRAMS
    prog = PROGRAMS[program]
    args = [_edge_arg(e) for e in edge_sets]
    on_dev = {a[2] for a in args if a[1]}
    if len(on_dev) > 1:
        raise DatalogError(1, "edge sets must all be host arrays or all CUDA tensors")
    count = len(args)
    ptrs = (C.c_void_p * max(count, 1))(*[C.c_void_p(a[0]) if a[0] else None for a in args])
    rows = (C.c_int64 * max(count, 1))(*[a[1] for a in args])
    opts = _options(wcc_stop, max_iterations)
    h = C.c_void_p()
    check(lib().dl_run_batch(engine.ctx, prog, ptrs, rows, count, on_dev.pop() if on_dev else 0, C.byref(opts),
                             C.byref(h)))
    with Session(engine, program, _handle=h) as s:
        return [s.result(i, output=output, labels=labels) for i in range(count)]
