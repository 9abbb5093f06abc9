"""ctypes wrapper over oracle/liboracle.so (the C restatement) -- TEST INFRASTRUCTURE.

Each function returns plain numpy arrays. Row layout matches the reference's
binary files: an ``(n, 2)`` int32 array, row order as the reference writes it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liboracle.so")
_lib = None

STOP_REFERENCE = 0
STOP_FIXPOINT = 1


def build() -> str:
    """Compile liboracle.so with gcc (no GPU needed)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB


def lib():
    global _lib
    if _lib is None:
        src = os.path.join(_HERE, "dl_oracle.c")
        if not os.path.exists(_LIB) or os.path.getmtime(_LIB) < os.path.getmtime(src):
            build()
        L = C.CDLL(_LIB)
        P32 = C.POINTER(C.POINTER(C.c_int32))
        P64 = C.POINTER(C.POINTER(C.c_int64))
        pi64 = C.POINTER(C.c_int64)
        pi32 = C.POINTER(C.c_int32)
        for name in ("oracle_tc", "oracle_sg", "oracle_tc_nl"):
            f = getattr(L, name)
            f.argtypes = [C.c_void_p, C.c_int64, P32, pi64, pi32, P64]
            f.restype = C.c_int
        L.oracle_wcc.argtypes = [C.c_void_p, C.c_int64, C.c_int32, P32, pi64, pi64, pi32, P64,
                                 P32, P32, pi64]
        L.oracle_wcc.restype = C.c_int
        L.oracle_single_join.argtypes = [C.c_int64, C.c_int32, P32, pi64]
        L.oracle_single_join.restype = C.c_int
        L.oracle_generate_rows.argtypes = [C.c_int64, C.c_int32, C.c_void_p]
        L.oracle_generate_rows.restype = None
        L.oracle_free.argtypes = [C.c_void_p]
        L.oracle_free.restype = None
        _lib = L
    return _lib


def _take(ptr, n, dtype, width=1) -> np.ndarray:
    count = int(n) * width
    if count == 0:
        out = np.zeros((0,) if width == 1 else (0, width), dtype=dtype)
    else:
        buf = np.ctypeslib.as_array(ptr, shape=(count,)).copy()
        out = buf.astype(dtype, copy=False).reshape((-1, width) if width > 1 else (-1,))
    lib().oracle_free(C.cast(ptr, C.c_void_p))
    return out


@dataclass
class FixpointResult:
    rows: np.ndarray          # (n, 2) int32, reference file order
    iterations: int
    deltas: np.ndarray        # int64, |delta| after each iteration


@dataclass
class WccResult:
    comp_rows: np.ndarray     # (c, 2) int32: (component_id, 0), ascending
    n_components: int
    largest: int
    iterations: int
    deltas: np.ndarray
    node_ids: np.ndarray      # int32, ascending
    labels: np.ndarray        # int32, final label per node


def _edges(edges) -> np.ndarray:
    e = np.ascontiguousarray(np.asarray(edges, dtype=np.int32).reshape(-1, 2))
    return e


def _fixpoint(fn, edges) -> FixpointResult:
    e = _edges(edges)
    out = C.POINTER(C.c_int32)()
    n = C.c_int64()
    it = C.c_int32()
    d = C.POINTER(C.c_int64)()
    rc = fn(e.ctypes.data, e.shape[0], C.byref(out), C.byref(n), C.byref(it), C.byref(d))
    if rc != 0:
        raise RuntimeError(f"oracle failed: {rc}")
    rows = _take(out, n.value, np.int32, 2)
    deltas = _take(d, it.value, np.int64)
    return FixpointResult(rows, it.value, deltas)


def tc(edges) -> FixpointResult:
    return _fixpoint(lib().oracle_tc, edges)


def sg(edges) -> FixpointResult:
    return _fixpoint(lib().oracle_sg, edges)


def wcc(edges, stop_mode: int = STOP_REFERENCE) -> WccResult:
    e = _edges(edges)
    comp = C.POINTER(C.c_int32)()
    nc = C.c_int64()
    big = C.c_int64()
    it = C.c_int32()
    d = C.POINTER(C.c_int64)()
    ids = C.POINTER(C.c_int32)()
    lab = C.POINTER(C.c_int32)()
    nn = C.c_int64()
    rc = lib().oracle_wcc(e.ctypes.data, e.shape[0], stop_mode, C.byref(comp), C.byref(nc), C.byref(big),
                          C.byref(it), C.byref(d), C.byref(ids), C.byref(lab), C.byref(nn))
    if rc != 0:
        raise RuntimeError(f"oracle failed: {rc}")
    return WccResult(_take(comp, nc.value, np.int32, 2), nc.value, big.value, it.value,
                     _take(d, it.value, np.int64), _take(ids, nn.value, np.int32),
                     _take(lab, nn.value, np.int32))


def single_join(rows: int, rand_range: int) -> np.ndarray:
    out = C.POINTER(C.c_int32)()
    n = C.c_int64()
    rc = lib().oracle_single_join(rows, rand_range, C.byref(out), C.byref(n))
    if rc != 0:
        raise RuntimeError(f"oracle failed: {rc}")
    return _take(out, n.value, np.int32, 2)


def generate_rows(rows: int, rand_range: int) -> np.ndarray:
    """The reference's synthetic single-join rows (glibc srand(1)/rand())."""
    out = np.empty((rows, 2), dtype=np.int32)
    lib().oracle_generate_rows(rows, rand_range, out.ctypes.data)
    return out
