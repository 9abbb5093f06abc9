"""B200-native semi-naive Datalog engine (TC, SG, WCC, single join).

The compute path is libmnmgdl.so (hand-written sm_100a CUDA behind a C-ABI,
include/mnmgdl.h); this package is its Python host mirror.
"""
from .capi import DatalogError, LIB_PATH
from .engine import Engine, HashTable, RunResult, generate_rows, read_edges, write_rows

__all__ = ["DatalogError", "Engine", "HashTable", "RunResult", "generate_rows", "read_edges", "write_rows",
           "LIB_PATH"]
