"""ctypes binding of libmnmgdl.so (declarations mirror include/mnmgdl.h).

The library is the only compute path: importing this module does not need a
GPU, but every compute call fails loudly (``DatalogError``) when the library
is missing or no CUDA device is visible. There is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libmnmgdl.so")

DL_OK = 0
STATUS_NAMES = {
    0: "DL_OK", 1: "DL_ERR_INVALID_ARGUMENT", 2: "DL_ERR_CUDA", 3: "DL_ERR_OUT_OF_MEMORY",
    4: "DL_ERR_DEVICE_TIMEOUT", 5: "DL_ERR_OVERFLOW", 6: "DL_ERR_NO_DEVICE", 7: "DL_ERR_INTERNAL",
}

PROGRAM_TC, PROGRAM_SG, PROGRAM_WCC, PROGRAM_SINGLE_JOIN = 0, 1, 2, 3
WCC_STOP_REFERENCE, WCC_STOP_FIXPOINT = 0, 1
DEDUP_AUTO, DEDUP_SORT, DEDUP_HASH, DEDUP_BITMAP = 0, 1, 2, 3

# Every symbol include/mnmgdl.h declares (checked by the CPU test suite).
EXPORTS = (
    "dl_status_string", "dl_last_error", "dl_version",
    "dl_context_create", "dl_context_destroy", "dl_context_synchronize", "dl_context_release_memory", "dl_free", "dl_memcpy",
    "dl_context_get_tuning", "dl_context_set_tuning",
    "dl_sort_unique", "dl_sort", "dl_set_difference", "dl_merge", "dl_diff_merge",
    "dl_unique_by_key_min", "dl_remove_self_pairs", "dl_partition",
    "dl_build_hash_table", "dl_hash_table_info", "dl_hash_table_destroy", "dl_join", "dl_join_sorted",
    "dl_run_program", "dl_run_tc", "dl_run_sg", "dl_run_wcc", "dl_run_single_join",
    "dl_run_get_info", "dl_run_copy_output", "dl_run_copy_deltas", "dl_run_copy_labels", "dl_run_destroy",
    "dl_run_copy_iteration_stats",
    "dl_generate_rows", "dl_profile_enable", "dl_profile_read",
    "dl_compat_get_hash_table", "dl_compat_get_join", "dl_compat_get_join_nl",
    "dl_sort_unique_noalloc", "dl_sort_unique_noalloc_max_rows",
    "dl_session_create", "dl_session_admit", "dl_session_admit_many", "dl_session_step", "dl_session_poll", "dl_session_get_info",
    "dl_session_copy_output", "dl_session_copy_deltas", "dl_session_copy_labels", "dl_session_release",
    "dl_session_memory", "dl_session_destroy", "dl_run_batch",
)


class DatalogError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class dl_options(C.Structure):
    _fields_ = [("wcc_stop", C.c_int32), ("max_iterations", C.c_int32), ("phase_timing", C.c_int32),
                ("dedup", C.c_int32), ("reserved", C.c_int32 * 4)]


class dl_run_info(C.Structure):
    _fields_ = [("program", C.c_int32), ("iterations", C.c_int32), ("input_rows", C.c_int64),
                ("output_rows", C.c_int64), ("output_tuples", C.c_int64), ("largest_component", C.c_int64),
                ("nodes", C.c_int64), ("seconds_total", C.c_double), ("seconds_init", C.c_double),
                ("seconds_join", C.c_double), ("seconds_dedup", C.c_double), ("seconds_merge", C.c_double),
                ("seconds_finalize", C.c_double), ("join_rows_total", C.c_int64), ("join_rows_max", C.c_int64)]


class dl_tuning(C.Structure):
    _fields_ = [("sort_algorithm", C.c_int32), ("sort_ranking", C.c_int32), ("sort_keys_per_thread", C.c_int32),
                ("dense_ratio", C.c_int32), ("small_ratio", C.c_int32), ("sort_input_tma", C.c_int32),
                ("hash_load_factor", C.c_double), ("join_first_pass", C.c_int32), ("bitmap_max_gib", C.c_int32),
                ("bitmap_unit_rows", C.c_int32), ("cache_max_gib", C.c_int32),
                ("bitmap_result", C.c_int32)]


class dl_kernel_stat(C.Structure):
    _fields_ = [("name", C.c_char * 32), ("launches", C.c_int64), ("timed_launches", C.c_int64),
                ("seconds", C.c_double), ("bytes", C.c_double)]


_lib = None


def lib():
    """Load libmnmgdl.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise DatalogError(7, f"{LIB_PATH} is missing; build it with `python -m mnmgdatalog_b200.build`")
    L = C.CDLL(LIB_PATH)
    vp, i64, i32, pi64 = C.c_void_p, C.c_int64, C.c_int32, C.POINTER(C.c_int64)
    pvp = C.POINTER(C.c_void_p)
    sig = {
        "dl_status_string": ([C.c_int], C.c_char_p),
        "dl_last_error": ([], C.c_char_p),
        "dl_version": ([], C.c_char_p),
        "dl_context_create": ([i32, vp, pvp], C.c_int),
        "dl_context_destroy": ([vp], C.c_int),
        "dl_context_synchronize": ([vp], C.c_int),
        "dl_context_release_memory": ([vp], C.c_int),
        "dl_free": ([vp, vp], C.c_int),
        "dl_memcpy": ([vp, vp, vp, i64], C.c_int),
        "dl_context_get_tuning": ([vp, C.POINTER(dl_tuning)], C.c_int),
        "dl_context_set_tuning": ([vp, C.POINTER(dl_tuning)], C.c_int),
        "dl_sort_unique": ([vp, vp, i64, pi64], C.c_int),
        "dl_sort": ([vp, vp, i64], C.c_int),
        "dl_set_difference": ([vp, vp, i64, vp, i64, vp, pi64], C.c_int),
        "dl_merge": ([vp, vp, i64, vp, i64, vp], C.c_int),
        "dl_diff_merge": ([vp, vp, i64, vp, i64, vp, vp, pi64], C.c_int),
        "dl_unique_by_key_min": ([vp, vp, i64, pi64], C.c_int),
        "dl_remove_self_pairs": ([vp, vp, i64, pi64], C.c_int),
        "dl_partition": ([vp, vp, i64, i32, i32, vp, vp], C.c_int),
        "dl_build_hash_table": ([vp, vp, i64, C.c_double, pvp], C.c_int),
        "dl_hash_table_info": ([vp, pi64, pi64, pi64], C.c_int),
        "dl_hash_table_destroy": ([vp], C.c_int),
        "dl_join": ([vp, vp, vp, i64, pvp, pi64], C.c_int),
        "dl_join_sorted": ([vp, vp, i64, vp, i64, pvp, pi64], C.c_int),
        "dl_run_program": ([vp, i32, vp, i64, i32, C.POINTER(dl_options), pvp], C.c_int),
        "dl_run_tc": ([vp, vp, i64, i32, C.POINTER(dl_options), pvp], C.c_int),
        "dl_run_sg": ([vp, vp, i64, i32, C.POINTER(dl_options), pvp], C.c_int),
        "dl_run_wcc": ([vp, vp, i64, i32, C.POINTER(dl_options), pvp], C.c_int),
        "dl_run_single_join": ([vp, vp, i64, i32, C.POINTER(dl_options), pvp], C.c_int),
        "dl_run_get_info": ([vp, C.POINTER(dl_run_info)], C.c_int),
        "dl_run_copy_output": ([vp, vp, i64, i32], C.c_int),
        "dl_run_copy_deltas": ([vp, vp, i64], C.c_int),
        "dl_run_copy_labels": ([vp, vp, vp, i64], C.c_int),
        "dl_run_copy_iteration_stats": ([vp, vp, vp, i64], C.c_int),
        "dl_run_destroy": ([vp], C.c_int),
        "dl_generate_rows": ([i64, i32, C.c_uint32, vp], C.c_int),
        "dl_profile_enable": ([vp, i32], C.c_int),
        "dl_sort_unique_noalloc": ([vp, i64, pi64, vp], C.c_int),
        "dl_sort_unique_noalloc_max_rows": ([], C.c_int64),
        "dl_profile_read": ([vp, C.POINTER(dl_kernel_stat), i32, C.POINTER(C.c_int32)], C.c_int),
        "dl_session_create": ([vp, i32, C.POINTER(dl_options), i64, pvp], C.c_int),
        "dl_session_admit": ([vp, vp, i64, i32, pi64], C.c_int),
        "dl_session_admit_many": ([vp, vp, vp, i64, i32, pi64], C.c_int),
        "dl_session_step": ([vp, pi64], C.c_int),
        "dl_session_poll": ([vp, vp, i64, pi64], C.c_int),
        "dl_session_get_info": ([vp, i64, C.POINTER(dl_run_info)], C.c_int),
        "dl_session_copy_output": ([vp, i64, vp, i64, i32], C.c_int),
        "dl_session_copy_deltas": ([vp, i64, vp, i64], C.c_int),
        "dl_session_copy_labels": ([vp, i64, vp, vp, i64], C.c_int),
        "dl_session_release": ([vp, i64], C.c_int),
        "dl_session_memory": ([vp, pi64, pi64], C.c_int),
        "dl_session_destroy": ([vp], C.c_int),
        "dl_run_batch": ([vp, i32, vp, vp, i64, i32, C.POINTER(dl_options), pvp], C.c_int),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _lib = L
    return L


def check(status: int) -> None:
    if status != DL_OK:
        msg = lib().dl_last_error().decode(errors="replace")
        raise DatalogError(status, msg)
