"""C-ABI library checks that need no GPU."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from conftest import ROOT


def _declared_symbols():
    names = set()
    for h in ("mnmgdl.h", "mnmgdl_compat.h"):
        txt = open(os.path.join(ROOT, "include", h)).read()
        names |= set(re.findall(r"DL_API[^;(]*?\b(dl_[a-z0-9_]+)\s*\(", txt))
    return names


def test_library_builds_and_exports_every_declared_symbol():
    from mnmgdatalog_b200 import build, capi
    build.build()
    lib = C.CDLL(capi.LIB_PATH)
    declared = _declared_symbols()
    assert declared, "no declarations parsed"
    missing = [s for s in sorted(declared) if not hasattr(lib, s)]
    assert not missing, missing
    assert declared == set(capi.EXPORTS)


def test_generate_rows_matches_c_library_rand():
    from mnmgdatalog_b200 import generate_rows
    from oracle import cpu
    for rows, rng in ((1, 7), (1000, 100), (50000, 1000000)):
        assert np.array_equal(generate_rows(rows, rng, 1), cpu.generate_rows(rows, rng))


def test_status_strings_and_version():
    from mnmgdatalog_b200 import capi
    L = capi.lib()
    assert L.dl_version().startswith(b"mnmgdl")
    for s in range(8):
        assert L.dl_status_string(s)


def test_invalid_arguments_are_rejected_without_a_device():
    from mnmgdatalog_b200 import capi
    L = capi.lib()
    assert L.dl_context_create(0, None, None) == 1  # out == NULL
    assert L.dl_run_program(None, 0, None, 0, 0, None, None) == 1
    assert L.dl_generate_rows(-1, 5, 1, None) == 1
    assert b"invalid" in L.dl_last_error() or L.dl_last_error()


@pytest.mark.skipif(os.environ.get("CUDA_VISIBLE_DEVICES", None) is None and
                    os.path.exists("/dev/nvidia0"), reason="a GPU is visible")
def test_no_device_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    from mnmgdatalog_b200 import DatalogError, Engine
    with pytest.raises(DatalogError):
        Engine(0)


def test_oracle_ops_restatement_basics():
    from oracle import ops
    a = np.array([[3, 1], [1, 2], [1, 2], [-1, 5], [1, -4]], np.int32)
    assert ops.sort_unique(a).tolist() == [[-1, 5], [1, -4], [1, 2], [3, 1]]
    b = ops.sort_unique(np.array([[1, 2], [9, 9]], np.int32))
    assert ops.set_difference(ops.sort_unique(a), b).tolist() == [[-1, 5], [1, -4], [3, 1]]
    assert ops.join(np.array([[1, 5], [1, 6], [2, 7]]), np.array([[1, 9], [3, 0], [2, 8]])).tolist() == \
        [[5, 9], [6, 9], [7, 8]]


def test_profile_classes_match_the_ncu_summary_classes():
    """Every kernel class of the library's live profile (dl_context.cu) is a
    class the ncu launch-list summary (mnmgdatalog_b200/profiling.py) can
    attribute kernels to, and the summary names no class the library lacks,
    so the committed launch lists and the bench's profile speak of the same
    classes."""
    import re

    from mnmgdatalog_b200 import profiling
    src = open(os.path.join(ROOT, "mnmgdatalog_b200", "csrc", "dl_context.cu")).read()
    block = src[src.index("static const char *names[K_COUNT]"):]
    block = block[:block.index("};")]
    lib_classes = {c for c in re.findall(r'"([a-z_A-Z]+)"', block) if not c.startswith("host_")}
    ncu_classes = {cls for _, cls in profiling.CLASSES} | {"prep"}
    assert ncu_classes <= lib_classes, sorted(ncu_classes - lib_classes)
    # a class with no pattern would have its kernels counted as "prep" in the summary
    assert not lib_classes - ncu_classes, sorted(lib_classes - ncu_classes)


@pytest.mark.parametrize("lang,std", [("c", "-std=c99"), ("c++", "-std=c++17")])
def test_public_header_compiles_as_plain_c_and_cpp(tmp_path, lang, std):
    """include/mnmgdl.h is usable from C (cgo, FFI generators) and C++ alike:
    it compiles with -pedantic and every warning enabled."""
    import shutil
    import subprocess
    cc = shutil.which("gcc" if lang == "c" else "g++")
    if cc is None:
        pytest.skip("no host compiler")
    src = tmp_path / ("use." + ("c" if lang == "c" else "cpp"))
    src.write_text('#include "mnmgdl.h"\n'
                   "int main(void) {\n"
                   "    dl_tuning t; dl_options o; dl_run_info i; dl_kernel_stat k;\n"
                   "    (void) t; (void) o; (void) i; (void) k;\n"
                   "    return dl_status_string(DL_OK) == 0;\n"
                   "}\n")
    r = subprocess.run([cc, std, "-Wall", "-Wextra", "-pedantic", "-Werror", "-fsyntax-only",
                        "-I", os.path.join(ROOT, "include"), str(src)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
