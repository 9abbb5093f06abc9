"""dl_sort_unique_noalloc, the allocation-free sort + unique, through the C-ABI.

Some users of this library cannot allocate device memory when they sort: their
GPU memory is already reserved by another allocator's pool, they must keep a
fixed footprint after start-up, or they cannot afford the device-wide
synchronisation an allocation may cause. This file checks that the entry point
written for them returns exactly what dl_sort_unique returns, and what the
oracle's restatement of the reference's thrust::sort + thrust::unique returns,
on two calls in a row (the second reusing the scratch array the first left
behind); that neither the first nor the second call changes the device's free
memory; and that inputs beyond its fixed maximum are refused with a clear
error.

The file is named to be collected last, so a run that stops at the first
failure has already run every other test.
"""
import ctypes as C
import os
import subprocess
import sys
import textwrap

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu


def _rows(rng, n, lo, hi):
    return rng.integers(lo, hi, size=(n, 2), dtype=np.int64).astype(np.int32)


@pytest.mark.parametrize("n,lo,hi", [(1, -5, 5), (1000, -100, 100), (300_000, -2**31, 2**31),
                                     (1 << 20, -3000, 3000)])
def test_noalloc_matches_sort_unique_on_two_calls(n, lo, hi):
    import torch

    from mnmgdatalog_b200 import Engine, capi
    from oracle import ops
    L = capi.lib()
    assert n <= L.dl_sort_unique_noalloc_max_rows()
    rng = np.random.default_rng(n)
    with Engine(0) as eng:
        for call in range(2):
            a = _rows(rng, n, lo, hi)
            mine = torch.from_numpy(a).cuda()
            theirs = mine.clone()
            torch.cuda.synchronize()
            n_out = C.c_int64()
            st = L.dl_sort_unique_noalloc(C.c_void_p(mine.data_ptr()), n, C.byref(n_out), None)
            assert st == 0, L.dl_last_error()
            got = mine[: n_out.value]
            want = eng.sort_unique(theirs)
            assert n_out.value == len(want), f"call {call}"
            assert torch.equal(got, want), f"call {call}: differs from dl_sort_unique"
            assert np.array_equal(got.cpu().numpy(), ops.sort_unique(a)), f"call {call}: differs from the oracle"


# Run in a fresh process without torch, with every CUDA module loaded when the
# library's runtime starts (CUDA_MODULE_LOADING=EAGER), so that the first call
# cannot hide an allocation behind the loading of the library's device code.
_PROBE = textwrap.dedent(r"""
    import ctypes as C, glob, json, os, sys
    import numpy as np
    sys.path.insert(0, sys.argv[1])
    from mnmgdatalog_b200 import capi
    from oracle import ops
    cands = sorted(glob.glob("/usr/local/cuda/lib64/libcudart.so*")) + sorted(glob.glob(
        os.path.join(sys.prefix, "lib", "python*", "site-packages", "nvidia", "cuda_runtime", "lib", "libcudart.so*")))
    rt = C.CDLL(cands[0])
    assert rt.cudaSetDevice(0) == 0 and rt.cudaFree(None) == 0
    L = capi.lib()
    h = C.c_void_p()
    assert L.dl_context_create(0, None, C.byref(h)) == 0   # starts the library's runtime: all modules load now
    assert L.dl_context_destroy(h) == 0
    n = 200_000
    rng = np.random.default_rng(7)
    dptr = C.c_void_p()
    assert rt.cudaMalloc(C.byref(dptr), C.c_size_t(n * 8)) == 0
    def free_bytes():
        assert rt.cudaDeviceSynchronize() == 0
        f, t = C.c_size_t(), C.c_size_t()
        assert rt.cudaMemGetInfo(C.byref(f), C.byref(t)) == 0
        return f.value
    out = {"free": [free_bytes()], "ok": []}
    for call in range(2):
        a = rng.integers(-5000, 5000, size=(n, 2), dtype=np.int64).astype(np.int32)
        assert rt.cudaMemcpy(dptr, a.ctypes.data_as(C.c_void_p), C.c_size_t(n * 8), 1) == 0
        k = C.c_int64()
        st = L.dl_sort_unique_noalloc(dptr, n, C.byref(k), None)
        assert st == 0, L.dl_last_error()
        out["free"].append(free_bytes())
        got = np.empty((k.value, 2), dtype=np.int32)
        assert rt.cudaMemcpy(got.ctypes.data_as(C.c_void_p), dptr, C.c_size_t(k.value * 8), 2) == 0
        out["ok"].append(bool(np.array_equal(got, ops.sort_unique(a))))
    print(json.dumps(out))
""")


def test_noalloc_first_and_second_call_allocate_nothing():
    env = dict(os.environ, CUDA_MODULE_LOADING="EAGER")
    r = subprocess.run([sys.executable, "-c", _PROBE, ROOT], capture_output=True, text=True, timeout=300, env=env)
    assert r.returncode == 0, r.stderr[-3000:]
    import json
    res = json.loads(r.stdout.strip().splitlines()[-1])
    assert res["ok"] == [True, True]
    f0, f1, f2 = res["free"]
    assert f1 == f0, f"the first call changed free device memory by {f0 - f1} bytes"
    assert f2 == f1, f"the second call changed free device memory by {f1 - f2} bytes"


def test_noalloc_refuses_more_than_its_maximum():
    import torch

    from mnmgdatalog_b200 import capi
    L = capi.lib()
    m = L.dl_sort_unique_noalloc_max_rows()
    t = torch.zeros((m + 1, 2), dtype=torch.int32, device="cuda")
    n_out = C.c_int64(-1)
    assert L.dl_sort_unique_noalloc(C.c_void_p(t.data_ptr()), m + 1, C.byref(n_out), None) == 1
    assert b"at most" in L.dl_last_error()
