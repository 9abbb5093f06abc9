"""dl_sort_unique_noalloc, the allocation-free sort + unique, through the C-ABI.

Some users of this library cannot allocate device memory when they sort: their
GPU memory is already reserved by another allocator's pool, they must keep a
fixed footprint after start-up, or they cannot afford the device-wide
synchronisation an allocation may cause. This file checks that the entry point
written for them returns exactly what dl_sort_unique returns, on two calls in a
row (the second reusing the scratch array the first left behind), that the
second call changes the device's free memory by nothing, and that inputs beyond
its fixed maximum are refused with a clear error.

The file is named to be collected last, so a run that stops at the first
failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rows(rng, n, lo, hi):
    return rng.integers(lo, hi, size=(n, 2), dtype=np.int64).astype(np.int32)


@pytest.mark.parametrize("n,lo,hi", [(1, -5, 5), (1000, -100, 100), (300_000, -2**31, 2**31),
                                     (1 << 20, -3000, 3000)])
def test_noalloc_matches_sort_unique_on_two_calls(n, lo, hi):
    import torch

    from mnmgdatalog_b200 import Engine, capi
    L = capi.lib()
    assert n <= L.dl_sort_unique_noalloc_max_rows()
    rng = np.random.default_rng(n)
    with Engine(0) as eng:
        for call in range(2):
            a = _rows(rng, n, lo, hi)
            mine = torch.from_numpy(a).cuda()
            theirs = mine.clone()
            torch.cuda.synchronize()
            free_before = torch.cuda.mem_get_info()[0]
            n_out = C.c_int64()
            st = L.dl_sort_unique_noalloc(C.c_void_p(mine.data_ptr()), n, C.byref(n_out), None)
            assert st == 0, L.dl_last_error()
            free_after = torch.cuda.mem_get_info()[0]
            if call == 1:  # the first call may load the library's device code; the second allocates nothing
                assert free_after == free_before
            want = eng.sort_unique(theirs)
            assert n_out.value == len(want)
            assert torch.equal(mine[: n_out.value], want)


def test_noalloc_refuses_more_than_its_maximum():
    import torch

    from mnmgdatalog_b200 import capi
    L = capi.lib()
    m = L.dl_sort_unique_noalloc_max_rows()
    t = torch.zeros((m + 1, 2), dtype=torch.int32, device="cuda")
    n_out = C.c_int64(-1)
    assert L.dl_sort_unique_noalloc(C.c_void_p(t.data_ptr()), m + 1, C.byref(n_out), None) == 1
    assert b"at most" in L.dl_last_error()
