"""Relational operators of the C-ABI against the numpy restatement of the
reference's thrust idioms and hash join (bit-exact)."""
import numpy as np
import pytest

from oracle import ops

pytestmark = pytest.mark.gpu

SIZES = [0, 1, 2, 7, 100, 4095, 4096, 4097, 6143, 6144, 6145, 50_000, 1_000_003]


def T(a):
    import torch
    a = np.ascontiguousarray(np.asarray(a, dtype=np.int32).reshape(-1, 2))
    return torch.from_numpy(a).cuda()


def H(t):
    return t.cpu().numpy().reshape(-1, 2)


def rand_rel(rng, n, lo=-1000, hi=1000):
    return rng.integers(lo, hi, size=(n, 2), dtype=np.int64).astype(np.int32)


@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("span", ["narrow", "full"])
def test_sort_unique(engine, n, span):
    rng = np.random.default_rng(n + (7 if span == "full" else 0))
    a = rand_rel(rng, n, -2**31, 2**31) if span == "full" else rand_rel(rng, n, -50, 50)
    got = H(engine.sort_unique(T(a)))
    assert np.array_equal(got, ops.sort_unique(a))


@pytest.mark.parametrize("n", [0, 1, 5000, 300_000])
def test_sort_keeps_duplicates(engine, n):
    rng = np.random.default_rng(11)
    a = rand_rel(rng, n, -5, 5)
    assert np.array_equal(H(engine.sort(T(a))), ops.sort(a))


def test_sort_constant_and_extreme_values(engine):
    a = np.array([[-2**31, 2**31 - 1]] * 9000 + [[2**31 - 1, -2**31]] * 10 + [[-1, -1]] * 5, np.int32)
    assert np.array_equal(H(engine.sort_unique(T(a))), ops.sort_unique(a))
    c = np.full((20000, 2), 42, np.int32)
    assert np.array_equal(H(engine.sort_unique(T(c))), [[42, 42]])


@pytest.mark.parametrize("na,nb", [(0, 0), (0, 10), (10, 0), (1000, 1000), (70_000, 5_000), (3_000, 200_000)])
def test_set_difference(engine, na, nb):
    rng = np.random.default_rng(na * 3 + nb)
    a = ops.sort_unique(rand_rel(rng, na, -300, 300))
    b = ops.sort_unique(np.concatenate([a[: len(a) // 2], rand_rel(rng, nb, -300, 300)]))
    got = H(engine.set_difference(T(a), T(b)))
    assert np.array_equal(got, ops.set_difference(a, b))


@pytest.mark.parametrize("na,nb", [(0, 0), (0, 5), (5, 0), (4096, 4096), (100_000, 33_333)])
def test_merge(engine, na, nb):
    rng = np.random.default_rng(na + 5 * nb)
    a = ops.sort(rand_rel(rng, na, -40, 40))
    b = ops.sort(rand_rel(rng, nb, -40, 40))
    assert np.array_equal(H(engine.merge(T(a), T(b))), ops.merge(a, b))


@pytest.mark.parametrize("nf,nj", [(0, 0), (0, 100), (100, 0), (5000, 5000), (500_000, 120_000), (20, 300_000)])
def test_diff_merge(engine, nf, nj):
    rng = np.random.default_rng(nf + nj)
    full = ops.sort_unique(rand_rel(rng, nf, -800, 800))
    j = ops.sort(np.concatenate([full[: len(full) // 3], rand_rel(rng, nj, -800, 800)]))
    fo, do = engine.diff_merge(T(full), T(j))
    assert np.array_equal(H(do), ops.set_difference(ops.sort_unique(j), full))
    assert np.array_equal(H(fo), ops.sort_unique(np.concatenate([full, j])))


@pytest.mark.parametrize("n", [0, 1, 10_000, 400_000])
def test_unique_by_key_min(engine, n):
    rng = np.random.default_rng(n)
    a = ops.sort(rand_rel(rng, n, -500, 500))
    assert np.array_equal(H(engine.unique_by_key_min(T(a))), ops.unique_by_key_min(a))


@pytest.mark.parametrize("n", [0, 3, 10_000, 400_000])
def test_remove_self_pairs(engine, n):
    rng = np.random.default_rng(n + 1)
    a = rand_rel(rng, n, -20, 20)
    assert np.array_equal(H(engine.remove_self_pairs(T(a))), ops.remove_self_pairs(a))


@pytest.mark.parametrize("nr,np_", [(0, 10), (10, 0), (1, 1), (1000, 1000), (50_000, 20_000), (200_000, 300_000)])
@pytest.mark.parametrize("lf", [0.0, 0.6, 0.9])
def test_hash_join(engine, nr, np_, lf):
    rng = np.random.default_rng(nr + np_)
    rel = rand_rel(rng, nr, -1, 3000)           # includes key -1 (the reference's empty sentinel)
    if nr > 10:
        rel[:10, 0] = 7                         # a hub key
    probe = rand_rel(rng, np_, -1, 3000)
    ht = engine.get_hash_table(T(rel), lf)
    assert ht.rows == nr
    got = H(engine.get_join(ht, T(probe)))
    ht.close()
    assert np.array_equal(got, ops.join(rel, probe))


@pytest.mark.parametrize("nr,np_", [(0, 10), (5, 5), (30_000, 70_000)])
def test_sorted_join(engine, nr, np_):
    rng = np.random.default_rng(3 * nr + np_)
    rel = ops.sort(rand_rel(rng, nr, -100, 2000))
    probe = rand_rel(rng, np_, -100, 2000)
    got = H(engine.get_join_nl(T(rel), T(probe)))
    assert np.array_equal(got, ops.join(rel, probe))


def test_skewed_join_hub(engine):
    # one key with 200k matches probed 50 times: load-balanced emit
    rel = np.stack([np.zeros(200_000, np.int32), np.arange(200_000, dtype=np.int32)], 1)
    probe = np.stack([np.zeros(50, np.int32), np.arange(50, dtype=np.int32)], 1)
    ht = engine.get_hash_table(T(rel))
    got = H(engine.get_join(ht, T(probe)))
    ht.close()
    assert got.shape == (10_000_000, 2)
    assert np.array_equal(got, ops.join(rel, probe))


def test_diff_merge_across_epoch_wrap():
    """The 14-bit look-back epoch wraps after 16383 launches and the wrap
    clears the look-back buffer; the merge-path split points of the launch
    that wraps must survive it. On a fresh context every dl_diff_merge call
    takes exactly one epoch, so call 16384 is the one that wraps."""
    import ctypes as C

    import torch

    from mnmgdatalog_b200 import Engine
    from mnmgdatalog_b200.capi import check, lib
    rng = np.random.default_rng(5)
    full = ops.sort_unique(rand_rel(rng, 9000))
    j = ops.sort(rand_rel(rng, 5000))
    want_delta = ops.set_difference(ops.sort_unique(j), full)
    want_full = ops.sort_unique(np.concatenate([full, j]))
    with Engine(0) as eng:
        df, dj = T(full), T(j)
        fo = torch.empty((len(full) + len(j), 2), dtype=torch.int32, device="cuda")
        do = torch.empty((len(j), 2), dtype=torch.int32, device="cuda")
        n = C.c_int64()
        args = (eng.ctx, C.c_void_p(df.data_ptr()), len(full), C.c_void_p(dj.data_ptr()), len(j),
                C.c_void_p(fo.data_ptr()), C.c_void_p(do.data_ptr()), C.byref(n))
        torch.cuda.synchronize()
        for call in range(1, 16400):
            fo.zero_()
            eng.synchronize()
            check(lib().dl_diff_merge(*args))
            assert n.value == len(want_delta), call
            if call >= 16380 or call % 4096 == 0:
                eng.synchronize()
                assert np.array_equal(H(fo[: len(full) + n.value]), want_full), call
                assert np.array_equal(H(do[: n.value]), want_delta), call
