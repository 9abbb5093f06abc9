"""numpy restatements of the reference's relational idioms -- TEST INFRASTRUCTURE.

Relations are (n, 2) int32 arrays in the reference's Entity layout. Order is
set_cmp (common/utils.cu:114-124): signed key, then signed value.
"""
from __future__ import annotations

import numpy as np


def _key(rel: np.ndarray) -> np.ndarray:
    r = np.asarray(rel, dtype=np.int64).reshape(-1, 2)
    hi = (r[:, 0] + 2**31).astype(np.uint64)
    lo = (r[:, 1] + 2**31).astype(np.uint64)
    return (hi << np.uint64(32)) | lo


def _rows(keys: np.ndarray) -> np.ndarray:
    k = np.asarray(keys, dtype=np.uint64)
    hi = (k >> np.uint64(32)).astype(np.int64) - 2**31
    lo = (k & np.uint64(0xFFFFFFFF)).astype(np.int64) - 2**31
    return np.stack([hi, lo], axis=1).astype(np.int32)


def sort(rel):
    """thrust::sort(set_cmp)."""
    return _rows(np.sort(_key(rel), kind="stable"))


def sort_unique(rel):
    """thrust::sort(set_cmp) + thrust::unique(is_equal) (tc.cu:250-253)."""
    return _rows(np.unique(_key(rel)))


def set_difference(a, b):
    """thrust::set_difference(set_cmp) for duplicate-free sorted inputs (tc.cu:260-263)."""
    ka, kb = _key(a), _key(b)
    return _rows(ka[~np.isin(ka, kb)])


def merge(a, b):
    """thrust::merge(set_cmp): stable, ties take `a` first (tc.cu:276-279)."""
    ka, kb = _key(a), _key(b)
    both = np.concatenate([ka, kb])
    src = np.concatenate([np.zeros(len(ka), np.int8), np.ones(len(kb), np.int8)])
    order = np.lexsort((src, both))
    return _rows(both[order])


def unique_by_key_min(rel):
    """thrust::unique(is_equal_key) on set_cmp-sorted input (wcc.cu:320-323)."""
    r = np.asarray(rel, dtype=np.int32).reshape(-1, 2)
    if len(r) == 0:
        return r
    keep = np.ones(len(r), bool)
    keep[1:] = r[1:, 0] != r[:-1, 0]
    return r[keep]


def remove_self_pairs(rel):
    """thrust::remove_if(is_key_equal_value) (sg.cu:176-179)."""
    r = np.asarray(rel, dtype=np.int32).reshape(-1, 2)
    return r[r[:, 0] != r[:, 1]]


def join(rel, probe):
    """get_join (common/join.cu:1-87): for probe (k, v) and rel (k, w) emit
    (w, v); grouped by probe row in probe order, matches by ascending w."""
    rel = np.asarray(rel, dtype=np.int32).reshape(-1, 2)
    probe = np.asarray(probe, dtype=np.int32).reshape(-1, 2)
    srt = rel[np.lexsort((rel[:, 1], rel[:, 0]))]
    keys = srt[:, 0]
    lo = np.searchsorted(keys, probe[:, 0], side="left")
    hi = np.searchsorted(keys, probe[:, 0], side="right")
    cnt = hi - lo
    out = np.empty((int(cnt.sum()), 2), dtype=np.int32)
    pos = 0
    for i in np.nonzero(cnt)[0]:
        c = int(cnt[i])
        out[pos:pos + c, 0] = srt[lo[i]:hi[i], 1]
        out[pos:pos + c, 1] = probe[i, 1]
        pos += c
    return out
