"""Seeded synthetic edge relations with the shapes of the reference's graphs.

The reference's headline graphs (com-dblp, fe_body, ...) are public datasets
that are not shipped here; these generators produce int32 edge rows of the
same scale and degree structure, deterministically from a seed:

* ``dag``        -- a DAG on 0..n-1: edge i->i+1 with probability p, plus
                    `extra` edges u->v, v uniform in (u, u+span]; duplicates
                    removed (the OL.cedge-scale TC input, ~5.5K edges).
* ``chung_lu``   -- a Chung-Lu power-law graph (expected degrees ~ rank^(-1/(gamma-1))),
                    each undirected edge stored once, oriented from the lower to
                    the higher node id of a seeded random relabelling, like
                    the once-per-edge storage of com-dblp; self loops and
                    duplicates removed.
* ``lattice3d``  -- an s^3 lattice with 6-neighbour directed edges kept with
                    probability p plus a fraction of random long edges (the
                    fe_body-like mesh of the SG config).
"""
from __future__ import annotations

import numpy as np


def _dedup(rows: np.ndarray) -> np.ndarray:
    if rows.size == 0:
        return rows.reshape(0, 2).astype(np.int32)
    key = (rows[:, 0].astype(np.int64) << 32) | (rows[:, 1].astype(np.int64) & 0xFFFFFFFF)
    _, idx = np.unique(key, return_index=True)
    return np.ascontiguousarray(rows[np.sort(idx)]).astype(np.int32)


def dag(n: int = 5000, p: float = 0.7, extra: int = 2000, span: int = 64, seed: int = 0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    chain = np.nonzero(rng.random(n - 1) < p)[0]
    e1 = np.stack([chain, chain + 1], axis=1)
    u = rng.integers(0, n, size=extra)
    v = u + rng.integers(1, span + 1, size=extra)
    keep = v < n
    e2 = np.stack([u[keep], v[keep]], axis=1)
    return _dedup(np.concatenate([e1, e2]).astype(np.int64))


def chung_lu(n: int = 317_000, m: int = 1_050_000, gamma: float = 2.5, orient_noise: float = 0.065,
             seed: int = 0) -> np.ndarray:
    """m distinct undirected edges, each stored once. An edge points from the
    endpoint with the smaller score to the larger, score = degree rank +
    orient_noise * n * U(0,1) (mostly hub -> leaf). At the defaults the
    closure holds ~1.9e9 tuples (com-dblp scale). Node ids are a seeded
    random relabelling of the ranks."""
    rng = np.random.default_rng(seed)
    w = np.arange(1, n + 1, dtype=np.float64) ** (-1.0 / (gamma - 1.0))
    cdf = np.cumsum(w)
    cdf /= cdf[-1]
    score = np.arange(n) + orient_noise * n * rng.random(n)
    ids = rng.permutation(n)
    out = np.zeros((0, 2), dtype=np.int64)
    while out.shape[0] < m:
        k = int((m - out.shape[0]) * 1.3) + 1024
        a = np.searchsorted(cdf, rng.random(k))
        b = np.searchsorted(cdf, rng.random(k))
        ok = a != b
        a, b = a[ok], b[ok]
        fwd = score[a] < score[b]
        src = np.where(fwd, a, b)
        dst = np.where(fwd, b, a)
        cand = np.concatenate([out, np.stack([src, dst], axis=1)])
        key = (cand[:, 0] << 32) | cand[:, 1]
        _, idx = np.unique(key, return_index=True)
        out = cand[np.sort(idx)]
    out = out[:m]
    return np.ascontiguousarray(ids[out]).astype(np.int32)


def lattice3d(side: int = 55, p: float = 0.15, long_frac: float = 0.01, seed: int = 0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    n = side ** 3
    idx = np.arange(n, dtype=np.int64)
    x, y, z = idx % side, (idx // side) % side, idx // (side * side)
    parts = []
    for dim, coord, step in ((0, x, 1), (1, y, side), (2, z, side * side)):
        for sgn in (1, -1):
            ok = (coord + sgn >= 0) & (coord + sgn < side)
            src = idx[ok]
            dst = src + sgn * step
            keep = rng.random(src.size) < p
            parts.append(np.stack([src[keep], dst[keep]], axis=1))
    local = np.concatenate(parts)
    nl = int(local.shape[0] * long_frac)
    lu = rng.integers(0, n, size=nl)
    lv = rng.integers(0, n, size=nl)
    ok = lu != lv
    rows = np.concatenate([local, np.stack([lu[ok], lv[ok]], axis=1)])
    return _dedup(rows)


def sized(program: str, edges: int, seed: int = 0) -> np.ndarray:
    """An input of about `edges` rows for one program, from the generators
    above: TC on a DAG (n = edges / 1.1, extra = 0.4 n), SG on a lattice
    (side = (edges / 0.9)^(1/3)), WCC on a Chung-Lu graph with exponent 2.3
    (n = edges / 3.3, the node/edge ratio of the TC-at-scale graph)."""
    if program == "tc":
        n = max(8, int(edges / 1.1))
        return dag(n=n, extra=int(0.4 * n), seed=seed)
    if program == "sg":
        return lattice3d(side=max(3, int(round((edges / 0.9) ** (1.0 / 3.0)))), seed=seed)
    if program == "wcc":
        return chung_lu(n=max(16, int(edges / 3.3)), m=edges, gamma=2.3, seed=seed)
    raise ValueError(program)


def log_uniform(count: int, lo: int, hi: int, rng: np.random.Generator) -> np.ndarray:
    return np.exp(rng.uniform(np.log(lo), np.log(hi), size=count)).astype(np.int64)


def batched_workload(count: int = 1024, lo: int = 1000, hi: int = 200_000, seed: int = 0) -> list:
    """The batched configuration: half TC on DAGs, half WCC on Chung-Lu
    graphs (exponent 2.3), edge counts log-uniform in [lo, hi].
    Returns [(program, edges), ...] with the TC instances first."""
    rng = np.random.default_rng(seed)
    sizes = log_uniform(count, lo, hi, rng)
    half = count // 2
    out = [("tc", sized("tc", int(sizes[i]), seed=seed * 100_003 + i)) for i in range(half)]
    out += [("wcc", sized("wcc", int(sizes[i]), seed=seed * 100_003 + i)) for i in range(half, count)]
    return out


CONFIGS = {
    # name: (program, generator, kwargs)
    "tc_dag_5k": ("tc", dag, {}),
    "tc_chung_lu_317k": ("tc", chung_lu, {}),
    "sg_lattice_55": ("sg", lattice3d, {}),
    # the TC-at-scale shape at 1/8 of the nodes (~3e7 closure tuples, a few
    # hundred MB: larger than L2, small enough for detailed counter captures)
    "tc_chung_lu_40k": ("tc", chung_lu, {"n": 40_000, "m": 132_500}),
    # 1/4 of the nodes (~1e8 closure tuples, ~4 GB on the device): join steps
    # of milliseconds for counter captures of the bit-matrix step
    "tc_chung_lu_80k": ("tc", chung_lu, {"n": 80_000, "m": 265_000}),
}


def make(name: str, seed: int = 0) -> tuple[str, np.ndarray]:
    prog, fn, kw = CONFIGS[name]
    return prog, fn(seed=seed, **kw)
