"""ORACLE - test infrastructure only: a numpy builder of Freudenthal lower-star
boundary matrices, for the CPU baseline arm of bench.py.

It builds the same kind of input as the engine's own generator (a G^3 grid of
seeded Gaussian white noise smoothed by a Gaussian of the given sigma,
'reflect' boundary, truncated at 4 sigma; every vertex, edge, triangle and
tetrahedron of the Freudenthal (Kuhn) triangulation; each simplex valued by
its largest vertex value; columns ordered by (value, dimension, lexicographic
vertex tuple), faces ascending, int32) without loading any of the engine's
libraries, so the baseline arm runs on plain numpy and the oracle.  Sizes and
the value distribution match the engine's generator exactly; the values
themselves come from numpy's generator, so individual columns differ.

The reference itself reads such matrices from PHAT files written by external
tools (src/main.cu:90-167); its CPU reduction is what the oracle restates.
"""
from __future__ import annotations

import numpy as np


def field(grid: int, sigma: float, seed: int) -> np.ndarray:
    """Smoothed white noise, shape (grid, grid, grid) indexed [z, y, x], float32."""
    from scipy.ndimage import gaussian_filter

    rng = np.random.default_rng(seed)
    f = rng.standard_normal((grid, grid, grid))
    return gaussian_filter(f, sigma, mode="reflect", truncate=4.0).astype(np.float32)


def _offset(mask: int, g: int) -> int:
    return (mask & 1) + g * ((mask >> 1) & 1) + g * g * ((mask >> 2) & 1)


def _bases(mask: int, g: int) -> np.ndarray:
    """Vertices v for which v + offset(mask) stays inside the grid."""
    lim = [g - 1 if (mask >> b) & 1 else g for b in range(3)]
    z, y, x = np.meshgrid(np.arange(lim[2]), np.arange(lim[1]), np.arange(lim[0]), indexing="ij")
    return (x + g * y + g * g * z).ravel().astype(np.int64)


def lowerstar(grid: int, sigma: float, seed: int):
    """(dims int32, col_ptr int64, rows int32) of the lower-star filtration."""
    g = grid
    val = field(g, sigma, seed).ravel()
    val = np.where(val == 0, np.float32(0), val)  # -0 reads as +0
    nv = g ** 3
    # simplices as (base vertex, chain of offset masks); keys identify them
    recs = []  # (key array, dim, tuple columns list)
    # vertices
    v = np.arange(nv, dtype=np.int64)
    recs.append((v, 0, [v]))
    chains1 = list(range(1, 8))
    chains2 = [(a, b) for b in range(1, 8) for a in range(1, 8) if a != b and (a & b) == a]
    chains3 = [(a, b, 7) for (a, b) in chains2 if b != 7 and bin(a).count("1") == 1 and bin(b).count("1") == 2]
    for m in chains1:
        b = _bases(m, g)
        recs.append((b * 8 + m, 1, [b, b + _offset(m, g)]))
    for (a, m) in chains2:
        b = _bases(m, g)
        recs.append((b * 64 + a * 8 + m, 2, [b, b + _offset(a, g), b + _offset(m, g)]))
    for (a, m, t) in chains3:
        b = _bases(t, g)
        recs.append((b * 512 + a * 64 + m * 8 + t, 3, [b, b + _offset(a, g), b + _offset(m, g), b + _offset(t, g)]))
    # per dimension: keys, tuples, values
    keys, dims, vals, tups = [], [], [], []
    for key, d, t in recs:
        keys.append((d, key))
        dims.append(np.full(key.shape[0], d, np.int32))
        vv = val[t[0]]
        for c in t[1:]:
            vv = np.maximum(vv, val[c])
        vals.append(vv)
        pad = t + [np.full(key.shape[0], -1, np.int64)] * (4 - len(t))
        tups.append(np.stack(pad, axis=1))
    dim = np.concatenate(dims)
    value = np.concatenate(vals)
    tup = np.concatenate(tups)
    order = np.lexsort((tup[:, 3], tup[:, 2], tup[:, 1], tup[:, 0], dim, value))
    n = order.shape[0]
    rank = np.empty(n, np.int64)
    rank[order] = np.arange(n)
    # column index of every simplex, by dimension and key
    starts = np.cumsum([0] + [k.shape[0] for (_, k) in keys])
    sorted_keys = []
    for i, (d, k) in enumerate(keys):
        sorted_keys.append((d, k, rank[starts[i]:starts[i + 1]]))

    by_dim = {}
    for d in (1, 2):
        ks = np.concatenate([k for (dd, k, _) in sorted_keys if dd == d])
        rs = np.concatenate([r for (dd, _, r) in sorted_keys if dd == d])
        o = np.argsort(ks, kind="stable")
        by_dim[d] = (ks[o], rs[o])

    def lookup(d, key):
        ks, rs = by_dim[d]
        pos = np.searchsorted(ks, key)
        assert np.all(ks[pos] == key)
        return rs[pos]

    # edges: both vertices
    # triangles / tetrahedra: the face with base and masks given by the chain
    cols = {}
    for i, (key, d, t) in enumerate(recs):
        cnt = key.shape[0]
        if d == 1:
            f = np.stack([t[0], t[1]], axis=1)
        elif d == 2:
            b = key // 64
            a = (key // 8) % 8
            m = key % 8
            f = np.stack([lookup(1, (b + _off_arr(a, g)) * 8 + (m & ~a)), lookup(1, b * 8 + m),
                          lookup(1, b * 8 + a)], axis=1)
        elif d == 3:
            b = key // 512
            a = (key // 64) % 8
            m = (key // 8) % 8
            t7 = key % 8
            f = np.stack([lookup(2, (b + _off_arr(a, g)) * 64 + (m & ~a) * 8 + (t7 & ~a)),
                          lookup(2, b * 64 + m * 8 + t7), lookup(2, b * 64 + a * 8 + t7),
                          lookup(2, b * 64 + a * 8 + m)], axis=1)
        else:
            f = np.zeros((cnt, 0), np.int64)
        if d == 1:
            f = rank[f]  # vertices: the column of vertex v is rank[v] (vertex records come first)
        cols[i] = (rank[starts[i]:starts[i + 1]], np.sort(f, axis=1))
    col_of = np.concatenate([cols[i][0] for i in range(len(recs))])
    width = np.concatenate([np.full(cols[i][0].shape[0], cols[i][1].shape[1], np.int64) for i in range(len(recs))])
    lens = np.empty(n, np.int64)
    lens[col_of] = width
    col_ptr = np.zeros(n + 1, np.int64)
    np.cumsum(lens, out=col_ptr[1:])
    rows = np.empty(col_ptr[-1], np.int32)
    for i in range(len(recs)):
        c, f = cols[i]
        if f.shape[1] == 0:
            continue
        idx = col_ptr[c][:, None] + np.arange(f.shape[1])[None, :]
        rows[idx.ravel()] = f.ravel()
    dims_out = np.empty(n, np.int32)
    dims_out[col_of] = np.concatenate([np.full(cols[i][0].shape[0], recs[i][1], np.int32) for i in range(len(recs))])
    return dims_out, col_ptr, rows


def _off_arr(mask, g):
    mask = np.asarray(mask, np.int64)
    return (mask & 1) + g * ((mask >> 1) & 1) + g * g * ((mask >> 2) & 1)
