"""Test helpers: small complexes and independent reference computations."""
from __future__ import annotations

import itertools

import numpy as np

from specseqplusplus_b200.gen import BoundaryMatrix


def flag_complex(nverts, edges, maxdim):
    """All cliques up to maxdim of a graph, as sorted vertex tuples."""
    adj = {v: set() for v in range(nverts)}
    for u, v in edges:
        adj[u].add(v)
        adj[v].add(u)
    simplices = [(v,) for v in range(nverts)]
    layer = simplices
    for _ in range(maxdim):
        nxt = []
        for s in layer:
            common = set.intersection(*(adj[v] for v in s))
            for w in common:
                if w > s[-1]:
                    nxt.append(s + (w,))
        simplices += nxt
        layer = nxt
    return simplices


def random_filtration(simplices, rng):
    """A random linear extension of the face order (faces before cofaces)."""
    idx = {s: i for i, s in enumerate(simplices)}
    indeg = {s: len(s) if len(s) > 1 else 0 for s in simplices}
    cofaces = {s: [] for s in simplices}
    for s in simplices:
        if len(s) > 1:
            for k in range(len(s)):
                cofaces[s[:k] + s[k + 1:]].append(s)
    ready = [s for s in simplices if indeg[s] == 0]
    order = []
    while ready:
        j = int(rng.integers(len(ready)))
        s = ready.pop(j)
        order.append(s)
        for c in cofaces[s]:
            indeg[c] -= 1
            if indeg[c] == 0:
                ready.append(c)
    assert len(order) == len(simplices)
    del idx
    return order


def boundary_matrix(order):
    pos = {s: i for i, s in enumerate(order)}
    dims, cols = [], []
    for s in order:
        dims.append(len(s) - 1)
        if len(s) == 1:
            cols.append([])
        else:
            cols.append(sorted(pos[s[:k] + s[k + 1:]] for k in range(len(s))))
    return BoundaryMatrix.from_columns(dims, cols)


def random_complex(rng, nverts, p, maxdim):
    edges = [(u, v) for u in range(nverts) for v in range(u + 1, nverts) if rng.random() < p]
    return boundary_matrix(random_filtration(flag_complex(nverts, edges, maxdim), rng))


def dense_standard_pairs(m):
    """Standard column reduction (no clearing, no twist) on a dense GF(2) matrix."""
    n = m.ncols
    R = np.zeros((n, n), dtype=np.uint8)
    for j in range(n):
        R[m.column(j), j] = 1
    low_owner = {}
    pairs = []
    for j in range(n):
        while True:
            nz = np.nonzero(R[:, j])[0]
            if len(nz) == 0:
                break
            low = int(nz[-1])
            if low in low_owner:
                R[:, j] ^= R[:, low_owner[low]]
            else:
                low_owner[low] = j
                pairs.append((low, j))
                break
    return np.array(sorted(pairs), dtype=np.int64).reshape(-1, 2)


def gf2_rank(A):
    A = A.copy() % 2
    r = 0
    rows, cols = A.shape
    for c in range(cols):
        piv = None
        for i in range(r, rows):
            if A[i, c]:
                piv = i
                break
        if piv is None:
            continue
        A[[r, piv]] = A[[piv, r]]
        for i in range(rows):
            if i != r and A[i, c]:
                A[i] ^= A[r]
        r += 1
        if r == rows:
            break
    return r


def rank_pairs(m):
    """Pairing lemma: (i, j) is a pair iff the rank function of the lower-left
    submatrices has a unit jump there (independent of any reduction)."""
    n = m.ncols
    D = np.zeros((n, n), dtype=np.uint8)
    for j in range(n):
        D[m.column(j), j] = 1

    def rk(i, j):  # rank of rows i.., columns ..j
        if i >= n or j < 0:
            return 0
        return gf2_rank(D[i:, : j + 1])

    pairs = []
    for j in range(n):
        for i in m.column(j):
            pass
        for i in range(j):
            if rk(i, j) - rk(i + 1, j) - rk(i, j - 1) + rk(i + 1, j - 1) == 1:
                pairs.append((i, j))
    return np.array(sorted(pairs), dtype=np.int64).reshape(-1, 2)


def essentials_from_pairs(n, pairs, dropped=None):
    paired = np.zeros(n, dtype=bool)
    if len(pairs):
        paired[pairs[:, 0]] = True
        paired[pairs[:, 1]] = True
    if dropped is not None:
        paired |= dropped
    return np.nonzero(~paired)[0].astype(np.int64)
