"""CPU tests of the complex builders' definition: the host generator (the
reference the device builders are compared with bit for bit) against a
brute-force construction written independently here - every clique of the
graph, values as maxima of float32 edge values, columns sorted by (value,
dimension, vertex tuple), facets looked up by tuple."""

import numpy as np
import pytest

from specseqplusplus_b200 import gen


def _matrix_from_simplices(simplices):
    """simplices: list of (value, tuple of vertices ascending)."""
    order = sorted(simplices, key=lambda s: (s[0], len(s[1]), s[1]))
    index = {s[1]: i for i, s in enumerate(order)}
    dims = np.array([len(t) - 1 for _, t in order], dtype=np.int32)
    col_ptr = [0]
    rows = []
    for _, t in order:
        if len(t) > 1:
            rows.extend(sorted(index[t[:q] + t[q + 1:]] for q in range(len(t))))
        col_ptr.append(len(rows))
    values = np.array([v for v, _ in order], dtype=np.float32)
    return dims, np.array(col_ptr, dtype=np.int64), np.array(rows, dtype=np.int32), values


def _cliques(n, adj, weight, maxdim, vertex_value):
    out = [(vertex_value(v), (v,)) for v in range(n)]
    nbrs = [sorted(u for u in range(v + 1, n) if adj[v][u]) for v in range(n)]

    def grow(t, w, cand):
        out.append((w, t))
        if len(t) > maxdim:
            return
        for u in cand:
            wu = w
            for x in t:
                wu = max(wu, weight[x][u])
            grow(t + (u,), wu, [c for c in cand if c > u and adj[u][c]])

    if maxdim >= 1:
        for v in range(n):
            for u in nbrs[v]:
                grow((v, u), weight[v][u], [c for c in nbrs[v] if c > u and adj[u][c]])
    return out


def _brute_rips(pts, radius, maxdim):
    pts = np.asarray(pts, dtype=np.float32)
    n, dim = pts.shape
    adj = [[False] * n for _ in range(n)]
    weight = [[np.float32(0)] * n for _ in range(n)]
    r = np.float32(radius)
    for i in range(n):
        for j in range(i + 1, n):
            s = np.float32(0.0)
            for d in range(dim):
                t = np.float32(pts[i, d] - pts[j, d])
                s = np.float32(s + np.float32(t * t))
            dist = np.float32(np.sqrt(s))
            if dist <= r:
                adj[i][j] = adj[j][i] = True
                weight[i][j] = weight[j][i] = dist
    return _matrix_from_simplices(_cliques(n, adj, weight, maxdim, lambda v: np.float32(0.0)))


def _brute_lowerstar(field, maxdim):
    f = np.asarray(field, dtype=np.float32)
    gz, gy, gx = f.shape
    val = np.where(f == 0, np.float32(0.0), f).reshape(-1)  # -0 read as +0
    n = gx * gy * gz
    coord = [(v % gx, (v // gx) % gy, v // (gx * gy)) for v in range(n)]
    adj = [[False] * n for _ in range(n)]
    weight = [[np.float32(0)] * n for _ in range(n)]
    for a in range(n):
        for b in range(a + 1, n):
            off = [coord[b][k] - coord[a][k] for k in range(3)]
            if all(o in (0, 1) for o in off) or all(o in (0, -1) for o in off):
                adj[a][b] = adj[b][a] = True
                weight[a][b] = weight[b][a] = max(val[a], val[b])
    return _matrix_from_simplices(_cliques(n, adj, weight, maxdim, lambda v: val[v]))


def _same(m, ref):
    dims, col_ptr, rows, values = ref
    assert np.array_equal(m.dims, dims)
    assert np.array_equal(m.col_ptr, col_ptr)
    assert np.array_equal(m.rows, rows)
    assert np.array_equal(m.values.view(np.uint32), values.view(np.uint32))


@pytest.mark.parametrize("case", range(6))
def test_rips_points_match_brute_force(case):
    rng = np.random.default_rng(100 + case)
    n, dim = [(25, 3), (30, 2), (18, 1), (22, 3), (28, 2), (16, 3)][case]
    pts = rng.random((n, dim), dtype=np.float32)
    if case == 3:  # unbounded coordinates, negative values
        pts = rng.normal(size=(n, dim)).astype(np.float32) * 3
    if case == 4:  # duplicated points: zero-length edges
        pts[10:20] = pts[0:10]
    radius = [0.45, 0.3, 0.2, 2.5, 0.25, 10.0][case]
    maxdim = [3, 2, 1, 3, 3, 3][case]
    _same(gen.rips_from_points(pts, radius, maxdim), _brute_rips(pts, radius, maxdim))


def test_rips_seeded_equals_its_points():
    for args in [(40, 3, 5, 0.4, 3), (60, 2, 6, 0.2, 2)]:
        a = gen.rips(*args)
        b = gen.rips_from_points(gen.points(args[0], args[1], args[2]), args[3], args[4])
        assert np.array_equal(a.rows, b.rows) and np.array_equal(a.values, b.values)
    _same(gen.rips(30, 3, 9, 0.45, 3), _brute_rips(gen.points(30, 3, 9), 0.45, 3))


@pytest.mark.parametrize("shape", [(2, 3, 4), (1, 4, 5), (3, 3, 3), (2, 2, 6)])
def test_lowerstar_field_matches_brute_force(shape):
    rng = np.random.default_rng(sum(shape))
    f = rng.normal(size=shape).astype(np.float32)
    _same(gen.lowerstar_from_field(f, 3), _brute_lowerstar(f, 3))


def test_lowerstar_ties_and_signed_zero():
    rng = np.random.default_rng(7)
    f = rng.integers(-2, 3, size=(3, 3, 4)).astype(np.float32)  # many equal values
    f[f == 0] = -0.0
    f[0, 0, 0] = 0.0
    _same(gen.lowerstar_from_field(f, 3), _brute_lowerstar(f, 3))
    _same(gen.lowerstar_from_field(f, 2), _brute_lowerstar(f, 2))


def test_lowerstar_seeded_equals_its_field():
    a = gen.lowerstar(6, 1.0, 3)
    b = gen.lowerstar_from_field(gen.field(6, 1.0, 3), 3)
    assert np.array_equal(a.rows, b.rows) and np.array_equal(a.values, b.values)
    assert int(np.sum((-1) ** a.dims.astype(np.int64))) == 1  # the triangulated cube is contractible
    assert np.count_nonzero(a.dims == 3) == 6 * 5 ** 3  # six tetrahedra per voxel


def test_rejects_bad_input():
    with pytest.raises(ValueError):
        gen.rips_from_points(np.array([[0.0, np.nan]], dtype=np.float32), 0.5, 2)
    with pytest.raises(ValueError):
        gen.lowerstar_from_field(np.full((2, 2, 2), np.nan, dtype=np.float32), 3)
