"""GPU tests of the device complex builders (sspp_load_rips / sspp_load_lowerstar
through the C ABI): the matrix built on the device equals the host generator's
bit for bit (dims, col_ptr, rows and float32 values), and reducing it gives the
same pairs as reducing the host matrix.  The host generator itself is pinned
against a brute-force clique construction on the CPU (test_gen.py)."""
import numpy as np
import pytest

import oracle
from specseqplusplus_b200 import Engine, Params, SsppError, gen

pytestmark = pytest.mark.gpu


def _same_matrix(a, b):
    assert a.ncols == b.ncols and a.nnz == b.nnz
    assert np.array_equal(a.dims, b.dims)
    assert np.array_equal(a.col_ptr, b.col_ptr)
    assert np.array_equal(a.rows, b.rows)
    assert np.array_equal(a.values.view(np.uint32), b.values.view(np.uint32))


def _built_rips(e, pts, radius, maxdim):
    e.load_rips(pts, radius, maxdim)
    return e.input_matrix(values=True)


def _built_lowerstar(e, f, maxdim=3):
    e.load_lowerstar(f, maxdim)
    return e.input_matrix(values=True)


RIPS = [  # (npts, space_dim, seed, radius, maxdim)
    (2000, 3, 1, 0.08, 3),        # the 2000-point 3-D Rips workload
    (100000, 3, 7, 0.016, 3),     # the 100k-point 3-D Rips workload
    (1500, 2, 5, 0.06, 2),
    (1500, 3, 9, gen.rips_radius_for_degree(1500, 3, 40), 3),  # mean degree 40
    (3000, 2, 4, 0.03, 1),
    (500, 1, 3, 0.01, 1),
    (700, 3, 6, 0.16, 0),
]


@pytest.mark.parametrize("args", RIPS)
def test_rips_matches_host(args):
    n, d, seed, r, maxdim = args
    with Engine(0) as e:
        got = _built_rips(e, gen.points(n, d, seed), r, maxdim)
    _same_matrix(got, gen.rips(n, d, seed, r, maxdim))


def test_rips_unusual_point_sets():
    rng = np.random.default_rng(11)
    clouds = [
        (rng.normal(size=(3000, 3)).astype(np.float32) * 5.0, 0.6, 3),        # unbounded, negative
        (np.repeat(rng.random((400, 2), dtype=np.float32), 3, axis=0), 0.05, 2),  # every point three times
        (rng.random((40, 3), dtype=np.float32), 10.0, 3),                    # complete graph
        (rng.random((800, 3), dtype=np.float32), 1e-4, 3),                   # (almost) no edges
        (np.repeat(rng.random((50, 3), dtype=np.float32), 2, axis=0), 0.0, 3),   # radius 0: duplicates only
        (rng.random((1, 2), dtype=np.float32), 0.5, 3),                      # one point
        (rng.random((5000, 3), dtype=np.float32) * 1e4 + 1e6, 150.0, 2),     # large offset coordinates
    ]
    with Engine(0) as e:
        for pts, r, maxdim in clouds:
            _same_matrix(_built_rips(e, pts, r, maxdim), gen.rips_from_points(pts, r, maxdim))


LOWERSTAR = [(12, 1.5, 4), (16, 2.0, 2), (32, 2.0, 2), (64, 2.0, 2)]  # the last is the 64^3 grid workload


@pytest.mark.parametrize("args", LOWERSTAR)
def test_lowerstar_matches_host(args):
    g, sigma, seed = args
    with Engine(0) as e:
        got = _built_lowerstar(e, gen.field(g, sigma, seed))
    _same_matrix(got, gen.lowerstar(g, sigma, seed))


def test_lowerstar_unusual_fields():
    rng = np.random.default_rng(12)
    ties = rng.integers(-3, 4, size=(9, 10, 11)).astype(np.float32)
    ties[ties == 0] = -0.0
    fields = [
        (rng.normal(size=(7, 5, 3)).astype(np.float32), 3),
        (rng.normal(size=(1, 40, 30)).astype(np.float32), 3),    # a 2-D image
        (rng.normal(size=(50, 1, 1)).astype(np.float32), 3),     # a 1-D signal
        (ties, 3),                                               # many equal values, signed zeros
        (ties, 2),
        (np.zeros((6, 6, 6), dtype=np.float32), 3),              # constant field
        (rng.normal(size=(2, 2, 2)).astype(np.float32), 1),
    ]
    with Engine(0) as e:
        for f, maxdim in fields:
            _same_matrix(_built_lowerstar(e, f, maxdim), gen.lowerstar_from_field(f, maxdim))


def test_built_complexes_reduce_like_loaded_ones():
    cases = [("r", (2000, 3, 1, 0.08, 3), Params()),
             ("r", (100000, 3, 7, 0.016, 3), Params(model=3, max_iteration=100, level1_capacity=100,
                                                    level2_capacity=250)),
             ("l", (32, 2.0, 2), Params(model=1, max_iteration=10)),
             ("l", (16, 1.0, 5), Params(dualize=1))]
    with Engine(0) as e:
        for kind, args, p in cases:
            if kind == "r":
                n, d, seed, r, maxdim = args
                m = gen.rips(*args)
                e.load_rips(gen.points(n, d, seed), r, maxdim)
            else:
                m = gen.lowerstar(*args)
                e.load_lowerstar(gen.field(*args))
            e.reduce(p)
            built = (e.pairs(), e.essentials())
            assert e.stats()["build_ms"] > 0
            e.load_csc(m)
            e.reduce(p)
            assert np.array_equal(built[0], e.pairs()) and np.array_equal(built[1], e.essentials())
    # and against the oracle on a small one
    m = gen.rips(600, 3, 2, 0.15, 3)
    ref = oracle.reduce(m)
    with Engine(0) as e:
        e.load_rips(gen.points(600, 3, 2), 0.15, 3)
        e.reduce(Params())
        assert np.array_equal(e.pairs(), ref.pairs) and np.array_equal(e.essentials(), ref.essential)


def test_device_resident_inputs_and_buffer_reuse():
    torch = pytest.importorskip("torch")
    pts = gen.points(20000, 3, 21)
    f = gen.field(24, 1.5, 22)
    with Engine(0) as e:
        # large, small, large again: the builder's buffers grow and are reused
        for _ in range(2):
            _same_matrix(_built_rips(e, torch.from_numpy(pts).cuda(), 0.03, 3),
                         gen.rips_from_points(pts, 0.03, 3))
            _same_matrix(_built_lowerstar(e, torch.from_numpy(f).cuda()), gen.lowerstar_from_field(f))
            _same_matrix(_built_rips(e, pts[:300], 0.2, 2), gen.rips_from_points(pts[:300], 0.2, 2))


def test_builders_reject_bad_input():
    with Engine(0) as e:
        bad = gen.points(100, 3, 1)
        bad[17, 2] = np.inf
        with pytest.raises(SsppError):
            e.load_rips(bad, 0.2, 3)
        f = gen.field(8, 1.0, 1)
        f[3, 4, 5] = np.nan
        with pytest.raises(SsppError):
            e.load_lowerstar(f)
        with pytest.raises(SsppError):
            e.load_rips(gen.points(10, 3, 1), 0.2, 4)  # maxdim above 3
        with pytest.raises(SsppError):
            e.reduce(Params())  # nothing loaded after a failed build
        # the context stays usable
        e.load_rips(gen.points(300, 2, 3), 0.1, 2)
        e.reduce(Params())
        with pytest.raises(SsppError):
            e.load_csc(gen.rips(50, 2, 1, 0.2, 2))
            e.input_matrix(values=True)  # values exist for built complexes only


def test_server_builds_point_cloud_and_field_requests():
    from specseqplusplus_b200 import Server

    rng = np.random.default_rng(13)
    clouds = [(gen.points(int(n), d, int(s)), float(r), 2 if d == 2 else 3)
              for n, d, s, r in [(900, 2, 1, 0.06), (1500, 3, 2, 0.09), (400, 3, 3, 0.2), (2500, 2, 4, 0.03)]]
    fields = [gen.field(12, 1.5, 5), gen.field(20, 2.0, 6), rng.normal(size=(7, 9, 5)).astype(np.float32)]
    mats = [gen.rips(700, 3, 7, 0.15, 3), gen.lowerstar(10, 1.0, 8)]
    want = {}
    with Engine(0) as e:
        for i, (pts, r, md) in enumerate(clouds):
            e.load_rips(pts, r, md)
            e.reduce(Params())
            want[("r", i)] = (e.pairs(), e.essentials(), e.input_matrix(values=True).values)
        for i, f in enumerate(fields):
            e.load_lowerstar(f)
            e.reduce(Params())
            want[("l", i)] = (e.pairs(), e.essentials(), e.input_matrix(values=True).values)
        for i, m in enumerate(mats):
            e.load_csc(m)
            e.reduce(Params())
            want[("m", i)] = (e.pairs(), e.essentials(), None)
    with Server(Params(autotune=2), workers=2) as srv:
        ids = {}
        for rep in range(2):  # interleaved kinds, twice
            for i, (pts, r, md) in enumerate(clouds):
                ids[("r", i, rep)] = srv.submit_rips(pts, r, md, values=(rep == 0))
            for i, m in enumerate(mats):
                ids[("m", i, rep)] = srv.submit(m)
            for i, f in enumerate(fields):
                ids[("l", i, rep)] = srv.submit_lowerstar(f, values=(rep == 1), copy=(rep == 0))
        bad = gen.field(6, 1.0, 9)
        bad[1, 2, 3] = np.nan
        bad_id = srv.submit_lowerstar(bad)
        for (k, i, rep), rid in ids.items():
            p, es, vals = want[(k, i)]
            assert np.array_equal(srv.pairs(rid), p), (k, i, rep)
            assert np.array_equal(srv.essentials(rid), es), (k, i, rep)
            if (k == "r" and rep == 0) or (k == "l" and rep == 1):
                assert np.array_equal(srv.values(rid).view(np.uint32), vals.view(np.uint32))
        with pytest.raises(SsppError):
            srv.pairs(bad_id)
    with Server(Params(), workers=1, memory_budget=1 << 20) as small:
        with pytest.raises(SsppError):
            small.submit_lowerstar(gen.field(40, 1.0, 1))  # larger than the budget: refused at submit


def test_built_batch_matches_separate_builds():
    # several point clouds and fields built one after another into one
    # block-diagonal batch: each complex's matrix values, pairs and essentials
    # equal those of building and reducing it alone
    reqs = [("rips", gen.points(900, 2, 1), 0.06, 2), ("lowerstar", gen.field(11, 1.5, 5), 3),
            ("rips", gen.points(1500, 3, 2), 0.09, 3), ("rips", gen.points(3, 3, 4), 0.01, 3),
            ("lowerstar", np.random.default_rng(3).normal(size=(6, 8, 5)).astype(np.float32), 2),
            ("rips", gen.points(600, 3, 8), gen.rips_radius_for_degree(600, 3, 30), 3)]
    want = []
    with Engine(0) as e:
        for r in reqs:
            if r[0] == "rips":
                e.load_rips(r[1], r[2], r[3])
            else:
                e.load_lowerstar(r[1], r[2])
            vals = e.input_matrix(values=True).values
            e.reduce(Params())
            want.append((e.pairs(), e.essentials(), vals))
        for p in (Params(), Params(autotune=2), Params(schedule=1)):
            e.load_built_batch(reqs)
            e.reduce(p)
            for i, (pw, ew, vw) in enumerate(want):
                assert np.array_equal(e.batch_pairs(i), pw), (p, i)
                assert np.array_equal(e.batch_essentials(i), ew), (p, i)
                assert np.array_equal(e.batch_values(i).view(np.uint32), vw.view(np.uint32)), (p, i)
        bad = gen.field(6, 1.0, 9)
        bad[1, 2, 3] = np.nan
        with pytest.raises(SsppError):
            e.load_built_batch([reqs[0], ("lowerstar", bad, 3)])
        e.load_built_batch([])
        e.reduce(Params())
