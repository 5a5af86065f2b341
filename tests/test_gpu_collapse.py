"""GPU parity of the Flag-complex edge collapse (model bit 2) against the oracle.

The oracle restates GUDHI's collapse (include/Flag_complex_edge_collapser.h,
pinned against the reference's own header in test_oracle.py) with edge
filtration = edge order (include/specseq.h:209-212), drops every edge that is
not kept and every higher simplex with a dropped facet (include/specseq.h:
410-436).  Every column is paired, essential or dropped, so equal pairs and
equal essentials also mean an equal dropped set; the dropped count is checked
as well.  The dense Rips cases make the order-dependent re-examinations long.
"""
import numpy as np
import pytest

import oracle
from helpers import random_complex
from specseqplusplus_b200 import Engine, Params, gen

pytestmark = pytest.mark.gpu


def run(m, p):
    with Engine(0) as e:
        e.load_csc(m)
        e.reduce(p)
        return e.pairs(), e.essentials(), e.stats()


def check(m, p):
    ref = oracle.reduce(m, dualize=p.dualize, model=p.model, max_iteration=p.max_iteration)
    pairs, ess, st = run(m, p)
    assert np.array_equal(pairs, ref.pairs)
    assert np.array_equal(ess, ref.essential)
    assert st["collapse_dropped"] == ref.stats["dropped"]
    return st, ref


@pytest.mark.parametrize("seed", range(16))
def test_collapse_random_flag_complexes(seed):
    rng = np.random.default_rng(3000 + seed)
    m = random_complex(rng, nverts=7 + seed % 6, p=0.5 + 0.05 * (seed % 5), maxdim=3)
    check(m, Params(model=2))
    check(m, Params(model=3, max_iteration=5, dualize=seed % 2, level1_capacity=32, level2_capacity=64))


def test_collapse_rips_2000():
    m = gen.rips(2000, 3, 1, 0.08, 3)
    st, ref = check(m, Params(model=2))
    assert st["collapse_dropped"] > 0
    check(m, Params(model=3, max_iteration=100))
    check(m, Params(model=3, max_iteration=100, dualize=1))


@pytest.mark.parametrize("npts,dim,deg,seed", [(1500, 3, 30, 1), (2500, 2, 40, 2), (600, 3, 60, 3)])
def test_collapse_dense_rips(npts, dim, deg, seed):
    m = gen.rips(npts, dim, seed, gen.rips_radius_for_degree(npts, dim, deg), min(dim, 3))
    st, _ = check(m, Params(model=2))
    assert st["collapse_dropped"] > 0


def test_collapse_lowerstar_grid():
    m = gen.lowerstar(12, 1.5, 6)
    check(m, Params(model=3, max_iteration=10))


def test_collapse_large_vr_100k_points():
    # 100,000 points in [0,1]^3, radius 0.016, dim <= 3, model 3, max_iteration
    # 100, queue 65536, level capacities 100/250
    m = gen.rips(100000, 3, 7, 0.016, 3)
    st, ref = check(m, Params(model=3, max_iteration=100, queue_size=65536, level1_capacity=100,
                              level2_capacity=250))
    assert st["collapse_dropped"] == ref.stats["dropped"] > 0


def test_collapse_in_batch():
    from specseqplusplus_b200 import workloads

    mats, _ = workloads.batch_of_rips(10, seed=21, n_min=100, n_max=800)
    with Engine(0) as e:
        e.load_batch(mats)
        e.reduce(Params(model=3, max_iteration=10))
        for i, m in enumerate(mats):
            assert np.array_equal(e.batch_pairs(i), oracle.reduce(m, model=3, max_iteration=10).pairs), i
