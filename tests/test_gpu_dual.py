"""GPU parity of the dualized reductions (dualize = 1 and 2) against the oracle.

The dual matrix is the anti-transpose of the cleared and compressed boundary
matrix (include/kernel.h:521-580, include/specseq.h:303-363); it is reduced
dimension by dimension from low to high and its pairs are mapped back through
n-1-x (include/specseq.h:1188).  The pairs must equal the primal pairs and the
oracle's, bit for bit.  The hub complexes give one vertex a coboundary of up
to 20,000 entries, so the dual pass's long-column sort (shared-memory chunks
plus merge rounds in global memory) runs; their dual reduction is a chain of m
additions on a column of about m entries, which the CTA tier runs in two
reused arena buffers.
"""
import numpy as np
import pytest

import oracle
from helpers import dense_standard_pairs, essentials_from_pairs, random_complex
from specseqplusplus_b200 import Engine, Params, SpecSeqPlusPlus, gen

pytestmark = pytest.mark.gpu


def run(m, p):
    with Engine(0) as e:
        e.load_csc(m)
        e.reduce(p)
        return e.pairs(), e.essentials(), e.stats()


def hub_complex(m):
    """Vertex 0 joined to leaves 1..m, a path through the leaves, and the
    triangles (0, i, i+1): the dual column of vertex 0 holds m entries."""
    dims = [0] * (m + 1)
    cols = [[] for _ in range(m + 1)]
    spoke = {}
    for i in range(1, m + 1):
        spoke[i] = len(cols)
        dims.append(1)
        cols.append([0, i])
    path = {}
    for i in range(1, m):
        path[i] = len(cols)
        dims.append(1)
        cols.append([i, i + 1])
    for i in range(1, m):
        dims.append(2)
        cols.append(sorted([spoke[i], spoke[i + 1], path[i]]))
    return gen.BoundaryMatrix.from_columns(dims, cols)


@pytest.mark.parametrize("seed", range(12))
def test_dual_random_small_complexes(seed):
    rng = np.random.default_rng(2000 + seed)
    m = random_complex(rng, nverts=6 + seed % 5, p=0.65, maxdim=3)
    want = dense_standard_pairs(m)
    pairs, ess, _ = run(m, Params(dualize=1, ss_block_size=1 + seed % 5, level1_capacity=32,
                                  level2_capacity=32 + 32 * (seed % 2)))
    assert np.array_equal(pairs, want)
    assert np.array_equal(ess, essentials_from_pairs(m.ncols, want))


def test_dual_rips_equals_primal_and_oracle():
    m = gen.rips(2000, 3, 1, 0.08, 3)
    ref = oracle.reduce(m, dualize=1)
    primal = oracle.reduce(m)
    assert np.array_equal(ref.pairs, primal.pairs)
    pairs, ess, _ = run(m, Params(dualize=1))
    assert np.array_equal(pairs, ref.pairs)
    assert np.array_equal(ess, ref.essential)


@pytest.mark.parametrize("p", [
    Params(dualize=1, ss_block_size=64, growth=1.2, level1_capacity=32, level2_capacity=64),
    Params(dualize=1, ss_block_size=1 << 30, level1_capacity=64, level2_capacity=96),
    Params(dualize=1, ss_block_size=7, growth=1.5, queue_size=33, level1_capacity=128, level2_capacity=2048),
])
def test_dual_schedule_and_tier_variants(p):
    for m in (gen.rips(1500, 2, 5, 0.06, 2), gen.rips(700, 3, 6, 0.16, 3), gen.lowerstar(12, 1.5, 4)):
        ref = oracle.reduce(m)
        pairs, ess, _ = run(m, p)
        assert np.array_equal(pairs, ref.pairs)
        assert np.array_equal(ess, ref.essential)


def test_dual_with_guided_clearing():
    for m in (gen.rips(1200, 3, 7, 0.12, 3), gen.lowerstar(16, 2.0, 2)):
        ref = oracle.reduce(m, dualize=1, model=1, max_iteration=10)
        pairs, ess, st = run(m, Params(dualize=1, model=1, max_iteration=10))
        assert st["highclear_cleared"] == ref.stats["highclear"]
        assert np.array_equal(pairs, ref.pairs)
        assert np.array_equal(ess, ref.essential)


def test_dual_lowerstar_32():
    m = gen.lowerstar(32, 2.0, 2)
    ref = oracle.reduce(m)
    pairs, ess, _ = run(m, Params(dualize=1))
    assert np.array_equal(pairs, ref.pairs)
    assert np.array_equal(ess, ref.essential)


@pytest.mark.parametrize("leaves", [700, 1500, 12000, 20000])
def test_dual_long_coboundary_sort(leaves):
    m = hub_complex(leaves)
    ref = oracle.reduce(m)
    for p in (Params(dualize=1), Params(dualize=1, level1_capacity=32, level2_capacity=64)):
        pairs, ess, _ = run(m, p)
        assert np.array_equal(pairs, ref.pairs)
        assert np.array_equal(ess, ref.essential)


def test_dual_batch_and_class_mirror():
    from specseqplusplus_b200 import workloads

    mats, _ = workloads.batch_of_rips(12, seed=11, n_min=100, n_max=900)
    with Engine(0) as e:
        e.load_batch(mats)
        e.reduce(Params(dualize=1))
        for i, m in enumerate(mats):
            assert np.array_equal(e.batch_pairs(i), oracle.reduce(m).pairs), i
    m = gen.rips(500, 3, 3, 0.15, 3)
    alg = SpecSeqPlusPlus(m, [0, 1000, 8000, 0], 1, 0, 0, 102400, 1.05, 65536)
    alg.GPU_Init()
    alg.GPU_Compute()
    assert np.array_equal(alg.GetPersistencePairs(), oracle.reduce(m).pairs)


# dualize = 2: the 0-dimensional pairs from the boundary matrix's edge columns,
# then the coboundary matrix from dimension 1 up; the pairs never change


@pytest.mark.parametrize("seed", range(12))
def test_mode2_random_small_complexes(seed):
    rng = np.random.default_rng(4000 + seed)
    m = random_complex(rng, nverts=6 + seed % 5, p=0.65, maxdim=3)
    want = dense_standard_pairs(m)
    pairs, ess, _ = run(m, Params(dualize=2, ss_block_size=1 + seed % 5, level1_capacity=32,
                                  level2_capacity=32 + 32 * (seed % 2)))
    assert np.array_equal(pairs, want)
    assert np.array_equal(ess, essentials_from_pairs(m.ncols, want))


@pytest.mark.parametrize("p", [
    Params(dualize=2),
    Params(dualize=2, ss_block_size=64, growth=1.2, level1_capacity=32, level2_capacity=64),
    Params(dualize=2, model=3, max_iteration=10),
    Params(dualize=2, model=1, max_iteration=100, level1_capacity=32, level2_capacity=8192),
])
def test_mode2_matches_primal(p):
    for m in (gen.rips(2000, 3, 1, 0.08, 3), gen.rips(1500, 2, 5, 0.06, 2), gen.lowerstar(16, 2.0, 2),
              hub_complex(1500)):
        ref = oracle.reduce(m, model=p.model, max_iteration=p.max_iteration)
        pairs, ess, _ = run(m, p)
        assert np.array_equal(pairs, ref.pairs)
        assert np.array_equal(ess, ref.essential)


def test_mode2_dense_rips_and_batch():
    from specseqplusplus_b200 import workloads

    m = gen.rips(1500, 3, 9, gen.rips_radius_for_degree(1500, 3, 35), 3)
    ref = oracle.reduce(m, dualize=1)
    pairs, ess, st = run(m, Params(dualize=2, level1_capacity=32))
    assert np.array_equal(pairs, ref.pairs)
    assert np.array_equal(ess, ref.essential)
    mats, _ = workloads.batch_of_rips(12, seed=13, n_min=100, n_max=900)
    with Engine(0) as e:
        e.load_batch(mats)
        e.reduce(Params(dualize=2, level1_capacity=32))
        for i, mm in enumerate(mats):
            assert np.array_equal(e.batch_pairs(i), oracle.reduce(mm).pairs), i
            assert np.array_equal(e.batch_essentials(i), oracle.reduce(mm).essential), i
