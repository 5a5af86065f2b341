"""GPU parity of the two ways of driving the spectral-sequence blocks.

schedule 1 is a host loop of per-block launches (the reference's
GPU_Compute structure); schedule 2 (the default) is one persistent launch that
drains a device queue of (complex, block) items, each complex with its own
block order and dimension gate.  Both must give the oracle's pairs and
essential classes bit for bit, on single complexes and on batches, in every
dualization mode and with both CTA sizes.
"""
import numpy as np
import pytest

import oracle
from helpers import dense_standard_pairs, essentials_from_pairs, random_complex
from specseqplusplus_b200 import Engine, Params, gen, workloads

pytestmark = pytest.mark.gpu


def _run(m, p):
    with Engine(0) as e:
        e.load_csc(m)
        e.reduce(p)
        return e.pairs(), e.essentials(), e.stats()


@pytest.mark.parametrize("schedule", [1, 2])
@pytest.mark.parametrize("seed", range(6))
def test_random_complexes_both_schedules(schedule, seed):
    rng = np.random.default_rng(7000 + seed)
    m = random_complex(rng, nverts=7 + seed % 4, p=0.7, maxdim=3)
    want = dense_standard_pairs(m)
    pairs, ess, _ = _run(m, Params(schedule=schedule, ss_block_size=1 + seed % 5, growth=1.0 + 0.2 * (seed % 2),
                                   level1_capacity=32, level2_capacity=64))
    assert np.array_equal(pairs, want)
    assert np.array_equal(ess, essentials_from_pairs(m.ncols, want))


@pytest.mark.parametrize("p", [
    Params(schedule=2),
    Params(schedule=2, ss_block_size=64, growth=1.2, level1_capacity=32, level2_capacity=64),
    Params(schedule=2, ss_block_size=7, growth=1.5, level1_capacity=128, level2_capacity=2048, heavy_threads=128),
    Params(schedule=2, dualize=1),
    Params(schedule=2, dualize=2, level1_capacity=32, level2_capacity=4096),
    Params(schedule=2, model=3, max_iteration=20),
])
def test_queue_matches_oracle(p):
    for m in (gen.rips(1500, 2, 5, 0.06, 2), gen.lowerstar(14, 1.5, 4), gen.rips(900, 3, 2, 0.12, 3)):
        ref = oracle.reduce(m, model=p.model, max_iteration=p.max_iteration)
        pairs, ess, st = _run(m, p)
        assert np.array_equal(pairs, ref.pairs)
        assert np.array_equal(ess, ref.essential)


def test_queue_and_host_loop_agree_on_32_grid():
    m = gen.lowerstar(32, 2.0, 2)
    ref = oracle.reduce(m, model=1, max_iteration=10)
    for s in (1, 2):
        pairs, ess, st = _run(m, Params(schedule=s, model=1, max_iteration=10, level1_capacity=32,
                                        level2_capacity=8192))
        assert np.array_equal(pairs, ref.pairs), s
        assert np.array_equal(ess, ref.essential), s


@pytest.mark.parametrize("p", [Params(schedule=2), Params(schedule=2, autotune=2), Params(schedule=2, dualize=2),
                               Params(schedule=1)])
def test_batch_queue_each_complex_exact(p):
    mats, _ = workloads.batch_of_rips(40, seed=13, n_min=60, n_max=1500)
    mats.append(gen.lowerstar(9, 1.0, 3))
    mats.append(gen.BoundaryMatrix.from_columns([0, 0], [[], []]))  # nothing to reduce
    mats.append(gen.BoundaryMatrix.from_columns([], []))            # no columns at all
    with Engine(0) as e:
        e.load_batch(mats)
        e.reduce(p)
        for i, m in enumerate(mats):
            ref = oracle.reduce(m)
            assert np.array_equal(e.batch_pairs(i), ref.pairs), i
            assert np.array_equal(e.batch_essentials(i), ref.essential), i


def test_queue_repeats_and_reports_items():
    m = gen.lowerstar(16, 2.0, 9)
    with Engine(0) as e:
        e.load_csc(m)
        e.reduce(Params(schedule=2, ss_block_size=512, growth=1.1))
        a = e.pairs()
        st = e.stats()
        assert st["ss_steps"] > 2  # one item per block
        e.reduce(Params(schedule=2, ss_block_size=512, growth=1.1))
        assert np.array_equal(a, e.pairs())
