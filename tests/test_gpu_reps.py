"""GPU tests of representative cycles (sspp_representative through the C ABI).

A reduction keeps no particular representative (any valid reduction order
gives the same pairs but different reduced columns), so each returned cycle is
checked against the definition instead of against a fixed answer: for a pair
(birth b, death d) the representative z is ascending, its youngest simplex is
b, it is a Z2 cycle (even size in dimension 0), and z + boundary(d) lies in the
span of the boundaries of the columns before d (so z is the boundary of a
chain whose youngest simplex is d).  Pairs must still equal the oracle's."""
import numpy as np
import pytest

import oracle
from helpers import random_complex
from specseqplusplus_b200 import Engine, Params, SsppError, gen

pytestmark = pytest.mark.gpu


def _rank2(A):
    """Rank over GF(2), eliminating all rows of a pivot column at once."""
    A = (A % 2).astype(np.uint8)
    r = 0
    for c in range(A.shape[1]):
        rows = np.nonzero(A[r:, c])[0]
        if len(rows) == 0:
            continue
        piv = r + rows[0]
        A[[r, piv]] = A[[piv, r]]
        hit = np.nonzero(A[:, c])[0]
        hit = hit[hit != r]
        A[hit] ^= A[r]
        r += 1
        if r == A.shape[0]:
            break
    return r


def _boundary_xor(m, chain):
    acc = set()
    for s in chain:
        acc ^= set(int(x) for x in m.column(int(s)))
    return acc


def _check_cycle(m, b, d, z, span_check):
    assert np.all(np.diff(z) > 0)
    assert z[-1] == b
    assert np.all(m.dims[z] == m.dims[b])
    if m.dims[b] == 0:
        assert len(z) % 2 == 0
    else:
        assert not _boundary_xor(m, z)
    if span_check:
        n = m.ncols
        B = np.zeros((n, d + 1), dtype=np.uint8)
        for j in range(d):
            B[m.column(j), j] = 1
        v = np.zeros(n, dtype=np.uint8)
        v[m.column(d)] ^= 1
        v[z] ^= 1
        B[:, d] = v
        assert _rank2(B[:, :d]) == _rank2(B)


def _reps(m, p, span_check, limit=None):
    span_check = span_check and m.ncols <= 400
    ref = oracle.reduce(m, model=p.model, max_iteration=p.max_iteration)
    with Engine(0) as e:
        e.load_csc(m)
        e.reduce(p)
        pairs = e.pairs()
        assert np.array_equal(pairs, ref.pairs)
        assert np.array_equal(e.essentials(), ref.essential)
        sel = pairs if limit is None else pairs[np.linspace(0, len(pairs) - 1, min(limit, len(pairs))).astype(int)]
        for b, d in sel:
            _check_cycle(m, int(b), int(d), e.representative(int(d)), span_check)
    return len(sel)


@pytest.mark.parametrize("seed", range(6))
def test_random_complexes(seed):
    rng = np.random.default_rng(9100 + seed)
    m = random_complex(rng, nverts=9, p=0.6, maxdim=3)
    p = Params(representatives=1, level1_capacity=32, level2_capacity=64, ss_block_size=1 + seed)
    assert _reps(m, p, span_check=True) > 0


@pytest.mark.parametrize("p", [Params(representatives=1), Params(representatives=1, model=1, max_iteration=10),
                               Params(representatives=1, autotune=2)])
def test_rips_and_grid(p):
    for m in (gen.rips(30, 3, 4, 0.4, 3), gen.lowerstar(3, 1.0, 2)):  # span-checked
        _reps(m, p, span_check=True, limit=40)
    for m in (gen.rips(400, 3, 4, 0.2, 3), gen.lowerstar(10, 1.0, 2)):
        _reps(m, p, span_check=False, limit=300)


def test_larger_inputs_use_both_tiers():
    # long chains (CTA tier) and the dimension gate on the 32^3 grid
    p = Params(representatives=1, level1_capacity=32, level2_capacity=4096)
    for m in (gen.lowerstar(32, 2.0, 2), gen.rips(3000, 3, 5, gen.rips_radius_for_degree(3000, 3, 30), 3)):
        _reps(m, p, span_check=False, limit=400)


def test_collapse_representatives_lie_in_the_complex():
    m = gen.rips(800, 3, 6, 0.14, 3)
    p = Params(representatives=1, model=3, max_iteration=10)
    _reps(m, p, span_check=False, limit=200)


def test_errors_and_autotune_stays_primal():
    m = gen.rips(300, 2, 1, 0.15, 2)
    with Engine(0) as e:
        e.load_csc(m)
        e.reduce(Params())
        with pytest.raises(SsppError):
            e.representative(int(e.pairs()[0][1]))  # the reduction kept no representatives
        with pytest.raises(SsppError):
            e.reduce(Params(representatives=1, dualize=1))
        e.reduce(Params(representatives=1, autotune=2))
        assert e.params().dualize == 0
        pairs = e.pairs()
        with pytest.raises(SsppError):
            e.representative(int(pairs[0][0]))  # a birth, not a death
        with pytest.raises(SsppError):
            e.representative(m.ncols + 5)
        plain = Engine(0)
        try:
            plain.load_csc(m)
            plain.reduce(Params())
            assert np.array_equal(plain.pairs(), pairs)  # keeping whole columns changes no pair
        finally:
            plain.close()
