"""CPU tests of the oracle (test infrastructure): pinned against the reference's
known-answer fixture, an independent dense standard reduction, the rank-based
pairing lemma, primal = dual, and the reference's own GUDHI edge collapser."""
import itertools
import os

import numpy as np
import pytest

import oracle
from helpers import (boundary_matrix, dense_standard_pairs, essentials_from_pairs, flag_complex, random_complex,
                     random_filtration, rank_pairs)
from specseqplusplus_b200 import gen

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _read_pairs(path):
    lines = [ln.split() for ln in open(path).read().split("\n") if ln.strip()]
    return np.array([(int(a), int(b)) for a, b in lines[1:]], dtype=np.int64).reshape(-1, 2)


def _matrix(path, binary):
    d, c, r = oracle.read_phat(path, binary)
    return gen.BoundaryMatrix(d, c, r)


@pytest.mark.parametrize("binary", [False, True])
def test_single_triangle_known_answer(binary):
    m = _matrix(os.path.join(GOLD, "single_triangle.bin" if binary else "single_triangle.dat"), binary)
    assert m.ncols == 7
    want = _read_pairs(os.path.join(GOLD, "single_triangle_pairs.dat"))
    for dual in (0, 1):
        for pre in (0, 1):
            r = oracle.reduce(m, dualize=dual, preprocess=pre)
            assert np.array_equal(r.pairs, want)
            assert list(r.essential) == [0]


def test_reader_semantics(tmp_path):
    p = tmp_path / "m.txt"
    p.write_text("# c\n0\n0  \n\n1 1 0 1\n   \n2\n")
    d, c, r = oracle.read_phat(str(p), False)
    assert list(d) == [0, 0, 1, 2]
    assert list(c) == [0, 0, 0, 2, 2]
    assert list(r) == [0, 1]


def test_standard_vs_rank_lemma_exhaustive_triangle():
    # every filtration of the filled triangle
    simplices = flag_complex(3, [(0, 1), (0, 2), (1, 2)], 2)
    seen = 0
    for perm in itertools.permutations(simplices):
        pos = {s: i for i, s in enumerate(perm)}
        if any(len(s) > 1 and any(pos[s[:k] + s[k + 1:]] > pos[s] for k in range(len(s))) for s in perm):
            continue
        m = boundary_matrix(list(perm))
        ref = rank_pairs(m)
        assert np.array_equal(dense_standard_pairs(m), ref)
        assert np.array_equal(oracle.reduce(m).pairs, ref)
        assert np.array_equal(oracle.reduce(m, dualize=1).pairs, ref)
        seen += 1
    assert seen > 10


@pytest.mark.parametrize("seed", range(12))
def test_oracle_vs_independent_reductions(seed):
    rng = np.random.default_rng(seed)
    m = random_complex(rng, nverts=7 + seed % 4, p=0.6, maxdim=3)
    want = dense_standard_pairs(m)
    if m.ncols <= 45:
        assert np.array_equal(rank_pairs(m), want)
    for dual in (0, 1):
        for pre in (0, 1):
            r = oracle.reduce(m, dualize=dual, preprocess=pre)
            assert np.array_equal(r.pairs, want), (dual, pre)
            assert np.array_equal(r.essential, essentials_from_pairs(m.ncols, want))


@pytest.mark.parametrize("seed", range(4))
def test_highclear_is_sound(seed):
    m = gen.rips(300, 3, seed, 0.25, 3)
    a = oracle.reduce(m, model=0, preprocess=0)
    b = oracle.reduce(m, model=1, max_iteration=50)
    assert b.stats["highclear"] > 0
    assert np.array_equal(a.pairs, b.pairs)
    assert np.array_equal(a.essential, b.essential)


def test_rips_and_lowerstar_primal_equals_dual():
    for m in (gen.rips(600, 3, 11, 0.15, 3), gen.rips(800, 2, 12, 0.07, 2), gen.lowerstar(8, 1.0, 3)):
        a = oracle.reduce(m)
        b = oracle.reduce(m, dualize=1)
        assert np.array_equal(a.pairs, b.pairs)


def test_generator_counts():
    m = gen.lowerstar(6, 1.0, 1)
    counts = np.bincount(m.dims)
    g = 6
    assert counts[0] == g ** 3
    assert counts[1] == 3 * g * g * (g - 1) + 3 * g * (g - 1) ** 2 + (g - 1) ** 3
    assert counts[3] == 6 * (g - 1) ** 3
    assert counts[0] - counts[1] + counts[2] - counts[3] == 1  # Euler characteristic of a cube
    # filtration order: faces precede cofaces, values non-decreasing
    for j in range(m.ncols):
        assert all(r < j for r in m.column(j))
    assert np.all(np.diff(m.values) >= 0)


def _edges(m):
    vid = -np.ones(m.ncols, dtype=np.int64)
    vs = np.nonzero(m.dims == 0)[0]
    vid[vs] = np.arange(len(vs))
    es = np.nonzero(m.dims == 1)[0]
    u = np.array([vid[m.column(j)[0]] for j in es], dtype=np.int32)
    v = np.array([vid[m.column(j)[1]] for j in es], dtype=np.int32)
    return len(vs), u, v


@pytest.mark.skipif(not oracle.ref_collapse_available(), reason="reference collapser not built (no reference tree)")
@pytest.mark.parametrize("seed", range(6))
def test_collapse_matches_reference_gudhi(seed):
    rng = np.random.default_rng(100 + seed)
    n = int(rng.integers(30, 200))
    m = gen.rips(n, 2 + seed % 2, seed, float(rng.uniform(0.1, 0.35)), 1)
    nv, u, v = _edges(m)
    ours = oracle.collapse_edges(nv, u, v)
    ref = oracle.ref_collapse_edges(u, v)
    assert np.array_equal(ours, ref)
    assert 0 < ours.sum() <= len(u)


def test_collapse_keeps_homology_of_flag_complex():
    # a collapse removes edges but never changes the homology of the full flag complex
    m = gen.rips(120, 2, 5, 0.2, 2)
    r0 = oracle.reduce(m, model=0)
    r2 = oracle.reduce(m, model=2)
    assert r2.stats["dropped"] > 0
    # essential classes of the final complex (Betti numbers) agree in every dimension
    b0 = np.bincount(m.dims[r0.essential], minlength=3)
    b2 = np.bincount(m.dims[r2.essential], minlength=3)
    assert b0[0] == b2[0]


# the reference tree's root comes from SSPP_REFERENCE; the check is skipped without it
REF_ALPHA = os.path.join(os.environ.get("SSPP_REFERENCE", "/nonexistent"), "data", "Alpha")


@pytest.mark.skipif(not os.path.isdir(REF_ALPHA), reason="reference tree absent (set SSPP_REFERENCE)")
def test_reference_highclear_artefacts_keep_the_pairs():
    # The reference's HIGHOUT build wrote each Alpha input again with its guided
    # clearing applied (cleared columns as dimension-only lines,
    # include/specseq.h:1108-1129); both files must give the same pairs.
    names = sorted(f for f in os.listdir(REF_ALPHA) if f.endswith(".txt") and not f.endswith("_maxclear.txt"))
    checked = 0
    for f in names:
        cleared = os.path.join(REF_ALPHA, f[:-4] + "_maxclear.txt")
        if not os.path.exists(cleared):
            continue
        mats = []
        for path in (os.path.join(REF_ALPHA, f), cleared):
            d, c, r = oracle.read_phat(path, False)
            mats.append(gen.BoundaryMatrix(d, c, r))
        assert mats[0].ncols == mats[1].ncols
        a, b = oracle.reduce(mats[0]), oracle.reduce(mats[1])
        assert np.array_equal(a.pairs, b.pairs), f
        checked += 1
    assert checked >= 3
