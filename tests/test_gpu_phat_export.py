"""GPU tests of the PHAT-style Python module and of the preprocessed-matrix
export (the reference's HIGHOUT build, include/specseq.h:1108-1129)."""
import os
import subprocess

import numpy as np
import pytest

import oracle
from helpers import dense_standard_pairs, random_complex
from specseqplusplus_b200 import ASCII, BINARY, Engine, Params, gen, phat
from specseqplusplus_b200.engine import read_phat

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden")
CLI = os.path.join(ROOT, "specseqplusplus_b200", "bin", "specseq++")


def test_phat_module_single_triangle():
    bm = phat.boundary_matrix(representation=phat.representations.vector_vector)
    bm.columns = [(0, []), (0, []), (1, [0, 1]), (0, []), (1, [1, 3]), (1, [0, 3]), (2, [2, 4, 5])]
    pairs = bm.compute_persistence_pairs()
    pairs.sort()
    assert list(pairs) == [(1, 2), (3, 4), (5, 6)]
    assert bm.compute_persistence_pairs_dualized(phat.reductions.chunk_reduction) == pairs
    # the reference's known-answer fixture, through load()
    other = phat.boundary_matrix()
    other.load(os.path.join(GOLD, "single_triangle.bin"), "b")
    assert list(other.compute_persistence_pairs()) == [(1, 3), (2, 4), (5, 6)]


@pytest.mark.parametrize("seed", range(4))
def test_phat_module_random_complexes(seed):
    rng = np.random.default_rng(5000 + seed)
    m = random_complex(rng, nverts=8, p=0.6, maxdim=3)
    bm = phat.boundary_matrix(columns=[(int(m.dims[j]), list(m.column(j))) for j in range(m.ncols)])
    assert np.array_equal(bm.compute_persistence_pairs().as_array(), dense_standard_pairs(m))


def _exported(m, p, tmp_path, fmt=ASCII):
    path = str(tmp_path / ("pre.txt" if fmt == ASCII else "pre.bin"))
    with Engine(0) as e:
        e.load_csc(m)
        e.export_preprocessed(path, p, fmt)
        st = e.stats()
    return read_phat(path, fmt), st


def _emptied(m, out):
    lens_in = np.diff(m.col_ptr)
    lens_out = np.diff(out.col_ptr)
    assert np.array_equal(m.dims, out.dims)
    kept = lens_out > 0
    assert np.array_equal(lens_in[kept], lens_out[kept])
    return int(np.count_nonzero((lens_in > 0) & (lens_out == 0)))


def test_export_guided_clearing_keeps_pairs(tmp_path):
    m = gen.rips(2000, 3, 1, 0.08, 3)
    p = Params(model=1, max_iteration=100)
    out, st = _exported(m, p, tmp_path)
    ref = oracle.reduce(m, model=1, max_iteration=100)
    assert _emptied(m, out) == st["highclear_cleared"] == ref.stats["highclear"] > 0
    with Engine(0) as e:
        e.load_csc(out)
        e.reduce(Params())
        assert np.array_equal(e.pairs(), ref.pairs)


def test_export_with_collapse_binary(tmp_path):
    m = gen.rips(1500, 3, 4, 0.1, 3)
    p = Params(model=3, max_iteration=10)
    out, st = _exported(m, p, tmp_path, BINARY)
    ref = oracle.reduce(m, model=3, max_iteration=10)
    assert _emptied(m, out) == st["highclear_cleared"] + st["collapse_dropped"]
    assert st["collapse_dropped"] == ref.stats["dropped"] > 0
    with Engine(0) as e:  # dropped simplices stay as empty columns: same pairs
        e.load_csc(out)
        e.reduce(Params())
        assert np.array_equal(e.pairs(), ref.pairs)


def test_cli_export_preprocessed(tmp_path):
    src = gen.rips(800, 3, 2, 0.14, 3)
    inp = tmp_path / "in.txt"
    from specseqplusplus_b200.engine import write_phat

    write_phat(str(inp), src, ASCII)
    out = tmp_path / "out.txt"
    r = subprocess.run([CLI, str(inp), str(out), "ascii", "ascii", "0", "1", "50", "102400", "1.05", "65536", "1000",
                        "8000", "--export-preprocessed"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    got = read_phat(str(out), ASCII)
    ref = oracle.reduce(src, model=1, max_iteration=50)
    assert _emptied(src, got) == ref.stats["highclear"]
