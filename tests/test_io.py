"""CPU checks of the library's PHAT reader and writers and of the PHAT-style
Python module (no GPU needed).

The reader must agree with the oracle's restatement of processFiles
(src/main.cu:90-167) on every file: comments, blank lines, trailing blanks and
carriage returns, unsorted and repeated faces, lines without a leading integer,
and files large enough to be cut into chunks parsed by several threads.
"""
import os

import numpy as np
import pytest

import oracle
from specseqplusplus_b200 import ASCII, BINARY, SsppError, gen
from specseqplusplus_b200.engine import read_phat, write_phat
from specseqplusplus_b200 import phat

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden")


def same_as_oracle(path, fmt):
    m = read_phat(path, fmt)
    d, c, r = oracle.read_phat(str(path), fmt == BINARY)
    assert np.array_equal(m.dims, d) and np.array_equal(m.col_ptr, c) and np.array_equal(m.rows, r)
    return m


def test_golden_single_triangle_both_formats():
    a = same_as_oracle(os.path.join(GOLD, "single_triangle.dat"), ASCII)
    b = same_as_oracle(os.path.join(GOLD, "single_triangle.bin"), BINARY)
    assert a.ncols == 7 and np.array_equal(a.rows, b.rows)


def test_messy_ascii_lines(tmp_path):
    text = ("# a comment\n\n0\n0   \n1 1 0\r\n0\n# another\n1 3 1 1\n1 0 3\n2 5 2 4 4\n"
            "x 1 2\n   \n3 2 4 5 junk 7\n")
    p = tmp_path / "messy.txt"
    p.write_text(text)
    m = same_as_oracle(p, ASCII)
    assert list(m.column(2)) == [0, 1] and list(m.column(4)) == [1, 3] and list(m.column(6)) == [2, 4, 5]


@pytest.mark.parametrize("fmt", [ASCII, BINARY])
def test_large_files_parsed_in_chunks_match_and_round_trip(tmp_path, fmt):
    # ~0.8 M columns: above the size at which the reader splits the file across threads
    m = gen.lowerstar(24, 1.5, 3)
    p = tmp_path / ("big.txt" if fmt == ASCII else "big.bin")
    write_phat(str(p), m, fmt)
    assert os.path.getsize(p) > (4 << 20)
    back = same_as_oracle(p, fmt)
    assert np.array_equal(back.dims, m.dims) and np.array_equal(back.col_ptr, m.col_ptr)
    assert np.array_equal(back.rows, m.rows)


def test_large_ascii_with_unsorted_columns_and_comments(tmp_path):
    rng = np.random.default_rng(5)
    lines = []
    for j in range(300000):
        if j % 997 == 0:
            lines.append("# comment line")
        k = int(rng.integers(0, 6))
        faces = rng.integers(0, max(j, 1), size=k)
        lines.append(" ".join([str(int(rng.integers(0, 4)))] + [str(int(x)) for x in faces]))
    p = tmp_path / "rand.txt"
    p.write_text("\n".join(lines) + "\n")
    assert os.path.getsize(p) > (4 << 20)
    same_as_oracle(p, ASCII)


def test_reader_errors(tmp_path):
    with pytest.raises(SsppError):
        read_phat(str(tmp_path / "missing.txt"))
    p = tmp_path / "trunc.bin"
    np.array([5, 1, 3, 0], dtype=np.int64).tofile(p)  # 5 columns announced, one truncated column
    with pytest.raises(SsppError):
        read_phat(str(p), BINARY)


def test_phat_module_interface(tmp_path):
    bm = phat.boundary_matrix(representation=phat.representations.vector_vector)
    bm.columns = [(0, []), (0, []), (1, [0, 1]), (0, []), (1, [1, 3]), (1, [0, 3]), (2, [2, 4, 5])]
    assert len(bm.columns) == 7 and len(bm) == 9
    assert bm.dimensions == [0, 0, 1, 0, 1, 1, 2]
    assert bm.columns[6].boundary == [2, 4, 5] and bm.columns[6].dimension == 2 and bm.columns[6].index == 6
    for mode in ("b", "t"):
        f = str(tmp_path / f"m.{mode}")
        assert bm.save(f, mode)
        other = phat.boundary_matrix()
        assert other.load(f, mode)
        assert other == bm
    copy = bm.convert(phat.representations.sparse_pivot_column)
    assert copy == bm and not (copy != bm)
    with pytest.raises(TypeError):
        bm.columns = [[0, 1]]
    pairs = phat.persistence_pairs(np.array([[5, 6], [1, 3], [2, 4]]))
    pairs.sort()
    assert list(pairs) == [(1, 3), (2, 4), (5, 6)] and len(pairs) == 3 and pairs.get_pair(0) == (1, 3)
    pairs.save(str(tmp_path / "p.txt"), "t")
    assert open(tmp_path / "p.txt").read() == open(os.path.join(GOLD, "single_triangle_pairs.dat")).read()
