"""The reference's own engine (src/main.cu with include/*.h, built from the
reference tree by oracle/Makefile into oracle/_ref/specseq_ref) run on the GPU
as a cross-check of the oracle: its pairs on the reference's known-answer
triangle and on the 2,000-point Rips workload (model 0, the reference's default
block sizes and level capacities 1000 / 8000) must equal the oracle's.

Skipped where the binary was not built (it needs the reference tree at build
time: SSPP_REFERENCE).
"""
import os
import subprocess

import numpy as np
import pytest

import oracle
from specseqplusplus_b200 import gen
from specseqplusplus_b200.engine import write_phat

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref", "specseq_ref")
GOLD = os.path.join(ROOT, "tests", "golden")
ARGS = ["ascii", "ascii", "0", "0", "0", "102400", "1.05", "65536", "1000", "8000"]


def _pairs(path):
    lines = [ln.split() for ln in open(path).read().split("\n") if ln.strip()]
    assert int(lines[0][0]) == len(lines) - 1
    return np.array(sorted((int(a), int(b)) for a, b in lines[1:]), dtype=np.int64).reshape(-1, 2)


def _run(inp, out):
    r = subprocess.run([REF, str(inp), str(out)] + ARGS, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    return _pairs(out)


@pytest.mark.skipif(not os.path.exists(REF), reason="reference engine not built (set SSPP_REFERENCE at build time)")
def test_reference_engine_known_triangle(tmp_path):
    got = _run(os.path.join(GOLD, "single_triangle.dat"), tmp_path / "p.txt")
    assert np.array_equal(got, _pairs(os.path.join(GOLD, "single_triangle_pairs.dat")))


@pytest.mark.skipif(not os.path.exists(REF), reason="reference engine not built (set SSPP_REFERENCE at build time)")
def test_reference_engine_rips_2000_equals_oracle(tmp_path):
    m = gen.rips(2000, 3, 1, 0.08, 3)
    inp = tmp_path / "rips2000.txt"
    write_phat(str(inp), m)
    got = _run(inp, tmp_path / "p.txt")
    assert np.array_equal(got, oracle.reduce(m).pairs)
