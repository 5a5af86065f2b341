"""GPU parity: the CUDA engine (through the C ABI) against the oracle, bit for bit.

Pairs are compared as sorted (birth, death) arrays in input indices; essential
simplices as sorted index arrays.  Sizes are small enough for the oracle to
finish in seconds, except the full 64^3 lower-star case whose oracle run takes
a few seconds on one core.
"""
import os
import subprocess

import numpy as np
import pytest

import oracle
from helpers import dense_standard_pairs, essentials_from_pairs, random_complex
from specseqplusplus_b200 import ASCII, BINARY, Engine, Params, SpecSeqPlusPlus, SsppError, gen

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden")
CLI = os.path.join(ROOT, "specseqplusplus_b200", "bin", "specseq++")


def run(m, p=None):
    with Engine(0) as e:
        e.load_csc(m)
        e.reduce(p or Params())
        return e.pairs(), e.essentials(), e.stats()


def assert_same(m, p=None, **oracle_kw):
    ref = oracle.reduce(m, **oracle_kw)
    pairs, ess, st = run(m, p)
    assert np.array_equal(pairs, ref.pairs)
    assert np.array_equal(ess, ref.essential)
    return st, ref


def _read_pairs(path):
    lines = [ln.split() for ln in open(path).read().split("\n") if ln.strip()]
    return np.array([(int(a), int(b)) for a, b in lines[1:]], dtype=np.int64).reshape(-1, 2)


@pytest.mark.parametrize("name,fmt", [("single_triangle.dat", ASCII), ("single_triangle.bin", BINARY)])
def test_single_triangle_known_answer(name, fmt):
    want = _read_pairs(os.path.join(GOLD, "single_triangle_pairs.dat"))
    with Engine(0) as e:
        e.load_phat(os.path.join(GOLD, name), fmt)
        e.reduce(Params())
        assert np.array_equal(e.pairs(), want)
        assert list(e.essentials()) == [0]


def test_cli_matches_reference_output_bytes(tmp_path):
    out = tmp_path / "pairs.txt"
    r = subprocess.run([CLI, os.path.join(GOLD, "single_triangle.dat"), str(out), "ascii", "ascii", "0", "0", "0",
                        "102400", "1.05", "65536", "1000", "8000"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert out.read_text() == open(os.path.join(GOLD, "single_triangle_pairs.dat")).read()
    outb = tmp_path / "pairs.bin"
    r = subprocess.run([CLI, os.path.join(GOLD, "single_triangle.bin"), str(outb), "binary", "binary", "0", "0", "0",
                        "102400", "1.05", "65536", "1000", "8000"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    raw = np.fromfile(str(outb), dtype=np.int64)
    assert raw[0] == 3 and list(raw[1:]) == [1, 3, 2, 4, 5, 6]


@pytest.mark.parametrize("seed", range(16))
def test_random_small_complexes(seed):
    rng = np.random.default_rng(1000 + seed)
    m = random_complex(rng, nverts=6 + seed % 5, p=0.65, maxdim=3)
    want = dense_standard_pairs(m)
    pairs, ess, _ = run(m, Params(ss_block_size=1 + seed % 7, growth=1.0 + 0.1 * (seed % 3), level1_capacity=32,
                                  level2_capacity=32 + 32 * (seed % 2)))
    assert np.array_equal(pairs, want)
    assert np.array_equal(ess, essentials_from_pairs(m.ncols, want))


def test_rips_2000_points_reference_params():
    # Vietoris-Rips, 2000 points in [0,1]^3, r = 0.08, dim <= 3, model 0
    m = gen.rips(2000, 3, 1, 0.08, 3)
    st, ref = assert_same(m, Params(), model=0)
    assert st["active_after_init"] == ref.stats["active_after_init"]
    assert st["apparent_pairs"] == ref.stats["apparent"]
    assert st["cleared_init"] == ref.stats["cleared_init"]


@pytest.mark.parametrize("p", [
    Params(ss_block_size=64, growth=1.2, level1_capacity=32, level2_capacity=64),
    Params(ss_block_size=1 << 30, level1_capacity=64, level2_capacity=96),
    Params(ss_block_size=7, growth=1.5, queue_size=33, level1_capacity=128, level2_capacity=2048),
])
def test_schedule_and_tier_variants(p):
    # small capacities force the CTA tier and its arena (global) buffers
    assert_same(gen.rips(1500, 2, 5, 0.06, 2), p)
    assert_same(gen.lowerstar(12, 1.5, 4), p)


def test_lowerstar_32():
    assert_same(gen.lowerstar(32, 2.0, 2), Params())


def test_lowerstar_64_full_size():
    # the 64^3 Freudenthal lower-star workload: 6,573,043 columns
    m = gen.lowerstar(64, 2.0, 2)
    assert m.ncols == 6573043
    ref = oracle.reduce(m, preprocess=0)
    pairs, ess, st = run(m, Params(model=0))
    assert np.array_equal(pairs, ref.pairs)
    assert np.array_equal(ess, ref.essential)
    # size-independent checks: every simplex is paired once or essential; the
    # grid is contractible, so one essential class (a vertex)
    assert 2 * len(pairs) + len(ess) == m.ncols
    assert len(ess) == 1 and m.dims[ess[0]] == 0


def test_dense_rips_many_additions():
    m = gen.rips(1200, 2, 9, 0.1, 2)
    st, _ = assert_same(m, Params(level1_capacity=64, level2_capacity=1024))
    assert st["additions"] > 100000


def test_reference_class_mirror():
    m = gen.rips(500, 3, 3, 0.15, 3)
    ref = oracle.reduce(m)
    alg = SpecSeqPlusPlus(m, [0, 1000, 8000, 0], 0, 0, 0, 102400, 1.05, 65536)
    t_init = alg.GPU_Init()
    t_comp = alg.GPU_Compute()
    assert t_init >= 0 and t_comp >= 0
    assert np.array_equal(alg.GetPersistencePairs(), ref.pairs)


def test_deterministic_repeats():
    m = gen.lowerstar(20, 1.0, 9)
    a = run(m)
    b = run(m)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


def test_context_reuse_across_sizes():
    with Engine(0) as e:
        for m in (gen.lowerstar(10, 1.0, 1), gen.rips(900, 3, 2, 0.12, 3), gen.lowerstar(6, 1.0, 2)):
            e.load_csc(m)
            e.reduce(Params())
            ref = oracle.reduce(m)
            assert np.array_equal(e.pairs(), ref.pairs)
            assert np.array_equal(e.essentials(), ref.essential)


def test_empty_and_vertex_only_inputs():
    m = gen.BoundaryMatrix.from_columns([0, 0, 0], [[], [], []])
    pairs, ess, _ = run(m)
    assert len(pairs) == 0 and list(ess) == [0, 1, 2]
    m0 = gen.BoundaryMatrix.from_columns([], [])
    pairs, ess, _ = run(m0)
    assert len(pairs) == 0 and len(ess) == 0


@pytest.mark.parametrize("dims,cols", [
    ([0, 0, 1], [[], [], [0, 5]]),        # face index out of range
    ([0, 0, 1], [[], [], [1, 0]]),        # unsorted
    ([0, 1, 1], [[], [0], [0, 1]]),       # face of the wrong dimension
    ([0, 0, 9], [[], [], []]),            # dimension out of range
    ([0, 0, 0, 1, 1, 1, 2], [[], [], [], [0, 1], [0, 2], [1, 2], [3, 9]]),   # triangle face out of range
    ([0, 0, 0, 1, 1, 1, 2], [[], [], [], [0, 1], [0, 2], [1, 2], [1, 3]]),   # triangle face of the wrong dimension
    ([0, 0, 0, 1, 1, 1, 2], [[], [], [], [0, 1], [0, 2], [1, 2], [-4, 5]]),  # negative face index
])
@pytest.mark.parametrize("model", [0, 1, 3])
def test_malformed_inputs_are_rejected(dims, cols, model):
    # guided clearing (model bit 1) reads the input columns beside the reorder:
    # a bad face must still end as a malformed-input error, not a fault
    col_ptr = np.zeros(len(cols) + 1, dtype=np.int64)
    for j, c in enumerate(cols):
        col_ptr[j + 1] = col_ptr[j] + len(c)
    rows = np.array([x for c in cols for x in c], dtype=np.int32)
    m = gen.BoundaryMatrix(np.array(dims, dtype=np.int32), col_ptr, rows)
    with Engine(0) as e:
        e.load_csc(m)
        with pytest.raises(SsppError) as ei:
            e.reduce(Params(model=model))
        assert ei.value.code == 1
        good = gen.lowerstar(4, 1.0, 1)  # the context stays usable
        e.load_csc(good)
        e.reduce(Params(model=model))
        ref = oracle.reduce(good, model=model)
        assert np.array_equal(e.pairs(), ref.pairs)


def test_bad_params_and_call_order():
    m = gen.lowerstar(4, 1.0, 1)
    with Engine(0) as e:
        with pytest.raises(SsppError) as ei:
            e.compute()
        assert ei.value.code == 5
        e.load_csc(m)
        for bad in (Params(growth=0.9), Params(ss_block_size=0), Params(queue_size=0), Params(model=7)):
            with pytest.raises(SsppError) as ei:
                e.reduce(bad)
            assert ei.value.code == 1
        e.reduce(Params())


@pytest.mark.parametrize("seed,npts,r,maxiter", [(0, 300, 0.25, 50), (1, 600, 0.2, 10), (2, 2000, 0.08, 100),
                                                  (3, 400, 0.3, 3), (4, 500, 0.28, 64), (5, 500, 0.28, 65)])
def test_highclear_matches_oracle(seed, npts, r, maxiter):
    # model 1: the cleared set size and the pairs match the oracle's restatement
    # (max_iteration <= 64 runs on candidate masks, above on neighbour-list search)
    m = gen.rips(npts, 3, seed, r, 3)
    ref = oracle.reduce(m, model=1, max_iteration=maxiter)
    pairs, ess, st = run(m, Params(model=1, max_iteration=maxiter))
    assert st["highclear_cleared"] == ref.stats["highclear"]
    assert np.array_equal(pairs, ref.pairs)
    assert np.array_equal(ess, ref.essential)
    assert st["active_after_init"] == ref.stats["active_after_init"]


def test_highclear_lowerstar_and_2d():
    for m in (gen.lowerstar(16, 2.0, 2), gen.rips(1500, 2, 3, 0.07, 2)):
        ref = oracle.reduce(m, model=1, max_iteration=10)
        pairs, ess, st = run(m, Params(model=1, max_iteration=10))
        assert st["highclear_cleared"] == ref.stats["highclear"]
        assert np.array_equal(pairs, ref.pairs)


def test_cpp_mirror_class_end_to_end(tmp_path):
    exe = tmp_path / "mirror"
    r = subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"),
                        os.path.join(ROOT, "tests", "cpp", "mirror_main.cpp"), "-o", str(exe),
                        "-L", os.path.join(ROOT, "specseqplusplus_b200"), "-lsspp",
                        "-Wl,-rpath," + os.path.join(ROOT, "specseqplusplus_b200")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(exe), os.path.join(GOLD, "single_triangle.dat")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert r.stdout == open(os.path.join(GOLD, "single_triangle_pairs.dat")).read()


def test_batch_matches_individual_reductions():
    from specseqplusplus_b200 import workloads

    mats, _ = workloads.batch_of_rips(24, seed=9, n_min=100, n_max=1200)
    mats.append(gen.lowerstar(10, 1.0, 3))
    mats.append(gen.BoundaryMatrix.from_columns([0, 0], [[], []]))
    with Engine(0) as e:
        e.load_batch(mats)
        e.reduce(Params(model=1, max_iteration=10))
        for i, m in enumerate(mats):
            assert np.array_equal(e.batch_pairs(i), oracle.reduce(m).pairs), i


def test_batch_device_concatenation():
    torch = pytest.importorskip("torch")
    mats = [gen.rips(300, 2, s, 0.12, 2) for s in range(5)]
    dims = np.concatenate([m.dims for m in mats])
    cps, rows, c0, e0 = [np.zeros(1, np.int64)], [], 0, 0
    for m in mats:
        cps.append(m.col_ptr[1:] + e0)
        rows.append(m.rows + c0)
        c0 += m.ncols
        e0 += m.nnz
    dev = torch.device("cuda", 0)
    d_d = torch.from_numpy(dims).to(dev)
    d_c = torch.from_numpy(np.concatenate(cps)).to(dev)
    d_r = torch.from_numpy(np.concatenate(rows).astype(np.int32)).to(dev)
    with Engine(0) as e:
        e.load_batch_device([m.ncols for m in mats], d_d.data_ptr(), d_c.data_ptr(), d_r.data_ptr())
        e.reduce(Params())
        for i, m in enumerate(mats):
            assert np.array_equal(e.batch_pairs(i), oracle.reduce(m).pairs)


@pytest.fixture(scope="module")
def lowerstar64_model1():
    # the benched workload: 64^3 Freudenthal lower-star, sigma 2, seed 2;
    # model 1 (guided clearing), max_iteration 10 -- the oracle runs once
    m = gen.lowerstar(64, 2.0, 2)
    return m, oracle.reduce(m, model=1, max_iteration=10)


@pytest.mark.parametrize("l1,l2", [(32, 8192), (1000, 8000)])
def test_lowerstar_64_model1_as_benched(lowerstar64_model1, l1, l2):
    # exactly the bench's configuration (ss_block_size 102400, growth 1.05,
    # queue 65536) with the bench's level capacities and the reference defaults
    m, ref = lowerstar64_model1
    p = Params(model=1, max_iteration=10, ss_block_size=102400, growth=1.05, queue_size=65536, level1_capacity=l1,
               level2_capacity=l2)
    pairs, ess, st = run(m, p)
    assert np.array_equal(pairs, ref.pairs)
    assert np.array_equal(ess, ref.essential)
    assert st["highclear_cleared"] == ref.stats["highclear"]
    assert st["active_after_init"] == ref.stats["active_after_init"]
    assert 2 * len(pairs) + len(ess) == m.ncols
