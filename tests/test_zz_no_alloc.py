"""GPU test of the allocation-free entry point, sspp_reduce_noalloc.

That entry point serves callers that must not have the library allocate
device memory: a server that hands all of its GPU memory to its own pool at
start-up, or a multi-stream pipeline that cannot afford the device-wide
synchronisation cudaMalloc and cudaFree impose.  Its working memory is one
fixed 64 MiB device array owned by the library, shared by every call, so this
test also checks that a call leaves nothing behind that changes the next one:
two calls in a row (and a repeat of the first) must each give exactly the
pairs of the regular context API and of the CPU oracle, and a call that fails
(malformed input, fill-in beyond the array) must leave the next call correct.

This file sorts last so that a run stopping at the first failure has run every
other test before it.
"""
import ctypes

import numpy as np
import pytest

import oracle
from specseqplusplus_b200 import Engine, Params, SsppError, gen
from specseqplusplus_b200.engine import load_library, reduce_noalloc
from specseqplusplus_b200.gen import BoundaryMatrix

pytestmark = pytest.mark.gpu


def _context_pairs(m):
    with Engine(0) as e:
        e.load_csc(m)
        e.reduce(Params())
        return e.pairs()


def _noalloc_raw(torch, ncols, dims, col_ptr, rows):
    dev = torch.device("cuda", 0)
    d_dims = torch.from_numpy(np.ascontiguousarray(dims, dtype=np.int32)).to(dev)
    d_colptr = torch.from_numpy(np.ascontiguousarray(col_ptr, dtype=np.int64)).to(dev)
    r = np.ascontiguousarray(rows, dtype=np.int32)
    d_rows = torch.from_numpy(r if r.size else np.zeros(1, dtype=np.int32)).to(dev)
    d_pairs = torch.full((2 * max(ncols, 1),), -7, dtype=torch.int64, device=dev)
    d_npairs = torch.full((1,), -7, dtype=torch.int64, device=dev)
    stream = torch.cuda.current_stream(dev)
    reduce_noalloc(ncols, int(r.size), d_dims.data_ptr(), d_colptr.data_ptr(), d_rows.data_ptr(),
                   d_pairs.data_ptr(), d_npairs.data_ptr(), stream.cuda_stream)
    k = int(d_npairs.item())
    return d_pairs[: 2 * k].cpu().numpy().reshape(k, 2)


def _noalloc_pairs(m, torch):
    return _noalloc_raw(torch, m.ncols, m.dims, m.col_ptr, m.rows)


def test_noalloc_matches_context_api_and_oracle_on_consecutive_calls():
    torch = pytest.importorskip("torch")
    a = gen.rips(700, 3, 21, 0.14, 3)
    b = gen.lowerstar(12, 1.5, 5)
    want_a = _context_pairs(a)
    want_b = _context_pairs(b)
    assert np.array_equal(oracle.reduce(a).pairs, want_a)
    assert np.array_equal(oracle.reduce(b).pairs, want_b)
    got_a = _noalloc_pairs(a, torch)
    got_b = _noalloc_pairs(b, torch)
    got_a2 = _noalloc_pairs(a, torch)
    assert np.array_equal(got_a, want_a)
    assert np.array_equal(got_b, want_b)
    assert np.array_equal(got_a2, want_a)


def _triangle():
    # vertices 0-2, edges 3-5, one triangle 6
    return BoundaryMatrix.from_columns([0, 0, 0, 1, 1, 1, 2], [[], [], [], [0, 1], [1, 2], [0, 2], [3, 4, 5]])


@pytest.mark.parametrize("case", ["negative_col_ptr", "unsorted_rows", "wrong_face_dim", "bad_last_col_ptr",
                                  "dim_too_large"])
def test_noalloc_rejects_malformed_matrix_then_recovers(case):
    torch = pytest.importorskip("torch")
    t = _triangle()
    dims, col_ptr, rows = t.dims.copy(), t.col_ptr.copy(), t.rows.copy()
    nnz = rows.size
    if case == "negative_col_ptr":
        # a column starting below entry 0: column 5 would read rows[-4..] if unchecked
        col_ptr[5] = -4
    elif case == "unsorted_rows":
        rows[col_ptr[6]:col_ptr[7]] = rows[col_ptr[6]:col_ptr[7]][::-1]
    elif case == "wrong_face_dim":
        rows[col_ptr[6]] = 0  # a vertex as a face of the triangle
    elif case == "bad_last_col_ptr":
        col_ptr[-1] = nnz - 1
    elif case == "dim_too_large":
        dims[2] = 8
    with pytest.raises(SsppError) as ei:
        _noalloc_raw(torch, t.ncols, dims, col_ptr, rows)
    assert ei.value.code == 1 and "malformed" in str(ei.value)
    # the failed call leaves nothing that changes the next one
    m = gen.rips(300, 3, 4, 0.2, 3)
    assert np.array_equal(_noalloc_pairs(m, torch), oracle.reduce(m).pairs)
    assert np.array_equal(_noalloc_pairs(t, torch), np.array([[1, 3], [2, 4], [5, 6]], dtype=np.int64))


def test_noalloc_fill_in_overflow_is_capacity_then_recovers():
    torch = pytest.importorskip("torch")
    # 4096 vertex columns and 2000 identical edge-like columns holding every
    # vertex (not a simplicial complex, but well formed: faces one dimension
    # down, ascending).  Each of the 1999 additions writes 8192 ints of fill-in
    # and nothing is reclaimed, so the 64 MiB array runs out after about 950.
    nv, ne = 4096, 2000
    dims = np.concatenate([np.zeros(nv, np.int32), np.ones(ne, np.int32)])
    col_ptr = np.concatenate([np.zeros(nv + 1, np.int64), nv * np.arange(1, ne + 1, dtype=np.int64)])
    rows = np.tile(np.arange(nv, dtype=np.int32), ne)
    with pytest.raises(SsppError) as ei:
        _noalloc_raw(torch, nv + ne, dims, col_ptr, rows)
    assert ei.value.code == 2 and "scratch" in str(ei.value)
    m = gen.lowerstar(10, 1.0, 9)
    assert np.array_equal(_noalloc_pairs(m, torch), oracle.reduce(m).pairs)


def test_noalloc_rejects_oversized_input():
    load_library()
    with pytest.raises(SsppError) as ei:
        reduce_noalloc(1 << 21, 0, 1, 1, 1, 1, 1)
    assert ei.value.code == 1 and "too many columns" in str(ei.value)
    with pytest.raises(SsppError) as ei:
        reduce_noalloc(1000, 20_000_000, 1, 1, 1, 1, 1)
    assert ei.value.code == 1 and "too large" in str(ei.value)
    assert ctypes.sizeof(ctypes.c_int64) == 8
