"""GPU test of the allocation-free entry point, sspp_reduce_noalloc.

That entry point serves callers that must not have the library allocate
device memory: a server that hands all of its GPU memory to its own pool at
start-up, or a multi-stream pipeline that cannot afford the device-wide
synchronisation cudaMalloc and cudaFree impose.  Its working memory is one
fixed 64 MiB device array owned by the library, shared by every call, so this
test also checks that a call leaves nothing behind that changes the next one:
two calls in a row (and a repeat of the first) must each give exactly the
pairs of the regular context API.

This file sorts last so that a run stopping at the first failure has run every
other test before it.
"""
import ctypes

import numpy as np
import pytest

from specseqplusplus_b200 import Engine, Params, SsppError, gen
from specseqplusplus_b200.engine import load_library, reduce_noalloc

pytestmark = pytest.mark.gpu


def _reference_pairs(m):
    with Engine(0) as e:
        e.load_csc(m)
        e.reduce(Params())
        return e.pairs()


def _noalloc_pairs(m, torch):
    dev = torch.device("cuda", 0)
    d_dims = torch.from_numpy(m.dims).to(dev)
    d_colptr = torch.from_numpy(m.col_ptr).to(dev)
    d_rows = torch.from_numpy(m.rows if m.nnz else np.zeros(1, dtype=np.int32)).to(dev)
    d_pairs = torch.full((2 * max(m.ncols, 1),), -7, dtype=torch.int64, device=dev)
    d_npairs = torch.full((1,), -7, dtype=torch.int64, device=dev)
    stream = torch.cuda.current_stream(dev)
    reduce_noalloc(m.ncols, m.nnz, d_dims.data_ptr(), d_colptr.data_ptr(), d_rows.data_ptr(), d_pairs.data_ptr(),
                   d_npairs.data_ptr(), stream.cuda_stream)
    k = int(d_npairs.item())
    return d_pairs[: 2 * k].cpu().numpy().reshape(k, 2)


def test_noalloc_matches_context_api_on_consecutive_calls():
    torch = pytest.importorskip("torch")
    a = gen.rips(700, 3, 21, 0.14, 3)
    b = gen.lowerstar(12, 1.5, 5)
    want_a = _reference_pairs(a)
    want_b = _reference_pairs(b)
    got_a = _noalloc_pairs(a, torch)
    got_b = _noalloc_pairs(b, torch)
    got_a2 = _noalloc_pairs(a, torch)
    assert np.array_equal(got_a, want_a)
    assert np.array_equal(got_b, want_b)
    assert np.array_equal(got_a2, want_a)


def test_noalloc_rejects_oversized_input():
    load_library()
    with pytest.raises(SsppError) as ei:
        reduce_noalloc(1 << 21, 0, 1, 1, 1, 1, 1)
    assert ei.value.code == 1 and "too many columns" in str(ei.value)
    with pytest.raises(SsppError) as ei:
        reduce_noalloc(1000, 20_000_000, 1, 1, 1, 1, 1)
    assert ei.value.code == 1 and "too large" in str(ei.value)
    assert ctypes.sizeof(ctypes.c_int64) == 8
