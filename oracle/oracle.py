"""ORACLE - test infrastructure only (ctypes front end of ``sspp_oracle.cpp``).

Imported only by tests/, ``__graft_entry__.smoke()`` and bench.py's CPU
baseline leg, always as the checker.  The product path never imports it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_lib = None
_ref = None


def build(quiet: bool = True) -> None:
    out = subprocess.run(["make", "-C", _HERE, "liboracle.so"], capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)


def _load():
    global _lib
    if _lib is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        lib = ctypes.CDLL(path)
        vp = ctypes.c_void_p
        lib.oracle_run.restype = vp
        lib.oracle_run.argtypes = [ctypes.c_int64, vp, vp, vp, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32]
        lib.oracle_num_pairs.restype = ctypes.c_int64
        lib.oracle_num_pairs.argtypes = [vp]
        lib.oracle_num_essential.restype = ctypes.c_int64
        lib.oracle_num_essential.argtypes = [vp]
        for f in ("oracle_pairs", "oracle_essential", "oracle_stats"):
            getattr(lib, f).restype = None
            getattr(lib, f).argtypes = [vp, vp]
        lib.oracle_flags.restype = None
        lib.oracle_flags.argtypes = [vp, vp, vp]
        lib.oracle_adds_per_col.restype = None
        lib.oracle_adds_per_col.argtypes = [vp, vp]
        lib.oracle_free.restype = None
        lib.oracle_free.argtypes = [vp]
        lib.oracle_collapse_edges.restype = None
        lib.oracle_collapse_edges.argtypes = [ctypes.c_int64, ctypes.c_int64, vp, vp, vp]
        lib.oracle_read_phat.restype = vp
        lib.oracle_read_phat.argtypes = [ctypes.c_char_p, ctypes.c_int32]
        lib.oracle_matrix_ncols.restype = ctypes.c_int64
        lib.oracle_matrix_ncols.argtypes = [vp]
        lib.oracle_matrix_nnz.restype = ctypes.c_int64
        lib.oracle_matrix_nnz.argtypes = [vp]
        lib.oracle_matrix_copy.restype = None
        lib.oracle_matrix_copy.argtypes = [vp, vp, vp, vp]
        lib.oracle_matrix_free.restype = None
        lib.oracle_matrix_free.argtypes = [vp]
        _lib = lib
    return _lib


STAT_KEYS = ("additions", "add_bytes", "active_after_init", "cleared_init", "apparent", "highclear", "dropped")


class OracleResult:
    adds_per_col = None

    def __init__(self, pairs, essential, flags, apparent, stats):
        self.pairs = pairs            # int64 [m, 2] sorted (birth, death), input indices
        self.essential = essential    # int64 [k] unpaired, not collapsed
        self.flags = flags            # uint8 per column (see sspp_oracle.cpp oracle_flags)
        self.apparent = apparent      # int32 per row: apparent pivot column or -1
        self.stats = stats            # dict


def reduce(m, dualize: int = 0, model: int = 0, max_iteration: int = 0, preprocess: int = 1) -> OracleResult:
    lib = _load()
    dims = np.ascontiguousarray(m.dims, dtype=np.int32)
    col_ptr = np.ascontiguousarray(m.col_ptr, dtype=np.int64)
    rows = np.ascontiguousarray(m.rows, dtype=np.int32)
    n = dims.shape[0]
    h = lib.oracle_run(n, dims.ctypes.data, col_ptr.ctypes.data, rows.ctypes.data, dualize, model, max_iteration, preprocess)
    try:
        npairs = lib.oracle_num_pairs(h)
        pairs = np.empty((npairs, 2), dtype=np.int64)
        if npairs:
            lib.oracle_pairs(h, pairs.ctypes.data)
        ness = lib.oracle_num_essential(h)
        ess = np.empty(ness, dtype=np.int64)
        if ness:
            lib.oracle_essential(h, ess.ctypes.data)
        flags = np.empty(n, dtype=np.uint8)
        apparent = np.empty(n, dtype=np.int32)
        if n:
            lib.oracle_flags(h, flags.ctypes.data, apparent.ctypes.data)
        st = np.empty(7, dtype=np.int64)
        lib.oracle_stats(h, st.ctypes.data)
        apc = np.zeros(n, dtype=np.int32)
        if n:
            lib.oracle_adds_per_col(h, apc.ctypes.data)
    finally:
        lib.oracle_free(h)
    r = OracleResult(pairs, ess, flags, apparent, dict(zip(STAT_KEYS, (int(x) for x in st))))
    r.adds_per_col = apc
    return r


def collapse_edges(nverts: int, u, v) -> np.ndarray:
    lib = _load()
    u = np.ascontiguousarray(u, dtype=np.int32)
    v = np.ascontiguousarray(v, dtype=np.int32)
    out = np.zeros(u.shape[0], dtype=np.uint8)
    lib.oracle_collapse_edges(nverts, u.shape[0], u.ctypes.data, v.ctypes.data, out.ctypes.data)
    return out


def read_phat(path: str, binary: bool):
    """Returns (dims, col_ptr, rows) as read by the reference's reader semantics."""
    lib = _load()
    h = lib.oracle_read_phat(path.encode(), 1 if binary else 0)
    if not h:
        raise OSError(f"cannot read {path}")
    try:
        n = lib.oracle_matrix_ncols(h)
        nnz = lib.oracle_matrix_nnz(h)
        dims = np.empty(n, dtype=np.int32)
        col_ptr = np.empty(n + 1, dtype=np.int64)
        rows = np.empty(nnz, dtype=np.int32)
        lib.oracle_matrix_copy(h, dims.ctypes.data, col_ptr.ctypes.data, rows.ctypes.data)
    finally:
        lib.oracle_matrix_free(h)
    return dims, col_ptr, rows


def ref_collapse_available() -> bool:
    return os.path.exists(os.path.join(_HERE, "_ref", "libref_collapse.so"))


def ref_collapse_edges(u, v) -> np.ndarray:
    """Surviving-edge flags from the reference's own vendored GUDHI collapser."""
    global _ref
    if _ref is None:
        _ref = ctypes.CDLL(os.path.join(_HERE, "_ref", "libref_collapse.so"))
        _ref.ref_collapse_edges.restype = None
        _ref.ref_collapse_edges.argtypes = [ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    u = np.ascontiguousarray(u, dtype=np.int32)
    v = np.ascontiguousarray(v, dtype=np.int32)
    out = np.zeros(u.shape[0], dtype=np.uint8)
    _ref.ref_collapse_edges(u.shape[0], u.ctypes.data, v.ctypes.data, out.ctypes.data)
    return out
