"""Python host mirror of the engine's C ABI (``include/sspp.h``).

``SpecSeqPlusPlus`` keeps the reference's class interface
(``include/specseq.h:486-512``: constructor with the matrix and the CLI
parameters, ``GPU_Init``, ``GPU_Compute``, ``GetPersistencePairs``); ``Engine``
is the lower-level context wrapper.  All computation happens in ``libsspp.so``
on the GPU: if the library cannot be loaded this module raises, there is no
CPU path.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, fields

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libsspp.so")

OK, ERR_BAD_INPUT, ERR_CAPACITY, ERR_CUDA, ERR_TIMEOUT, ERR_STATE, ERR_IO = range(7)
ASCII, BINARY = 0, 1
_ERR_NAMES = {1: "BAD_INPUT", 2: "CAPACITY", 3: "CUDA", 4: "TIMEOUT", 5: "STATE", 6: "IO"}


class SsppError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{_ERR_NAMES.get(code, code)}] {msg}")
        self.code = code


class _Config(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int32), ("arena_bytes", ctypes.c_int64), ("verbose", ctypes.c_int32),
                ("profile", ctypes.c_int32), ("host_threads", ctypes.c_int32), ("sm_share", ctypes.c_int32)]


class _Params(ctypes.Structure):
    _fields_ = [("dualize", ctypes.c_int32), ("model", ctypes.c_int32), ("max_iteration", ctypes.c_int32),
                ("ss_block_size", ctypes.c_int32), ("growth", ctypes.c_float), ("queue_size", ctypes.c_int32),
                ("level1_capacity", ctypes.c_int32), ("level2_capacity", ctypes.c_int32),
                ("autotune", ctypes.c_int32), ("heavy_threads", ctypes.c_int32), ("representatives", ctypes.c_int32),
                ("schedule", ctypes.c_int32)]


class _BuildSpec(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("maxdim", ctypes.c_int32), ("size", ctypes.c_int64 * 3),
                ("data", ctypes.c_void_p), ("radius", ctypes.c_float)]


class _Stats(ctypes.Structure):
    _fields_ = [(k, ctypes.c_int64) for k in (
        "ncols", "nnz", "active_after_init", "apparent_pairs", "cleared_init", "highclear_cleared",
        "collapse_dropped", "additions", "add_ints", "published_ints", "displaced", "ss_steps", "npairs",
        "nessential")] + [("init_ms", ctypes.c_double), ("compute_ms", ctypes.c_double), ("launches", ctypes.c_int64)] + [
        (k, ctypes.c_double) for k in ("init_gpu_ms", "light_gpu_ms", "heavy_gpu_ms", "pairs_gpu_ms")] + [
        ("light_launches", ctypes.c_int64), ("heavy_launches", ctypes.c_int64), ("arena_ints_used", ctypes.c_int64),
        ("tuned_candidate", ctypes.c_int64), ("heavy_additions", ctypes.c_int64), ("build_ms", ctypes.c_double),
        ("heavy_fast_inline", ctypes.c_int64), ("heavy_fast_slot", ctypes.c_int64)]


class _ServerConfig(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int32), ("workers", ctypes.c_int32), ("memory_budget", ctypes.c_int64),
                ("max_batch_cols", ctypes.c_int64), ("max_batch_requests", ctypes.c_int32),
                ("batch_window_ms", ctypes.c_double)]


class _ServerStats(ctypes.Structure):
    _fields_ = [(k, ctypes.c_int64) for k in ("submitted", "completed", "failed", "rejected", "batches", "columns")] + [
        (k, ctypes.c_double) for k in ("wall_s", "cols_per_s", "p50_ms", "p95_ms", "p99_ms", "max_ms", "mean_ms",
                                       "mean_batch_requests", "load_s", "reduce_s", "results_s")]


@dataclass
class Params:
    """The reference's CLI parameters (src/main.cu:281-294, README.md:26-51)."""

    dualize: int = 0
    model: int = 0
    max_iteration: int = 0
    ss_block_size: int = 102400
    growth: float = 1.05
    queue_size: int = 65536
    level1_capacity: int = 1000
    level2_capacity: int = 8000
    autotune: int = 0
    heavy_threads: int = 0
    representatives: int = 0
    schedule: int = 0  # 1 (= 0) host loop of per-block launches, 2 one persistent device work-queue launch

    def _c(self) -> _Params:
        return _Params(*(getattr(self, f.name) for f in fields(self)))


_lib = None


def load_library():
    """Loads libsspp.so; raises if it is missing (no fallback path exists)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with __graft_entry__.build()")
    lib = ctypes.CDLL(LIB_PATH)
    vp, i32, i64 = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64
    sig = {
        "sspp_create": (vp, [ctypes.POINTER(_Config)]),
        "sspp_destroy": (None, [vp]),
        "sspp_last_error": (ctypes.c_char_p, [vp]),
        "sspp_default_params": (None, [ctypes.POINTER(_Params)]),
        "sspp_load_phat": (i32, [vp, ctypes.c_char_p, i32]),
        "sspp_load_csc": (i32, [vp, i64, vp, vp, vp]),
        "sspp_load_csc_device": (i32, [vp, i64, vp, vp, vp]),
        "sspp_load_rips": (i32, [vp, i64, i32, vp, ctypes.c_float, i32]),
        "sspp_load_lowerstar": (i32, [vp, i64, i64, i64, vp, i32]),
        "sspp_input_size": (i32, [vp, vp, vp]),
        "sspp_input_copy": (i32, [vp, vp, vp, vp, vp]),
        "sspp_representative": (i64, [vp, i64, vp, i64]),
        "sspp_server_submit_rips": (i64, [vp, i64, i32, vp, ctypes.c_float, i32, i32]),
        "sspp_server_submit_lowerstar": (i64, [vp, i64, i64, i64, vp, i32, i32]),
        "sspp_server_values": (i64, [vp, i64, vp, i64]),
        "sspp_init": (i32, [vp, ctypes.POINTER(_Params), vp]),
        "sspp_compute": (i32, [vp, vp]),
        "sspp_reduce": (i32, [vp, ctypes.POINTER(_Params), vp]),
        "sspp_num_pairs": (i64, [vp]),
        "sspp_pairs": (i64, [vp, vp, i64]),
        "sspp_num_essential": (i64, [vp]),
        "sspp_essentials": (i64, [vp, vp, i64]),
        "sspp_write_pairs": (i32, [vp, ctypes.c_char_p, i32]),
        "sspp_get_stats": (i32, [vp, ctypes.POINTER(_Stats)]),
        "sspp_reduce_noalloc": (i32, [i64, i64, vp, vp, vp, vp, vp, vp, ctypes.c_char_p, i32]),
        "sspp_load_batch": (i32, [vp, i32, vp, vp, vp, vp]),
        "sspp_load_batch_device": (i32, [vp, i32, vp, vp, vp, vp]),
        "sspp_load_built_batch": (i32, [vp, i32, vp]),
        "sspp_batch_values": (i64, [vp, i32, vp, i64]),
        "sspp_batch_num_pairs": (i64, [vp, i32]),
        "sspp_batch_pairs": (i64, [vp, i32, vp, i64]),
        "sspp_get_params": (i32, [vp, ctypes.POINTER(_Params)]),
        "sspp_batch_num_essential": (i64, [vp, i32]),
        "sspp_batch_essentials": (i64, [vp, i32, vp, i64]),
        "sspp_batch_counts": (i32, [vp, vp, vp]),
        "sspp_batch_copy": (i32, [vp, vp, vp]),
        "sspp_server_create": (vp, [ctypes.POINTER(_ServerConfig), ctypes.POINTER(_Params)]),
        "sspp_server_destroy": (None, [vp]),
        "sspp_server_last_error": (ctypes.c_char_p, [vp]),
        "sspp_server_submit": (i64, [vp, i64, vp, vp, vp, i32]),
        "sspp_server_wait": (i32, [vp, i64, ctypes.c_double]),
        "sspp_server_state": (i32, [vp, i64]),
        "sspp_server_result": (i32, [vp, i64, ctypes.c_char_p, i32]),
        "sspp_server_num_pairs": (i64, [vp, i64]),
        "sspp_server_pairs": (i64, [vp, i64, vp, i64]),
        "sspp_server_num_essential": (i64, [vp, i64]),
        "sspp_server_essentials": (i64, [vp, i64, vp, i64]),
        "sspp_server_latency_ms": (ctypes.c_double, [vp, i64]),
        "sspp_server_release": (i32, [vp, i64]),
        "sspp_server_get_stats": (i32, [vp, ctypes.POINTER(_ServerStats)]),
        "sspp_server_reset_stats": (i32, [vp]),
        "sspp_export_preprocessed": (i32, [vp, ctypes.POINTER(_Params), ctypes.c_char_p, i32]),
        "sspp_phat_read": (vp, [ctypes.c_char_p, i32, ctypes.c_char_p, i32]),
        "sspp_phat_ncols": (i64, [vp]),
        "sspp_phat_nnz": (i64, [vp]),
        "sspp_phat_copy": (i32, [vp, vp, vp, vp]),
        "sspp_phat_free": (None, [vp]),
        "sspp_phat_write": (i32, [ctypes.c_char_p, i32, i64, vp, vp, vp, ctypes.c_char_p, i32]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


EXPORTED = ("sspp_create", "sspp_destroy", "sspp_last_error", "sspp_default_params", "sspp_load_phat",
            "sspp_load_csc", "sspp_load_csc_device", "sspp_init", "sspp_compute", "sspp_reduce", "sspp_num_pairs",
            "sspp_pairs", "sspp_num_essential", "sspp_essentials", "sspp_write_pairs", "sspp_get_stats",
            "sspp_reduce_noalloc", "sspp_load_batch", "sspp_load_batch_device", "sspp_load_built_batch",
            "sspp_batch_values", "sspp_batch_num_pairs",
            "sspp_batch_pairs", "sspp_get_params", "sspp_batch_num_essential", "sspp_batch_essentials",
            "sspp_batch_counts", "sspp_batch_copy",
            "sspp_server_create", "sspp_server_destroy", "sspp_server_last_error", "sspp_server_submit",
            "sspp_server_wait", "sspp_server_state", "sspp_server_result", "sspp_server_num_pairs",
            "sspp_server_pairs", "sspp_server_num_essential", "sspp_server_essentials", "sspp_server_latency_ms",
            "sspp_server_release", "sspp_server_get_stats", "sspp_server_reset_stats", "sspp_phat_read",
            "sspp_phat_ncols", "sspp_phat_nnz", "sspp_phat_copy", "sspp_phat_free", "sspp_phat_write",
            "sspp_export_preprocessed", "sspp_load_rips", "sspp_load_lowerstar", "sspp_input_size",
            "sspp_input_copy", "sspp_representative", "sspp_server_submit_rips", "sspp_server_submit_lowerstar",
            "sspp_server_values")


class Engine:
    """One device context (include/sspp.h)."""

    def __init__(self, device: int = 0, arena_bytes: int = 0, verbose: int = 0, profile: int = 0):
        self._lib = load_library()
        cfg = _Config(device, arena_bytes, verbose, profile)
        self._h = self._lib.sspp_create(ctypes.byref(cfg))
        if not self._h:
            raise SsppError(ERR_CUDA, "sspp_create failed (no usable CUDA device?)")

    def close(self):
        if getattr(self, "_h", None):
            self._lib.sspp_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, rc: int):
        if rc != OK:
            raise SsppError(rc, self._lib.sspp_last_error(self._h).decode(errors="replace"))

    def load_csc(self, m) -> None:
        dims = np.ascontiguousarray(m.dims, dtype=np.int32)
        col_ptr = np.ascontiguousarray(m.col_ptr, dtype=np.int64)
        rows = np.ascontiguousarray(m.rows, dtype=np.int32)
        self._check(self._lib.sspp_load_csc(self._h, dims.shape[0], dims.ctypes.data, col_ptr.ctypes.data,
                                            rows.ctypes.data))
        self._batch_k = 0

    def load_csc_device(self, ncols: int, d_dims: int, d_col_ptr: int, d_rows: int) -> None:
        self._check(self._lib.sspp_load_csc_device(self._h, ncols, d_dims, d_col_ptr, d_rows))

    @staticmethod
    def _float_buffer(x, shape_ndim: int):
        """(pointer, shape, keep-alive) of a float32 array: a CUDA tensor is read in place."""
        if hasattr(x, "data_ptr") and getattr(x, "is_cuda", False):
            import torch

            if x.dtype != torch.float32 or not x.is_contiguous() or x.dim() != shape_ndim:
                raise ValueError(f"expected a contiguous float32 tensor of {shape_ndim} dimensions")
            return x.data_ptr(), tuple(x.shape), x
        a = np.ascontiguousarray(x, dtype=np.float32)
        if a.ndim != shape_ndim:
            raise ValueError(f"expected an array of {shape_ndim} dimensions")
        return a.ctypes.data, a.shape, a

    def load_rips(self, points, radius: float, maxdim: int = 3) -> None:
        """Builds the Vietoris-Rips complex of ``points`` [npts, D] (float32, D = 1..3; a numpy array or a
        CUDA tensor) on the device and loads it; same matrix as ``gen.rips_from_points``."""
        ptr, shape, keep = self._float_buffer(points, 2)
        self._check(self._lib.sspp_load_rips(self._h, shape[0], shape[1], ptr if shape[0] else None,
                                             float(radius), int(maxdim)))
        del keep
        self._batch_k = 0

    def load_lowerstar(self, values, maxdim: int = 3) -> None:
        """Builds the Freudenthal lower-star filtration of the field ``values`` [gz, gy, gx] (float32, x
        fastest; a numpy array or a CUDA tensor) on the device and loads it; same matrix as
        ``gen.lowerstar_from_field``."""
        ptr, shape, keep = self._float_buffer(values, 3)
        gz, gy, gx = shape
        self._check(self._lib.sspp_load_lowerstar(self._h, gx, gy, gz, ptr, int(maxdim)))
        del keep
        self._batch_k = 0

    def representative(self, death: int) -> np.ndarray:
        """Representative cycle (input indices, ascending) of the pair whose death is ``death``;
        needs a reduction with ``Params(representatives=1)`` (dualize 0)."""
        n = self._lib.sspp_representative(self._h, int(death), None, 0)
        if n < 0:
            raise SsppError(ERR_BAD_INPUT, self._lib.sspp_last_error(self._h).decode(errors="replace"))
        out = np.empty(max(n, 1), dtype=np.int64)
        self._lib.sspp_representative(self._h, int(death), out.ctypes.data, n)
        return out[:n]

    def input_matrix(self, values: bool = False):
        """The loaded matrix copied back (with its filtration values for a built complex)."""
        from .gen import BoundaryMatrix

        n = ctypes.c_int64()
        z = ctypes.c_int64()
        self._check(self._lib.sspp_input_size(self._h, ctypes.byref(n), ctypes.byref(z)))
        dims = np.empty(n.value, dtype=np.int32)
        col_ptr = np.empty(n.value + 1, dtype=np.int64)
        rows = np.empty(max(z.value, 1), dtype=np.int32)
        vals = np.empty(max(n.value, 1), dtype=np.float32) if values else None
        self._check(self._lib.sspp_input_copy(self._h, dims.ctypes.data, col_ptr.ctypes.data, rows.ctypes.data,
                                              vals.ctypes.data if values else None))
        return BoundaryMatrix(dims, col_ptr, rows[:z.value], vals[:n.value] if values else None)

    def load_batch(self, matrices) -> None:
        """k independent complexes reduced together (block-diagonal concatenation)."""
        ms = list(matrices)
        k = len(ms)
        keep = [(np.ascontiguousarray(m.dims, dtype=np.int32), np.ascontiguousarray(m.col_ptr, dtype=np.int64),
                 np.ascontiguousarray(m.rows if m.nnz else np.zeros(1, np.int32), dtype=np.int32)) for m in ms]
        ncols = np.array([m.ncols for m in ms], dtype=np.int64)
        arr = lambda i: (ctypes.c_void_p * max(k, 1))(*[t[i].ctypes.data for t in keep])
        self._check(self._lib.sspp_load_batch(self._h, k, ncols.ctypes.data, arr(0), arr(1), arr(2)))
        self._batch_k = k

    def load_built_batch(self, requests) -> None:
        """Builds several complexes on the device and loads them as one batch: each request is
        ("rips", points [npts, D], radius, maxdim) or ("lowerstar", field [gz, gy, gx], maxdim), as
        load_rips / load_lowerstar take them; results come back per complex (batch_pairs ...)."""
        reqs = list(requests)
        specs = (_BuildSpec * max(len(reqs), 1))()
        keep = []
        for i, r in enumerate(reqs):
            if r[0] == "rips":
                ptr, shape, k_ = self._float_buffer(r[1], 2)
                specs[i].kind = 0
                specs[i].size[0], specs[i].size[1], specs[i].size[2] = shape[0], shape[1], 0
                specs[i].radius = float(r[2])
                specs[i].maxdim = int(r[3])
            elif r[0] == "lowerstar":
                ptr, shape, k_ = self._float_buffer(r[1], 3)
                specs[i].kind = 1
                specs[i].size[0], specs[i].size[1], specs[i].size[2] = shape[2], shape[1], shape[0]
                specs[i].maxdim = int(r[2])
            else:
                raise ValueError(f"unknown request kind {r[0]!r}")
            specs[i].data = ptr
            keep.append(k_)
        self._check(self._lib.sspp_load_built_batch(self._h, len(reqs), specs))
        del keep
        self._batch_k = len(reqs)

    def batch_values(self, i: int) -> np.ndarray:
        """Column filtration values of complex i of a built batch."""
        n = self._lib.sspp_batch_values(self._h, i, None, 0)
        if n < 0:
            self._check(ERR_STATE)
        out = np.empty(max(n, 1), dtype=np.float32)
        self._lib.sspp_batch_values(self._h, i, out.ctypes.data, n)
        return out[:n]

    def load_batch_device(self, ncols, d_dims: int, d_col_ptr: int, d_rows: int) -> None:
        nc = np.ascontiguousarray(ncols, dtype=np.int64)
        self._check(self._lib.sspp_load_batch_device(self._h, nc.shape[0], nc.ctypes.data, d_dims, d_col_ptr, d_rows))
        self._batch_k = int(nc.shape[0])

    def batch_pairs(self, i: int) -> np.ndarray:
        n = self._lib.sspp_batch_num_pairs(self._h, i)
        if n < 0:
            self._check(ERR_STATE)
        out = np.empty((n, 2), dtype=np.int64)
        if self._lib.sspp_batch_pairs(self._h, i, out.ctypes.data, n) != n:
            self._check(ERR_CUDA)
        return out

    def batch_results(self) -> list:
        """[(pairs, essentials)] of every complex of the batch, in one staged copy."""
        k = getattr(self, "_batch_k", 0)
        np_ = np.zeros(max(k, 1), dtype=np.int64)
        ne_ = np.zeros(max(k, 1), dtype=np.int64)
        self._check(self._lib.sspp_batch_counts(self._h, np_.ctypes.data, ne_.ctypes.data))
        outs = [(np.empty((int(np_[i]), 2), dtype=np.int64), np.empty(int(ne_[i]), dtype=np.int64)) for i in range(k)]
        po = (ctypes.c_void_p * max(k, 1))(*[o[0].ctypes.data for o in outs])
        eo = (ctypes.c_void_p * max(k, 1))(*[o[1].ctypes.data for o in outs])
        self._check(self._lib.sspp_batch_copy(self._h, po, eo))
        return outs

    def batch_essentials(self, i: int) -> np.ndarray:
        n = self._lib.sspp_batch_num_essential(self._h, i)
        if n < 0:
            self._check(ERR_STATE)
        out = np.empty(n, dtype=np.int64)
        if self._lib.sspp_batch_essentials(self._h, i, out.ctypes.data, n) != n:
            self._check(ERR_CUDA)
        return out

    def export_preprocessed(self, path: str, params: Params | None = None, fmt: int = ASCII) -> None:
        """Writes the loaded matrix with guided clearing / edge collapse applied (cleared and dropped
        columns as dimension-only lines), as the reference's HIGHOUT build does."""
        p = (params or Params())._c()
        self._check(self._lib.sspp_export_preprocessed(self._h, ctypes.byref(p), str(path).encode(), fmt))

    def load_phat(self, path: str, fmt: int = ASCII) -> None:
        self._check(self._lib.sspp_load_phat(self._h, path.encode(), fmt))

    def init(self, params: Params | None = None, stream: int = 0) -> None:
        p = (params or Params())._c()
        self._check(self._lib.sspp_init(self._h, ctypes.byref(p), stream or None))

    def compute(self, stream: int = 0) -> None:
        self._check(self._lib.sspp_compute(self._h, stream or None))

    def reduce(self, params: Params | None = None, stream: int = 0) -> None:
        p = (params or Params())._c()
        self._check(self._lib.sspp_reduce(self._h, ctypes.byref(p), stream or None))

    def num_pairs(self) -> int:
        return int(self._lib.sspp_num_pairs(self._h))

    def num_essential(self) -> int:
        return int(self._lib.sspp_num_essential(self._h))

    def pairs(self, out: np.ndarray | None = None) -> np.ndarray:
        """Sorted (birth, death) pairs; `out` (int64, >= 2 * npairs entries, e.g. pinned) is filled if given."""
        n = self._lib.sspp_num_pairs(self._h)
        if n < 0:
            self._check(ERR_STATE)
        if out is None:
            out = np.empty((n, 2), dtype=np.int64)
        got = self._lib.sspp_pairs(self._h, out.ctypes.data, n)
        if got != n:
            self._check(ERR_CUDA)
        return out.reshape(-1)[: 2 * n].reshape(n, 2)

    def essentials(self, out: np.ndarray | None = None) -> np.ndarray:
        n = self._lib.sspp_num_essential(self._h)
        if n < 0:
            self._check(ERR_STATE)
        if out is None:
            out = np.empty(n, dtype=np.int64)
        got = self._lib.sspp_essentials(self._h, out.ctypes.data, n)
        if got != n:
            self._check(ERR_CUDA)
        return out[:n]

    def write_pairs(self, path: str, fmt: int = ASCII) -> None:
        self._check(self._lib.sspp_write_pairs(self._h, path.encode(), fmt))

    def stats(self) -> dict:
        st = _Stats()
        self._check(self._lib.sspp_get_stats(self._h, ctypes.byref(st)))
        return {k: getattr(st, k) for k, _ in _Stats._fields_}

    def params(self) -> Params:
        """Parameters of the last init, autotuned values included."""
        p = _Params()
        self._check(self._lib.sspp_get_params(self._h, ctypes.byref(p)))
        return Params(*(getattr(p, f) for f, _ in _Params._fields_))


def reduce_noalloc(ncols: int, nnz: int, d_dims: int, d_col_ptr: int, d_rows: int, d_pairs: int, d_npairs: int,
                   stream: int = 0) -> None:
    """Allocation-free reduction on device buffers (sspp_reduce_noalloc in include/sspp.h).

    For callers that must not have the library allocate device memory: all
    working memory is a fixed 64 MiB device array owned by the library.  All
    pointers are device addresses; d_pairs needs room for 2 * ncols int64.
    """
    lib = load_library()
    msg = ctypes.create_string_buffer(256)
    rc = lib.sspp_reduce_noalloc(ncols, nnz, d_dims, d_col_ptr, d_rows, d_pairs, d_npairs, stream or None, msg, 256)
    if rc != OK:
        raise SsppError(rc, msg.value.decode(errors="replace"))


def compute_persistence_pairs(m, params: Params | None = None, device: int = 0):
    """Sorted (birth, death) pairs and essential simplices of a boundary matrix."""
    with Engine(device) as e:
        e.load_csc(m)
        e.reduce(params)
        return e.pairs(), e.essentials()


class SpecSeqPlusPlus:
    """Mirror of the reference's host class (include/specseq.h:486-512, 513, 592, 1182).

    ``level_capacity`` is the reference's 4-entry array whose entries 1 and 2 are
    the CLI's level-1/level-2 capacities (src/main.cu:292-294).
    """

    def __init__(self, matrix, level_capacity, dualize, model, highclear_maxneighbors, ss_block_size,
                 block_size_growth_rate, queue_size, device: int = 0):
        self.params = Params(dualize=int(dualize), model=int(model), max_iteration=int(highclear_maxneighbors),
                             ss_block_size=int(ss_block_size), growth=float(block_size_growth_rate),
                             queue_size=int(queue_size), level1_capacity=int(level_capacity[1]),
                             level2_capacity=int(level_capacity[2]))
        self._e = Engine(device)
        self._e.load_csc(matrix)

    def GPU_Init(self) -> float:
        self._e.init(self.params)
        return self._e.stats()["init_ms"] / 1000.0

    def GPU_Compute(self) -> float:
        self._e.compute()
        return self._e.stats()["compute_ms"] / 1000.0

    def GetPersistencePairs(self) -> np.ndarray:
        return self._e.pairs()

    def GetEssentials(self) -> np.ndarray:
        return self._e.essentials()

    def stats(self) -> dict:
        return self._e.stats()


REQ_QUEUED, REQ_RUNNING, REQ_DONE, REQ_FAILED = 0, 1, 2, 3


class Server:
    """Resident request loop with continuous batching (sspp_server_* in include/sspp.h).

    submit() queues a complex and returns its id; workers reduce queued
    requests in batches as they free up; wait() / pairs() / essentials() read
    one request's results in its own indices.  With copy=False the matrix's
    arrays are referenced, not copied, and kept alive here until release().
    """

    def __init__(self, params: Params | None = None, device: int = 0, workers: int = 2, memory_budget: int = 0,
                 max_batch_cols: int = 0, max_batch_requests: int = 0, batch_window_ms: float = 0.0):
        self._lib = load_library()
        cfg = _ServerConfig(device, workers, memory_budget, max_batch_cols, max_batch_requests, batch_window_ms)
        p = (params or Params())._c()
        self._h = self._lib.sspp_server_create(ctypes.byref(cfg), ctypes.byref(p))
        if not self._h:
            raise SsppError(ERR_CUDA, "sspp_server_create failed (no usable CUDA device)")
        self._keep = {}

    def close(self) -> None:
        if self._h:
            self._lib.sspp_server_destroy(self._h)
            self._h = None
            self._keep.clear()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, m, copy: bool = True) -> int:
        dims = np.ascontiguousarray(m.dims, dtype=np.int32)
        col_ptr = np.ascontiguousarray(m.col_ptr, dtype=np.int64)
        rows = np.ascontiguousarray(m.rows if m.nnz else np.zeros(1, np.int32), dtype=np.int32)
        rid = self._lib.sspp_server_submit(self._h, dims.shape[0], dims.ctypes.data, col_ptr.ctypes.data,
                                           rows.ctypes.data, 0 if copy else 1)
        if rid < 0:
            raise SsppError(-rid, self._lib.sspp_server_last_error(self._h).decode(errors="replace"))
        if not copy:
            self._keep[rid] = (dims, col_ptr, rows)
        return int(rid)

    def _submitted(self, rid: int, keep) -> int:
        if rid < 0:
            raise SsppError(-rid, self._lib.sspp_server_last_error(self._h).decode(errors="replace"))
        if keep is not None:
            self._keep[rid] = keep
        return int(rid)

    def submit_rips(self, points, radius: float, maxdim: int = 3, values: bool = False, copy: bool = True) -> int:
        """A point cloud [npts, D] (float32) whose Rips complex the server builds and reduces."""
        pts = np.ascontiguousarray(points, dtype=np.float32)
        flags = (0 if copy else 1) | (2 if values else 0)
        rid = self._lib.sspp_server_submit_rips(self._h, pts.shape[0], pts.shape[1], pts.ctypes.data if pts.size else None,
                                                float(radius), int(maxdim), flags)
        return self._submitted(rid, None if copy else pts)

    def submit_lowerstar(self, field, maxdim: int = 3, values: bool = False, copy: bool = True) -> int:
        """A field [gz, gy, gx] (float32, x fastest) whose Freudenthal lower-star filtration the server builds
        and reduces."""
        f = np.ascontiguousarray(field, dtype=np.float32)
        gz, gy, gx = f.shape
        flags = (0 if copy else 1) | (2 if values else 0)
        rid = self._lib.sspp_server_submit_lowerstar(self._h, gx, gy, gz, f.ctypes.data, int(maxdim), flags)
        return self._submitted(rid, None if copy else f)

    def values(self, rid: int) -> np.ndarray:
        """Filtration values of a built request's matrix (submitted with values=True)."""
        self.wait(rid)
        n = self._lib.sspp_server_values(self._h, rid, None, 0)
        if n < 0:
            raise SsppError(ERR_STATE, "no values kept for this request")
        out = np.empty(max(n, 1), dtype=np.float32)
        self._lib.sspp_server_values(self._h, rid, out.ctypes.data, n)
        return out[:n]

    def wait(self, rid: int, timeout_ms: float = -1.0) -> bool:
        rc = self._lib.sspp_server_wait(self._h, rid, timeout_ms)
        if rc == ERR_TIMEOUT:
            return False
        if rc != OK:
            raise SsppError(rc, "unknown request id")
        return True

    def state(self, rid: int) -> int:
        return int(self._lib.sspp_server_state(self._h, rid))

    def _raise_failed(self, rid: int) -> None:
        buf = ctypes.create_string_buffer(512)
        rc = self._lib.sspp_server_result(self._h, rid, buf, 512)
        if rc != OK:
            raise SsppError(rc, buf.value.decode(errors="replace"))

    def pairs(self, rid: int) -> np.ndarray:
        self.wait(rid)
        self._raise_failed(rid)
        n = self._lib.sspp_server_num_pairs(self._h, rid)
        out = np.empty((max(n, 0), 2), dtype=np.int64)
        if n > 0:
            self._lib.sspp_server_pairs(self._h, rid, out.ctypes.data, n)
        return out

    def essentials(self, rid: int) -> np.ndarray:
        self.wait(rid)
        self._raise_failed(rid)
        n = self._lib.sspp_server_num_essential(self._h, rid)
        out = np.empty(max(n, 0), dtype=np.int64)
        if n > 0:
            self._lib.sspp_server_essentials(self._h, rid, out.ctypes.data, n)
        return out

    def latency_ms(self, rid: int) -> float:
        return float(self._lib.sspp_server_latency_ms(self._h, rid))

    def release(self, rid: int) -> None:
        self._lib.sspp_server_release(self._h, rid)
        self._keep.pop(rid, None)

    def stats(self) -> dict:
        st = _ServerStats()
        self._lib.sspp_server_get_stats(self._h, ctypes.byref(st))
        return {k: getattr(st, k) for k, _ in _ServerStats._fields_}

    def reset_stats(self) -> None:
        self._lib.sspp_server_reset_stats(self._h)


def read_phat(path: str, fmt: int = ASCII):
    """PHAT boundary matrix from a file, read on the host by the library's reader
    (processFiles semantics: 0-based faces, columns sorted and de-duplicated)."""
    from .gen import BoundaryMatrix

    lib = load_library()
    err = ctypes.create_string_buffer(256)
    h = lib.sspp_phat_read(str(path).encode(), fmt, err, 256)
    if not h:
        raise SsppError(ERR_IO, err.value.decode(errors="replace"))
    try:
        n, nnz = lib.sspp_phat_ncols(h), lib.sspp_phat_nnz(h)
        dims = np.empty(n, dtype=np.int32)
        col_ptr = np.empty(n + 1, dtype=np.int64)
        rows = np.empty(max(nnz, 1), dtype=np.int32)
        lib.sspp_phat_copy(h, dims.ctypes.data, col_ptr.ctypes.data, rows.ctypes.data)
    finally:
        lib.sspp_phat_free(h)
    return BoundaryMatrix(dims, col_ptr, rows[:nnz])


def write_phat(path: str, m, fmt: int = ASCII) -> None:
    """Writes a boundary matrix in PHAT ascii or binary format."""
    lib = load_library()
    dims = np.ascontiguousarray(m.dims, dtype=np.int32)
    col_ptr = np.ascontiguousarray(m.col_ptr, dtype=np.int64)
    rows = np.ascontiguousarray(m.rows if m.nnz else np.zeros(1, np.int32), dtype=np.int32)
    err = ctypes.create_string_buffer(256)
    rc = lib.sspp_phat_write(str(path).encode(), fmt, dims.shape[0], dims.ctypes.data, col_ptr.ctypes.data,
                             rows.ctypes.data, err, 256)
    if rc != OK:
        raise SsppError(rc, err.value.decode(errors="replace"))
