"""Synthetic filtered complexes as PHAT boundary matrices (input side).

Thin ctypes front end of ``csrc/sspp_gen.cpp``: Vietoris-Rips complexes of
point clouds (seeded uniform, or the caller's) and Freudenthal lower-star
filtrations of scalar fields (seeded smoothed Gaussian noise, or the caller's), ordered by (filtration value, dimension, lexicographic vertex
tuple) with int32 face indices.  These are the synthetic stand-ins for the
reference's PHAT input files (read by ``src/main.cu:90-167``).
"""
from __future__ import annotations

import ctypes
import math
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_lib = None


def _load():
    global _lib
    if _lib is None:
        path = os.path.join(_HERE, "libsspp_gen.so")
        if not os.path.exists(path):
            raise RuntimeError(f"{path} is missing: run __graft_entry__.build() first")
        lib = ctypes.CDLL(path)
        lib.sspp_gen_rips.restype = ctypes.c_void_p
        lib.sspp_gen_rips.argtypes = [ctypes.c_int64, ctypes.c_int32, ctypes.c_uint64, ctypes.c_float, ctypes.c_int32]
        lib.sspp_gen_lowerstar.restype = ctypes.c_void_p
        lib.sspp_gen_lowerstar.argtypes = [ctypes.c_int32, ctypes.c_float, ctypes.c_uint64]
        lib.sspp_gen_ncols.restype = ctypes.c_int64
        lib.sspp_gen_ncols.argtypes = [ctypes.c_void_p]
        lib.sspp_gen_nnz.restype = ctypes.c_int64
        lib.sspp_gen_nnz.argtypes = [ctypes.c_void_p]
        lib.sspp_gen_copy.restype = ctypes.c_int32
        lib.sspp_gen_copy.argtypes = [ctypes.c_void_p] + [ctypes.c_void_p] * 4
        lib.sspp_gen_free.restype = None
        lib.sspp_gen_free.argtypes = [ctypes.c_void_p]
        lib.sspp_gen_rips_points.restype = ctypes.c_void_p
        lib.sspp_gen_rips_points.argtypes = [ctypes.c_int64, ctypes.c_int32, ctypes.c_void_p, ctypes.c_float,
                                             ctypes.c_int32]
        lib.sspp_gen_lowerstar_field.restype = ctypes.c_void_p
        lib.sspp_gen_lowerstar_field.argtypes = [ctypes.c_int32] * 3 + [ctypes.c_void_p, ctypes.c_int32]
        lib.sspp_gen_points.restype = ctypes.c_int32
        lib.sspp_gen_points.argtypes = [ctypes.c_int64, ctypes.c_int32, ctypes.c_uint64, ctypes.c_void_p]
        lib.sspp_gen_field.restype = ctypes.c_int32
        lib.sspp_gen_field.argtypes = [ctypes.c_int32, ctypes.c_float, ctypes.c_uint64, ctypes.c_void_p]
        _lib = lib
    return _lib


@dataclass
class BoundaryMatrix:
    """A filtered boundary matrix in PHAT column order (0-based face indices)."""

    dims: np.ndarray      # int32 [ncols]
    col_ptr: np.ndarray   # int64 [ncols + 1]
    rows: np.ndarray      # int32 [nnz], ascending within each column
    values: np.ndarray | None = None  # float32 [ncols] filtration values, if known

    @property
    def ncols(self) -> int:
        return int(self.dims.shape[0])

    @property
    def nnz(self) -> int:
        return int(self.rows.shape[0])

    def column(self, j: int) -> np.ndarray:
        return self.rows[self.col_ptr[j]:self.col_ptr[j + 1]]

    @staticmethod
    def from_columns(dims, columns) -> "BoundaryMatrix":
        dims = np.asarray(dims, dtype=np.int32)
        cols = [sorted(set(int(x) for x in c)) for c in columns]
        col_ptr = np.zeros(len(cols) + 1, dtype=np.int64)
        for j, c in enumerate(cols):
            col_ptr[j + 1] = col_ptr[j] + len(c)
        rows = np.zeros(int(col_ptr[-1]), dtype=np.int32)
        for j, c in enumerate(cols):
            rows[col_ptr[j]:col_ptr[j + 1]] = c
        return BoundaryMatrix(dims, col_ptr, rows)


def _take(h) -> BoundaryMatrix:
    lib = _load()
    if not h:
        raise ValueError("invalid generator arguments")
    try:
        n = lib.sspp_gen_ncols(h)
        nnz = lib.sspp_gen_nnz(h)
        dims = np.empty(n, dtype=np.int32)
        col_ptr = np.empty(n + 1, dtype=np.int64)
        rows = np.empty(nnz, dtype=np.int32)
        values = np.empty(n, dtype=np.float32)
        lib.sspp_gen_copy(h, dims.ctypes.data, col_ptr.ctypes.data, rows.ctypes.data, values.ctypes.data)
    finally:
        lib.sspp_gen_free(h)
    return BoundaryMatrix(dims, col_ptr, rows, values)


def rips(npts: int, space_dim: int, seed: int, radius: float, maxdim: int = 3) -> BoundaryMatrix:
    """Vietoris-Rips complex of ``npts`` points i.i.d. uniform in [0,1]^space_dim."""
    return _take(_load().sspp_gen_rips(int(npts), int(space_dim), int(seed) & (2**64 - 1), float(radius), int(maxdim)))


def lowerstar(grid: int, sigma: float, seed: int) -> BoundaryMatrix:
    """Lower-star filtration of the Freudenthal triangulation of a grid^3 lattice."""
    return _take(_load().sspp_gen_lowerstar(int(grid), float(sigma), int(seed) & (2**64 - 1)))


def points(npts: int, space_dim: int, seed: int) -> np.ndarray:
    """The seeded point cloud of ``rips(npts, space_dim, seed, ...)``: float32 [npts, space_dim]."""
    out = np.empty((int(npts), int(space_dim)), dtype=np.float32)
    if _load().sspp_gen_points(int(npts), int(space_dim), int(seed) & (2**64 - 1), out.ctypes.data):
        raise ValueError("invalid generator arguments")
    return out


def field(grid: int, sigma: float, seed: int) -> np.ndarray:
    """The smoothed noise of ``lowerstar(grid, sigma, seed)``: float32 [grid, grid, grid] as [z, y, x]."""
    out = np.empty((int(grid),) * 3, dtype=np.float32)
    if _load().sspp_gen_field(int(grid), float(sigma), int(seed) & (2**64 - 1), out.ctypes.data):
        raise ValueError("invalid generator arguments")
    return out


def rips_from_points(pts, radius: float, maxdim: int = 3) -> BoundaryMatrix:
    """Vietoris-Rips complex of the float32 points ``pts`` [npts, D] (D = 1..3)."""
    pts = np.ascontiguousarray(pts, dtype=np.float32)
    n, d = pts.shape
    return _take(_load().sspp_gen_rips_points(n, d, pts.ctypes.data, float(radius), int(maxdim)))


def lowerstar_from_field(values, maxdim: int = 3) -> BoundaryMatrix:
    """Freudenthal lower-star filtration of the float32 field ``values`` [gz, gy, gx] (x fastest)."""
    v = np.ascontiguousarray(values, dtype=np.float32)
    gz, gy, gx = v.shape
    return _take(_load().sspp_gen_lowerstar_field(gx, gy, gz, v.ctypes.data, int(maxdim)))


def rips_radius_for_degree(npts: int, space_dim: int, mean_degree: float) -> float:
    """Radius giving an expected mean degree k for n uniform points: r = (k / (n c_D))^(1/D)."""
    c = math.pi if space_dim == 2 else 4.0 * math.pi / 3.0
    return float((mean_degree / (npts * c)) ** (1.0 / space_dim))
