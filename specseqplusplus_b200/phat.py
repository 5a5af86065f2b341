"""PHAT-style Python interface to the B200 engine.

The reference ships a Python binding of PHAT (phat-highclear/python/phat.py:
`boundary_matrix` with `columns`, `dimensions`, `load` / `save` and
`compute_persistence_pairs` / `compute_persistence_pairs_dualized`, plus the
`representations` and `reductions` enums and a `persistence_pairs` result).
This module keeps those names and their meaning so that code written against
that binding runs here; the reduction itself is the engine's (libsspp.so on
the GPU).  The representation and reduction arguments are accepted for
compatibility: every combination gives the same pairs, so they do not change
what is computed.
"""
from __future__ import annotations

import enum

import numpy as np

from .engine import ASCII, BINARY, Engine, Params, read_phat, write_phat
from .gen import BoundaryMatrix

__all__ = ["boundary_matrix", "persistence_pairs", "representations", "reductions"]


class representations(enum.Enum):
    """Column storage names of PHAT (accepted, not used: the engine has one layout)."""
    bit_tree_pivot_column = 1
    sparse_pivot_column = 2
    full_pivot_column = 3
    vector_vector = 4
    vector_heap = 5
    vector_set = 6
    vector_list = 7


class reductions(enum.Enum):
    """Reduction names of PHAT (accepted: all give the same pairs)."""
    twist_reduction = 1
    chunk_reduction = 2
    standard_reduction = 3
    row_reduction = 4
    spectral_sequence_reduction = 5


class persistence_pairs:
    """(birth, death) pairs, as PHAT's persistence_pairs."""

    def __init__(self, pairs: np.ndarray | None = None):
        self._p = np.zeros((0, 2), dtype=np.int64) if pairs is None else np.asarray(pairs, dtype=np.int64).reshape(-1, 2)

    def __len__(self):
        return int(self._p.shape[0])

    def __iter__(self):
        return ((int(b), int(d)) for b, d in self._p)

    def __getitem__(self, i):
        b, d = self._p[i]
        return int(b), int(d)

    def get_num_pairs(self) -> int:
        return len(self)

    def get_pair(self, i: int):
        return self[i]

    def sort(self) -> None:
        self._p = self._p[np.lexsort((self._p[:, 1], self._p[:, 0]))]

    def as_array(self) -> np.ndarray:
        return self._p

    def __eq__(self, other):
        return isinstance(other, persistence_pairs) and np.array_equal(self._p, other._p)

    def save(self, file_name: str, mode: str = "b") -> bool:
        with open(file_name, "w" if mode == "t" else "wb") as f:
            if mode == "t":
                f.write(f"{len(self)}\n" + "".join(f"{b} {d}\n" for b, d in self._p))
            elif mode == "b":
                np.array([len(self)], dtype=np.int64).tofile(f)
                self._p.astype(np.int64).tofile(f)
            else:
                raise ValueError("Only 'b' - binary and 't' - text modes are supported")
        return True


class column:
    """A view on one column of a boundary_matrix."""

    def __init__(self, matrix: "boundary_matrix", index: int):
        self._matrix = matrix
        self._index = index

    @property
    def index(self) -> int:
        return self._index

    @property
    def dimension(self) -> int:
        return int(self._matrix._m.dims[self._index])

    @property
    def boundary(self) -> list:
        return [int(x) for x in self._matrix._m.column(self._index)]

    def __str__(self):
        return f"(dimension={self.dimension}, boundary={self.boundary})"


class boundary_matrix:
    """Boundary matrix of a filtered cell complex, in PHAT's column order."""

    def __init__(self, representation=representations.bit_tree_pivot_column, source=None, columns=None):
        self._representation = representation
        self._m = BoundaryMatrix(np.zeros(0, np.int32), np.zeros(1, np.int64), np.zeros(0, np.int32))
        if source is not None:
            self._m = BoundaryMatrix(source._m.dims.copy(), source._m.col_ptr.copy(), source._m.rows.copy())
        elif columns:
            self.columns = columns

    @property
    def columns(self):
        return [column(self, i) for i in range(self._m.ncols)]

    @columns.setter
    def columns(self, columns):
        dims, cols = [], []
        for col in columns:
            if isinstance(col, column):
                dims.append(col.dimension)
                cols.append(col.boundary)
            elif isinstance(col, tuple):
                dims.append(int(col[0]))
                cols.append(list(col[1]))
            else:
                raise TypeError("All columns must be column objects, or (dimension, values) tuples")
        self._m = BoundaryMatrix.from_columns(dims, cols)

    @property
    def dimensions(self):
        return [int(d) for d in self._m.dims]

    @dimensions.setter
    def dimensions(self, dimensions):
        d = np.asarray(dimensions, dtype=np.int32)
        if d.shape[0] != self._m.ncols:  # PHAT resizes to the new number of columns, all empty
            self._m = BoundaryMatrix(d, np.zeros(d.shape[0] + 1, np.int64), np.zeros(0, np.int32))
        else:
            self._m = BoundaryMatrix(d, self._m.col_ptr, self._m.rows)

    def __eq__(self, other):
        return (isinstance(other, boundary_matrix) and np.array_equal(self._m.dims, other._m.dims)
                and np.array_equal(self._m.col_ptr, other._m.col_ptr) and np.array_equal(self._m.rows, other._m.rows))

    def __ne__(self, other):
        return not self == other

    def __len__(self):
        return self._m.nnz

    @property
    def matrix(self) -> BoundaryMatrix:
        """The columns as engine arrays (dims, col_ptr, rows)."""
        return self._m

    def load(self, file_name: str, mode: str = "b") -> bool:
        if mode not in ("b", "t"):
            raise ValueError("Only 'b' - binary and 't' - text modes are supported")
        self._m = read_phat(file_name, BINARY if mode == "b" else ASCII)
        return True

    def save(self, file_name: str, mode: str = "b") -> bool:
        if mode not in ("b", "t"):
            raise ValueError("Only 'b' - binary and 't' - text modes are supported")
        write_phat(file_name, self._m, BINARY if mode == "b" else ASCII)
        return True

    def _reduce(self, dualize: int) -> persistence_pairs:
        with Engine(0) as e:
            e.load_csc(self._m)
            e.reduce(Params(dualize=dualize))
            return persistence_pairs(e.pairs())

    def compute_persistence_pairs(self, reduction=reductions.twist_reduction) -> persistence_pairs:
        """Persistence pairs (birth, death) of the matrix, sorted by birth."""
        return self._reduce(0)

    def compute_persistence_pairs_dualized(self, reduction=reductions.twist_reduction) -> persistence_pairs:
        """The same pairs, computed from the dualized (coboundary) matrix."""
        return self._reduce(1)

    def convert(self, representation) -> "boundary_matrix":
        return boundary_matrix(representation, self)
