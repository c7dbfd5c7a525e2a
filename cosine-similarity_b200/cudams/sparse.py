"""Sparse score container.

The reference returns sparsestack.StackedSparseArray for array_type="sparse"
(cudams/similarity/CudaCosineGreedy.py:207-226, CudaFingerprintSimilarity.py
:178-183).  When sparsestack is installed it is used as is; otherwise this
module provides a small stand-in with the calls the reference and its tests
use: add_sparse_data, add_dense_matrix, to_array(name), shape, row/col/data.
"""
from __future__ import annotations

import numpy as np

try:  # pragma: no cover - depends on the environment
    from sparsestack import StackedSparseArray  # type: ignore
    HAVE_SPARSESTACK = True
except ImportError:
    HAVE_SPARSESTACK = False

    class StackedSparseArray:  # type: ignore[no-redef]
        """Minimal COO stack of named score layers over an (n_row, n_col) grid."""

        def __init__(self, n_row: int, n_col: int):
            self.shape = (int(n_row), int(n_col))
            self.row = np.zeros(0, dtype=np.int64)
            self.col = np.zeros(0, dtype=np.int64)
            self._layers: dict[str, np.ndarray] = {}

        @property
        def score_names(self):
            return tuple(self._layers)

        @property
        def data(self):
            if not self._layers:
                return np.zeros(0)
            names = list(self._layers)
            return np.rec.fromarrays([self._layers[n] for n in names], names=names)

        def _set_coords(self, row, col):
            row = np.asarray(row, dtype=np.int64).ravel()
            col = np.asarray(col, dtype=np.int64).ravel()
            if self._layers and (row.shape != self.row.shape or (row != self.row).any()
                                 or (col != self.col).any()):
                raise ValueError("new layer must share the coordinates of existing layers")
            self.row, self.col = row, col

        def add_sparse_data(self, row, col, data, name: str):
            self._set_coords(row, col)
            data = np.asarray(data)
            if data.dtype.names:
                for f in data.dtype.names:
                    self._layers[f"{name}_{f}" if name else f] = np.asarray(data[f]).ravel()
            else:
                self._layers[name] = data.ravel()

        def add_dense_matrix(self, matrix, name: str):
            matrix = np.asarray(matrix)
            if matrix.shape != self.shape:
                raise ValueError("matrix shape differs from the array shape")
            if matrix.dtype.names:
                keep = np.zeros(self.shape, dtype=bool)
                for f in matrix.dtype.names:
                    keep |= matrix[f] != 0
            else:
                keep = matrix != 0
            row, col = np.nonzero(keep)
            self.add_sparse_data(row, col, matrix[row, col], name)

        def to_array(self, name: str | None = None):
            if name is None:
                if len(self._layers) != 1:
                    names = list(self._layers)
                    out = np.zeros(self.shape, dtype=[(n, self._layers[n].dtype) for n in names])
                    for n in names:
                        out[n][self.row, self.col] = self._layers[n]
                    return out
                name = next(iter(self._layers))
            vals = self._layers[name]
            out = np.zeros(self.shape, dtype=vals.dtype)
            out[self.row, self.col] = vals
            return out

        def __repr__(self):
            return (f"StackedSparseArray(shape={self.shape}, entries={self.row.shape[0]}, "
                    f"layers={list(self._layers)})")

__all__ = ["StackedSparseArray", "HAVE_SPARSESTACK"]
