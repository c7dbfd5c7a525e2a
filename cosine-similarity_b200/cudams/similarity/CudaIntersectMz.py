"""CudaIntersectMz: matchms' IntersectMz on the device.

The reference prototypes it beside its CUDA classes
(notebooks/prototyping/other_similarities.ipynb imports it from matchms,
its requirement matchms >= 0.24.0).  matchms' definition, restated: with A
and B the sets of a pair's peak m/z values (exact float64, so repeated
values count once),

    score = scaling * |A & B| / |A | B|,  0 when both spectra have no peaks,

in float64 (scaling * |A & B| first, then the division).  The score is
symmetric bit for bit, so is_symmetric=True computes the full matrix.  The
device kernel is cms_intersect_mz (csrc/metadata_match.cu); it merges the two
sorted m/z lists, so the peaks of each spectrum must be sorted by m/z, as
matchms keeps them.
"""
from __future__ import annotations

from typing import List

import numpy as np

from .. import _native, kernels
from ..sparse import StackedSparseArray
from ._base import BaseSimilarity


def pack_mz64(spectra):
    """(mz float64 [P], offsets int64 [n + 1]) of matchms-like spectra,
    checking that each spectrum's m/z are sorted."""
    arrays = [np.asarray(s.peaks.mz, dtype=np.float64) for s in spectra]
    off = np.zeros(len(arrays) + 1, dtype=np.int64)
    if arrays:
        off[1:] = np.cumsum([a.shape[0] for a in arrays])
    mz = np.concatenate(arrays) if arrays else np.zeros(0, dtype=np.float64)
    for i, a in enumerate(arrays):
        if a.shape[0] > 1 and not np.all(a[1:] >= a[:-1]):
            raise ValueError(f"spectrum {i}: peak m/z values are not sorted")
    return mz, off


class CudaIntersectMz(BaseSimilarity):
    """Share of distinct m/z values two spectra have in common."""
    is_commutative = True
    score_datatype = np.float64

    def __init__(self, scaling: float = 1.0, device=None):
        self.scaling = scaling
        self._device_index = device

    def _compute(self, references, queries) -> np.ndarray:
        import torch

        rm, ro = pack_mz64(references)
        qm, qo = pack_mz64(queries)
        dev = _native.require_cuda(self._device_index)
        t = lambda x: torch.from_numpy(x).to(dev)  # noqa: E731
        out = kernels.intersect_mz_matrix(t(rm), t(ro), t(qm), t(qo), float(self.scaling),
                                          check_errors=True)
        return out.cpu().numpy()

    def pair(self, reference, query) -> float:
        return float(self._compute([reference], [query])[0, 0])

    def matrix(self, references: List, queries: List, array_type: str = "numpy",
               is_symmetric: bool = False):
        """float64 matrix [R, Q] (or a StackedSparseArray of the nonzero
        scores for array_type="sparse")."""
        if array_type not in ("numpy", "sparse"):
            raise NotImplementedError("Output array type is not yet implemented.")
        if is_symmetric and len(references) != len(queries):
            raise ValueError(f"Found unequal number of spectra {len(references)} and "
                             f"{len(queries)} while `is_symmetric` is True.")
        scores = self._compute(references, queries)
        if array_type == "sparse":
            scores_array = StackedSparseArray(len(references), len(queries))
            scores_array.add_dense_matrix(scores, "")
            return scores_array
        return scores
