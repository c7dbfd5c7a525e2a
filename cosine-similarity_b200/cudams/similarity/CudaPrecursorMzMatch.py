"""CudaPrecursorMzMatch and CudaParentMassMatch: matchms' PrecursorMzMatch and
ParentMassMatch on the device.

The reference prototypes both beside its CUDA classes
(notebooks/prototyping/other_similarities.ipynb imports them from matchms,
its requirement matchms >= 0.24.0, next to CudaCosineGreedy).  matchms'
definitions, restated:

  ParentMassMatch(tolerance=0.1): a pair matches when
      |parent_mass(ref) - parent_mass(query)| <= tolerance;
  PrecursorMzMatch(tolerance=0.1, tolerance_type="Dalton"): the same on
      precursor_mz, or with tolerance_type="ppm" when
      |mz_r - mz_q| / ((mz_r + mz_q) / 2) * 1e6 <= tolerance;

every operation in IEEE float64, scores of type bool, and a missing value
stops the call with matchms' assertion message.  Every expression is
symmetric in (ref, query) bit for bit, so is_symmetric=True computes the
full matrix.  The device kernel is cms_mass_match (csrc/metadata_match.cu).
"""
from __future__ import annotations

from typing import List

import numpy as np

from .. import _native, kernels
from ..sparse import StackedSparseArray
from ._base import BaseSimilarity


def metadata_values(spectra, key: str, message: str) -> np.ndarray:
    """The float64 metadata field `key` of matchms-like spectra
    (``.get(key)``), asserting that every spectrum has it."""
    out = np.empty(len(spectra), dtype=np.float64)
    for i, s in enumerate(spectra):
        get = getattr(s, "get", None)
        v = get(key) if callable(get) else getattr(s, key, None)
        assert v is not None, message
        out[i] = float(v)
    return out


class _MassMatch(BaseSimilarity):
    is_commutative = True
    score_datatype = bool
    _key = ""
    _missing = ""

    def __init__(self, tolerance: float = 0.1, ppm: bool = False, device=None):
        self.tolerance = tolerance
        self._ppm = ppm
        self._device_index = device

    def _compute(self, references, queries) -> np.ndarray:
        import torch

        r = metadata_values(references, self._key, self._missing)
        q = metadata_values(queries, self._key, self._missing)
        dev = _native.require_cuda(self._device_index)
        out = kernels.mass_match_matrix(torch.from_numpy(r).to(dev), torch.from_numpy(q).to(dev),
                                        float(self.tolerance), self._ppm)
        return out.cpu().numpy().astype(bool)

    def pair(self, reference, query) -> bool:
        return bool(self._compute([reference], [query])[0, 0])

    def matrix(self, references: List, queries: List, array_type: str = "numpy",
               is_symmetric: bool = False):
        """Boolean matrix [R, Q] (or a StackedSparseArray of the matching
        pairs for array_type="sparse")."""
        if array_type not in ("numpy", "sparse"):
            raise NotImplementedError("Output array type is not yet implemented.")
        if is_symmetric and len(references) != len(queries):
            raise ValueError(f"Found unequal number of spectra {len(references)} and "
                             f"{len(queries)} while `is_symmetric` is True.")
        scores = self._compute(references, queries)
        if array_type == "sparse":
            rows, cols = np.nonzero(scores)
            scores_array = StackedSparseArray(len(references), len(queries))
            scores_array.add_sparse_data(rows, cols, scores[rows, cols], "")
            return scores_array
        return scores


class CudaParentMassMatch(_MassMatch):
    """True for pairs whose parent masses differ by at most `tolerance`."""
    _key = "parent_mass"
    _missing = "Missing parent mass."

    def __init__(self, tolerance: float = 0.1, device=None):
        super().__init__(tolerance, False, device)


class CudaPrecursorMzMatch(_MassMatch):
    """True for pairs whose precursor m/z differ by at most `tolerance`
    (Dalton, or ppm of the pair's mean m/z)."""
    _key = "precursor_mz"
    _missing = "Missing precursor m/z."

    def __init__(self, tolerance: float = 0.1, tolerance_type: str = "Dalton", device=None):
        assert tolerance_type in ["Dalton", "ppm"], "Expected type from ['Dalton', 'ppm']"
        super().__init__(tolerance, tolerance_type == "ppm", device)
        self.tolerance_type = tolerance_type
