"""CudaFingerprintSimilarity: Jaccard / Dice / cosine of molecular fingerprints.

Drop-in for the reference class (cudams/similarity/CudaFingerprintSimilarity
.py:13-186).  Fingerprints (``spectrum.get("fingerprint")``, 0/1 vectors)
are bit-packed on the host and compared by the popcount kernel of
libcudams_b200.so; results are bit-identical to the reference's float32
torch expressions (vector_similarity_functions.py:12-119).  Spectra without
a fingerprint get `set_empty_scores` ("nan" -> NaN, a number -> that number)
in every pair they take part in, written by the kernel itself instead of a
host-side scatter.
"""
from __future__ import annotations

from typing import List, Union

import numpy as np

from .. import _native, kernels
from ..packing import pack_fingerprints
from ..sparse import StackedSparseArray
from ._base import BaseSimilarity


class CudaFingerprintSimilarity(BaseSimilarity):
    """Calculate similarity between molecules based on their fingerprints.

    similarity_measure: "cosine", "dice" or "jaccard" (default "jaccard").
    set_empty_scores: score used where a fingerprint is missing; "nan"
        (default) gives NaN.
    """

    is_commutative = True
    score_datatype = np.float32

    def __init__(
        self,
        similarity_measure: str = "jaccard",
        set_empty_scores: Union[float, int, str] = "nan",
        device=None,
    ):
        self.set_empty_scores = set_empty_scores
        assert similarity_measure in [
            "cosine",
            "dice",
            "jaccard",
        ], "Unknown similarity measure."
        self.similarity_measure = similarity_measure
        self._device_index = device

    def _fill(self) -> float:
        if self.set_empty_scores == "nan":
            return float("nan")
        if isinstance(self.set_empty_scores, (float, int)) and not isinstance(
                self.set_empty_scores, bool):
            return float(self.set_empty_scores)
        return 0.0  # reference: the matrix starts as zeros (create_full_matrix)

    def _compute(self, fps_ref, fps_qry, symmetric: bool = False) -> np.ndarray:
        import torch

        dev = _native.require_cuda(self._device_index)
        rb, rv, nbits_r = pack_fingerprints(fps_ref)
        qb, qv, nbits_q = pack_fingerprints(fps_qry)
        if rv.any() and qv.any() and nbits_r != nbits_q:
            raise ValueError(f"fingerprint lengths differ: {nbits_r} vs {nbits_q}")
        n_words = max(rb.shape[1], qb.shape[1])
        if rb.shape[1] != n_words:
            rb = np.zeros((rb.shape[0], n_words), np.uint32)
        if qb.shape[1] != n_words:
            qb = np.zeros((qb.shape[0], n_words), np.uint32)
        t = lambda x: torch.from_numpy(np.ascontiguousarray(x)).to(dev)  # noqa: E731
        r_bits, r_valid = t(rb), t(rv)
        if symmetric and np.array_equal(rb, qb) and np.array_equal(rv, qv):
            # one set against itself: the same device arrays on both sides let
            # the library compute the full matrix directly (bit-identical to
            # the mirrored one, and faster than half the tiles plus the mirror)
            q_bits, q_valid = r_bits, r_valid
        else:
            q_bits, q_valid = t(qb), t(qv)
        out = kernels.fingerprint_matrix(self.similarity_measure, r_bits, r_valid, q_bits,
                                         q_valid, n_words, self._fill(), symmetric=symmetric)
        return out.cpu().numpy()

    def pair(self, reference, query) -> np.ndarray:
        """Score of one pair as a [1, 1] float32 array (the reference returns the
        1 x 1 matrix of its vector functions, CudaFingerprintSimilarity.py:88-111)."""
        return np.asarray(self._compute([reference.get("fingerprint")],
                                        [query.get("fingerprint")]), dtype=self.score_datatype)

    def matrix(
        self,
        references: List,
        queries: List,
        array_type: str = "numpy",
        is_symmetric: bool = False,
    ):
        """Matrix of fingerprint similarities [R, Q] (float32), or a
        StackedSparseArray for array_type="sparse".

        is_symmetric=True (matchms semantics; the reference ignores the flag):
        R == Q, pairs (i, j) with i <= j are computed and mirrored to (j, i);
        for one set against itself the full matrix is computed directly (the
        same values, and faster than half the tiles plus the mirror copy)."""
        fps_ref = [s.get("fingerprint") for s in references]
        fps_qry = [s.get("fingerprint") for s in queries]
        n_ref = sum(fp is not None for fp in fps_ref)
        n_qry = sum(fp is not None for fp in fps_qry)
        assert n_ref > 0 and n_qry > 0, (
            "Not enough molecular fingerprints.",
            "Apply 'add_fingerprint'filter first.",
        )
        if array_type not in ("numpy", "sparse"):
            raise NotImplementedError("Output array type is not yet implemented.")
        if is_symmetric and len(references) != len(queries):
            raise ValueError(f"Found unequal number of spectra {len(references)} and "
                             f"{len(queries)} while `is_symmetric` is True.")
        similarity_matrix = self._compute(fps_ref, fps_qry, symmetric=is_symmetric)
        if array_type == "sparse":
            scores_array = StackedSparseArray(len(references), len(queries))
            scores_array.add_dense_matrix(similarity_matrix.astype(self.score_datatype), "")
            return scores_array
        return similarity_matrix.astype(self.score_datatype)
