"""CudaModifiedCosine: matchms ModifiedCosine on B200, in the mould of CudaCosineGreedy.

The reference has no CUDA ModifiedCosine: it prototypes matchms'
ModifiedCosine beside its CUDA classes (notebooks/prototyping/
other_similarities.ipynb) and carries the shift such a score needs in its
kernel (cudams/similarity/spectrum_similarity_functions.py:14,133).  This
class computes matchms' definition: the peak matches at shift 0 and at the
pair's precursor difference (precursor_mz of the reference minus that of the
query) are concatenated in that order, sorted once by descending product
(stable, so on equal products a shifted match precedes an unshifted one and
a later-generated one an earlier one) and assigned greedily; the score is the
sum of the assigned products over the two spectra's norms.  As in
CudaCosineGreedy, spectra are truncated to `n_max_peaks` (at most 32767
here), m/z and intensities are rounded to float32, and a pair whose
concatenated candidate list reaches `match_limit` is flagged as overflowed.
"""
from __future__ import annotations

from typing import List, Literal, Optional

import numpy as np

from .. import autotune, kernels
from ..packing import PackedSpectra
from ..sparse import StackedSparseArray
from ..utils import CudaTimer
from .CudaCosineGreedy import CudaCosineGreedy

MAX_PEAKS = 32767


def precursors_of(spectra) -> np.ndarray:
    """precursor_mz (float64) of matchms-like spectra (``.get("precursor_mz")``
    or a ``precursor_mz`` attribute)."""
    out = np.empty(len(spectra), dtype=np.float64)
    for i, s in enumerate(spectra):
        v = None
        if s is not None:
            get = getattr(s, "get", None)
            v = get("precursor_mz") if callable(get) else getattr(s, "precursor_mz", None)
        assert v is not None, "Precursor_mz missing. Apply 'add_precursor_mz' filter first."
        out[i] = float(v)
    return out


class CudaModifiedCosine(CudaCosineGreedy):
    score_datatype = CudaCosineGreedy.score_datatype

    def __init__(self, tolerance: float = 0.1, mz_power: float = 0.0,
                 intensity_power: float = 1.0, batch_size: int = 2048, n_max_peaks: int = 1024,
                 match_limit: int = 2048, sparse_threshold: float = .75, verbose=False,
                 device=None, config: Optional[dict] = None,
                 max_device_bytes: Optional[int] = None):
        if n_max_peaks is None or not (1 <= n_max_peaks <= MAX_PEAKS):
            raise ValueError(f"n_max_peaks must be in [1, {MAX_PEAKS}] for modified cosine")
        super().__init__(tolerance=tolerance, mz_power=mz_power, intensity_power=intensity_power,
                         shift=0, batch_size=batch_size, n_max_peaks=n_max_peaks,
                         match_limit=match_limit, sparse_threshold=sparse_threshold,
                         verbose=verbose, device=device, config=config,
                         max_device_bytes=max_device_bytes)

    def __str__(self) -> str:
        return (f"CudaModifiedCosine(tolerance={self.tolerance}, mz_power={self.mz_power}, "
                f"intensity_power={self.int_power}, n_max_peaks={self.n_max_peaks}, "
                f"match_limit={self.match_limit}, sparse_threshold={self.sparse_threshold})")

    def _split(self, spectra):
        """(PackedSpectra, precursor float64[n]) from matchms-like spectra or a
        (PackedSpectra, precursors) pair."""
        if isinstance(spectra, tuple) and len(spectra) == 2 and isinstance(spectra[0],
                                                                           PackedSpectra):
            packed, prec = spectra
            prec = np.ascontiguousarray(prec, dtype=np.float64)
            if prec.shape != (packed.n,):
                raise ValueError("one precursor m/z per spectrum")
            return self.pack(packed), prec
        return self.pack(spectra), precursors_of(spectra)

    def _config_for(self, ref: PackedSpectra, qry: PackedSpectra) -> dict:
        if self.config is not None:
            return dict(self.config)
        cfg = autotune.choose_config(ref, qry, float(self.tolerance), 0.0)
        if cfg.get("cand_per_pair"):  # the shifted pass adds about as many again
            cfg["cand_per_pair"] = 2.0 * cfg["cand_per_pair"]
            cfg["tile_spectra"] = max(32, (cfg.get("tile_spectra", 64) // 2 + 31) // 32 * 32)
        return cfg

    def _compute_mod(self, ref, rprec, qry, qprec, symmetric: bool = False):
        import torch

        dev = self._torch_device()
        R, Q = ref.n, qry.n
        score = np.zeros((R, Q), dtype=np.float32)
        matches = np.zeros((R, Q), dtype=np.int32)
        overflow = np.zeros((R, Q), dtype=np.uint8)
        self.kernel_time = 0.0
        if R == 0 or Q == 0:
            return score, matches, overflow
        cfg = self._config_for(ref, qry)
        rows = self._row_block(R, Q, dev)
        stream = torch.cuda.current_stream(dev)
        one_block = rows >= R
        if symmetric and one_block:
            cfg = dict(cfg, symmetric=1)
        qd = qry.to_device(dev)
        qp = torch.from_numpy(qprec).to(dev)
        bufs = None
        for r0 in range(0, R, rows):
            r1 = min(R, r0 + rows)
            rd = (ref if one_block else ref.subset(r0, r1)).to_device(dev)
            rp = torch.from_numpy(np.ascontiguousarray(rprec[r0:r1])).to(dev)
            if bufs is None or bufs[0].shape[0] != r1 - r0:
                bufs = tuple(torch.empty((r1 - r0, Q), dtype=t, device=dev)
                             for t in (torch.float32, torch.int32, torch.uint8))
            timer = CudaTimer(stream)
            timer.start()
            kernels.modified_cosine_dense(rd, rp, qd, qp, self.tolerance, self.match_limit,
                                          out=bufs, config=cfg, stream=stream,
                                          check_errors=True)
            timer.stop()
            self.kernel_time += timer.elapsed_seconds()
            score[r0:r1] = bufs[0].cpu().numpy()
            matches[r0:r1] = bufs[1].cpu().numpy()
            overflow[r0:r1] = bufs[2].cpu().numpy()
        if symmetric and not one_block:
            # matchms semantics: (j, i) takes the result of (i, j), i < j
            lower = np.tril_indices(R, -1)
            for a in (score, matches, overflow):
                a[lower] = a.T[lower]
        return score, matches, overflow

    def pair(self, reference, query) -> np.ndarray:
        result_mat = self.matrix([reference], [query])
        return np.asarray(result_mat.squeeze(), dtype=self.score_datatype)

    def matrix(self, references: List, queries: List,
               array_type: Literal["numpy", "sparse"] = "numpy", is_symmetric: bool = False):
        """All-vs-all modified cosine.  references / queries: matchms-like
        spectra with precursor_mz metadata, or (PackedSpectra, precursors).
        array_type and is_symmetric as in CudaCosineGreedy.matrix."""
        assert self.kernel is not None, "Kernel isn't compiled - use .compile() first"
        if array_type == "sparse":
            assert self.sparse_threshold is not None, (
                "When using array_type `sparse` you have to set `score_threshold`. "
                "Scores below this will get discarded.")
            assert 0 <= self.sparse_threshold <= 1, "Score threshold must be in [0, 1] range."
        elif array_type != "numpy":
            raise NotImplementedError("Output array type is not yet implemented.")
        ref, rprec = self._split(references)
        qry, qprec = self._split(queries)
        if is_symmetric and ref.n != qry.n:
            raise ValueError(f"Found unequal number of spectra {ref.n} and {qry.n} while "
                             "`is_symmetric` is True.")
        if array_type == "numpy":
            score, matches, overflow = self._compute_mod(ref, rprec, qry, qprec, is_symmetric)
            return np.rec.fromarrays([score, matches, overflow], dtype=self.score_datatype)
        return self._sparse_mod(ref, rprec, qry, qprec, is_symmetric)

    def _sparse_mod(self, ref, rprec, qry, qprec, symmetric: bool):
        import torch

        R, Q = ref.n, qry.n
        sp = StackedSparseArray(R, Q)
        thr = float(self.sparse_threshold)
        if thr <= 0.0 or R == 0 or Q == 0:
            score, matches, overflow = self._compute_mod(ref, rprec, qry, qprec, symmetric)
            r, q = np.nonzero(score >= thr)
            s, m, o = score[r, q], matches[r, q], overflow[r, q]
        else:
            dev = self._torch_device()
            cfg = self._config_for(ref, qry)
            if symmetric:
                cfg = dict(cfg, symmetric=1)
            stream = torch.cuda.current_stream(dev)
            timer = CudaTimer(stream)
            timer.start()
            hits = kernels.modified_cosine_sparse(
                ref.to_device(dev), torch.from_numpy(rprec).to(dev), qry.to_device(dev),
                torch.from_numpy(qprec).to(dev), self.tolerance, self.match_limit, thr,
                config=cfg, stream=stream)
            timer.stop()
            self.kernel_time = timer.elapsed_seconds()
            r, q, s, m, o = hits.to_host(sort=True)
        sp.add_sparse_data(
            r.astype(np.int64), q.astype(np.int64),
            np.rec.fromarrays([s.astype(np.float32), m.astype(np.int32), o.astype(bool)],
                              names=["score", "matches", "overflow"]),
            name="sparse")
        return sp
