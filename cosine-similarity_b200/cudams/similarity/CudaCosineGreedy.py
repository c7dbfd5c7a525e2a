"""CudaCosineGreedy: greedy cosine similarity on B200, matchms plug-in.

Drop-in for the reference class of the same name
(cudams/similarity/CudaCosineGreedy.py:17-226): same constructor keywords,
same `pair` / `matrix` calls, same structured outputs
(score float32, matches int32, overflow uint8).  Scores follow matchms
CosineGreedy in float64 (window, key order, greedy assignment) and are
rounded to float32; matches and overflow are exact.  The reference kernel's
input rules are kept: spectra are truncated to their first `n_max_peaks`
peaks, m/z and intensities are rounded to float32, and a pair whose
candidate list reaches `match_limit` is flagged as overflowed (its score is
then a lower bound, computed from the first match_limit candidates in
generation order).
"""
from __future__ import annotations

import warnings
from typing import List, Literal, Optional

import numpy as np

from .. import _native, autotune, kernels
from ..packing import PackedSpectra, _peaks_of, pack_spectra
from ..sparse import StackedSparseArray
from ..utils import CudaTimer
from ._base import BaseSimilarity

_BYTES_PER_PAIR = 9  # score f32 + matches i32 + overflow u8 on the device


class CudaCosineGreedy(BaseSimilarity):
    score_datatype = [
        ("score", np.float32),
        ("matches", np.int32),
        ("overflow", np.uint8),
    ]

    def __init__(
        self,
        tolerance: float = 0.1,
        mz_power: float = 0.0,
        intensity_power: float = 1.0,
        shift: float = 0,
        batch_size: int = 2048,
        n_max_peaks: int = 1024,
        match_limit: int = 2048,
        sparse_threshold: float = .75,
        verbose=False,
        device=None,
        config: Optional[dict] = None,
        max_device_bytes: Optional[int] = None,
    ):
        """Keywords as in the reference (CudaCosineGreedy.py:24-35).

        batch_size: kept for compatibility; the device kernels tile the
            problem themselves, so it is only a lower bound on the number of
            reference rows computed per device pass.
        device: CUDA device index (default: current device).
        config: fixed cms_cosine_config fields (default: chosen per workload).
        max_device_bytes: cap on the device memory used for dense outputs of
            one pass (default: a quarter of the free memory).
        """
        if match_limit < 1:
            raise ValueError("match_limit must be >= 1")
        if tolerance < 0:
            raise ValueError("tolerance must be >= 0")
        if n_max_peaks is not None and not (1 <= n_max_peaks <= 65535):
            raise ValueError("n_max_peaks must be in [1, 65535]")
        self.tolerance = tolerance
        self.mz_power = mz_power
        self.int_power = intensity_power
        self.shift = shift
        self.batch_size = batch_size
        self.match_limit = match_limit
        self.verbose = verbose
        self.n_max_peaks = n_max_peaks
        self.kernel_time = 0  # device seconds of the last matrix() call
        self.sparse_threshold = sparse_threshold
        self.config = config
        self.max_device_bytes = max_device_bytes
        self._device_index = device
        self.kernel = self._compute  # the reference asserts kernel is not None
        try:
            import torch

            self.device = "cuda" if torch.cuda.is_available() else "cpu"
        except ImportError:  # pragma: no cover
            self.device = "cpu"
        if self.device != "cuda":
            warnings.warn(f"{self.__class__}: CUDA device seems unavailable.")

    def __str__(self) -> str:
        return (f"CudaCosineGreedy(tolerance={self.tolerance}, mz_power={self.mz_power}, "
                f"intensity_power={self.int_power}, shift={self.shift}, "
                f"n_max_peaks={self.n_max_peaks}, match_limit={self.match_limit}, "
                f"sparse_threshold={self.sparse_threshold})")

    # -- packing ---------------------------------------------------------------
    def pack(self, spectra) -> PackedSpectra:
        """Pack spectra with this object's n_max_peaks and powers."""
        if isinstance(spectra, PackedSpectra):
            if (spectra.mz_power != float(self.mz_power)
                    or spectra.intensity_power != float(self.int_power)):
                raise ValueError("PackedSpectra was packed with other mz/intensity powers")
            return spectra.truncate(self.n_max_peaks)
        return pack_spectra(spectra, self.n_max_peaks, self.mz_power, self.int_power)

    def _spectra_peaks_to_tensor(self, spectra: list):
        """Reference layout [2, n, n_max_peaks] float32 plus int32 lengths
        (compatibility helper; padding is zero instead of uninitialised)."""
        peaks = [_peaks_of(s) for s in spectra]
        width = self.n_max_peaks or max((0 if m is None else m.shape[0]) for m, _ in peaks)
        out = np.zeros((2, len(spectra), width), dtype=np.float32)
        lens = np.zeros(len(spectra), dtype=np.int32)
        for i, (m, it) in enumerate(peaks):
            if m is None:
                continue
            n = min(m.shape[0], width)
            out[0, i, :n] = m[:n]
            out[1, i, :n] = it[:n]
            lens[i] = n
        return out, lens

    # -- compute ---------------------------------------------------------------
    def _torch_device(self):
        return _native.require_cuda(self._device_index)

    def _config_for(self, ref: PackedSpectra, qry: PackedSpectra) -> dict:
        if self.config is not None:
            return dict(self.config)
        return autotune.choose_config(ref, qry, float(self.tolerance), float(self.shift))

    def _row_block(self, n_ref: int, n_q: int, dev) -> int:
        import torch

        budget = self.max_device_bytes
        if budget is None:
            free, _ = torch.cuda.mem_get_info(dev)
            budget = max(1 << 28, free // 4)
        rows = max(1, int(budget // max(1, n_q * _BYTES_PER_PAIR)))
        return max(min(n_ref, rows), min(n_ref, int(self.batch_size or 1)))

    def _compute(self, ref: PackedSpectra, qry: PackedSpectra, symmetric: bool = False):
        """Dense result on the host: (score, matches, overflow) [n_ref, n_q].

        symmetric: only pairs (i, j) with i <= j are computed and (j, i) gets
        the same result (matchms is_symmetric=True; needs n_ref == n_q)."""
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
        if symmetric and rows < R:
            return self._compute_symmetric_blocked(ref, qry, cfg, rows, dev, stream,
                                                   (score, matches, overflow))
        if symmetric:
            cfg = dict(cfg, symmetric=1)
        qd = qry.to_device(dev)
        bufs = None
        for r0 in range(0, R, rows):
            r1 = min(R, r0 + rows)
            rd = (ref if (r0 == 0 and r1 == R) else ref.subset(r0, r1)).to_device(dev)
            if bufs is None or bufs[0].shape[0] != r1 - r0:
                bufs = (torch.empty((r1 - r0, Q), dtype=torch.float32, device=dev),
                        torch.empty((r1 - r0, Q), dtype=torch.int32, device=dev),
                        torch.empty((r1 - r0, Q), dtype=torch.uint8, device=dev))
            timer = CudaTimer(stream)
            timer.start()
            kernels.cosine_greedy_dense(rd, qd, self.tolerance, self.shift, self.match_limit,
                                        out=bufs, config=cfg, stream=stream, check_errors=True)
            timer.stop()
            self.kernel_time += timer.elapsed_seconds()
            score[r0:r1] = bufs[0].cpu().numpy()
            matches[r0:r1] = bufs[1].cpu().numpy()
            overflow[r0:r1] = bufs[2].cpu().numpy()
        return score, matches, overflow

    def _compute_symmetric_blocked(self, ref, qry, cfg, rows, dev, stream, out):
        """Symmetric result when the matrix does not fit the device at once:
        row block [r0, r1) computes its diagonal square symmetrically and the
        columns right of it fully; the columns left of r0 are the transpose of
        blocks already computed."""
        import torch

        score, matches, overflow = out
        R = ref.n
        for r0 in range(0, R, rows):
            r1 = min(R, r0 + rows)
            rd = ref.subset(r0, r1).to_device(dev)
            parts = [(qry.subset(r0, r1), r0, dict(cfg, symmetric=1))]
            if r1 < R:
                parts.append((qry.subset(r1, R), r1, dict(cfg)))
            for qpart, c0, c in parts:
                qd = qpart.to_device(dev)
                bufs = (torch.empty((r1 - r0, qd.n), dtype=torch.float32, device=dev),
                        torch.empty((r1 - r0, qd.n), dtype=torch.int32, device=dev),
                        torch.empty((r1 - r0, qd.n), dtype=torch.uint8, device=dev))
                timer = CudaTimer(stream)
                timer.start()
                kernels.cosine_greedy_dense(rd, qd, self.tolerance, self.shift,
                                            self.match_limit, out=bufs, config=c,
                                            stream=stream, check_errors=True)
                timer.stop()
                self.kernel_time += timer.elapsed_seconds()
                c1 = c0 + qd.n
                score[r0:r1, c0:c1] = bufs[0].cpu().numpy()
                matches[r0:r1, c0:c1] = bufs[1].cpu().numpy()
                overflow[r0:r1, c0:c1] = bufs[2].cpu().numpy()
            if r0 > 0:
                score[r0:r1, :r0] = score[:r0, r0:r1].T
                matches[r0:r1, :r0] = matches[:r0, r0:r1].T
                overflow[r0:r1, :r0] = overflow[:r0, r0:r1].T
        return score, matches, overflow

    def pair(self, reference, query) -> np.ndarray:
        result_mat = self.matrix([reference], [query])
        return np.asarray(result_mat.squeeze(), dtype=self.score_datatype)

    def matrix(
        self,
        references: List,
        queries: List,
        array_type: Literal["numpy", "sparse"] = "numpy",
        is_symmetric: bool = False,
    ):
        """All-vs-all greedy cosine (reference CudaCosineGreedy.py:107-226).

        array_type "numpy": np.recarray [R, Q] with fields score/matches/overflow.
        array_type "sparse": StackedSparseArray(R, Q) holding, under the name
        "sparse", every pair with score >= sparse_threshold.
        is_symmetric=True (matchms semantics; the reference warns and ignores
        it, CudaCosineGreedy.py:131-132): R == Q, pairs (i, j) with i <= j are
        scored as (references[i], queries[j]) and (j, i) gets the same result.
        """
        assert self.kernel is not None, "Kernel isn't compiled - use .compile() first"
        if array_type == "sparse":
            assert self.sparse_threshold is not None, (
                "When using array_type `sparse` you have to set `score_threshold`. "
                "Scores below this will get discarded.")
            assert 0 <= self.sparse_threshold <= 1, "Score threshold must be in [0, 1] range."
        elif array_type != "numpy":
            raise NotImplementedError("Output array type is not yet implemented.")

        ref = self.pack(references)
        qry = self.pack(queries)
        if is_symmetric and ref.n != qry.n:
            raise ValueError(f"Found unequal number of spectra {ref.n} and {qry.n} while "
                             "`is_symmetric` is True.")
        if array_type == "numpy":
            score, matches, overflow = self._compute(ref, qry, symmetric=is_symmetric)
            return np.rec.fromarrays([score, matches, overflow], dtype=self.score_datatype)
        return self._sparse(ref, qry, symmetric=is_symmetric)

    def _sparse(self, ref: PackedSpectra, qry: PackedSpectra, symmetric: bool = False):
        import torch

        R, Q = ref.n, qry.n
        sp = StackedSparseArray(R, Q)
        thr = float(self.sparse_threshold)
        if thr <= 0.0 or R == 0 or Q == 0:
            # every pair qualifies (scores are >= 0): dense result, all entries
            score, matches, overflow = self._compute(ref, qry, symmetric=symmetric)
            keep = score >= thr
            r, q = np.nonzero(keep)
            s, m, o = score[r, q], matches[r, q], overflow[r, q]
        else:
            dev = self._torch_device()
            cfg = self._config_for(ref, qry)
            if symmetric:
                cfg = dict(cfg, symmetric=1)
            stream = torch.cuda.current_stream(dev)
            timer = CudaTimer(stream)
            timer.start()
            hits = kernels.cosine_greedy_sparse(ref.to_device(dev), qry.to_device(dev),
                                                self.tolerance, self.shift, self.match_limit,
                                                thr, config=cfg, stream=stream)
            timer.stop()
            self.kernel_time = timer.elapsed_seconds()
            r, q, s, m, o = hits.to_host(sort=True)
        sp.add_sparse_data(
            r.astype(np.int64), q.astype(np.int64),
            np.rec.fromarrays([s.astype(np.float32), m.astype(np.int32), o.astype(bool)],
                              names=["score", "matches", "overflow"]),
            name="sparse")
        return sp
