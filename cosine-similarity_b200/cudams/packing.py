"""Spectrum and fingerprint packers (host side, vectorised numpy).

Spectra become a CSR layout:
    mz       float32 [P]   m/z, ascending within each spectrum
    a        float64 [P]   mz ** mz_power        (None when mz_power == 0)
    b        float64 [P]   intensity ** intensity_power
    offsets  int64   [N+1]

This replaces the reference's padded [2, n, n_max_peaks] float32 tensor
(cudams/similarity/CudaCosineGreedy.py:63-87), keeping its two input rules:
each spectrum is truncated to its first ``n_max_peaks`` peaks (the lowest m/z,
:82) and m/z and intensities are rounded to float32 (:74-77).  The per-peak
powers are taken on the host with numpy (the same libm ``pow`` that matchms
uses through numba) from the float32-rounded values, so the device only
multiplies.  Unlike the reference (which leaves ``lens`` uninitialised for a
``None`` spectrum, :78-85), ``None`` packs as an empty spectrum.

Fingerprints become rows of uint32 words (bit k in word k // 32 at bit
k % 32), with a validity flag per row for spectra without a fingerprint
(CudaFingerprintSimilarity.py:137-145).
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Iterable, Optional, Sequence

import numpy as np

MAX_PEAKS = 65535  # peak indices are packed in 16 bits on the device


def _peaks_of(s):
    """(mz, intensities) of a matchms-like Spectrum, a (mz, int) pair or None."""
    if s is None:
        return None, None
    peaks = getattr(s, "peaks", None)
    if peaks is not None:
        return np.asarray(peaks.mz), np.asarray(peaks.intensities)
    if isinstance(s, (tuple, list)) and len(s) == 2:
        return np.asarray(s[0]), np.asarray(s[1])
    arr = np.asarray(s)
    if arr.ndim == 2 and arr.shape[1] == 2:
        return arr[:, 0], arr[:, 1]
    raise TypeError(f"cannot read peaks from {type(s).__name__}")


@dataclass
class PackedSpectra:
    mz: np.ndarray
    a: Optional[np.ndarray]
    b: np.ndarray
    offsets: np.ndarray
    mz_power: float
    intensity_power: float
    n_max_peaks: Optional[int]
    _device: dict = field(default_factory=dict, repr=False, compare=False)
    # float32 intensities when b is exactly their float64 widening (intensity
    # power 1, set by pack_csr): uploads then send 4 bytes a peak instead of 8
    # and widen on the device
    _b32: Optional[np.ndarray] = field(default=None, repr=False, compare=False)

    @property
    def n(self) -> int:
        return int(self.offsets.shape[0] - 1)

    @property
    def n_peaks(self) -> int:
        return int(self.mz.shape[0])

    @property
    def lengths(self) -> np.ndarray:
        return np.diff(self.offsets)

    def host_bytes(self) -> int:
        """Bytes that to_device copies from the host."""
        b = self._b32 if self._b32 is not None and self._b32.shape == self.b.shape else self.b
        return int(self.mz.nbytes + b.nbytes + self.offsets.nbytes
                   + (self.a.nbytes if self.a is not None else 0))

    def to_device(self, device, non_blocking: bool = False):
        """DeviceSpectra on `device` (cached per device).  Large arrays go through
        the pinned staging ring (`cudams.staging`): the copies are enqueued on
        the current stream, so work on that stream sees the data; use another
        stream only after synchronising (or pass non_blocking=False, the
        default, which waits for the copies)."""
        import torch

        from . import staging

        key = str(device)
        if key not in self._device:
            def up(x):
                if x is None:
                    return None
                return staging.upload(np.ascontiguousarray(x), device)

            if self._b32 is not None and self._b32.shape == self.b.shape:
                b = up(self._b32).to(torch.float64)
            else:
                b = up(self.b)
            self._device[key] = DeviceSpectra(up(self.mz), up(self.a), b,
                                              up(self.offsets), self.n, self.n_peaks)
            if not non_blocking:
                torch.cuda.current_stream(device).synchronize()
        return self._device[key]

    def truncate(self, n_max_peaks: Optional[int]) -> "PackedSpectra":
        """Keep the first `n_max_peaks` peaks of every spectrum (self if none is longer)."""
        if n_max_peaks is None or self.n == 0:
            return self
        lengths = self.lengths
        if lengths.max(initial=0) <= n_max_peaks:
            return self
        keep = np.minimum(lengths, int(n_max_peaks))
        off = np.zeros(self.n + 1, dtype=np.int64)
        np.cumsum(keep, out=off[1:])
        seg = np.repeat(np.arange(self.n), keep)
        idx = self.offsets[:-1][seg] + (np.arange(off[-1]) - off[:-1][seg])
        return PackedSpectra(self.mz[idx], None if self.a is None else self.a[idx], self.b[idx],
                             off, self.mz_power, self.intensity_power, int(n_max_peaks),
                             _b32=None if self._b32 is None else self._b32[idx])

    def take(self, indices) -> "PackedSpectra":
        """The spectra at `indices` (in that order) as a new packed set."""
        idx = np.asarray(indices, dtype=np.int64)
        keep = self.lengths[idx]
        off = np.zeros(idx.shape[0] + 1, dtype=np.int64)
        np.cumsum(keep, out=off[1:])
        seg = np.repeat(np.arange(idx.shape[0]), keep)
        pk = self.offsets[:-1][idx][seg] + (np.arange(off[-1]) - off[:-1][seg])
        return PackedSpectra(self.mz[pk], None if self.a is None else self.a[pk], self.b[pk],
                             off, self.mz_power, self.intensity_power, self.n_max_peaks,
                             _b32=None if self._b32 is None else self._b32[pk])

    def subset(self, start: int, stop: int) -> "PackedSpectra":
        """Spectra [start, stop) as a new packed set (peaks re-based to 0)."""
        lo, hi = int(self.offsets[start]), int(self.offsets[stop])
        return PackedSpectra(self.mz[lo:hi], None if self.a is None else self.a[lo:hi],
                             self.b[lo:hi], self.offsets[start:stop + 1] - lo, self.mz_power,
                             self.intensity_power, self.n_max_peaks,
                             _b32=None if self._b32 is None else self._b32[lo:hi])


@dataclass
class DeviceSpectra:
    mz: "object"
    a: "object"
    b: "object"
    offsets: "object"
    n: int
    n_peaks: int


def _weights(mz32: np.ndarray, int32: np.ndarray, mz_power: float, intensity_power: float):
    a = None if mz_power == 0 else np.power(mz32.astype(np.float64), float(mz_power))
    b = np.power(int32.astype(np.float64), float(intensity_power))
    return a, b


def pack_csr(mz, intensities, offsets, n_max_peaks: Optional[int] = 1024,
             mz_power: float = 0.0, intensity_power: float = 1.0,
             check: bool = True) -> PackedSpectra:
    """Pack spectra already laid out as CSR arrays (fully vectorised).

    mz / intensities: 1-D arrays of all peaks; offsets: int array [N+1].
    """
    offsets = np.asarray(offsets, dtype=np.int64)
    if offsets.ndim != 1 or offsets.shape[0] < 1:
        raise ValueError("offsets must be a 1-D array of length n_spectra + 1")
    mz = np.asarray(mz)
    intensities = np.asarray(intensities)
    if mz.shape != intensities.shape or mz.ndim != 1:
        raise ValueError("mz and intensities must be 1-D arrays of equal length")
    lengths = np.diff(offsets)
    if (lengths < 0).any() or offsets[0] < 0 or offsets[-1] > mz.shape[0]:
        raise ValueError("offsets must be non-decreasing and within the peak arrays")
    if n_max_peaks is not None:
        if n_max_peaks < 1:
            raise ValueError("n_max_peaks must be >= 1")
        keep = np.minimum(lengths, int(n_max_peaks))
    else:
        keep = lengths
    if keep.size and keep.max(initial=0) > MAX_PEAKS:
        raise ValueError(f"a spectrum has more than {MAX_PEAKS} peaks; set n_max_peaks")
    new_off = np.zeros(offsets.shape[0], dtype=np.int64)
    np.cumsum(keep, out=new_off[1:])
    if (keep == lengths).all() and offsets[0] == 0 and offsets[-1] == mz.shape[0]:
        sel_mz, sel_int = mz, intensities
    else:
        # first `keep[s]` peaks of every spectrum
        seg = np.repeat(np.arange(keep.shape[0]), keep)
        idx = offsets[:-1][seg] + (np.arange(new_off[-1]) - new_off[:-1][seg])
        sel_mz, sel_int = mz[idx], intensities[idx]
    mz32 = np.ascontiguousarray(sel_mz, dtype=np.float32)
    int32 = np.ascontiguousarray(sel_int, dtype=np.float32)
    if check:
        if not np.isfinite(mz32).all() or not np.isfinite(int32).all():
            raise ValueError("m/z and intensities must be finite")
        if mz32.shape[0] > 1:
            d = np.diff(mz32)
            starts = new_off[1:-1]
            bad = d < 0
            if bad.any():
                # differences across spectrum boundaries do not count
                boundary = np.zeros(d.shape[0], dtype=bool)
                inner = starts[(starts > 0) & (starts <= d.shape[0])]
                boundary[inner - 1] = True
                if (bad & ~boundary).any():
                    raise ValueError("m/z values must be sorted ascending within each spectrum")
    a, b = _weights(mz32, int32, mz_power, intensity_power)
    return PackedSpectra(mz32, a, b, new_off, float(mz_power), float(intensity_power),
                         None if n_max_peaks is None else int(n_max_peaks),
                         _b32=int32 if float(intensity_power) == 1.0 else None)


def pack_spectra(spectra: Sequence, n_max_peaks: Optional[int] = 1024, mz_power: float = 0.0,
                 intensity_power: float = 1.0, check: bool = True) -> PackedSpectra:
    """Pack a list of matchms-like spectra (``.peaks.mz`` / ``.peaks.intensities``),
    ``(mz, intensities)`` pairs or ``None`` (empty)."""
    mzs, ints = [], []
    lens = np.empty(len(spectra), dtype=np.int64)
    for i, s in enumerate(spectra):
        m, it = _peaks_of(s)
        if m is None:
            lens[i] = 0
            continue
        n = m.shape[0] if n_max_peaks is None else min(m.shape[0], int(n_max_peaks))
        if it.shape[0] != m.shape[0]:
            raise ValueError(f"spectrum {i}: mz and intensities differ in length")
        lens[i] = n
        mzs.append(m[:n])
        ints.append(it[:n])
    offsets = np.zeros(len(spectra) + 1, dtype=np.int64)
    np.cumsum(lens, out=offsets[1:])
    mz = np.concatenate(mzs) if mzs else np.zeros(0, np.float32)
    it = np.concatenate(ints) if ints else np.zeros(0, np.float32)
    packed = pack_csr(mz, it, offsets, None, mz_power, intensity_power, check=check)
    packed.n_max_peaks = None if n_max_peaks is None else int(n_max_peaks)
    return packed


def pack_fingerprints(fingerprints: Iterable, n_bits: Optional[int] = None):
    """Bit-pack fingerprints.

    Returns (bits uint32 [N, W], valid uint8 [N], n_bits) where W = ceil(n_bits/32).
    ``None`` entries are rows without a fingerprint (valid = 0, bits zero).
    Fingerprint values must be 0/1 (the reference's matrices are 0/1 vectors).
    """
    fps = list(fingerprints)
    n = len(fps)
    valid = np.array([fp is not None for fp in fps], dtype=np.uint8)
    lengths = {int(np.asarray(fp).shape[-1]) for fp in fps if fp is not None}
    if n_bits is None:
        if len(lengths) > 1:
            raise ValueError(f"fingerprints have different lengths: {sorted(lengths)}")
        n_bits = lengths.pop() if lengths else 0
    elif lengths and lengths != {n_bits}:
        raise ValueError("fingerprint length differs from n_bits")
    n_words = (n_bits + 31) // 32
    bits = np.zeros((n, n_words), dtype=np.uint32)
    if valid.any() and n_words:
        dense = np.zeros((n, n_words * 32), dtype=np.uint8)
        rows = np.flatnonzero(valid)
        stacked = np.stack([np.asarray(fps[i]).reshape(-1) for i in rows])
        if not np.isin(stacked, (0, 1)).all():
            raise ValueError("fingerprints must be binary (0/1) vectors")
        dense[rows, :n_bits] = stacked.astype(np.uint8)
        packed = np.packbits(dense, axis=1, bitorder="little")  # [n, n_words*4] bytes
        bits = np.ascontiguousarray(packed).view("<u4").reshape(n, n_words).astype(np.uint32)
    return bits, valid, int(n_bits)


def pack_fingerprint_matrix(dense: np.ndarray):
    """Bit-pack a dense 0/1 matrix [N, n_bits] (all rows valid)."""
    dense = np.asarray(dense)
    if dense.ndim != 2:
        raise ValueError("expected a 2-D 0/1 matrix")
    if not np.isin(dense, (0, 1)).all():
        raise ValueError("fingerprints must be binary (0/1) vectors")
    n, n_bits = dense.shape
    n_words = (n_bits + 31) // 32
    pad = np.zeros((n, n_words * 32), dtype=np.uint8)
    pad[:, :n_bits] = dense
    packed = np.packbits(pad, axis=1, bitorder="little")
    bits = np.ascontiguousarray(packed).view("<u4").reshape(n, n_words).astype(np.uint32)
    return bits, np.ones(n, dtype=np.uint8), int(n_bits)
