"""Seeded synthetic spectra and fingerprints with the shapes of the benchmark
workloads (no public dataset is available offline; these stand in for the
GNPS library the reference benchmarks on).

All generators use numpy.random.default_rng(seed) and return packed CSR sets
(cudams.packing.PackedSpectra) built directly from arrays, so that 100k- and
1M-spectrum sets are generated without Python loops.

Workloads
  uniform_spectra    peaks ~ U{10..200}, m/z U(50, 1000) float32 sorted,
                     intensities U(0, 1] scaled to max 1        (1024 x 1024,
                     tolerance 0.1, powers (0, 1), match_limit 2048)
  lognormal_spectra  peaks = round(lognormal(median 60, sigma 1.0)) clipped to
                     [5, 1000], m/z U(50, 2000), intensities Exp(1) scaled to
                     max 1                                     (100k x 100k,
                     tolerance 0.01, powers (0, 1), match_limit 4096; and the
                     1M-spectrum served library)
  clustered_spectra  peaks ~ U{1000..2000}; one global set of 200 centres
                     U(50, 1000); each peak = random centre + N(0, 0.02^2),
                     sorted; intensities U(0, 1] scaled to max 1 (20k x 20k,
                     tolerance 0.05, powers (3, 0.6), match_limit 1024,
                     n_max_peaks 2048)
  fingerprints       2048-bit fingerprints, per-fingerprint density
                     U(5%, 15%), bits iid, packed as uint32 words
  analog_spectra     families of structural analogues for modified cosine:
                     a base spectrum (lognormal peak count, m/z below the
                     precursor) and members whose precursor and upper
                     fragments move by one mass difference, with jitter,
                     dropped and added peaks; returns the spectra and their
                     precursor m/z
"""
from __future__ import annotations

import numpy as np

from .packing import PackedSpectra, pack_csr

LOGNORMAL_SIGMA = 1.0


def _segments(lengths: np.ndarray):
    off = np.zeros(lengths.shape[0] + 1, dtype=np.int64)
    np.cumsum(lengths, out=off[1:])
    seg = np.repeat(np.arange(lengths.shape[0], dtype=np.int64), lengths)
    return off, seg


def _sort_within(mz: np.ndarray, seg: np.ndarray) -> np.ndarray:
    # segments are contiguous: sorting by (seg, mz) sorts inside each segment
    order = np.lexsort((mz, seg))
    return mz[order]


def sorted_uniform(rng, lengths: np.ndarray, lo: float, hi: float) -> np.ndarray:
    """Ascending U(lo, hi) samples per spectrum in O(P): the order statistics of
    n uniforms are the normalised partial sums of n + 1 exponential spacings."""
    lengths = np.asarray(lengths, dtype=np.int64)
    n = lengths.shape[0]
    ext = lengths + 1
    e = rng.exponential(1.0, int(ext.sum()))
    c = np.cumsum(e)
    ends = np.cumsum(ext) - 1
    starts = ends - lengths
    base = np.where(starts > 0, c[np.maximum(starts - 1, 0)], 0.0)
    total = c[ends] - base
    seg = np.repeat(np.arange(n), lengths)
    # output j of segment s is the partial sum at index starts[s] + j
    first_out = np.concatenate([[0], np.cumsum(lengths)[:-1]])
    within = np.arange(int(lengths.sum())) - first_out[seg]
    pos = starts[seg] + within
    u = (c[pos] - base[seg]) / total[seg]
    return (lo + (hi - lo) * u).astype(np.float32)


def _scale_to_max(x: np.ndarray, off: np.ndarray) -> np.ndarray:
    nonempty = off[1:] > off[:-1]
    mx = np.ones(off.shape[0] - 1, dtype=x.dtype)
    if nonempty.any():
        mx[nonempty] = np.maximum.reduceat(x, off[:-1][nonempty])
    lengths = np.diff(off)
    return (x / np.repeat(mx, lengths)).astype(np.float32)


def _build(lengths, mz, inten, n_max_peaks, mz_power, intensity_power,
           presorted: bool = False) -> PackedSpectra:
    off, seg = _segments(lengths)
    mz = mz.astype(np.float32) if presorted else _sort_within(mz.astype(np.float32), seg)
    inten = _scale_to_max(inten.astype(np.float32), off)
    return pack_csr(mz, inten, off, n_max_peaks, mz_power, intensity_power, check=False)


def uniform_spectra(n: int, seed: int = 0, n_max_peaks: int = 1024, mz_power: float = 0.0,
                    intensity_power: float = 1.0) -> PackedSpectra:
    rng = np.random.default_rng(seed)
    lengths = rng.integers(10, 201, n).astype(np.int64)
    p = int(lengths.sum())
    mz = sorted_uniform(rng, lengths, 50.0, 1000.0)
    inten = 1.0 - rng.uniform(0.0, 1.0, p)  # (0, 1]
    return _build(lengths, mz, inten, n_max_peaks, mz_power, intensity_power, presorted=True)


def lognormal_lengths(rng, n: int, median: float = 60.0, sigma: float = LOGNORMAL_SIGMA,
                      lo: int = 5, hi: int = 1000) -> np.ndarray:
    return np.clip(np.round(rng.lognormal(np.log(median), sigma, n)), lo, hi).astype(np.int64)


def lognormal_spectra(n: int, seed: int = 0, n_max_peaks: int = 1024, mz_power: float = 0.0,
                      intensity_power: float = 1.0, sigma: float = LOGNORMAL_SIGMA) -> PackedSpectra:
    rng = np.random.default_rng(seed)
    lengths = lognormal_lengths(rng, n, sigma=sigma)
    p = int(lengths.sum())
    mz = sorted_uniform(rng, lengths, 50.0, 2000.0)
    inten = rng.exponential(1.0, p)
    return _build(lengths, mz, inten, n_max_peaks, mz_power, intensity_power, presorted=True)


def cluster_centres(seed: int = 12345, n_centres: int = 200) -> np.ndarray:
    return np.random.default_rng(seed).uniform(50.0, 1000.0, n_centres)


def clustered_spectra(n: int, seed: int = 0, centres=None, n_max_peaks: int = 2048,
                      mz_power: float = 3.0, intensity_power: float = 0.6,
                      min_peaks: int = 1000, max_peaks: int = 2000) -> PackedSpectra:
    rng = np.random.default_rng(seed)
    centres = cluster_centres() if centres is None else np.asarray(centres)
    lengths = rng.integers(min_peaks, max_peaks + 1, n).astype(np.int64)
    p = int(lengths.sum())
    mz = centres[rng.integers(0, centres.shape[0], p)] + rng.normal(0.0, 0.02, p)
    inten = 1.0 - rng.uniform(0.0, 1.0, p)
    return _build(lengths, mz, inten, n_max_peaks, mz_power, intensity_power)


def fingerprints(n: int, n_bits: int = 2048, seed: int = 0, dmin: float = 0.05,
                 dmax: float = 0.15, chunk: int = 8192) -> np.ndarray:
    """Packed uint32 [n, ceil(n_bits/32)] fingerprints."""
    rng = np.random.default_rng(seed)
    n_words = (n_bits + 31) // 32
    out = np.zeros((n, n_words), dtype=np.uint32)
    dens = rng.uniform(dmin, dmax, n)
    for s in range(0, n, chunk):
        e = min(n, s + chunk)
        dense = np.zeros((e - s, n_words * 32), dtype=np.uint8)
        dense[:, :n_bits] = rng.random((e - s, n_bits)) < dens[s:e, None]
        packed = np.packbits(dense, axis=1, bitorder="little")
        out[s:e] = np.ascontiguousarray(packed).view("<u4").reshape(e - s, n_words)
    return out


def analog_spectra(n: int, seed: int = 0, family_size: int = 8, n_max_peaks: int = 1024,
                   mz_power: float = 0.0, intensity_power: float = 1.0, median_peaks: float = 60.0):
    """(PackedSpectra, precursor_mz float64[n]): families of `family_size`
    analogues.  Member k of a family shares the base spectrum's peaks; peaks
    above a random cut move by the member's mass difference d (one in four
    members has d = 0), every peak is jittered by N(0, 0.002^2), a tenth are
    dropped and a few noise peaks are added; its precursor is the base
    precursor + d."""
    rng = np.random.default_rng(seed)
    spectra, prec = [], np.empty(n, np.float64)
    base = None
    for i in range(n):
        if i % family_size == 0:
            k = int(np.clip(np.round(rng.lognormal(np.log(median_peaks), 0.6)), 5, 600))
            p0 = rng.uniform(300.0, 1500.0)
            bmz = np.sort(rng.uniform(50.0, p0 - 5.0, k))
            bint = rng.exponential(1.0, k)
            cut = rng.uniform(0.3, 0.8) * p0
            base = (bmz, bint, p0, cut)
        bmz, bint, p0, cut = base
        d = 0.0 if rng.random() < 0.25 else float(rng.uniform(-40.0, 40.0))
        keep = rng.random(bmz.shape[0]) >= 0.1
        mz = np.where(bmz > cut, bmz + d, bmz)[keep] + rng.normal(0.0, 0.002, int(keep.sum()))
        it = bint[keep] * rng.uniform(0.7, 1.3, int(keep.sum()))
        extra = int(rng.integers(0, 6))
        mz = np.concatenate([mz, rng.uniform(50.0, p0 + d, extra)])
        it = np.concatenate([it, rng.exponential(0.3, extra)])
        mz = np.clip(mz, 1.0, None)
        order = np.argsort(mz, kind="stable")
        spectra.append((mz[order], it[order] / max(it.max(), 1e-12)))
        prec[i] = p0 + d
    lengths = np.array([m.shape[0] for m, _ in spectra], np.int64)
    mz = np.concatenate([m for m, _ in spectra]).astype(np.float32)
    inten = np.concatenate([x for _, x in spectra])
    off, seg = _segments(lengths)
    mz = _sort_within(mz, seg)  # float32 rounding can reorder near-equal m/z
    packed = pack_csr(mz, inten.astype(np.float32), off, n_max_peaks, mz_power, intensity_power,
                      check=False)
    return packed, prec
