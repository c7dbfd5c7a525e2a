"""Pure-Python restatement of matchms CosineGreedy for small cases.

TEST INFRASTRUCTURE ONLY (see oracle/cosine_greedy_oracle.c).

matchms (>= 0.24.0, pinned by the reference's requirements.txt:1) is not
vendored in the reference and not installed here.  This restates its
published CosineGreedy algorithm, as the reference calls it in
cudams/similarity/spectrum_similarity_functions.py:306-317:
collect_peak_pairs (find_matches window + power products), numpy's stable
argsort(kind="mergesort")[::-1] on the products, then score_best_matches
(greedy over the sorted pairs, normalised by the two spectra's norms).  It
works on float64 arrays as given (no float32 rounding, no truncation, no
match_limit), so it checks the C oracle's ordering and tie rules
independently of the C code and of the packer.
"""
from __future__ import annotations

import numpy as np


def find_matches(mz1: np.ndarray, mz2: np.ndarray, tolerance: float, shift: float = 0.0):
    lowest_idx = 0
    matches = []
    for peak1_idx in range(mz1.shape[0]):
        mz = mz1[peak1_idx]
        low_bound = mz - tolerance
        high_bound = mz + tolerance
        for peak2_idx in range(lowest_idx, mz2.shape[0]):
            mz_2 = mz2[peak2_idx] + shift
            if mz_2 > high_bound:
                break
            if mz_2 < low_bound:
                lowest_idx = peak2_idx
            else:
                matches.append((peak1_idx, peak2_idx))
    return matches


def collect_peak_pairs(spec1, spec2, tolerance, shift=0.0, mz_power=0.0, intensity_power=1.0):
    matches = find_matches(spec1[:, 0], spec2[:, 0], tolerance, shift)
    if not matches:
        return None
    rows = []
    for i1, i2 in matches:
        prod = (spec1[i1, 0] ** mz_power * spec1[i1, 1] ** intensity_power
                * spec2[i2, 0] ** mz_power * spec2[i2, 1] ** intensity_power)
        rows.append([i1, i2, prod])
    return np.array(rows, dtype=np.float64)


def score_best_matches(pairs, spec1, spec2, mz_power=0.0, intensity_power=1.0):
    score = 0.0
    used = 0
    used1, used2 = set(), set()
    for i in range(pairs.shape[0]):
        a, b = pairs[i, 0], pairs[i, 1]
        if a not in used1 and b not in used2:
            score += pairs[i, 2]
            used1.add(a)
            used2.add(b)
            used += 1
    p1 = spec1[:, 0] ** mz_power * spec1[:, 1] ** intensity_power
    p2 = spec2[:, 0] ** mz_power * spec2[:, 1] ** intensity_power
    score = score / (np.sum(p1 ** 2) ** 0.5 * np.sum(p2 ** 2) ** 0.5)
    return score, used


def cosine_greedy_pair(mz1, int1, mz2, int2, tolerance=0.1, mz_power=0.0, intensity_power=1.0,
                       shift=0.0):
    """(score float64, matches int) of one pair, matchms semantics."""
    spec1 = np.stack([np.asarray(mz1, np.float64), np.asarray(int1, np.float64)], axis=1)
    spec2 = np.stack([np.asarray(mz2, np.float64), np.asarray(int2, np.float64)], axis=1)
    pairs = collect_peak_pairs(spec1, spec2, tolerance, shift, mz_power, intensity_power)
    if pairs is None:
        return 0.0, 0
    pairs = pairs[np.argsort(pairs[:, 2], kind="mergesort")[::-1], :]
    return score_best_matches(pairs, spec1, spec2, mz_power, intensity_power)


def modified_cosine_pair(mz1, int1, mz2, int2, precursor1, precursor2, tolerance=0.1,
                         mz_power=0.0, intensity_power=1.0):
    """(score float64, matches int) of one pair, matchms ModifiedCosine
    semantics: the matches at shift 0 and at shift precursor1 - precursor2,
    concatenated, sorted once (stable, reversed), then one greedy."""
    spec1 = np.stack([np.asarray(mz1, np.float64), np.asarray(int1, np.float64)], axis=1)
    spec2 = np.stack([np.asarray(mz2, np.float64), np.asarray(int2, np.float64)], axis=1)
    zero = collect_peak_pairs(spec1, spec2, tolerance, 0.0, mz_power, intensity_power)
    shifted = collect_peak_pairs(spec1, spec2, tolerance, float(precursor1) - float(precursor2),
                                 mz_power, intensity_power)
    parts = [x for x in (zero, shifted) if x is not None]
    if not parts:
        return 0.0, 0
    pairs = np.concatenate(parts, axis=0)
    pairs = pairs[np.argsort(pairs[:, 2], kind="mergesort")[::-1], :]
    return score_best_matches(pairs, spec1, spec2, mz_power, intensity_power)
