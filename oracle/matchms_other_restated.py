"""Pure-Python restatement of matchms' ParentMassMatch, PrecursorMzMatch and
IntersectMz, the other similarities the reference prototypes beside its CUDA
classes (notebooks/prototyping/other_similarities.ipynb).

TEST INFRASTRUCTURE ONLY: tests use it as the checker of the device kernels
in csrc/metadata_match.cu; the product never imports it.

Parity unpinned: matchms (>= 0.24.0, the reference's requirements.txt:1) is
neither vendored in the reference nor installed here, and the reference holds
no golden vectors for these three scores.  The definitions below restate
matchms' published algorithms:

  ParentMassMatch.pair / parentmass_scores:   abs(mass_r - mass_q) <= tolerance
  PrecursorMzMatch (tolerance_type "Dalton"): abs(mz_r - mz_q) <= tolerance
  PrecursorMzMatch (tolerance_type "ppm"):    mean = (mz_r + mz_q) / 2;
                                              abs(mz_r - mz_q) / mean * 1e6 <= tolerance
  IntersectMz.pair:  A = set(mz_r), B = set(mz_q); 0 if A | B is empty, else
                     scaling * len(A & B) / len(A | B)

each in Python float64 arithmetic (the order of operations as written), one
pair at a time.
"""
from __future__ import annotations

import numpy as np


def mass_match(ref_values, q_values, tolerance: float, ppm: bool = False) -> np.ndarray:
    """Boolean matrix [R, Q] of ParentMassMatch / PrecursorMzMatch."""
    out = np.zeros((len(ref_values), len(q_values)), dtype=bool)
    for i, r in enumerate(ref_values):
        r = float(r)
        for j, q in enumerate(q_values):
            q = float(q)
            if ppm:
                mean_mz = (r + q) / 2
                out[i, j] = abs(r - q) / mean_mz * 1e6 <= tolerance
            else:
                out[i, j] = abs(r - q) <= tolerance
    return out


def intersect_mz(ref_mz_lists, q_mz_lists, scaling: float = 1.0) -> np.ndarray:
    """float64 matrix [R, Q] of IntersectMz; *_mz_lists are per-spectrum
    float64 m/z arrays."""
    out = np.zeros((len(ref_mz_lists), len(q_mz_lists)), dtype=np.float64)
    ref_sets = [set(float(x) for x in a) for a in ref_mz_lists]
    q_sets = [set(float(x) for x in b) for b in q_mz_lists]
    for i, a in enumerate(ref_sets):
        for j, b in enumerate(q_sets):
            union = len(a | b)
            out[i, j] = 0.0 if union == 0 else scaling * len(a & b) / union
    return out
