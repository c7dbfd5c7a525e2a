"""Generate golden fixtures from the reference implementation itself.

Run where the reference package (a checkout of tornikeo/cosine-similarity)
is readable; its root is given by --reference or, when that is omitted, by
the CUDAMS_REFERENCE environment variable (one of the two is required):

    python tests/golden/make_golden.py --reference <path to the checkout>

Greedy cosine: the reference's Numba kernel (cudams/similarity/
spectrum_similarity_functions.py:39-278) is run under numba's CUDA simulator
(NUMBA_ENABLE_CUDASIM=1), with its packing (CudaCosineGreedy._spectra_peaks_to_
tensor, CudaCosineGreedy.py:63-87).  matchms and sparsestack are not
installed, so stub modules stand in for the names the reference imports; the
kernel itself does not use them.  The launcher is called directly because the
reference's CudaTimer does not work in the simulator.

Fingerprints: the reference's torch functions (cudams/similarity/
vector_similarity_functions.py:12-119) run on CPU torch with ndarray inputs.

Outputs: tests/golden/cosine_<case>.npz and fingerprint_<case>.npz holding
the raw float64 inputs as passed to the reference, the parameters, and the
reference's outputs.  Nothing at test time reads the reference.
"""
from __future__ import annotations

import argparse
import os
import sys
import time
import types
from pathlib import Path

import numpy as np

OUT = Path(__file__).resolve().parent


def _install_stubs():
    def stub(name, **attrs):
        m = types.ModuleType(name)
        m.__dict__.update(attrs)
        sys.modules[name] = m
        return m

    class BaseSimilarity:
        pass

    class _Peaks:
        def __init__(self, mz, it):
            self.mz = mz
            self.intensities = it

        def __len__(self):
            return len(self.mz)

    class Spectrum:
        def __init__(self, mz, intensities, metadata=None):
            self._peaks = _Peaks(np.asarray(mz, float), np.asarray(intensities, float))
            self.peaks = self._peaks

    stub("matchms", Spectrum=Spectrum)
    stub("matchms.similarity")
    stub("matchms.similarity.BaseSimilarity", BaseSimilarity=BaseSimilarity)
    stub("matchms.similarity.spectrum_similarity_functions", collect_peak_pairs=None,
         score_best_matches=None)
    stub("matchms.typing", SpectrumType=object)
    stub("matchms.filtering", **{k: None for k in (
        "add_losses normalize_intensities reduce_to_number_of_peaks "
        "require_minimum_number_of_peaks select_by_mz select_by_relative_intensity").split()})
    stub("sparsestack", StackedSparseArray=object)
    return Spectrum


# ---------------------------------------------------------------- inputs
def _uniform(rng, n, lo_peaks=10, hi_peaks=200, mz_lo=50.0, mz_hi=1000.0):
    spectra = []
    for _ in range(n):
        k = int(rng.integers(lo_peaks, hi_peaks + 1))
        mz = np.sort(rng.uniform(mz_lo, mz_hi, k).astype(np.float32)).astype(np.float64)
        it = (1.0 - rng.uniform(0, 1, k)).astype(np.float32)
        it = (it / it.max()).astype(np.float32).astype(np.float64)
        spectra.append((mz, it))
    return spectra


def _lognormal(rng, n):
    spectra = []
    for _ in range(n):
        k = int(np.clip(np.round(rng.lognormal(np.log(60), 1.0)), 5, 1000))
        mz = np.sort(rng.uniform(50, 2000, k).astype(np.float32)).astype(np.float64)
        it = rng.exponential(1.0, k).astype(np.float32)
        it = (it / it.max()).astype(np.float32).astype(np.float64)
        spectra.append((mz, it))
    return spectra


def _clustered(rng, n, centres, lo_peaks, hi_peaks):
    spectra = []
    for _ in range(n):
        k = int(rng.integers(lo_peaks, hi_peaks + 1))
        mz = centres[rng.integers(0, centres.shape[0], k)] + rng.normal(0, 0.02, k)
        mz = np.sort(mz.astype(np.float32)).astype(np.float64)
        it = (1.0 - rng.uniform(0, 1, k)).astype(np.float32)
        it = (it / it.max()).astype(np.float32).astype(np.float64)
        spectra.append((mz, it))
    return spectra


def _ties(rng, n):
    """Spectra whose products tie often: intensities on a coarse grid."""
    spectra = []
    for _ in range(n):
        k = int(rng.integers(5, 40))
        mz = np.sort(rng.choice(np.arange(100.0, 140.0, 0.25), k, replace=False))
        it = rng.choice(np.array([0.25, 0.5, 1.0]), k)
        it[rng.integers(0, k)] = 1.0
        spectra.append((mz, it))
    return spectra


KNOWN = [
    # tests/similarity/test_cosine_greedy.py:27-94 (peaks, tolerance, mz_power, intensity_power)
    (([100, 200, 300, 500, 510], [0.1, 0.2, 1.0, 0.3, 0.4]),
     ([100, 200, 290, 490, 510], [0.1, 0.2, 1.0, 0.3, 0.4]), 0.1, 0.0, 1.0),
    (([100, 299, 300, 301, 510], [0.1, 1.0, 0.2, 0.3, 0.4]),
     ([100, 300, 301, 511], [0.1, 1.0, 0.3, 0.4]), 0.2, 0.0, 1.0),
    (([100, 299, 300, 301, 510], [0.1, 1.0, 0.2, 0.3, 0.4]),
     ([100, 300, 301, 511], [0.1, 1.0, 0.3, 0.4]), 2.0, 0.0, 1.0),
    (([100, 200, 300, 500, 510], [0.1, 0.2, 1.0, 0.3, 0.4]),
     ([100, 200, 290, 490, 510], [0.1, 0.2, 1.0, 0.3, 0.4]), 1.0, 0.5, 2.0),
]


def _mgf_spectra(path: Path):
    """(m/z, intensity) float64 arrays of an MGF file's spectra: peaks sorted
    by m/z, intensities scaled to a maximum of 1 (matchms'
    normalize_intensities, which the reference's tests apply to their MGF
    spectra before scoring)."""
    spectra, cur, inside = [], [], False
    for line in path.read_text(errors="replace").splitlines():
        line = line.strip()
        if line.upper() == "BEGIN IONS":
            inside, cur = True, []
        elif line.upper() == "END IONS":
            inside = False
            arr = np.array(cur, float).reshape(-1, 2)
            arr = arr[np.argsort(arr[:, 0], kind="stable")]
            if arr.shape[0] and arr[:, 1].max() > 0:
                arr[:, 1] = arr[:, 1] / arr[:, 1].max()
            spectra.append((arr[:, 0].copy(), arr[:, 1].copy()))
        elif inside and line and (line[0].isdigit() or line[0] in "+-."):
            parts = line.split()
            cur.append((float(parts[0]), float(parts[1])))
    return spectra


def cosine_cases(reference: Path = None):
    rng = np.random.default_rng(20261203)
    cases = []
    for i, (s1, s2, tol, p, q) in enumerate(KNOWN):
        a = (np.array(s1[0], float), np.array(s1[1], float))
        b = (np.array(s2[0], float), np.array(s2[1], float))
        cases.append((f"known{i}", [a, b], [a, b], dict(tolerance=tol, mz_power=p,
                                                         intensity_power=q, shift=0.0,
                                                         match_limit=2048, n_max_peaks=16)))
    cases.append(("uniform", _uniform(rng, 20), _uniform(rng, 20),
                  dict(tolerance=0.1, mz_power=0.0, intensity_power=1.0, shift=0.0,
                       match_limit=2048, n_max_peaks=1024)))
    cases.append(("lognormal", _lognormal(rng, 20), _lognormal(rng, 20),
                  dict(tolerance=0.01, mz_power=0.0, intensity_power=1.0, shift=0.0,
                       match_limit=4096, n_max_peaks=1024)))
    centres = rng.uniform(50, 1000, 40)
    cases.append(("clustered_overflow", _clustered(rng, 10, centres, 60, 160),
                  _clustered(rng, 10, centres, 60, 160),
                  dict(tolerance=0.05, mz_power=3.0, intensity_power=0.6, shift=0.0,
                       match_limit=96, n_max_peaks=256)))
    cases.append(("truncation", _uniform(rng, 12, 20, 90), _uniform(rng, 12, 20, 90),
                  dict(tolerance=0.5, mz_power=0.0, intensity_power=1.0, shift=0.0,
                       match_limit=2048, n_max_peaks=32)))
    empty = (np.zeros(0), np.zeros(0))
    mix = _uniform(rng, 6, 5, 30)
    cases.append(("empty", [empty] + mix[:3], mix[3:] + [empty],
                  dict(tolerance=2.0, mz_power=0.0, intensity_power=1.0, shift=0.0,
                       match_limit=2048, n_max_peaks=64)))
    ties = _ties(rng, 14)
    cases.append(("ties", ties, ties, dict(tolerance=0.3, mz_power=0.0, intensity_power=1.0,
                                           shift=0.0, match_limit=2048, n_max_peaks=64)))
    cases.append(("shift", _uniform(rng, 10, 10, 60), _uniform(rng, 10, 10, 60),
                  dict(tolerance=0.6, mz_power=0.5, intensity_power=2.0, shift=0.5,
                       match_limit=2048, n_max_peaks=128)))
    cases.append(("limit_exact", [KNOWN[0][0]], [KNOWN[0][0]],
                  dict(tolerance=0.1, mz_power=0.0, intensity_power=1.0, shift=0.0,
                       match_limit=5, n_max_peaks=16)))
    # measured spectra: the reference's own test data (tests/data/pesticides.mgf),
    # all 76 against all 76 with the reference's default parameters
    mgf = None if reference is None else reference / "tests" / "data" / "pesticides.mgf"
    if mgf is not None and mgf.is_file():
        pest = _mgf_spectra(mgf)
        cases.append(("pesticides", pest, pest,
                      dict(tolerance=0.1, mz_power=0.0, intensity_power=1.0, shift=0.0,
                           match_limit=2048, n_max_peaks=1024)))
    return cases


def _csr(spectra):
    lens = np.array([len(m) for m, _ in spectra], np.int64)
    off = np.zeros(len(spectra) + 1, np.int64)
    np.cumsum(lens, out=off[1:])
    mz = np.concatenate([np.asarray(m, float) for m, _ in spectra]) if lens.sum() else np.zeros(0)
    it = np.concatenate([np.asarray(i, float) for _, i in spectra]) if lens.sum() else np.zeros(0)
    return mz, it, off


def run_reference_cosine(Spectrum, CudaCosineGreedy, refs, qrys, params):
    B = max(len(refs), len(qrys))
    k = CudaCosineGreedy(batch_size=B, tolerance=params["tolerance"], mz_power=params["mz_power"],
                         intensity_power=params["intensity_power"], shift=params["shift"],
                         n_max_peaks=params["n_max_peaks"], match_limit=params["match_limit"])
    R = [Spectrum(m, i) for m, i in refs]
    Q = [Spectrum(m, i) for m, i in qrys]
    rs, rl = k._spectra_peaks_to_tensor(R)
    qs, ql = k._spectra_peaks_to_tensor(Q)
    lens = np.zeros((2, B), np.int32)
    lens[0, :len(rl)] = rl
    lens[1, :len(ql)] = ql
    pad = lambda x: np.concatenate([x, np.zeros((2, B - x.shape[1], x.shape[2]), x.dtype)],  # noqa
                                   axis=1) if x.shape[1] < B else x
    out = np.zeros((3, B, B), np.float32)
    k.kernel(pad(rs), pad(qs), lens, out)
    return out[:, :len(refs), :len(qrys)]


def make_cosine(reference: Path, Spectrum, only_case=None):
    sys.path.insert(0, str(reference))
    from cudams.similarity import CudaCosineGreedy  # the reference package

    for name, refs, qrys, params in cosine_cases(reference):
        if only_case and name != only_case:
            continue
        t = time.time()
        out = run_reference_cosine(Spectrum, CudaCosineGreedy, refs, qrys, params)
        rmz, rit, roff = _csr(refs)
        qmz, qit, qoff = _csr(qrys)
        np.savez_compressed(OUT / f"cosine_{name}.npz", r_mz=rmz, r_int=rit, r_off=roff,
                            q_mz=qmz, q_int=qit, q_off=qoff,
                            params=np.array([params[k] for k in PARAM_KEYS], np.float64),
                            score=out[0].astype(np.float32), matches=out[1].astype(np.int32),
                            overflow=out[2].astype(np.uint8))
        print(f"cosine_{name}: {len(refs)}x{len(qrys)} in {time.time() - t:.1f}s; "
              f"mean matches {out[1].mean():.2f}, overflow {out[2].mean():.3f}", flush=True)


PARAM_KEYS = ["tolerance", "mz_power", "intensity_power", "shift", "match_limit", "n_max_peaks"]


def make_fingerprints(reference: Path):
    sys.path.insert(0, str(reference))
    from cudams.similarity.vector_similarity_functions import (cosine_similarity_matrix,
                                                               dice_similarity_matrix,
                                                               jaccard_similarity_matrix)

    rng = np.random.default_rng(7)
    f1 = np.array([1, 1, 0, 0, 0, 1, 0, 0, 1, 0, 0, 1, 0, 0, 0, 0])
    f2 = np.array([0, 1, 1, 0, 0, 1, 0, 0, 1, 0, 1, 1, 0, 0, 0, 1])
    f3 = np.array([0, 0, 1, 0, 0, 1, 0, 0, 1, 0, 1, 1, 0, 0, 0, 0])
    z = np.zeros(16, int)
    cases = {"tests16": (np.stack([f1, f2, f3, z]), np.stack([f2, f1, z, f3]))}

    def rand(n, bits):
        d = rng.uniform(0.05, 0.15, n)
        return (rng.random((n, bits)) < d[:, None]).astype(np.int64)

    a = rand(64, 2048)
    b = rand(48, 2048)
    a[5] = 0
    b[7] = 0
    cases["random2048"] = (a, b)
    cases["odd100"] = (rand(33, 100), rand(17, 100))
    dense = (rng.random((20, 256)) < 0.9).astype(np.int64)
    cases["dense256"] = (dense, dense[::-1].copy())
    for name, (r, q) in cases.items():
        res = {}
        for m, fn in (("jaccard", jaccard_similarity_matrix), ("dice", dice_similarity_matrix),
                      ("cosine", cosine_similarity_matrix)):
            res[m] = np.asarray(fn(np.asarray(r), np.asarray(q)), np.float32)
        np.savez_compressed(OUT / f"fingerprint_{name}.npz", ref=r.astype(np.uint8),
                            qry=q.astype(np.uint8), **res)
        print(f"fingerprint_{name}: {r.shape[0]}x{q.shape[0]}x{r.shape[1]}", flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("CUDAMS_REFERENCE"),
                    help="root of the reference checkout (default: $CUDAMS_REFERENCE)")
    ap.add_argument("--only", choices=["cosine", "fingerprint"], default=None)
    ap.add_argument("--case", default=None, help="only this cosine case (e.g. pesticides)")
    args = ap.parse_args()
    if not args.reference:
        ap.error("give --reference or set CUDAMS_REFERENCE to the reference checkout")
    ref = Path(args.reference)
    if not (ref / "cudams").is_dir():
        sys.exit(f"reference package not found under {ref}")
    # before numba is imported anywhere: the simulator is chosen at import
    os.environ["NUMBA_ENABLE_CUDASIM"] = "1"
    Spectrum = _install_stubs()
    if args.only in (None, "fingerprint"):
        make_fingerprints(ref)
    if args.only in (None, "cosine"):
        make_cosine(ref, Spectrum, args.case)


if __name__ == "__main__":
    main()
