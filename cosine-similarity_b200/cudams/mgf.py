"""MGF (Mascot Generic Format) reader straight into the packed CSR layout.

The reference's tests load spectra from MGF files through matchms
(`matchms.importing.load_from_mgf`, e.g. tests/usecase/test_tutorial_pesticide.py)
and then pack them one Python object at a time (CudaCosineGreedy.py:63-87).
This reader skips the per-spectrum objects: it collects the peak lines of all
spectra, converts them to numbers in one numpy call where every peak line has
two columns (a per-line split otherwise), sorts each spectrum's peaks by m/z
(stable, as matchms requires ascending m/z) and hands the CSR arrays to
`pack_csr`.  Metadata lines (`KEY=value`) are returned per spectrum with
lower-cased keys; `PEPMASS` also gives `precursor_mz` (its first number).
"""
from __future__ import annotations

import io
import os
from typing import Iterable, List, Optional, Tuple, Union

import numpy as np

from .packing import PackedSpectra, pack_csr


def _lines(source) -> Iterable[str]:
    if isinstance(source, (str, os.PathLike)):
        with open(source, "r", encoding="utf-8", errors="replace") as f:
            yield from f
    elif isinstance(source, io.IOBase) or hasattr(source, "read"):
        yield from source
    else:
        yield from source


def read_mgf(source: Union[str, os.PathLike, Iterable[str]], n_max_peaks: Optional[int] = 1024,
             mz_power: float = 0.0, intensity_power: float = 1.0
             ) -> Tuple[PackedSpectra, List[dict]]:
    """Spectra of an MGF file (path, open text file or iterable of lines).

    Returns (PackedSpectra, metadata): one metadata dict per BEGIN/END IONS
    block, in file order; peaks sorted by m/z within each spectrum, the first
    `n_max_peaks` of them kept (after sorting, as the reference keeps the first
    n_max_peaks of its m/z-sorted matchms spectra).  Peak lines hold m/z and
    intensity; further columns (annotations) are ignored."""
    meta: List[dict] = []
    counts: List[int] = []
    peak_lines: List[str] = []
    inside = False
    cur: dict = {}
    n_peaks = 0
    for raw in _lines(source):
        line = raw.strip()
        if not line:
            continue
        head = line[0]
        if inside and (head.isdigit() or head in "+-."):
            peak_lines.append(line)
            n_peaks += 1
            continue
        if head in "#;!/":
            continue
        if not inside:
            if line.upper() == "BEGIN IONS":
                inside, cur, n_peaks = True, {}, 0
            continue
        if line.upper() == "END IONS":
            inside = False
            meta.append(cur)
            counts.append(n_peaks)
            continue
        key, sep, value = line.partition("=")
        if sep:
            k = key.strip().lower()
            v = value.strip()
            cur[k] = v
            if k == "pepmass":
                try:
                    cur["precursor_mz"] = float(v.split()[0])
                except (ValueError, IndexError):
                    pass
    if inside:
        raise ValueError("MGF ends inside a BEGIN IONS block")

    peaks = None
    if peak_lines:
        # fast path: every peak line is "mz intensity" -> one bulk conversion
        toks = " ".join(peak_lines).split()
        if len(toks) == 2 * len(peak_lines):
            try:
                peaks = np.array(toks, dtype=np.float64).reshape(-1, 2)
            except ValueError:
                peaks = None
        if peaks is None:
            peaks = np.empty((len(peak_lines), 2))
            for i, line in enumerate(peak_lines):
                parts = line.split()
                peaks[i, 0] = float(parts[0])
                peaks[i, 1] = float(parts[1]) if len(parts) > 1 else 0.0
    else:
        peaks = np.zeros((0, 2))
    n = len(counts)
    lengths = np.asarray(counts, dtype=np.int64)
    offsets = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(lengths, out=offsets[1:])
    # sort peaks by m/z inside each spectrum (stable)
    if peaks.shape[0]:
        spec = np.repeat(np.arange(n), lengths)
        idx = np.lexsort((peaks[:, 0], spec))
        peaks = peaks[idx]
    packed = pack_csr(peaks[:, 0], peaks[:, 1], offsets, n_max_peaks, mz_power, intensity_power)
    return packed, meta
