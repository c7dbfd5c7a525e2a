"""Choice of the tiled kernel's shape for a workload.

Two decisions matter for cms_cosine_greedy:
  * mode: the indexed join (mode 1) wins when pairs have few candidates, the
    pair kernel over the whole matrix (mode 2) when nearly every pair has
    hundreds (dense, overflow-heavy spectra);
  * tile_spectra: the join keeps every candidate of (reference, query tile)
    in a 256-entry shared-memory pool, so the tile must be small enough that
    the pool rarely overflows, and large enough that the bucket lookups per
    reference peak are amortised over many queries.

Both follow from the expected number of candidates per pair, which is
measured here on a seeded sample of pairs with numpy (exact window counts,
no model of the m/z distribution), bucketed by peak count so that long
spectra are not under-represented.  Tuned settings can be pinned per
workload key in an on-disk cache (JSON) by `Tuner.record`, which the
benchmark's tuning pass fills with measured timings.
"""
from __future__ import annotations

import json
import os
import threading
from dataclasses import dataclass
from pathlib import Path
from typing import Optional

import numpy as np

from .packing import PackedSpectra

POOL = 256
DENSE_CANDIDATES = 48.0  # mean candidates per pair above which mode 2 is used


@dataclass
class WorkloadStats:
    cand_per_pair: float      # mean candidates per pair (sampled)
    cand_per_pair_p99: float  # 99th percentile
    mean_peaks_ref: float
    mean_peaks_qry: float


def sample_candidates(ref: PackedSpectra, qry: PackedSpectra, tolerance: float,
                      shift: float = 0.0, n_pairs: int = 512, seed: int = 0) -> np.ndarray:
    """Exact candidate counts of `n_pairs` random (ref, query) pairs."""
    rng = np.random.default_rng(seed)
    if ref.n == 0 or qry.n == 0:
        return np.zeros(0)
    ri = rng.integers(0, ref.n, n_pairs)
    qi = rng.integers(0, qry.n, n_pairs)
    counts = np.empty(n_pairs, dtype=np.int64)
    for k in range(n_pairs):
        r0, r1 = ref.offsets[ri[k]], ref.offsets[ri[k] + 1]
        q0, q1 = qry.offsets[qi[k]], qry.offsets[qi[k] + 1]
        mr = ref.mz[r0:r1].astype(np.float64)
        mq = qry.mz[q0:q1].astype(np.float64) + shift
        lo = np.searchsorted(mq, mr - tolerance, side="left")
        hi = np.searchsorted(mq, mr + tolerance, side="right")
        counts[k] = int((hi - lo).sum())
    return counts


def workload_stats(ref: PackedSpectra, qry: PackedSpectra, tolerance: float,
                   shift: float = 0.0, n_pairs: int = 512, seed: int = 0) -> WorkloadStats:
    c = sample_candidates(ref, qry, tolerance, shift, n_pairs, seed)
    return WorkloadStats(float(c.mean()) if c.size else 0.0,
                         float(np.percentile(c, 99)) if c.size else 0.0,
                         float(ref.lengths.mean()) if ref.n else 0.0,
                         float(qry.lengths.mean()) if qry.n else 0.0)


# work items (reference spectrum x query tile) wanted per launch: several per
# resident warp of the join kernel (148 SMs x 32 warps), so that small
# problems still fill the GPU
TARGET_ITEMS = 40_000


def heuristic_config(stats: WorkloadStats, n_q: int, n_ref: int = 1 << 30) -> dict:
    if stats.cand_per_pair >= DENSE_CANDIDATES:
        return {"mode": 2}
    per_pair = max(stats.cand_per_pair, 1e-4)
    # measured optimum on B200: ~70 expected candidates per (reference, tile)
    tile = int(70.0 / per_pair)
    tile = min(tile, max(32, (n_ref * n_q) // TARGET_ITEMS))
    tile = max(32, min(4096, tile))
    tile = (tile + 31) // 32 * 32
    tile = min(tile, max(32, (n_q + 31) // 32 * 32))
    return {"mode": 1, "tile_spectra": tile, "cand_per_pair": float(stats.cand_per_pair)}


class Tuner:
    """Heuristic config plus an optional on-disk cache of measured choices."""

    def __init__(self, cache_path: Optional[str] = None):
        self.cache_path = Path(cache_path or os.environ.get(
            "CUDAMS_TUNE_CACHE", Path.home() / ".cache" / "cudams_b200_tune.json"))
        self._lock = threading.Lock()
        self._cache: Optional[dict] = None

    @staticmethod
    def key(stats: WorkloadStats, gpu: str) -> str:
        # bucket the workload: log2 of candidates per pair and of mean peaks
        def b(x):
            return int(np.floor(np.log2(max(x, 1e-6))))

        return f"{gpu}|c{b(stats.cand_per_pair)}|r{b(stats.mean_peaks_ref)}|q{b(stats.mean_peaks_qry)}"

    def _load(self) -> dict:
        if self._cache is None:
            try:
                self._cache = json.loads(self.cache_path.read_text())
            except (OSError, ValueError):
                self._cache = {}
        return self._cache

    def lookup(self, stats: WorkloadStats, gpu: str, n_q: int, n_ref: int = 1 << 30) -> dict:
        with self._lock:
            hit = self._load().get(self.key(stats, gpu))
        if hit:
            cfg = dict(hit)
            if cfg.get("tile_spectra"):
                cfg["tile_spectra"] = min(cfg["tile_spectra"], max(32, n_q))
            return cfg
        return heuristic_config(stats, n_q, n_ref)

    def record(self, stats: WorkloadStats, gpu: str, config: dict) -> None:
        with self._lock:
            cache = self._load()
            cache[self.key(stats, gpu)] = dict(config)
            try:
                self.cache_path.parent.mkdir(parents=True, exist_ok=True)
                self.cache_path.write_text(json.dumps(cache, indent=1, sort_keys=True))
            except OSError:
                pass


_default = Tuner()


def choose_config(ref: PackedSpectra, qry: PackedSpectra, tolerance: float, shift: float = 0.0,
                  gpu: str = "B200") -> dict:
    stats = workload_stats(ref, qry, tolerance, shift)
    return _default.lookup(stats, gpu, qry.n, ref.n)
