"""Choice of the tiled kernel's shape for a workload.

Two decisions matter for cms_cosine_greedy:
  * mode: the indexed join (mode 1) wins when pairs have few candidates, the
    pair kernel over the whole matrix (mode 2) when nearly every pair has
    hundreds (dense, overflow-heavy spectra);
  * tile_spectra: the join keeps every candidate of (reference, query tile)
    in a 256-entry shared-memory pool, so the tile must be small enough that
    the pool rarely overflows, and large enough that the bucket lookups per
    reference peak are amortised over many queries.

Both follow from the expected number of candidates per pair.  Its mean is
estimated at the peak level: the probability that a random reference peak
and a random query peak fall within the window (exact window counts of a
seeded peak sample against a sorted sample of query peaks, with numpy),
times the peaks per spectrum of each side.  Sampling whole pairs instead
gives a noisy mean when peak counts are heavy-tailed; the pair sample is
kept for the 99th percentile.  That estimate gives the starting point
(`heuristic_config`).

`Tuner.measure` then chooses by timed trials on the device (CUDA events, a
sample of the workload): first the tile size among neighbours of the
estimate, then, per peak-count bucket of the reference spectra (length
class = bit length of the peak count), the width of the first query
sub-range swept per candidate-pool fill (cms_cosine_config.width_by_class:
narrower ranges keep a large spectrum's candidates in the shared-memory
pool, wider ones amortise its bucket lookups over more queries).  The
winners are recorded per workload key in an on-disk cache (JSON,
`Tuner.record`) that `choose_config` consults first.
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
    cand_per_pair: float      # mean candidates per pair (peak-level estimate)
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


def mean_candidates(ref: PackedSpectra, qry: PackedSpectra, tolerance: float,
                    shift: float = 0.0, n_ref_peaks: int = 20_000, n_qry_peaks: int = 400_000,
                    seed: int = 0) -> float:
    """Mean candidates per (reference, query) pair from a peak-level sample:
    P_ref * P_qry * p / (n_ref * n_qry), p = P(|mz_q + shift - mz_r| <= tol)
    for a random reference peak and a random query peak."""
    p_r, p_q = int(ref.mz.shape[0]), int(qry.mz.shape[0])
    if ref.n == 0 or qry.n == 0 or p_r == 0 or p_q == 0:
        return 0.0
    rng = np.random.default_rng(seed)
    mr = ref.mz if p_r <= n_ref_peaks else ref.mz[rng.integers(0, p_r, n_ref_peaks)]
    mq = qry.mz if p_q <= n_qry_peaks else qry.mz[rng.integers(0, p_q, n_qry_peaks)]
    mr = mr.astype(np.float64)
    mq = np.sort(mq.astype(np.float64) + shift)
    hits = (np.searchsorted(mq, mr + tolerance, side="right")
            - np.searchsorted(mq, mr - tolerance, side="left")).sum()
    p = float(hits) / (float(mr.shape[0]) * float(mq.shape[0]))
    return p * p_r * p_q / (float(ref.n) * float(qry.n))


def workload_stats(ref: PackedSpectra, qry: PackedSpectra, tolerance: float,
                   shift: float = 0.0, n_pairs: int = 512, seed: int = 0) -> WorkloadStats:
    c = sample_candidates(ref, qry, tolerance, shift, n_pairs, seed)
    return WorkloadStats(mean_candidates(ref, qry, tolerance, shift, seed=seed),
                         float(np.percentile(c, 99)) if c.size else 0.0,
                         float(ref.lengths.mean()) if ref.n else 0.0,
                         float(qry.lengths.mean()) if qry.n else 0.0)


# work items (reference spectrum x query tile) wanted per launch: tens per
# resident warp of the join kernel (148 SMs x 24 warps), so that small
# problems still fill the GPU and the last items do not leave it idle
TARGET_ITEMS = 100_000
# expected candidates per work item: measured on B200 with lognormal spectra
# (tol 0.01, ~0.1 candidates per pair, 100k x 100k, whole query tiles) the
# time per pair falls from 7.75 ps at ~130 candidates per item (1312 queries)
# to 7.09 ps at ~200 (2048); below ~75 the per-peak bucket lookups dominate
CANDIDATES_PER_ITEM = 200.0
# largest automatic tile: the join's per-warp query counters grow with the
# tile, and above ~2300 queries three CTAs no longer fit an SM
MAX_AUTO_TILE = 2048


def heuristic_config(stats: WorkloadStats, n_q: int, n_ref: int = 1 << 30) -> dict:
    if stats.cand_per_pair >= DENSE_CANDIDATES:
        return {"mode": 2}
    per_pair = max(stats.cand_per_pair, 1e-4)
    tile = int(CANDIDATES_PER_ITEM / per_pair)
    tile = min(tile, max(32, (n_ref * n_q) // TARGET_ITEMS))
    tile = max(32, min(MAX_AUTO_TILE, tile))
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


    def measure(self, ref: PackedSpectra, qry: PackedSpectra, tolerance: float,
                shift: float = 0.0, match_limit: int = 2048, device=None, gpu: str = "B200",
                sample_ref: int = 100000, tiles_per_trial: int = 3, class_sample: int = 1024,
                reps: int = 3, record: bool = True, seed: int = 0):
        """Choose tile_spectra and width_by_class by timed trials on the device.

        Tile trials sweep (a sample of at most sample_ref of) the reference
        spectra over the first tiles_per_trial tiles of queries, so that every
        tile is swept by as many references as at full size (how often a tile
        stream is reused decides how much its first load from DRAM costs);
        tiles are ranked by time per pair.  Width trials then time, per length
        class of the references, up to class_sample spectra of that class over
        the same query tiles.  Returns (config, report); report lists every
        trial (ms on its sample) and the chosen setting per bucket."""
        import time

        import torch

        from . import _native, kernels

        dev = _native.require_cuda(device)
        t_start = time.perf_counter()
        stats = workload_stats(ref, qry, tolerance, shift)
        base = heuristic_config(stats, qry.n, ref.n)
        report = {"heuristic": dict(base), "trials": [], "buckets": {}}
        if base["mode"] == 2 or ref.n == 0 or qry.n == 0:
            report["seconds"] = time.perf_counter() - t_start
            return base, report
        rng = np.random.default_rng(seed)
        lengths = ref.lengths
        classes = np.where(lengths > 0, np.floor(np.log2(np.maximum(lengths, 1))).astype(int) + 1, 0)
        if ref.n > sample_ref:
            rs = ref.take(np.sort(rng.choice(ref.n, sample_ref, replace=False)))
        else:
            rs = ref
        rd = rs.to_device(dev)
        t0 = base["tile_spectra"]
        tiles = sorted({max(32, min(MAX_AUTO_TILE, (int(t) + 31) // 32 * 32))
                        for t in (t0 / 2, 0.75 * t0, t0, 1.5 * t0, 2 * t0)})
        nq_max = min(qry.n, tiles_per_trial * max(tiles))
        out = tuple(torch.empty((max(rs.n, class_sample), nq_max), dtype=t, device=dev)
                    for t in (torch.float32, torch.int32, torch.uint8))

        def timed(rdev, n_rows, qdev, n_q, cfg):
            o = tuple(x[:n_rows, :n_q] for x in out)
            run = lambda: kernels.cosine_greedy_dense(rdev, qdev, tolerance, shift,  # noqa: E731
                                                      match_limit, out=o, config=cfg)
            run()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(reps):
                run()
            e1.record()
            torch.cuda.synchronize()
            return e0.elapsed_time(e1) / reps

        # 1) tile size: the estimate and its neighbours (at most MAX_AUTO_TILE:
        # larger tiles cost the join a CTA per SM), tiles_per_trial tiles each
        best_tile, best_ns = t0, float("inf")
        for t in tiles:
            n_q = min(qry.n, tiles_per_trial * t)
            qs = qry.subset(0, n_q)
            ms = timed(rd, rs.n, qs.to_device(dev), n_q, dict(base, tile_spectra=t))
            ns_pair = 1e6 * ms / (rs.n * n_q)
            report["trials"].append({"tile_spectra": t, "ms": ms, "ns_per_pair": ns_pair})
            if ns_pair < best_ns:
                best_tile, best_ns = t, ns_pair
        tile = min(best_tile, max(32, qry.n))
        n_q = min(qry.n, tiles_per_trial * tile)
        qd = qry.subset(0, n_q).to_device(dev)
        # 2) first sub-range width per reference length class
        widths = [0] * 17
        for c in range(17):
            members = np.nonzero(classes == c)[0]
            if members.size < 16:
                continue
            sel = np.sort(rng.choice(members, min(members.size, class_sample), replace=False))
            sub = ref.take(sel)
            sd = sub.to_device(dev)
            options = [0] + sorted({max(32, (tile // d) // 32 * 32) for d in (1, 2, 4, 8)},
                                   reverse=True)
            res = []
            for w in options:
                wbc = [0] * 17
                wbc[c] = w
                ms = timed(sd, sub.n, qd, n_q, dict(base, tile_spectra=tile, width_by_class=wbc))
                res.append((ms, w))
                report["trials"].append({"class": c, "width": w, "ms": ms})
            ms0 = res[0][0]
            ms_best, w_best = min(res)
            # keep the estimate unless a width is measurably faster (>= 2%)
            if w_best and ms_best < 0.98 * ms0:
                widths[c] = w_best
            report["buckets"][c] = {"spectra": int(members.size),
                                    "peaks": [1 << max(c - 1, 0), (1 << c) - 1],
                                    "width": widths[c], "ms_default": ms0,
                                    "ms_chosen": min(ms0, ms_best) if widths[c] else ms0}
        cfg = dict(base, tile_spectra=tile, width_by_class=widths)
        report["seconds"] = time.perf_counter() - t_start
        if record:
            self.record(stats, gpu, cfg)
        return cfg, report


_default = Tuner()


def measure(ref: PackedSpectra, qry: PackedSpectra, tolerance: float, shift: float = 0.0,
            match_limit: int = 2048, device=None, gpu: str = "B200", **kw):
    """Timed per-bucket tuning of the default tuner (see Tuner.measure)."""
    return _default.measure(ref, qry, tolerance, shift, match_limit, device, gpu, **kw)


def choose_config(ref: PackedSpectra, qry: PackedSpectra, tolerance: float, shift: float = 0.0,
                  gpu: str = "B200") -> dict:
    stats = workload_stats(ref, qry, tolerance, shift)
    return _default.lookup(stats, gpu, qry.n, ref.n)
