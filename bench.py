"""Benchmark: batched greedy cosine, pairs/s, on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (one "step"): greedy cosine over every pair of 100k reference x 100k
query spectra (1e10 pairs) with lognormal peak counts (median 60, sigma 1.0,
clipped to [5, 1000]), m/z U(50, 2000) float32, intensities Exp(1) scaled to
max 1, tolerance 0.01, mz_power 0, intensity_power 1, match_limit 4096;
seeded synthetic data (the reference benchmarks on GNPS, which is not
available offline).  Dense outputs (score f32, matches i32, overflow u8 per
pair) are written to device buffers reused across row blocks.  Inputs are
larger than L2 (no flush needed).

Reported (one JSON line, rank 0):
  value       pairs/s with inputs resident in HBM (device time, max over ranks)
  e2e         pairs/s through the public API (CudaCosineGreedy.matrix,
              array_type="sparse") from host spectra, H2D + D2H included
  plain       pairs/s of the one-pair-per-thread kernel on a row sample
  roofline    join kernel: algorithmic bytes / its live CUDA-event duration
              vs measured HBM copy bandwidth
  cpu_baseline  the CPU oracle (C restatement, all host threads) on a row
              sample of the same workload (rank 0, N=1 only)
Multi-GPU (torchrun): each rank computes its own 100k-reference shard against
the same queries; no collective on the data path ("scaling": "weak").

--impl reference times the reference's CPU implementation of the path: the
reference is a Python/Numba package without a CPU path of its own for this
kernel, so its CPU restatement (oracle/, C + OpenMP, every host thread)
stands in, on row samples of the same workload.  The reference's own Numba
CUDA kernel (installed under baseline/_ref) is timed beside ours on the
1024 x 1024 workload (other_workloads.uniform_1k.reference_numba_kernel).

--only NAME runs one of the other workloads alone (fingerprint, symmetric,
uniform, overflow, modified, metadata) and prints its result dict: the command
profiler captures of those kernels use.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "cosine-similarity_b200"))
sys.path.insert(0, str(ROOT))

METRIC = "cosine-greedy pairs/s (batched, 1 B200, |err|<=1e-5)"
UNIT = "pairs/s"
TOL, MATCH_LIMIT, N_MAX_PEAKS = 0.01, 4096, 1024
WORKLOAD = ("batched greedy cosine 100k x 100k, lognormal peaks (median 60, sigma 1.0, "
            "clip 5-1000), m/z U(50,2000), tol 0.01, powers (0,1), match_limit 4096")
BYTES_PER_PAIR = 9
# DRAM bytes per pair of join_kernel (read + write), from an ncu capture of the
# 20k x 20k case of this workload (profiles/join_kernel_batched_cosine_20k.txt);
# traffic grows with pairs, so a full launch is scaled by its pair count.
JOIN_TRAFFIC_BYTES_PER_PAIR = 11.37
# issue activity and the long-scoreboard share of stalls in the same capture
# (quoted, not measured by a bench run)
JOIN_PROFILE = "profiles/join_kernel_batched_cosine_20k.txt (20k x 20k capture)"
JOIN_PROFILE_FIGURES = {"issue_active_pct": 38.5, "long_scoreboard_stall_pct": 40.0}


def parse():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawTextHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--spectra", dest="n", type=int, default=100_000, help="spectra per side (default 100k)")
    ap.add_argument("--seed", type=int, default=2026)
    ap.add_argument("--plain-rows", type=int, default=0, help="rows for the plain sample (0=auto)")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--config", type=str, default="", help="JSON cms_cosine_config override")
    ap.add_argument("--no-extra", action="store_true", help="skip the other workloads")
    ap.add_argument("--no-served", action="store_true", help="skip the served workload")
    ap.add_argument("--overflow-rows", type=int, default=1000,
                    help="reference rows of the overflow-stress sample (20000: the whole matrix)")
    ap.add_argument("--only", choices=["fingerprint", "symmetric", "uniform", "overflow",
                                       "modified", "metadata"],
                    default="", help="run only this one of the other workloads (for profiler "
                                     "captures) and print its result instead of the bench line")
    return ap.parse_args()


# ----------------------------------------------------------------------------
def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def make_data(args, rank):
    from cudams import synthetic

    ref = synthetic.lognormal_spectra(args.n, seed=args.seed + 1000 * (rank + 1))
    qry = synthetic.lognormal_spectra(args.n, seed=args.seed)
    return ref, qry


# ----------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clock/throttle samples (every 50 ms, timestamped).  Started
    before the warm-up so that it is sampling when the timed region begins;
    `mark_start` / `mark_end` bracket the timed region and the summary keeps
    the samples taken inside it."""

    FIELDS = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self._t = None
        self.lines = []
        self.t0 = self.t1 = None

    def mark_start(self):
        self.t0 = time.time()

    def mark_end(self):
        self.t1 = time.time()

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.time(), line.strip()))

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                self.proc.wait(timeout=5)
            if self._t is not None:
                self._t.join(timeout=5)
            self.proc.stdout.close()
            self.proc = None

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        lines = self.lines
        if self.t0 is not None and self.t1 is not None:
            # samples read inside the timed region (a sample line is read within
            # a few ms of being taken)
            inside = [x for x in lines if self.t0 <= x[0] <= self.t1]
            lines = inside or lines
        for _, ln in lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 10:
                continue
            try:
                sm.append(float(parts[2]))
                mx = max(mx, float(parts[3]))
            except ValueError:
                continue
            for n, v in zip(names, parts[6:10]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    try:
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    except (OSError, ValueError, KeyError):
        return 6650.0, "fallback"


def lane_issue_frac(dev, visits_per_s: float) -> dict:
    """Greedy-cosine lane-issue roofline: peak visits per second of a two-pointer
    sweep of every pair, sum over pairs of (n_ref + n_query), against one
    visit per lane per clock (SMs x 128 lanes x max SM clock)."""
    mhz, src = sm_max_mhz()
    peak = sm_count(dev) * 128 * mhz * 1e6
    return {"achieved_visits_per_s": visits_per_s, "peak_visits_per_s": peak,
            "frac": visits_per_s / peak, "peak_basis": f"SMs x 128 lanes x {mhz:.0f} MHz ({src})"}


def measured_bf16_tflops():
    """Dense bf16 GEMM throughput (burst) from MEASURED_PEAKS.json, else the
    pool's fallback figure."""
    try:
        d = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
        return float(d["bf16_tflops"]), "measured"
    except (OSError, ValueError, KeyError):
        return 1590.0, "fallback"


def sm_max_mhz(clock_summary=None):
    """Maximum SM clock: MEASURED_PEAKS.json's record when it has one, else the
    clocks.max.sm that nvidia-smi reported during the run."""
    try:
        d = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
        for k, v in d.items():
            if "sm" in k.lower() and "max" in k.lower() and "mhz" in k.lower():
                return float(v), "MEASURED_PEAKS.json " + k
    except (OSError, ValueError, TypeError):
        pass
    if clock_summary and clock_summary.get("sm_max_mhz"):
        return float(clock_summary["sm_max_mhz"]), "nvidia-smi clocks.max.sm"
    return 1965.0, "B200 nominal clocks.max.sm"


def sm_count(dev):
    import torch

    return int(torch.cuda.get_device_properties(dev).multi_processor_count)


# ----------------------------------------------------------------------------
def cpu_baseline(ref, qry, seconds: float):
    """CPU oracle on a row sample of the workload, all host threads."""
    from oracle import oracle

    threads = oracle.available_threads()
    rows = 4
    while True:
        sub = ref.subset(0, rows)
        t = time.perf_counter()
        oracle.cosine_greedy(sub, qry, TOL, 0.0, MATCH_LIMIT, threads=threads)
        dt = time.perf_counter() - t
        if dt >= seconds / 4 or rows >= ref.n:
            break
        rows = min(ref.n, max(rows * 2, int(rows * (seconds / 4) / max(dt, 1e-3))))
    rate = rows * qry.n / dt
    return {"value": rate, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{rows} reference rows x {qry.n} queries ({rows * qry.n} pairs), "
                      f"{dt:.1f} s, C restatement (oracle/) with OpenMP"}


def run_reference_arm(args, world, rank):
    if rank != 0:
        return
    ref, qry = make_data(args, 0)
    from oracle import oracle

    threads = oracle.available_threads()
    # size one step to ~args.cpu_seconds / (steps + warmup) of CPU work
    probe_rows = 4
    t = time.perf_counter()
    oracle.cosine_greedy(ref.subset(0, probe_rows), qry, TOL, 0.0, MATCH_LIMIT, threads=threads)
    per_row = (time.perf_counter() - t) / probe_rows
    budget = max(2.0, 120.0 / max(1, args.steps + args.warmup))
    rows = max(1, min(ref.n, int(budget / max(per_row, 1e-6))))
    for w in range(args.warmup):
        oracle.cosine_greedy(ref.subset(w * rows % ref.n, min(ref.n, w * rows % ref.n + 1)), qry,
                             TOL, 0.0, MATCH_LIMIT, threads=threads)
    times = []
    for k in range(args.steps):
        r0 = (k * rows) % max(1, ref.n - rows + 1)
        t = time.perf_counter()
        oracle.cosine_greedy(ref.subset(r0, r0 + rows), qry, TOL, 0.0, MATCH_LIMIT,
                             threads=threads)
        times.append(time.perf_counter() - t)
    total = sum(times)
    rate = rows * qry.n * args.steps / total
    sample = (f"{rows} reference rows x {qry.n} queries per step, C restatement of the "
              f"reference algorithm (oracle/, OpenMP, {threads} threads)")
    line = {"metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * total / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "impl": "reference",
            "config": {"workload": WORKLOAD, "n_ref": args.n, "n_query": args.n},
            "cpu_baseline": {"value": rate, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": sample},
            "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------
def run_ours(args, world, rank, local):
    import numpy as np
    import torch

    from cudams import _native, kernels
    from cudams.similarity import CudaCosineGreedy

    dev = _native.require_cuda(local)
    torch.cuda.set_device(dev)
    if args.only:  # one of the other workloads alone (profiler captures)
        if rank == 0:
            print(json.dumps(other_workloads(dev, args, only=args.only)), flush=True)
        return
    ref, qry = make_data(args, rank)
    cfg = json.loads(args.config) if args.config else None
    tune_report = None
    if cfg is None:
        from cudams import autotune

        # timed trials on a sample of this workload: tile, then per peak-count
        # bucket of the reference spectra the first sub-range width
        cfg, tune_report = autotune.measure(ref, qry, TOL, 0.0, MATCH_LIMIT, device=dev,
                                            record=False)
    rd, qd = ref.to_device(dev), qry.to_device(dev)
    R, Q = ref.n, qry.n
    free, _ = torch.cuda.mem_get_info(dev)
    rows = int(min(R, max(1024, (free * 0.6) // (Q * BYTES_PER_PAIR))))
    blocks = [(r0, min(R, r0 + rows)) for r0 in range(0, R, rows)]
    sub = [ref.subset(a, b).to_device(dev) if (a, b) != (0, R) else rd for a, b in blocks]
    out = (torch.empty((rows, Q), dtype=torch.float32, device=dev),
           torch.empty((rows, Q), dtype=torch.int32, device=dev),
           torch.empty((rows, Q), dtype=torch.uint8, device=dev))
    stream = torch.cuda.current_stream(dev)
    ctx = _native.context(dev.index)

    def step():
        for (a, b), s in zip(blocks, sub):
            o = tuple(t[: b - a] for t in out)
            kernels.cosine_greedy_dense(s, qd, TOL, 0.0, MATCH_LIMIT, out=o, config=cfg,
                                        stream=stream)

    clocks = ClockSampler(dev.index).__enter__()
    for _ in range(args.warmup):
        step()
    bits = ctx.take_device_error(_native.stream_handle(stream))
    if bits:
        clocks.__exit__()
        raise RuntimeError(f"device error word {bits} during warm-up")
    ctx.profile_read(reset=True)
    ctx.profile_enable(True)
    barrier(world)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    try:
        clocks.mark_start()
        e0.record(stream)
        for _ in range(args.steps):
            step()
        e1.record(stream)
        torch.cuda.synchronize()
        clocks.mark_end()
    finally:
        clocks.__exit__()
    barrier(world)
    ms = e0.elapsed_time(e1)
    stage_ms, stage_n = ctx.profile_read(reset=True)
    ctx.profile_enable(False)
    ms_max = max_over_ranks(ms, world)
    pairs_rank = R * Q * args.steps
    value = pairs_rank * world / (ms_max / 1000.0)

    # roofline of the dominant kernel (join: HBM-write bound dense output)
    names = _native.PROFILE_STAGE_NAMES
    dom = int(np.argmax(stage_ms))
    join_launches = max(1, int(stage_n[3]))
    join_ms = stage_ms[3] / join_launches
    pairs_per_launch = R * Q * args.steps / join_launches
    peaks_bytes = 12 * (ref.n_peaks / len(blocks) + qry.n_peaks)
    alg_bytes = BYTES_PER_PAIR * pairs_per_launch + peaks_bytes
    hbm, peak_kind = measured_peaks()
    achieved = alg_bytes / (join_ms / 1000.0) / 1e9
    roofline = {"bound": "hbm", "kernel": "join_kernel", "achieved": achieved, "peak": hbm,
                "unit": "GB/s", "frac": achieved / hbm,
                "traffic": JOIN_TRAFFIC_BYTES_PER_PAIR * pairs_per_launch,
                "traffic_source": "ncu dram bytes of a 20k x 20k capture, scaled by pairs",
                "peak_source": f"{peak_kind} hbm_gbs (copy)",
                "algorithmic_bytes_per_launch": alg_bytes, "launch_ms": join_ms,
                "stage_ms_per_step": {n: float(v) / args.steps for n, v in zip(names, stage_ms)},
                "dominant_stage": names[dom]}
    # the lane-issue roofline of greedy cosine: peak visits a two-pointer sweep of
    # every pair would make, sum over pairs of (n_ref + n_query) = Q * P_ref +
    # R * P_query, per second of the join, against one visit per lane per clock
    # (148 SMs x 128 lanes x max SM clock).  The indexed join skips most of that
    # work, so this is an equivalence, not a count of what the kernel executes.
    visits = (Q * ref.n_peaks + R * qry.n_peaks) * args.steps / join_launches
    clk = clocks.summary()
    mhz, mhz_src = sm_max_mhz(clk)
    n_sm = sm_count(dev)
    lane_peak = n_sm * 128 * mhz * 1e6
    roofline["lane_issue_equivalent"] = {
        "achieved_visits_per_s": visits / (join_ms / 1000.0), "peak_visits_per_s": lane_peak,
        "frac": visits / (join_ms / 1000.0) / lane_peak,
        "peak_basis": f"{n_sm} SMs (device properties) x 128 lanes x {mhz:.0f} MHz ({mhz_src})",
        "ncu_profile": {"note": "not measured by this run: figures of the committed ncu capture",
                        "source": JOIN_PROFILE, **JOIN_PROFILE_FIGURES}}
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded; stands in for GNPS)",
            "config": {"workload": WORKLOAD, "n_ref_per_rank": R, "n_query": Q,
                       "pairs_per_step_per_rank": R * Q, "row_blocks": len(blocks),
                       "tuning": cfg,
                       "tuning_measured": None if tune_report is None else {
                           "seconds": tune_report["seconds"],
                           "heuristic": tune_report["heuristic"],
                           "tile_trials_ns_per_pair": {
                               str(t["tile_spectra"]): round(t["ns_per_pair"], 6)
                               for t in tune_report["trials"] if "tile_spectra" in t},
                           "buckets": tune_report["buckets"]},
                       "l2": "inputs larger than L2 (no flush)",
                       "parallelism": f"row shards x{world}, no collective"},
            "gpu_launches": int(stage_n.sum()),
            "roofline": roofline, "clocks": clk}

    # plain comparator (same inputs, row sample)
    if not args.no_plain:
        prow = args.plain_rows or max(256, min(R, 2048))
        psub = ref.subset(0, prow).to_device(dev)
        pout = tuple(t[:prow] for t in out)
        kernels.cosine_greedy_plain(psub, qd, TOL, 0.0, MATCH_LIMIT, N_MAX_PEAKS, out=pout)
        torch.cuda.synchronize()
        p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        p0.record(stream)
        kernels.cosine_greedy_plain(psub, qd, TOL, 0.0, MATCH_LIMIT, N_MAX_PEAKS, out=pout)
        p1.record(stream)
        torch.cuda.synchronize()
        pms = p0.elapsed_time(p1)
        plain_rate = prow * Q / (pms / 1000.0)
        line["plain"] = {"value": plain_rate, "unit": UNIT,
                         "sample": f"{prow} reference rows x {Q} queries, one launch"}
        try:
            line["plain"]["reference_numba_kernel"] = time_reference_kernel(
                ref, qry, TOL, MATCH_LIMIT, N_MAX_PEAKS, 2048)
        except Exception as e:  # noqa: BLE001 - reported, not fatal
            line["plain"]["reference_numba_kernel"] = {"unavailable":
                                                       f"{type(e).__name__}: {e}"[:300]}
        line["speedup_vs_plain"] = value / world / plain_rate

    # end to end through the public API from host spectra
    if not args.no_e2e:
        k = CudaCosineGreedy(tolerance=TOL, match_limit=MATCH_LIMIT, n_max_peaks=N_MAX_PEAKS,
                             sparse_threshold=0.75, config=cfg)
        h2d = ref.host_bytes() + qry.host_bytes()
        times, hits = [], 0
        for i in range(1 + max(1, min(args.steps, 2))):
            ref._device.clear()
            qry._device.clear()
            torch.cuda.synchronize()
            t = time.perf_counter()
            sp = k.matrix(ref, qry, array_type="sparse")
            torch.cuda.synchronize()
            if i > 0:
                times.append(time.perf_counter() - t)
            hits = sp.row.shape[0] if hasattr(sp, "row") else 0
        e2e_s = max_over_ranks(statistics.median(times), world)
        e2e = R * Q * world / e2e_s
        line["e2e"] = {"value": e2e, "unit": UNIT,
                       "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(hits * 17 + 8),
                       "path": "CudaCosineGreedy.matrix(array_type='sparse', threshold 0.75)",
                       "hits": int(hits)}

    if rank == 0 and world == 1 and not args.no_cpu:
        line["cpu_baseline"] = cpu_baseline(ref, qry, args.cpu_seconds)
    del out, sub, rd, qd
    ref._device.clear()
    qry._device.clear()
    torch.cuda.empty_cache()
    if rank == 0 and not args.no_extra:
        line["other_workloads"] = other_workloads(dev, args)
    if rank == 0 and not args.no_served:
        line["served"] = served_workload(dev, args)
    if rank == 0:
        print(json.dumps(line), flush=True)


REF_SSF = ROOT / "baseline" / "_ref" / "cudams" / "similarity" / "spectrum_similarity_functions.py"


def reference_gpu_kernel():
    """The reference's own Numba kernel factory (cosine_greedy_kernel,
    spectrum_similarity_functions.py:12-278) from the unmodified install in
    baseline/_ref, or (None, reason).  Its module imports matchms only for the
    CPU helpers the kernel does not use; stand-ins fill those names."""
    import importlib.util
    import types

    if not REF_SSF.exists():
        return None, "reference not installed in baseline/_ref"
    try:
        from numba import cuda

        if not cuda.is_available():
            return None, "numba reports no CUDA device"
        for name, attrs in (("matchms", {}), ("matchms.similarity", {}),
                            ("matchms.similarity.spectrum_similarity_functions",
                             {"collect_peak_pairs": None, "score_best_matches": None})):
            if name not in sys.modules:
                m = types.ModuleType(name)
                m.__dict__.update(attrs)
                sys.modules[name] = m
        spec = importlib.util.spec_from_file_location("cudams_reference_ssf", REF_SSF)
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        return mod.cosine_greedy_kernel, ""
    except Exception as e:  # noqa: BLE001 - reported, not fatal
        return None, f"{type(e).__name__}: {str(e)[:200]}"


def time_reference_kernel(packed_r, packed_q, tol, match_limit, n_max_peaks, batch):
    """pairs/s of the reference kernel on one batch x batch launch (its own
    padded [2, B, n_max_peaks] layout, CudaCosineGreedy.py:63-87), inputs on
    the device; or {"unavailable": reason}."""
    import numpy as np
    import torch

    factory, why = reference_gpu_kernel()
    if factory is None:
        return {"unavailable": why}
    from numba import cuda

    def padded(p, n):
        spec = np.zeros((2, batch, n_max_peaks), np.float32)
        lens = np.zeros(batch, np.int32)
        for i in range(min(n, p.n)):
            a, b = p.offsets[i], min(p.offsets[i + 1], p.offsets[i] + n_max_peaks)
            spec[0, i, :b - a] = p.mz[a:b]
            spec[1, i, :b - a] = p.b[a:b]
            lens[i] = b - a
        return spec, lens

    nr, nq = min(batch, packed_r.n), min(batch, packed_q.n)
    rs, rl = padded(packed_r, nr)
    qs, ql = padded(packed_q, nq)
    dev = torch.device("cuda", torch.cuda.current_device())
    rspec = torch.from_numpy(rs).to(dev)
    qspec = torch.from_numpy(qs).to(dev)
    lens = torch.from_numpy(np.stack([rl, ql])).to(dev)
    out = torch.empty((3, batch, batch), dtype=torch.float32, device=dev)
    kern = factory(tolerance=tol, shift=0.0, mz_power=0.0, int_power=1.0,
                   match_limit=match_limit, batch_size=batch, n_max_peaks=n_max_peaks)
    args = [cuda.as_cuda_array(t) for t in (rspec, qspec, lens, out)]
    kern(*args)  # JIT compile + warm-up
    cuda.synchronize()
    t0 = time.perf_counter()
    kern(*args)
    cuda.synchronize()
    dt = time.perf_counter() - t0
    return {"pairs_per_s": nr * nq / dt, "ms": 1e3 * dt, "batch": batch,
            "sample": f"{nr} x {nq} pairs in one {batch} x {batch} launch",
            "source": "baseline/_ref (unmodified reference), numba.cuda JIT for this GPU"}


class _Peaks:
    def __init__(self, mz, intensities):
        self.mz, self.intensities = mz, intensities


class _Spectrum:
    """A matchms-like spectrum (peaks.mz / peaks.intensities, float64)."""

    def __init__(self, mz, intensities):
        self.peaks = _Peaks(mz, intensities)


def _as_spectra(packed):
    import numpy as np

    off = packed.offsets
    return [_Spectrum(packed.mz[off[i]:off[i + 1]].astype(np.float64),
                      packed.b[off[i]:off[i + 1]].astype(np.float64)) for i in range(packed.n)]


def _time_ms(fn, reps=3):
    import torch

    fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def other_workloads(dev, args, only=""):
    """The other workloads, each bounded to seconds: device-resident pairs/s.
    only: run just the named one ("fingerprint", "symmetric", "uniform",
    "overflow", "modified", "metadata")."""
    res = {}
    for name, fn in (("fingerprint", _fingerprint_workload), ("symmetric", _symmetric_workload),
                     ("uniform", _uniform_workload), ("overflow", _overflow_workload),
                     ("modified", _modified_workload), ("metadata", _metadata_workload)):
        if only in ("", name):
            res.update(fn(dev, args))
    return res


def _fingerprint_workload(dev, args):
    import numpy as np
    import torch

    from cudams import kernels, synthetic

    res = {}
    # fingerprint similarity, 100k x 100k 2048-bit, jaccard/dice/cosine
    n_fp = min(args.n, 100_000)
    bits = synthetic.fingerprints(2 * n_fp, seed=args.seed)
    rb = torch.from_numpy(bits[:n_fp]).to(dev)
    qb = torch.from_numpy(bits[n_fp:]).to(dev)
    fout = torch.empty((n_fp, n_fp), dtype=torch.float32, device=dev)
    fp = {}
    for m in ("jaccard", "dice", "cosine"):
        ms = _time_ms(lambda: kernels.fingerprint_matrix(m, rb, None, qb, None, 64, float("nan"),
                                                         out=fout))
        fp[m] = n_fp * n_fp / (ms / 1e3)
    # is_symmetric=True on one set: upper triangle + mirror copy
    ms_sym = _time_ms(lambda: kernels.fingerprint_matrix("jaccard", rb, None, rb, None, 64,
                                                         float("nan"), out=fout, symmetric=True))
    del fout
    torch.cuda.empty_cache()
    # the reference's own torch formulation (float32 GEMM + elementwise) on a 20k tile
    nt = min(20_000, n_fp)
    R = torch.from_numpy(np.unpackbits(bits[:nt].view(np.uint8), axis=1,
                                       bitorder="little")).to(dev).float()
    Q = torch.from_numpy(np.unpackbits(bits[n_fp:n_fp + nt].view(np.uint8), axis=1,
                                       bitorder="little")).to(dev).float()

    def torch_jaccard():
        inter = R @ Q.T
        u = R.sum(1, keepdim=True) + Q.sum(1, keepdim=True).T
        u -= inter
        return inter.div(u).nan_to_num()

    tms = _time_ms(torch_jaccard)
    del R, Q
    torch.cuda.empty_cache()
    # the same torch formulation on the host cores (the reference's CPU
    # fingerprint path), on a 4096 x 4096 tile
    nc = min(4096, n_fp)
    Rc = torch.from_numpy(np.unpackbits(bits[:nc].view(np.uint8), axis=1,
                                        bitorder="little")).float()
    Qc = torch.from_numpy(np.unpackbits(bits[n_fp:n_fp + nc].view(np.uint8), axis=1,
                                        bitorder="little")).float()

    def torch_cpu_jaccard():
        inter = Rc @ Qc.T
        u = Rc.sum(1, keepdim=True) + Qc.sum(1, keepdim=True).T
        u -= inter
        return inter.div(u).nan_to_num()

    torch_cpu_jaccard()
    t0 = time.perf_counter()
    torch_cpu_jaccard()
    cpu_s = time.perf_counter() - t0
    del Rc, Qc
    # tensor-core kernel: 2 ops (multiply, add) per bit per pair on 4-bit float
    # operands (kind::mxf4); the fp4 reference is four times the measured dense
    # bf16 rate (the ratio of the nominal dense figures, 9 PFLOP/s : 2.25; no
    # fp4 GEMM is measured).  Neither the tensor pipe nor HBM bounds this
    # kernel: the shared-memory traffic of the operand expansion, the tensor
    # core's operand reads and the epilogue's staging does (see profiles/).
    bf16, bf16_kind = measured_bf16_tflops()
    ops_per_pair = 2 * 32 * bits.shape[1]
    fp4_peak = 4 * bf16 * 1e12
    res["fingerprint_100k"] = {
        "workload": f"{n_fp} x {n_fp} fingerprints, 2048 bits, density U(5%,15%)",
        "pairs_per_s": fp, "unit": "pairs/s",
        "ms_per_measure": {m: n_fp * n_fp / v * 1e3 for m, v in fp.items()},
        "roofline": {"bound": "shared memory (tensor fp4 and HBM fractions below)",
                     "kernel": "fp_umma_kernel",
                     "achieved_fp4_ops_per_s": ops_per_pair * fp["jaccard"],
                     "peak_fp4_ops_per_s": fp4_peak,
                     "frac": ops_per_pair * fp["jaccard"] / fp4_peak,
                     "peak_source": f"4 x {bf16_kind} bf16_tflops (dense fp4 : bf16 = 4 : 1)",
                     "hbm_frac_output": 4 * fp["jaccard"] / (measured_peaks()[0] * 1e9),
                     # (4 R Q + 256 (R + Q)) bytes per measure over the measured copy rate
                     "hbm_frac": (4.0 * n_fp * n_fp + 256.0 * 2 * n_fp) / (n_fp * n_fp / fp["jaccard"])
                                 / (measured_peaks()[0] * 1e9)},
        "reference_torch_cuda_jaccard_pairs_per_s": nt * nt / (tms / 1e3),
        "reference_torch_sample": f"{nt} x {nt}",
        "reference_torch_cpu_jaccard_pairs_per_s": nc * nc / cpu_s,
        "reference_torch_cpu_sample": f"{nc} x {nc}, {torch.get_num_threads()} threads",
        "symmetric_jaccard_output_pairs_per_s": n_fp * n_fp / (ms_sym / 1e3)}
    return res


def _symmetric_workload(dev, args):
    import torch

    from cudams import autotune, kernels, synthetic

    res = {}
    # is_symmetric=True greedy cosine on one set of the headline distribution:
    # upper triangle + mirror copy, against the full matrix of the same set
    n_sym = min(args.n, 40_000)
    sset = synthetic.lognormal_spectra(n_sym, seed=args.seed + 5)
    s_cfg = autotune.choose_config(sset, sset, TOL)
    sd = sset.to_device(dev)
    sout = tuple(torch.empty((n_sym, n_sym), dtype=t, device=dev)
                 for t in (torch.float32, torch.int32, torch.uint8))
    ms_full = _time_ms(lambda: kernels.cosine_greedy_dense(sd, sd, TOL, 0.0, MATCH_LIMIT,
                                                            out=sout, config=s_cfg), reps=2)
    ms_half = _time_ms(lambda: kernels.cosine_greedy_dense(sd, sd, TOL, 0.0, MATCH_LIMIT,
                                                            out=sout,
                                                            config=dict(s_cfg, symmetric=1)),
                       reps=2)
    res["symmetric_cosine_40k"] = {
        "workload": f"{n_sym} x {n_sym}, one set (lognormal peaks, tol 0.01), is_symmetric",
        "full_output_pairs_per_s": n_sym * n_sym / (ms_full / 1e3),
        "symmetric_output_pairs_per_s": n_sym * n_sym / (ms_half / 1e3),
        "full_ms": ms_full, "symmetric_ms": ms_half}
    del sout, sd
    sset._device.clear()
    torch.cuda.empty_cache()
    return res


def _uniform_workload(dev, args):
    import torch

    from cudams import autotune, kernels, synthetic

    res = {}
    # 1024 x 1024 uniform spectra, tol 0.1 (the reference's CPU-runnable case)
    u_r = synthetic.uniform_spectra(1024, seed=args.seed + 1).to_device(dev)
    u_q = synthetic.uniform_spectra(1024, seed=args.seed + 2).to_device(dev)
    u_cfg = autotune.choose_config(synthetic.uniform_spectra(1024, seed=args.seed + 1),
                                   synthetic.uniform_spectra(1024, seed=args.seed + 2), 0.1)
    u_out = tuple(torch.empty((1024, 1024), dtype=t, device=dev)
                  for t in (torch.float32, torch.int32, torch.uint8))
    ms_t = _time_ms(lambda: kernels.cosine_greedy_dense(u_r, u_q, 0.1, 0.0, 2048, out=u_out,
                                                        config=u_cfg), reps=20)
    # the same call replayed from a captured CUDA graph (cms_graph_enable)
    from cudams import _native as _nat

    gctx = _nat.context(dev.index)
    gctx.graph_enable(True)
    try:
        ms_g = _time_ms(lambda: kernels.cosine_greedy_dense(u_r, u_q, 0.1, 0.0, 2048, out=u_out,
                                                            config=u_cfg), reps=20)
    finally:
        gctx.graph_enable(False)
    ms_p = _time_ms(lambda: kernels.cosine_greedy_plain(u_r, u_q, 0.1, 0.0, 2048, 1024))
    # end to end from matchms-like Spectrum objects, as the reference's
    # published timings are taken: per-spectrum packing, H2D, kernels, D2H of
    # the dense [3, 1024, 1024] result into a structured array
    from cudams.similarity import CudaCosineGreedy

    sr = _as_spectra(synthetic.uniform_spectra(1024, seed=args.seed + 1))
    sq = _as_spectra(synthetic.uniform_spectra(1024, seed=args.seed + 2))
    cg = CudaCosineGreedy(tolerance=0.1, match_limit=2048)
    cg.matrix(sr, sq)
    e2e_s = []
    for _ in range(5):
        t0 = time.perf_counter()
        cg.matrix(sr, sq)
        e2e_s.append(time.perf_counter() - t0)
    try:
        ref_k = time_reference_kernel(synthetic.uniform_spectra(1024, seed=args.seed + 1),
                                      synthetic.uniform_spectra(1024, seed=args.seed + 2), 0.1,
                                      2048, 1024, 1024)
    except Exception as e:  # noqa: BLE001 - reported, not fatal
        ref_k = {"unavailable": f"{type(e).__name__}: {e}"[:300]}
    u_visits = 1024.0 * (u_r.n_peaks + u_q.n_peaks)  # sum over pairs of (n_ref + n_query)
    res["uniform_1k"] = {"workload": "1024 x 1024, peaks U{10..200}, tol 0.1, match_limit 2048",
                         "tiled_pairs_per_s": 1024 * 1024 / (ms_t / 1e3),
                         "lane_issue_equivalent": lane_issue_frac(dev, u_visits / (ms_t / 1e3)),
                         "tiled_graph_pairs_per_s": 1024 * 1024 / (ms_g / 1e3),
                         "plain_pairs_per_s": 1024 * 1024 / (ms_p / 1e3),
                         "reference_numba_kernel": ref_k, "tiled_ms": ms_t,
                         "tiled_graph_ms": ms_g, "tuning": u_cfg,
                         "e2e_from_spectrum_objects": {
                             "pairs_per_s": 1024 * 1024 / statistics.median(e2e_s),
                             "ms": 1e3 * statistics.median(e2e_s),
                             "path": "CudaCosineGreedy.matrix(list of Spectrum objects) -> "
                                     "numpy structured array (packing + H2D + kernels + D2H)"}}

    return res


def _modified_workload(dev, args):
    """Modified cosine (matchms ModifiedCosine) on 20k x 20k analogue families
    (shared peaks shifted by precursor differences), beside greedy cosine on
    the same spectra."""
    import torch

    from cudams import autotune, kernels, synthetic

    n = min(args.n, 20_000)
    r, rp = synthetic.analog_spectra(n, seed=args.seed + 20)
    q, qp = synthetic.analog_spectra(n, seed=args.seed + 21)
    cfg = autotune.choose_config(r, q, TOL)
    mcfg = dict(cfg)
    if mcfg.get("cand_per_pair"):  # the shifted pass adds about as many again
        mcfg["cand_per_pair"] = 2.0 * mcfg["cand_per_pair"]
        mcfg["tile_spectra"] = max(32, (mcfg.get("tile_spectra", 64) // 2 + 31) // 32 * 32)
    rd, qd = r.to_device(dev), q.to_device(dev)
    rpd, qpd = torch.from_numpy(rp).to(dev), torch.from_numpy(qp).to(dev)
    out = tuple(torch.empty((n, n), dtype=t, device=dev)
                for t in (torch.float32, torch.int32, torch.uint8))
    ms_m = _time_ms(lambda: kernels.modified_cosine_dense(rd, rpd, qd, qpd, TOL, 2048, out=out,
                                                          config=mcfg))
    ms_c = _time_ms(lambda: kernels.cosine_greedy_dense(rd, qd, TOL, 0.0, 2048, out=out,
                                                        config=cfg))
    del out
    torch.cuda.empty_cache()
    return {"modified_cosine_20k": {
        "workload": f"{n} x {n} analogue families (8 per family, precursor shifts U(-40, 40)), "
                    f"tol {TOL}, match_limit 2048",
        "modified_pairs_per_s": n * n / (ms_m / 1e3), "modified_ms": ms_m,
        "greedy_cosine_pairs_per_s_same_spectra": n * n / (ms_c / 1e3),
        "tuning": mcfg}}


def _metadata_workload(dev, args):
    """matchms PrecursorMzMatch (Dalton and ppm) on 100k x 100k precursor
    values (one byte per pair: output bandwidth) and IntersectMz on 20k x 20k
    lognormal spectra with m/z rounded to 0.01 (so that exact matches occur)."""
    import numpy as np
    import torch

    from cudams import kernels, synthetic

    n = min(args.n, 100_000)
    rng = np.random.default_rng(args.seed + 30)
    rv = torch.from_numpy(rng.uniform(100.0, 1500.0, n)).to(dev)
    qv = torch.from_numpy(rng.uniform(100.0, 1500.0, n)).to(dev)
    out = torch.empty((n, n), dtype=torch.uint8, device=dev)
    ms_d = _time_ms(lambda: kernels.mass_match_matrix(rv, qv, 0.1, False, out=out))
    ms_p = _time_ms(lambda: kernels.mass_match_matrix(rv, qv, 20.0, True, out=out))
    del out
    torch.cuda.empty_cache()
    m = min(args.n, 20_000)
    sr = synthetic.lognormal_spectra(m, seed=args.seed + 31)
    sq = synthetic.lognormal_spectra(m, seed=args.seed + 32)

    def csr(s):
        return (torch.from_numpy(np.round(s.mz.astype(np.float64), 2)).to(dev),
                torch.from_numpy(s.offsets.astype(np.int64)).to(dev))

    ix_out = torch.empty((m, m), dtype=torch.float64, device=dev)
    (rm, ro), (qm, qo) = csr(sr), csr(sq)
    ms_i = _time_ms(lambda: kernels.intersect_mz_matrix(rm, ro, qm, qo, 1.0, out=ix_out))
    del ix_out
    torch.cuda.empty_cache()
    peak = measured_peaks()[0] * 1e9
    return {"metadata_similarities": {
        "workload": f"PrecursorMzMatch {n} x {n} (tolerance 0.1 Da / 20 ppm); IntersectMz "
                    f"{m} x {m} lognormal spectra, m/z rounded to 0.01",
        "precursor_match_dalton_pairs_per_s": n * n / (ms_d / 1e3),
        "precursor_match_ppm_pairs_per_s": n * n / (ms_p / 1e3),
        "precursor_match_hbm_frac": n * n / (ms_d / 1e3) / peak,
        "intersect_mz_pairs_per_s": m * m / (ms_i / 1e3),
        "intersect_mz_ms": ms_i}}


def _overflow_workload(dev, args):
    import torch

    from cudams import autotune, kernels, synthetic

    res = {}
    # overflow stress: clustered dense spectra, 20k x 20k, nearly every pair overflows
    c_r = synthetic.clustered_spectra(20_000, seed=args.seed + 3)
    c_q = synthetic.clustered_spectra(20_000, seed=args.seed + 4)
    cfg = autotune.choose_config(c_r, c_q, 0.05)
    rows = max(1, min(c_r.n, args.overflow_rows))
    cr_sub = c_r.subset(0, rows).to_device(dev)
    cq = c_q.to_device(dev)
    cout = tuple(torch.empty((rows, c_q.n), dtype=t, device=dev)
                 for t in (torch.float32, torch.int32, torch.uint8))
    ms_o = _time_ms(lambda: kernels.cosine_greedy_dense(cr_sub, cq, 0.05, 0.0, 1024, out=cout,
                                                         config=cfg), reps=1)
    ovf = float(cout[2].float().mean().item())
    prow = 64
    cr_p = c_r.subset(0, prow).to_device(dev)
    pout = tuple(t[:prow] for t in cout)
    ms_pl = _time_ms(lambda: kernels.cosine_greedy_plain(cr_p, cq, 0.05, 0.0, 1024, 2048,
                                                          out=pout), reps=1)
    res["overflow_stress_20k"] = {
        "workload": "20k x 20k clustered (200 centres, sigma 0.02), 1000-2000 peaks, tol 0.05, "
                    "powers (3, 0.6), match_limit 1024",
        "tiled_pairs_per_s": rows * c_q.n / (ms_o / 1e3), "tiled_sample": f"{rows} x {c_q.n}",
        "lane_issue_equivalent": lane_issue_frac(
            dev, (c_q.n * float(c_r.lengths[:rows].sum()) + rows * float(c_q.n_peaks)) / (ms_o / 1e3)),
        "plain_pairs_per_s": prow * c_q.n / (ms_pl / 1e3), "plain_sample": f"{prow} x {c_q.n}",
        "overflow_fraction": ovf, "tuning": cfg}
    return res


def _offered_load(srv, pool, rng, rate_1k: float, rate_bg: float, seconds: float):
    """Poisson arrivals for `seconds`: 1000-query batches at rate_1k/s plus
    background batches of log-uniform size in [1, 4096] at rate_bg/s."""
    import numpy as np

    futs, kinds = [], []
    t0 = time.perf_counter()
    nxt1 = t0 + rng.exponential(1 / rate_1k)
    nxt2 = t0 + (rng.exponential(1 / rate_bg) if rate_bg > 0 else float("inf"))
    off = 0
    while True:
        now = time.perf_counter()
        if now - t0 >= seconds:
            break
        if now >= nxt1:
            futs.append(srv.submit(pool.subset(off % 59000, off % 59000 + 1000)))
            kinds.append(1000)
            off += 1000
            nxt1 += rng.exponential(1 / rate_1k)
        if now >= nxt2:
            k = int(np.exp(rng.uniform(0.0, np.log(4096.0))))
            futs.append(srv.submit(pool.subset(off % 55000, off % 55000 + k)))
            kinds.append(k)
            off += k
            nxt2 += rng.exponential(1 / rate_bg)
        time.sleep(max(0.0, min(nxt1, nxt2) - time.perf_counter() - 2e-4))
    res = [f.result() for f in futs]
    elapsed = time.perf_counter() - t0
    lat_1k = np.array([r.latency_s for r, k in zip(res, kinds) if k == 1000]) * 1e3
    lat = np.array([r.latency_s for r in res]) * 1e3
    return {"offered_1k_per_s": rate_1k, "offered_background_per_s": rate_bg,
            "seconds": seconds, "requests": len(res), "requests_1k": int(lat_1k.size),
            "p50_ms_1k": float(np.percentile(lat_1k, 50)),
            "p99_ms_1k": float(np.percentile(lat_1k, 99)),
            "p99_ms_all": float(np.percentile(lat, 99)),
            "pairs_per_s": sum(r.pairs for r in res) / elapsed,
            "hits": int(sum(r.ref.shape[0] for r in res))}


def _saturated(srv, pool, clients: int, seconds: float):
    """Closed loop: `clients` threads each submit a 1000-query batch as soon as
    their previous one returns, for `seconds`."""
    import numpy as np

    lats, pairs = [], [0]
    lock = threading.Lock()
    t_end = time.perf_counter() + seconds

    def client(i):
        off = 1000 * i
        while time.perf_counter() < t_end:
            r = srv.submit(pool.subset(off % 59000, off % 59000 + 1000)).result()
            off += 1000 * clients
            with lock:
                lats.append(r.latency_s * 1e3)
                pairs[0] += r.pairs

    t0 = time.perf_counter()
    ts = [threading.Thread(target=client, args=(i,)) for i in range(clients)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    elapsed = time.perf_counter() - t0
    return {"clients": clients, "seconds": seconds, "requests": len(lats),
            "pairs_per_s": pairs[0] / elapsed, "p50_ms_1k": float(np.percentile(lats, 50)),
            "p99_ms_1k": float(np.percentile(lats, 99))}


def served_workload(dev, args, library_size: int = 1_000_000):
    """Resident 1M-spectrum library, sparse output of scores >= 0.7: latency of
    one 1000-query batch alone; p50/p99 under two Poisson offered loads
    (1000-query batches plus log-uniform [1, 4096]-query background batches);
    saturated throughput from closed-loop clients."""
    import numpy as np
    import torch

    from cudams import synthetic
    from cudams.serving import Server, SpectrumLibrary

    libp = synthetic.lognormal_spectra(library_size, seed=args.seed + 10)
    t = time.perf_counter()
    lib = SpectrumLibrary(libp, tolerance=TOL, match_limit=MATCH_LIMIT, n_max_peaks=N_MAX_PEAKS)
    torch.cuda.synchronize()
    build_s = time.perf_counter() - t
    pool = synthetic.lognormal_spectra(60_000, seed=args.seed + 11)
    rng = np.random.default_rng(args.seed + 12)
    alone = []
    for i in range(5):
        alone.append(lib.search(pool.subset(1000 * i, 1000 * (i + 1)), 0.7).latency_s)
    try:
        with Server(lib, threshold=0.7, slots=4) as srv:
            loads = [_offered_load(srv, pool, rng, r1, 20.0, 10.0) for r1 in (20.0, 60.0)]
            sat = _saturated(srv, pool, clients=8, seconds=8.0)
            concurrent = srv.max_concurrent
    finally:
        lib.close()
    base = loads[0]
    return {
        "workload": f"resident library of {library_size} lognormal spectra, tol {TOL}, "
                    f"match_limit {MATCH_LIMIT}; sparse output score >= 0.7; 4 slots; "
                    "offered loads: Poisson 1000-query batches at 20/s or 60/s plus "
                    "log-uniform [1, 4096]-query batches at 20/s, 10 s each; saturated: 8 "
                    "closed-loop clients of 1000-query batches, 8 s",
        "library_build_s": build_s,
        "latency_1k_alone_ms": float(1e3 * np.median(alone)),
        "p50_ms_1k": base["p50_ms_1k"], "p99_ms_1k": base["p99_ms_1k"],
        "offered_loads": loads, "saturated": sat,
        "pairs_per_s": base["pairs_per_s"], "max_concurrent_requests": concurrent}


def main():
    args = parse()
    world, rank, local = dist_setup(args)
    try:
        if args.impl == "reference":
            run_reference_arm(args, world, rank)
        else:
            run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
