"""Serving: a device-resident spectral library and a continuous-batching server.

The reference computes similarity matrices in one call (CudaCosineGreedy.matrix,
cudams/similarity/CudaCosineGreedy.py:107-226) and has no server.  Here the
library (the "references") is packed, uploaded and indexed once
(cms_library_create) and stays on the device; query batches are searched
against it with sparse output (pairs with score >= threshold,
cms_library_search), as the sparse branch of matrix() would return them.

Server: requests (query batches of any size) are queued as they arrive.  Each
of `slots` worker threads owns a library context and two CUDA streams (high
and low priority); a worker takes the next request as soon as it is free and
the request's estimated device memory fits in the free HBM (minus a reserve),
so requests that arrive while others are on the GPU start immediately.
Their work overlaps on the device: a search launches short-lived CTAs (each
warp takes a few work items and exits), so SM slots free up continuously and
the CTAs of searches on other streams are scheduled in between; requests of
at most `chunk` queries run on the high-priority stream, so their CTAs are
dispatched ahead of the pending CTAs of larger batches (which run
`chunk` queries at a time on the low-priority one).  Every request's result
depends only on its own queries: it is the same alone or in the mix.
"""
from __future__ import annotations

import ctypes
import queue
import threading
import time
from concurrent.futures import Future
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import _native, autotune
from ._native import CosineConfig, check, ptr, stream_handle
from .packing import PackedSpectra, pack_spectra


@dataclass
class SearchResult:
    """Hits of one query batch, sorted by (query, library index)."""

    ref: np.ndarray      # library index (int32)
    query: np.ndarray    # query index within the batch (int32)
    score: np.ndarray    # float32
    matches: np.ndarray  # int32
    overflow: np.ndarray  # uint8
    n_queries: int
    n_library: int
    latency_s: float = 0.0      # submit -> result on the host (Server), or call time
    queued_s: float = 0.0       # time spent waiting for a slot / memory
    extra: dict = field(default_factory=dict)

    @property
    def pairs(self) -> int:
        return self.n_queries * self.n_library

    def as_set(self):
        return set(zip(self.ref.tolist(), self.query.tolist(), self.score.view(np.uint32).tolist(),
                       self.matches.tolist(), self.overflow.tolist()))


class SpectrumLibrary:
    """A spectrum set resident on one device, indexed for greedy-cosine search."""

    def __init__(self, spectra, tolerance: float = 0.1, mz_power: float = 0.0,
                 intensity_power: float = 1.0, shift: float = 0.0, match_limit: int = 2048,
                 n_max_peaks: Optional[int] = 1024, device=None, config: Optional[dict] = None):
        import torch

        self.device = _native.require_cuda(device)
        self.tolerance, self.shift, self.match_limit = float(tolerance), float(shift), int(match_limit)
        self.mz_power, self.intensity_power, self.n_max_peaks = mz_power, intensity_power, n_max_peaks
        if isinstance(spectra, PackedSpectra):
            packed = spectra.truncate(n_max_peaks)
        else:
            packed = pack_spectra(spectra, n_max_peaks, mz_power, intensity_power)
        self.packed = packed
        self.n = packed.n
        self._dev = packed.to_device(self.device)
        cfg = dict(config or {})
        if "cand_per_pair" not in cfg:
            cfg["cand_per_pair"] = autotune.workload_stats(packed, packed, tolerance,
                                                           shift).cand_per_pair
        c = CosineConfig.from_dict(cfg)
        self.config = cfg
        ctx = _native.context(self.device.index)
        h = ctypes.c_void_p()
        s = torch.cuda.current_stream(self.device)
        d = self._dev
        check(_native.load().cms_library_create(
            ctx.handle, ptr(d.mz), ptr(d.a), ptr(d.b), ptr(d.offsets), d.n, d.n_peaks,
            self.tolerance, self.shift, self.match_limit, ctypes.byref(c), ctypes.byref(h),
            stream_handle(s)), "cms_library_create")
        self._handle = h

    def pack_queries(self, queries) -> PackedSpectra:
        if isinstance(queries, PackedSpectra):
            if (queries.mz_power != float(self.mz_power)
                    or queries.intensity_power != float(self.intensity_power)):
                raise ValueError("queries were packed with other mz/intensity powers")
            return queries.truncate(self.n_max_peaks)
        return pack_spectra(queries, self.n_max_peaks, self.mz_power, self.intensity_power)

    def estimate_bytes(self, q: PackedSpectra, capacity: int) -> int:
        """Device bytes one search of `q` needs beyond the library itself."""
        return int(2 * q.host_bytes() + 17 * capacity + 24 * q.n + (1 << 20))

    def search(self, queries, threshold: float = 0.7, stream=None,
               capacity: Optional[int] = None, chunk: int = 0) -> SearchResult:
        """All (library, query) pairs with score >= threshold.  Runs on `stream`
        (default: the current stream) and synchronises it.  chunk > 0 searches
        the batch `chunk` queries at a time (a long batch then shares the GPU
        with concurrent requests between chunks); results are identical."""
        t0 = time.perf_counter()
        q = self.pack_queries(queries)
        if chunk <= 0 or q.n <= chunk:
            res = self._search_once(q, threshold, stream, capacity)
        else:
            parts = [self._search_once(q.subset(c, min(q.n, c + chunk)), threshold, stream,
                                       capacity) for c in range(0, q.n, chunk)]
            offs = range(0, q.n, chunk)
            res = SearchResult(np.concatenate([p.ref for p in parts]),
                               np.concatenate([p.query + o for p, o in zip(parts, offs)]),
                               np.concatenate([p.score for p in parts]),
                               np.concatenate([p.matches for p in parts]),
                               np.concatenate([p.overflow for p in parts]), q.n, self.n)
        res.latency_s = time.perf_counter() - t0
        return res

    def _search_once(self, q: PackedSpectra, threshold: float, stream, capacity) -> SearchResult:
        import torch

        t0 = time.perf_counter()
        s = stream if stream is not None else torch.cuda.current_stream(self.device)
        with torch.cuda.stream(s):
            qd = _upload(q, self.device)
            cap = int(capacity) if capacity else max(4096, 64 * max(1, q.n))
            count = torch.zeros(1, dtype=torch.int64, device=self.device)
            ctx = _native.context(self.device.index)
            while True:
                bufs = (torch.empty(cap, dtype=torch.int32, device=self.device),
                        torch.empty(cap, dtype=torch.int32, device=self.device),
                        torch.empty(cap, dtype=torch.float32, device=self.device),
                        torch.empty(cap, dtype=torch.int32, device=self.device),
                        torch.empty(cap, dtype=torch.uint8, device=self.device))
                check(_native.load().cms_library_search(
                    ctx.handle, self._handle, ptr(qd.mz), ptr(qd.a), ptr(qd.b), ptr(qd.offsets),
                    qd.n, qd.n_peaks, float(threshold), *[ptr(b) for b in bufs], cap, ptr(count),
                    stream_handle(s)), "cms_library_search")
                bits = ctx.take_device_error(stream_handle(s))  # synchronises s
                if bits:
                    raise _native.NativeError(f"library search: device error bits {bits}",
                                              _native.CMS_ERR_DEVICE)
                n = int(count.item())
                if n <= cap:
                    break
                cap = n
            host = [b[:n].cpu().numpy() for b in bufs]
        r, qq, sc, mt, ov = host
        o = np.lexsort((r, qq))
        return SearchResult(r[o], qq[o], sc[o], mt[o], ov[o], q.n, self.n,
                            latency_s=time.perf_counter() - t0)

    def close(self):
        if getattr(self, "_handle", None):
            _native.load().cms_library_destroy(self._handle)
            self._handle = None

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass


def _upload(p: PackedSpectra, device, slot: int = 0):
    """DeviceSpectra of `p`, copied on the current stream: small arrays from
    pageable memory, large ones through the slot's pinned staging ring."""
    from . import staging
    from .packing import DeviceSpectra

    def up(x):
        if x is None:
            return None
        return staging.upload(np.ascontiguousarray(x), device, slot=slot)

    return DeviceSpectra(up(p.mz), up(p.a), up(p.b), up(p.offsets), p.n, p.n_peaks)


@dataclass
class _Request:
    queries: PackedSpectra
    threshold: float
    future: Future
    t_submit: float
    est_bytes: int
    seq: int = 0


class Server:
    """Continuous-batching search server over one SpectrumLibrary."""

    def __init__(self, library: SpectrumLibrary, threshold: float = 0.7, slots: int = 4,
                 reserve_bytes: int = 4 << 30, warmup_queries: int = 4096, chunk: int = 1024,
                 trace_capacity: int = 0):
        """slots: concurrent searches (one context and stream pair each).
        warmup_queries: each slot first searches this many copies of a library
        spectrum, so that its device scratch and pinned staging are sized for
        the largest expected batch before requests arrive (allocations
        synchronise the device and would otherwise land on request latency).
        trace_capacity > 0: every result carries extra["trace"], the device
        timing records of its work items (cms_trace_enable; tag = request
        number), for studies of how requests overlap on the device."""
        import torch

        self.library = library
        self.trace_capacity = int(trace_capacity)
        self._seq = 0
        self._seq_lock = threading.Lock()
        self.warmup_queries = int(warmup_queries)
        self.chunk = int(chunk)
        self._ready = threading.Barrier(int(slots) + 1)
        self.threshold = float(threshold)
        self.reserve_bytes = int(reserve_bytes)
        self._q: "queue.Queue[Optional[_Request]]" = queue.Queue()
        self._mem_lock = threading.Condition()
        self._in_flight_bytes = 0
        self._running = 0
        self.max_concurrent = 0
        self._closed = False
        self._workers = []
        for i in range(int(slots)):
            t = threading.Thread(target=self._worker, name=f"cudams-slot-{i}", daemon=True)
            t.start()
            self._workers.append(t)
        self._ready.wait()
        # admission budget: the HBM free once every slot holds its scratch.
        # Measured here, not per request: querying the driver on the request
        # path serialises the worker threads.
        self._budget = self._free_bytes() - self.reserve_bytes
        self._start_budget = self._budget

    # -- client side ------------------------------------------------------------
    def submit(self, queries, threshold: Optional[float] = None) -> Future:
        """Queue a query batch; the future resolves to a SearchResult."""
        if self._closed:
            raise RuntimeError("server is closed")
        t = time.perf_counter()
        q = self.library.pack_queries(queries)
        f: Future = Future()
        cap = max(4096, 64 * max(1, q.n))
        with self._seq_lock:
            self._seq += 1
            seq = self._seq
        self._q.put(_Request(q, self.threshold if threshold is None else float(threshold), f, t,
                             self.library.estimate_bytes(q, cap), seq))
        return f

    def close(self):
        self._closed = True
        for _ in self._workers:
            self._q.put(None)
        for t in self._workers:
            t.join()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- admission ----------------------------------------------------------------
    def _free_bytes(self) -> int:
        import torch

        free, _ = torch.cuda.mem_get_info(self.library.device)
        return int(free)

    def _admit(self, req: _Request) -> None:
        """Block until the request's estimated memory fits in the HBM budget
        (re-measured only when a request does not fit)."""
        with self._mem_lock:
            remeasured = False
            while True:
                if self._in_flight_bytes + req.est_bytes <= self._budget or self._running == 0:
                    self._in_flight_bytes += req.est_bytes
                    self._running += 1
                    self.max_concurrent = max(self.max_concurrent, self._running)
                    return
                if not remeasured:
                    # free memory plus what the running requests hold, but never
                    # above the budget measured at start: an admitted request
                    # may not have allocated yet, so free memory can overstate
                    # what is left, and taken at face value it admits more
                    # than fits
                    self._budget = min(self._start_budget,
                                       self._free_bytes() + self._in_flight_bytes
                                       - self.reserve_bytes)
                    remeasured = True
                    continue
                self._mem_lock.wait(timeout=0.05)

    def _release(self, req: _Request) -> None:
        with self._mem_lock:
            self._in_flight_bytes -= req.est_bytes
            self._running -= 1
            self._mem_lock.notify_all()

    def _worker(self):
        import torch

        urgent = stream = trace = None
        try:
            torch.cuda.set_device(self.library.device)
            # lower number = higher priority; out-of-range values are clamped
            urgent = torch.cuda.Stream(self.library.device, priority=-5)
            stream = torch.cuda.Stream(self.library.device, priority=0)
            if self.trace_capacity > 0:
                trace = (torch.zeros((self.trace_capacity, 4), dtype=torch.int64,
                                     device=self.library.device),
                         torch.zeros(1, dtype=torch.int64, device=self.library.device))
            if self.warmup_queries > 0:
                one = self.library.packed.subset(0, 1)
                k = self.warmup_queries
                reps = PackedSpectra(np.tile(one.mz, k), None if one.a is None else np.tile(one.a, k),
                                     np.tile(one.b, k), np.arange(k + 1, dtype=np.int64) * one.n_peaks,
                                     one.mz_power, one.intensity_power, one.n_max_peaks)
                self.library.search(reps, 1.0, stream=stream)
        finally:
            self._ready.wait()
        while True:
            req = self._q.get()
            if req is None:
                return
            t_deq = time.perf_counter()
            if req.future.set_running_or_notify_cancel() is False:
                continue
            self._admit(req)
            t_start = time.perf_counter()
            try:
                small = req.queries.n <= self.chunk
                target = urgent if small else stream
                if trace is not None:
                    ctx = _native.context(self.library.device.index)
                    with torch.cuda.stream(target):
                        trace[1].zero_()
                    ctx.trace_enable(trace[0], trace[1], req.seq)
                res = self.library.search(req.queries, req.threshold, stream=target,
                                          chunk=self.chunk)
                res.queued_s = t_start - req.t_submit
                res.latency_s = time.perf_counter() - req.t_submit
                res.extra.update(dequeue_s=t_deq - req.t_submit, admit_s=t_start - t_deq,
                                 search_s=res.latency_s - res.queued_s, seq=req.seq,
                                 priority="high" if small else "low")
                if trace is not None:
                    ctx.trace_disable()
                    n = min(int(trace[1].item()), self.trace_capacity)
                    res.extra["trace"] = trace[0][:n].cpu().numpy()
                req.future.set_result(res)
            except BaseException as e:  # noqa: BLE001 - forwarded to the caller
                req.future.set_exception(e)
            finally:
                self._release(req)
