"""Host side of the continuous-batching server, on CPU: the GPU work is a fake
library whose search sleeps, so that admission by memory, concurrency across
slots, result routing and error forwarding are checked without a device."""
import threading
import time

import numpy as np
import pytest


class _FakeLibrary:
    """Stands in for SpectrumLibrary: search() records how many bytes of
    admitted work overlap, sleeps, and echoes the batch size."""

    def __init__(self):
        from cudams import synthetic

        self.device = "cpu"
        self.packed = synthetic.uniform_spectra(2, seed=1)
        self._lock = threading.Lock()
        self.live_bytes = 0
        self.max_live_bytes = 0
        self.live = 0
        self.max_live = 0

    def pack_queries(self, q):
        return q

    def estimate_bytes(self, q, capacity):
        return q.n * 1000

    def search(self, q, threshold, stream=None, chunk=0):
        from cudams.serving import SearchResult

        if threshold < 0:
            raise ValueError("bad threshold")
        with self._lock:
            self.live += 1
            self.live_bytes += q.n * 1000
            self.max_live = max(self.max_live, self.live)
            self.max_live_bytes = max(self.max_live_bytes, self.live_bytes)
        time.sleep(0.02)
        with self._lock:
            self.live -= 1
            self.live_bytes -= q.n * 1000
        z = np.zeros(q.n, np.int32)
        return SearchResult(z, np.arange(q.n, dtype=np.int32), z.astype(np.float32), z,
                            z.astype(np.uint8), q.n, 2)


@pytest.fixture
def fake_cuda(monkeypatch):
    import torch

    budget = {"free": 10_000}
    monkeypatch.setattr(torch.cuda, "set_device", lambda d: None)
    monkeypatch.setattr(torch.cuda, "Stream", lambda d=None, priority=0: None)
    monkeypatch.setattr(torch.cuda, "mem_get_info", lambda d=None: (budget["free"], 1 << 40))
    return budget


def test_admission_keeps_in_flight_work_within_the_memory_budget(fake_cuda):
    from cudams import synthetic
    from cudams.serving import Server

    lib = _FakeLibrary()
    # budget 10,000 "bytes": at most two 4-query requests (4,000 each) at once,
    # although four slots are free
    with Server(lib, slots=4, reserve_bytes=0, warmup_queries=0) as srv:
        futs = [srv.submit(synthetic.uniform_spectra(4, seed=10 + i)) for i in range(12)]
        res = [f.result(timeout=30) for f in futs]
    assert [r.n_queries for r in res] == [4] * 12
    assert lib.max_live_bytes <= 10_000
    assert lib.max_live == 2
    assert all(r.latency_s >= r.queued_s >= 0 for r in res)


def test_small_requests_overlap_and_oversized_one_runs_alone(fake_cuda):
    from cudams import synthetic
    from cudams.serving import Server

    lib = _FakeLibrary()
    with Server(lib, slots=4, reserve_bytes=0, warmup_queries=0) as srv:
        small = [srv.submit(synthetic.uniform_spectra(1, seed=30 + i)) for i in range(8)]
        big = srv.submit(synthetic.uniform_spectra(20, seed=40))  # 20,000 > budget
        assert [f.result(timeout=30).n_queries for f in small] == [1] * 8
        assert big.result(timeout=30).n_queries == 20
    assert lib.max_live == 4          # four slots busy with small requests at once
    assert srv.max_concurrent == 4


def test_errors_reach_the_caller_and_the_server_keeps_serving(fake_cuda):
    from cudams import synthetic
    from cudams.serving import Server

    lib = _FakeLibrary()
    with Server(lib, slots=2, reserve_bytes=0, warmup_queries=0) as srv:
        bad = srv.submit(synthetic.uniform_spectra(2, seed=50), threshold=-1.0)
        good = srv.submit(synthetic.uniform_spectra(3, seed=51))
        with pytest.raises(ValueError, match="bad threshold"):
            bad.result(timeout=30)
        assert good.result(timeout=30).n_queries == 3
    with pytest.raises(RuntimeError, match="closed"):
        srv.submit(synthetic.uniform_spectra(1, seed=52))
