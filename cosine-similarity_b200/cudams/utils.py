"""Batching and timing helpers kept from the reference's cudams.utils.

argbatch (reference cudams/utils.py:24-35), Timer (:267-273) and CudaTimer
(:322-362, there on numba events; here on torch CUDA events of the stream the
kernels run on).
"""
from __future__ import annotations

import time
from typing import Iterable


def argbatch(lst, batch_size: int) -> Iterable[tuple[int, int]]:
    """Yield (start, start + batch_size) index pairs over `lst`."""
    for i in range(0, len(lst), batch_size):
        yield i, i + batch_size


class Timer:
    """Wall-clock context manager: `with Timer() as t: ...; t.duration` (s)."""

    def __enter__(self):
        self.duration = -time.perf_counter()
        return self

    def __exit__(self, *args):
        self.duration += time.perf_counter()


class CudaTimer:
    """Device time between start() and stop() on a CUDA stream."""

    def __init__(self, stream=None):
        import torch

        self._stream = stream
        self._start = torch.cuda.Event(enable_timing=True)
        self._stop = torch.cuda.Event(enable_timing=True)

    def start(self):
        self._start.record(self._stream)

    def stop(self):
        self._stop.record(self._stream)

    def elapsed(self) -> float:
        """Milliseconds (synchronises on the stop event)."""
        self._stop.synchronize()
        return self._start.elapsed_time(self._stop)

    def elapsed_seconds(self) -> float:
        return self.elapsed() / 1000.0
