"""Host -> device uploads through a reusable pinned staging ring.

A plain `torch.from_numpy(x).to(device)` from pageable memory ran at ~11 GB/s
on the B200 hosts, and `pin_memory()` per call at ~1.4 GB/s (it allocates
pinned memory every time).  A `Stager` keeps a few pinned buffers for the life
of the process: each chunk of the source array is copied into a free buffer by
several host threads at once (numpy releases the GIL for these copies), then
sent with an asynchronous copy on the caller's stream while the next chunk is
being staged.  A buffer is reused only after the copy that read it has
finished (a CUDA event per buffer).
"""
from __future__ import annotations

import os
import threading
from concurrent.futures import ThreadPoolExecutor
from typing import Dict, Optional

import numpy as np

_TORCH_DTYPES = None
_pool: Optional[ThreadPoolExecutor] = None
_pool_lock = threading.Lock()
_stagers: Dict[str, "Stager"] = {}
_stagers_lock = threading.Lock()

# arrays below this size go through the plain path (staging would not pay)
MIN_STAGED_BYTES = 4 << 20


def _threads() -> int:
    return max(1, min(8, os.cpu_count() or 1))


def _copy_pool() -> ThreadPoolExecutor:
    global _pool
    with _pool_lock:
        if _pool is None:
            _pool = ThreadPoolExecutor(_threads(), thread_name_prefix="cudams-stage")
        return _pool


def _torch_dtype(dt: np.dtype):
    global _TORCH_DTYPES
    import torch

    if _TORCH_DTYPES is None:
        _TORCH_DTYPES = {np.dtype(np.float32): torch.float32, np.dtype(np.float64): torch.float64,
                         np.dtype(np.int64): torch.int64, np.dtype(np.int32): torch.int32,
                         np.dtype(np.uint8): torch.uint8, np.dtype(np.int16): torch.int16}
    return _TORCH_DTYPES.get(np.dtype(dt))


class Stager:
    """A pinned staging ring for uploads to one device (one upload at a time)."""

    def __init__(self, chunk_bytes: int = 16 << 20, n_buffers: int = 3):
        import torch

        self.chunk = int(chunk_bytes)
        self.bufs = [torch.empty(self.chunk, dtype=torch.uint8, pin_memory=True)
                     for _ in range(n_buffers)]
        self.views = [b.numpy() for b in self.bufs]
        self.events = [None] * n_buffers
        self.lock = threading.Lock()

    def upload(self, arr: np.ndarray, device, stream=None):
        """Device copy of `arr` (a new tensor; the copy is enqueued on `stream`,
        default the current stream of `device`)."""
        import torch

        arr = np.ascontiguousarray(arr)
        tdt = _torch_dtype(arr.dtype)
        if tdt is None or arr.nbytes < MIN_STAGED_BYTES:
            return torch.from_numpy(arr).to(device)
        stream = stream if stream is not None else torch.cuda.current_stream(device)
        src = arr.reshape(-1).view(np.uint8)
        dst = torch.empty(arr.nbytes, dtype=torch.uint8, device=device)
        pool = _copy_pool()
        parts = _threads()
        with self.lock, torch.cuda.stream(stream):
            for k, off in enumerate(range(0, src.shape[0], self.chunk)):
                b = k % len(self.bufs)
                if self.events[b] is not None:
                    self.events[b].synchronize()
                n = min(self.chunk, src.shape[0] - off)
                step = (n + parts - 1) // parts
                view, piece = self.views[b], src[off:off + n]
                list(pool.map(lambda i: np.copyto(view[i * step:min(n, (i + 1) * step)],
                                                  piece[i * step:min(n, (i + 1) * step)]),
                              range(parts)))
                dst[off:off + n].copy_(self.bufs[b][:n], non_blocking=True)
                ev = torch.cuda.Event()
                ev.record(stream)
                self.events[b] = ev
        return dst.view(tdt).reshape(arr.shape)


def stager(device, slot: int = 0) -> Stager:
    """The process-wide stager for (device, slot); create it on first use."""
    key = f"{device}/{slot}"
    with _stagers_lock:
        s = _stagers.get(key)
        if s is None:
            s = _stagers[key] = Stager()
        return s


def upload(arr: np.ndarray, device, stream=None, slot: int = 0):
    """Upload through the (device, slot) stager; see Stager.upload."""
    return stager(device, slot).upload(arr, device, stream)
