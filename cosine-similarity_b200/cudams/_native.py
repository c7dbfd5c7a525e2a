"""ctypes binding of libcudams_b200.so (the C ABI in include/cudams_b200.h).

The library is loaded lazily from this package directory.  If it is missing,
or no sm_100 device is present, every compute call raises NativeError: there
is deliberately no CPU fallback.
"""
from __future__ import annotations

import ctypes
import threading
from ctypes import POINTER, c_double, c_float, c_int, c_int32, c_int64, c_uint32, c_void_p
from pathlib import Path

LIB_PATH = Path(__file__).resolve().with_name("libcudams_b200.so")

CMS_OK = 0
CMS_ERR_INVALID = 1
CMS_ERR_CUDA = 2
CMS_ERR_UNSUPPORTED = 3
CMS_ERR_NOMEM = 4
CMS_ERR_CAPACITY = 5
CMS_ERR_DEVICE = 6

# device error word bits (csrc/cms_internal.cuh)
DEVERR_SPECTRUM_TOO_LONG = 1
DEVERR_SPILL_OVERRUN = 2
DEVERR_BAD_OFFSETS = 4
DEVERR_PIPELINE_TIMEOUT = 8

FP_MEASURES = {"jaccard": 0, "dice": 1, "cosine": 2}

PROFILE_STAGES = 5
PROFILE_STAGE_NAMES = ["validate_norms", "order", "index", "join", "pair"]

# Every exported symbol with its ctypes signature: (restype, argtypes).
_p = c_void_p
SIGNATURES = {
    "cms_version": (c_int, []),
    "cms_last_error": (ctypes.c_char_p, []),
    "cms_create": (c_int, [POINTER(c_void_p), c_int]),
    "cms_destroy": (c_int, [_p]),
    "cms_take_device_error": (c_int, [_p, POINTER(c_uint32), _p]),
    "cms_cosine_greedy_plain": (c_int, [
        _p, _p, _p, _p, c_int64,            # reference mz, a, b, off, n
        _p, _p, _p, _p, c_int64,            # query mz, a, b, off, n
        c_double, c_double, c_int, c_int,   # tol, shift, match_limit, n_max_peaks
        _p, _p, _p, c_int64, _p]),          # score, matches, overflow, ld, stream
    "cms_cosine_greedy": (c_int, [
        _p, _p, _p, _p, _p, c_int64, c_int64,
        _p, _p, _p, _p, c_int64, c_int64,
        c_double, c_double, c_int,
        _p, _p, _p, c_int64, _p, _p]),
    "cms_cosine_greedy_sparse": (c_int, [
        _p, _p, _p, _p, _p, c_int64, c_int64,
        _p, _p, _p, _p, c_int64, c_int64,
        c_double, c_double, c_int, c_float,
        _p, _p, _p, _p, _p, c_int64, _p, _p, _p]),
    "cms_modified_cosine": (c_int, [
        _p, _p, _p, _p, _p, _p, c_int64, c_int64,   # ctx, reference mz, a, b, off, precursor
        _p, _p, _p, _p, _p, c_int64, c_int64,       # query mz, a, b, off, precursor
        c_double, c_int,
        _p, _p, _p, c_int64, _p, _p]),
    "cms_modified_cosine_sparse": (c_int, [
        _p, _p, _p, _p, _p, _p, c_int64, c_int64,
        _p, _p, _p, _p, _p, c_int64, c_int64,
        c_double, c_int, c_float,
        _p, _p, _p, _p, _p, c_int64, _p, _p, _p]),
    "cms_cosine_greedy_noalloc": (c_int, [
        _p, _p, _p, _p, c_int64, c_int64,
        _p, _p, _p, _p, c_int64, c_int64,
        c_double, c_double, c_int,
        _p, _p, _p, c_int64, _p, _p]),
    "cms_library_create": (c_int, [
        _p, _p, _p, _p, _p, c_int64, c_int64, c_double, c_double, c_int, _p,
        POINTER(c_void_p), _p]),
    "cms_library_search": (c_int, [
        _p, _p, _p, _p, _p, _p, c_int64, c_int64, c_float,
        _p, _p, _p, _p, _p, c_int64, _p, _p]),
    "cms_library_destroy": (c_int, [_p]),
    "cms_profile_enable": (c_int, [_p, c_int]),
    "cms_trace_enable": (c_int, [_p, _p, c_int64, _p, c_uint32]),
    "cms_graph_enable": (c_int, [_p, c_int]),
    "cms_profile_read": (c_int, [_p, _p, _p, c_int]),
    "cms_fingerprint": (c_int, [
        c_int, _p, _p, c_int64, _p, _p, c_int64, c_int, c_float, _p, c_int64, _p]),
    "cms_fingerprint_take_error": (c_int, [POINTER(c_uint32), _p]),
    "cms_fingerprint_arith_check": (c_int, [POINTER(ctypes.c_uint64), _p]),
    "cms_mass_match": (c_int, [_p, c_int64, _p, c_int64, c_double, c_int, _p, c_int64, _p]),
    "cms_intersect_mz": (c_int, [
        _p, _p, c_int64, c_int64, _p, _p, c_int64, c_int64, c_double, _p, c_int64, _p, _p]),
    "cms_fingerprint_symmetric": (c_int, [
        c_int, _p, _p, _p, _p, c_int64, c_int, c_float, _p, c_int64, _p]),
}


class NativeError(RuntimeError):
    """A call into libcudams_b200.so failed (message from cms_last_error)."""

    def __init__(self, msg: str, code: int = CMS_ERR_CUDA):
        super().__init__(msg)
        self.code = code


class CosineConfig(ctypes.Structure):
    """cms_cosine_config (zero fields = automatic; symmetric=1 computes i <= j only)."""

    _fields_ = [
        ("tile_spectra", c_int32),
        ("bucket_width", c_double),
        ("n_buckets", c_int32),
        ("mode", c_int32),
        ("pair_threads", c_int32),
        ("cand_per_pair", c_double),
        ("symmetric", c_int32),
        ("width_by_class", c_int32 * 17),
    ]

    @classmethod
    def from_dict(cls, config: dict) -> "CosineConfig":
        c = cls()
        for k, v in config.items():
            if k == "width_by_class":
                w = [int(x) for x in v][:17]
                c.width_by_class = (c_int32 * 17)(*(w + [0] * (17 - len(w))))
            else:
                setattr(c, k, v)
        return c


_lib = None
_lib_lock = threading.Lock()


def load() -> ctypes.CDLL:
    """Load libcudams_b200.so and declare every signature (no GPU needed)."""
    global _lib
    if _lib is not None:
        return _lib
    with _lib_lock:
        if _lib is None:
            if not LIB_PATH.exists():
                raise NativeError(
                    f"{LIB_PATH.name} is not built; run "
                    "`python cosine-similarity_b200/build_native.py` (needs nvcc)",
                    CMS_ERR_UNSUPPORTED)
            lib = ctypes.CDLL(str(LIB_PATH))
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(lib, name)
                fn.restype = res
                fn.argtypes = args
            _lib = lib
    return _lib


def last_error() -> str:
    msg = load().cms_last_error()
    return msg.decode(errors="replace") if msg else ""


def check(rc: int, what: str) -> None:
    if rc != CMS_OK:
        raise NativeError(f"{what} failed (code {rc}): {last_error()}", rc)


class Context:
    """One cms_ctx (device scratch + error word) for one device."""

    def __init__(self, device: int):
        lib = load()
        h = c_void_p()
        check(lib.cms_create(ctypes.byref(h), int(device)), "cms_create")
        self.handle = h
        self.device = int(device)

    def take_device_error(self, stream) -> int:
        bits = c_uint32(0)
        check(load().cms_take_device_error(self.handle, ctypes.byref(bits), stream),
              "cms_take_device_error")
        return int(bits.value)

    def graph_enable(self, on: bool = True) -> None:
        """Capture repeated identical cms_cosine_greedy(_sparse) calls of this
        context into CUDA graphs and replay them (cms_graph_enable)."""
        check(load().cms_graph_enable(self.handle, 1 if on else 0), "cms_graph_enable")

    def trace_enable(self, records, count, tag: int) -> None:
        """Record every join work item of this context into `records` (device
        int64 tensor [cap, 4]: tag | SM id << 32, item, start ns, end ns);
        `count` (device int64 [1]) is advanced per record (cms_trace_enable)."""
        check(load().cms_trace_enable(self.handle, c_void_p(records.data_ptr()),
                                      int(records.shape[0]), c_void_p(count.data_ptr()),
                                      int(tag) & 0xFFFFFFFF), "cms_trace_enable")

    def trace_disable(self) -> None:
        check(load().cms_trace_enable(self.handle, None, 0, None, 0), "cms_trace_enable")

    def profile_enable(self, on: bool = True) -> None:
        check(load().cms_profile_enable(self.handle, 1 if on else 0), "cms_profile_enable")

    def profile_read(self, reset: bool = True):
        """(stage_ms[5], stage_launches[5]); synchronises the recorded events."""
        import numpy as np

        ms = np.zeros(PROFILE_STAGES, np.float64)
        n = np.zeros(PROFILE_STAGES, np.int64)
        check(load().cms_profile_read(self.handle, c_void_p(ms.ctypes.data),
                                      c_void_p(n.ctypes.data), 1 if reset else 0),
              "cms_profile_read")
        return ms, n

    def close(self) -> None:
        if self.handle:
            load().cms_destroy(self.handle)
            self.handle = c_void_p()

    def __del__(self):  # pragma: no cover - interpreter shutdown order
        try:
            self.close()
        except Exception:
            pass


_ctx_local = threading.local()


def context(device: int) -> Context:
    """Per-thread, per-device context (contexts must not be shared by threads)."""
    d = getattr(_ctx_local, "ctx", None)
    if d is None:
        d = _ctx_local.ctx = {}
    if device not in d:
        d[device] = Context(device)
    return d[device]


def ptr(t) -> c_void_p:
    """Device pointer of a torch tensor (or None -> NULL)."""
    if t is None:
        return c_void_p(0)
    return c_void_p(t.data_ptr())


def stream_handle(stream) -> c_void_p:
    return c_void_p(int(stream.cuda_stream))


def require_cuda(device=None):
    """Return a torch.device on a B200, or raise (no CPU fallback).  device:
    None (the current device), an index, or a torch.device."""
    import torch

    if not torch.cuda.is_available():
        raise NativeError("no CUDA device is available; cudams has no CPU fallback",
                          CMS_ERR_UNSUPPORTED)
    if isinstance(device, torch.device):
        device = device.index
    dev = torch.device("cuda", torch.cuda.current_device() if device is None else device)
    major, _ = torch.cuda.get_device_capability(dev)
    if major != 10:
        raise NativeError(f"{torch.cuda.get_device_name(dev)} is not an sm_100 device; "
                          "libcudams_b200.so is built for sm_100a only", CMS_ERR_UNSUPPORTED)
    load()
    return dev
