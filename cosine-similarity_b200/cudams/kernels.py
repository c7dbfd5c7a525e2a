"""Device calls: torch tensors as buffers, libcudams_b200.so for the compute.

These functions are the only place that hands device pointers to the C ABI.
They enqueue work on the current (or given) torch CUDA stream and return
device tensors; `check=True` synchronises the stream and raises if a kernel
reported bad input through the context's error word.
"""
from __future__ import annotations

import ctypes
from typing import Optional

import torch

from . import _native
from ._native import CosineConfig, NativeError, check, ptr, stream_handle
from .packing import DeviceSpectra


def _cfg(config: Optional[dict]):
    if not config:
        return None
    return CosineConfig.from_dict(config)


def _stream(device, stream):
    return stream if stream is not None else torch.cuda.current_stream(device)


def _raise_device_error(bits: int, what: str) -> None:
    if not bits:
        return
    parts = []
    if bits & _native.DEVERR_SPECTRUM_TOO_LONG:
        parts.append("a spectrum has more than 65535 peaks")
    if bits & _native.DEVERR_BAD_OFFSETS:
        parts.append("spectrum offsets are not non-decreasing within the peak arrays")
    if bits & _native.DEVERR_SPILL_OVERRUN:
        parts.append("spill list overrun")
    if bits & _native.DEVERR_PIPELINE_TIMEOUT:
        parts.append("a bounded wait between the pair kernel's warps ran out")
    raise NativeError(f"{what}: device reported an error ({'; '.join(parts)})",
                      _native.CMS_ERR_DEVICE)


def take_device_error(device, stream=None) -> int:
    s = _stream(device, stream)
    return _native.context(device.index).take_device_error(stream_handle(s))


def cosine_greedy_dense(ref: DeviceSpectra, qry: DeviceSpectra, tolerance: float, shift: float,
                        match_limit: int, *, out=None, config: Optional[dict] = None,
                        stream=None, check_errors: bool = False):
    """Greedy cosine for all pairs -> (score f32, matches i32, overflow u8) [n_ref, n_q]."""
    lib = _native.load()
    device = ref.mz.device if ref.mz is not None else qry.mz.device
    s = _stream(device, stream)
    if out is None:
        out = (torch.empty((ref.n, qry.n), dtype=torch.float32, device=device),
               torch.empty((ref.n, qry.n), dtype=torch.int32, device=device),
               torch.empty((ref.n, qry.n), dtype=torch.uint8, device=device))
    score, matches, overflow = out
    ld = score.stride(0) if score.dim() == 2 else qry.n
    ctx = _native.context(device.index)
    cfg = _cfg(config)
    rc = lib.cms_cosine_greedy(
        ctx.handle, ptr(ref.mz), ptr(ref.a), ptr(ref.b), ptr(ref.offsets), ref.n, ref.n_peaks,
        ptr(qry.mz), ptr(qry.a), ptr(qry.b), ptr(qry.offsets), qry.n, qry.n_peaks,
        float(tolerance), float(shift), int(match_limit), ptr(score), ptr(matches),
        ptr(overflow), int(ld), None if cfg is None else _ctypes_ref(cfg), stream_handle(s))
    check(rc, "cms_cosine_greedy")
    if check_errors:
        bits = ctx.take_device_error(stream_handle(s))
        if bits & _native.DEVERR_SPILL_OVERRUN and not (config or {}).get("mode") == 2:
            # rare: too many long-candidate pairs for the spill list; redo with
            # the pair kernel over the whole matrix
            cfg2 = dict(config or {})
            cfg2["mode"] = 2
            return cosine_greedy_dense(ref, qry, tolerance, shift, match_limit, out=out,
                                       config=cfg2, stream=stream, check_errors=True)
        _raise_device_error(bits, "cms_cosine_greedy")
    return score, matches, overflow


def _ctypes_ref(obj):
    import ctypes

    return ctypes.byref(obj)


def cosine_greedy_plain(ref: DeviceSpectra, qry: DeviceSpectra, tolerance: float, shift: float,
                        match_limit: int, n_max_peaks: int, *, out=None, stream=None):
    """The plain one-pair-per-thread kernel (benchmark comparator)."""
    lib = _native.load()
    device = ref.mz.device
    s = _stream(device, stream)
    if out is None:
        out = (torch.empty((ref.n, qry.n), dtype=torch.float32, device=device),
               torch.empty((ref.n, qry.n), dtype=torch.int32, device=device),
               torch.empty((ref.n, qry.n), dtype=torch.uint8, device=device))
    score, matches, overflow = out
    ld = score.stride(0)
    rc = lib.cms_cosine_greedy_plain(
        ptr(ref.mz), ptr(ref.a), ptr(ref.b), ptr(ref.offsets), ref.n,
        ptr(qry.mz), ptr(qry.a), ptr(qry.b), ptr(qry.offsets), qry.n,
        float(tolerance), float(shift), int(match_limit), int(n_max_peaks),
        ptr(score), ptr(matches), ptr(overflow), int(ld), stream_handle(s))
    check(rc, "cms_cosine_greedy_plain")
    return score, matches, overflow


class SparseHits:
    """Device hit arrays of one sparse call (the first `count` entries are valid)."""

    def __init__(self, r, q, score, matches, overflow, count):
        self.r, self.q, self.score, self.matches, self.overflow = r, q, score, matches, overflow
        self.count = count

    def to_host(self, sort: bool = True):
        import numpy as np

        n = int(self.count)
        r = self.r[:n].cpu().numpy()
        q = self.q[:n].cpu().numpy()
        sc = self.score[:n].cpu().numpy()
        mt = self.matches[:n].cpu().numpy()
        ov = self.overflow[:n].cpu().numpy()
        if sort and n:
            o = np.lexsort((q, r))
            r, q, sc, mt, ov = r[o], q[o], sc[o], mt[o], ov[o]
        return r, q, sc, mt, ov


def cosine_greedy_sparse(ref: DeviceSpectra, qry: DeviceSpectra, tolerance: float, shift: float,
                         match_limit: int, threshold: float, *, capacity: Optional[int] = None,
                         config: Optional[dict] = None, stream=None) -> SparseHits:
    """Pairs with score >= threshold (> 0).  Synchronises the stream (it must
    read the hit count) and grows the hit buffers until every hit fits."""
    lib = _native.load()
    device = ref.mz.device if ref.mz is not None else qry.mz.device
    s = _stream(device, stream)
    ctx = _native.context(device.index)
    cap = int(capacity) if capacity else max(1024, min(ref.n * qry.n, 1 << 22))
    count = torch.zeros(1, dtype=torch.int64, device=device)
    cfg = _cfg(config)
    while True:
        bufs = (torch.empty(cap, dtype=torch.int32, device=device),
                torch.empty(cap, dtype=torch.int32, device=device),
                torch.empty(cap, dtype=torch.float32, device=device),
                torch.empty(cap, dtype=torch.int32, device=device),
                torch.empty(cap, dtype=torch.uint8, device=device))
        rc = lib.cms_cosine_greedy_sparse(
            ctx.handle, ptr(ref.mz), ptr(ref.a), ptr(ref.b), ptr(ref.offsets), ref.n, ref.n_peaks,
            ptr(qry.mz), ptr(qry.a), ptr(qry.b), ptr(qry.offsets), qry.n, qry.n_peaks,
            float(tolerance), float(shift), int(match_limit), float(threshold),
            *[ptr(b) for b in bufs], cap, ptr(count),
            None if cfg is None else _ctypes_ref(cfg), stream_handle(s))
        check(rc, "cms_cosine_greedy_sparse")
        bits = ctx.take_device_error(stream_handle(s))  # synchronises s
        if bits & _native.DEVERR_SPILL_OVERRUN and not (config or {}).get("mode") == 2:
            config = dict(config or {})
            config["mode"] = 2
            cfg = _cfg(config)
            continue
        _raise_device_error(bits, "cms_cosine_greedy_sparse")
        n = int(count.item())
        if n <= cap:
            return SparseHits(*bufs, n)
        cap = n


def fingerprint_error(stream=None, device=None) -> int:
    """Read and clear the fingerprint kernels' error bits (synchronises)."""
    lib = _native.load()
    s = _stream(device or torch.device("cuda", torch.cuda.current_device()), stream)
    bits = ctypes.c_uint32(0)
    check(lib.cms_fingerprint_take_error(ctypes.byref(bits), stream_handle(s)),
          "cms_fingerprint_take_error")
    return int(bits.value)


def fingerprint_matrix(measure: str, r_bits, r_valid, q_bits, q_valid, n_words: int, fill: float,
                       *, out=None, stream=None, symmetric: bool = False,
                       check_errors: bool = False):
    """Fingerprint similarity [n_ref, n_q] float32 on the device.

    symmetric: n_ref == n_q; only pairs (i, j) with i <= j are computed and
    (j, i) gets the same value (matchms is_symmetric=True).
    check_errors: synchronise and raise NativeError if a kernel reported a
    pipeline timeout."""
    out = _fingerprint_matrix(measure, r_bits, r_valid, q_bits, q_valid, n_words, fill, out=out,
                              stream=stream, symmetric=symmetric)
    if check_errors:
        bits = fingerprint_error(stream, r_bits.device)
        if bits:
            raise _native.NativeError(f"fingerprint kernel error bits {bits:#x} (pipeline timeout)")
    return out


def _fingerprint_matrix(measure: str, r_bits, r_valid, q_bits, q_valid, n_words: int, fill: float,
                        *, out=None, stream=None, symmetric: bool = False):
    lib = _native.load()
    device = r_bits.device
    s = _stream(device, stream)
    n_r, n_q = int(r_bits.shape[0]), int(q_bits.shape[0])
    if symmetric and n_r != n_q:
        raise ValueError(f"symmetric fingerprint matrix needs n_ref == n_q ({n_r} != {n_q})")
    if out is None:
        out = torch.empty((n_r, n_q), dtype=torch.float32, device=device)
    if symmetric:
        rc = lib.cms_fingerprint_symmetric(_native.FP_MEASURES[measure], ptr(r_bits),
                                           ptr(r_valid), ptr(q_bits), ptr(q_valid), n_r,
                                           int(n_words), float(fill), ptr(out),
                                           int(out.stride(0)), stream_handle(s))
        check(rc, "cms_fingerprint_symmetric")
        return out
    rc = lib.cms_fingerprint(_native.FP_MEASURES[measure], ptr(r_bits), ptr(r_valid), n_r,
                             ptr(q_bits), ptr(q_valid), n_q, int(n_words), float(fill), ptr(out),
                             int(out.stride(0)), stream_handle(s))
    check(rc, "cms_fingerprint")
    return out


def modified_cosine_dense(ref: DeviceSpectra, ref_precursor, qry: DeviceSpectra, qry_precursor,
                          tolerance: float, match_limit: int, *, out=None,
                          config: Optional[dict] = None, stream=None,
                          check_errors: bool = False):
    """Modified cosine for all pairs -> (score f32, matches i32, overflow u8)
    [n_ref, n_q]; *_precursor are device float64 tensors, one per spectrum."""
    lib = _native.load()
    device = ref.mz.device if ref.mz is not None else qry.mz.device
    s = _stream(device, stream)
    if out is None:
        out = (torch.empty((ref.n, qry.n), dtype=torch.float32, device=device),
               torch.empty((ref.n, qry.n), dtype=torch.int32, device=device),
               torch.empty((ref.n, qry.n), dtype=torch.uint8, device=device))
    score, matches, overflow = out
    ld = score.stride(0) if score.dim() == 2 else qry.n
    ctx = _native.context(device.index)
    cfg = _cfg(config)
    rc = lib.cms_modified_cosine(
        ctx.handle, ptr(ref.mz), ptr(ref.a), ptr(ref.b), ptr(ref.offsets), ptr(ref_precursor),
        ref.n, ref.n_peaks, ptr(qry.mz), ptr(qry.a), ptr(qry.b), ptr(qry.offsets),
        ptr(qry_precursor), qry.n, qry.n_peaks, float(tolerance), int(match_limit), ptr(score),
        ptr(matches), ptr(overflow), int(ld), None if cfg is None else _ctypes_ref(cfg),
        stream_handle(s))
    check(rc, "cms_modified_cosine")
    if check_errors:
        bits = ctx.take_device_error(stream_handle(s))
        if bits & _native.DEVERR_SPILL_OVERRUN and not (config or {}).get("mode") == 2:
            return modified_cosine_dense(ref, ref_precursor, qry, qry_precursor, tolerance,
                                         match_limit, out=out, config=dict(config or {}, mode=2),
                                         stream=stream, check_errors=True)
        if bits & _native.DEVERR_SPECTRUM_TOO_LONG:
            raise NativeError("cms_modified_cosine: a spectrum has more than 32767 peaks",
                              _native.CMS_ERR_DEVICE)
        _raise_device_error(bits, "cms_modified_cosine")
    return score, matches, overflow


def modified_cosine_sparse(ref: DeviceSpectra, ref_precursor, qry: DeviceSpectra, qry_precursor,
                           tolerance: float, match_limit: int, threshold: float, *,
                           capacity: Optional[int] = None, config: Optional[dict] = None,
                           stream=None) -> SparseHits:
    """Modified-cosine pairs with score >= threshold (> 0); synchronises."""
    lib = _native.load()
    device = ref.mz.device if ref.mz is not None else qry.mz.device
    s = _stream(device, stream)
    ctx = _native.context(device.index)
    cap = int(capacity) if capacity else max(1024, min(ref.n * qry.n, 1 << 22))
    count = torch.zeros(1, dtype=torch.int64, device=device)
    while True:
        cfg = _cfg(config)
        bufs = (torch.empty(cap, dtype=torch.int32, device=device),
                torch.empty(cap, dtype=torch.int32, device=device),
                torch.empty(cap, dtype=torch.float32, device=device),
                torch.empty(cap, dtype=torch.int32, device=device),
                torch.empty(cap, dtype=torch.uint8, device=device))
        rc = lib.cms_modified_cosine_sparse(
            ctx.handle, ptr(ref.mz), ptr(ref.a), ptr(ref.b), ptr(ref.offsets), ptr(ref_precursor),
            ref.n, ref.n_peaks, ptr(qry.mz), ptr(qry.a), ptr(qry.b), ptr(qry.offsets),
            ptr(qry_precursor), qry.n, qry.n_peaks, float(tolerance), int(match_limit),
            float(threshold), *[ptr(b) for b in bufs], cap, ptr(count),
            None if cfg is None else _ctypes_ref(cfg), stream_handle(s))
        check(rc, "cms_modified_cosine_sparse")
        bits = ctx.take_device_error(stream_handle(s))  # synchronises s
        if bits & _native.DEVERR_SPILL_OVERRUN and not (config or {}).get("mode") == 2:
            config = dict(config or {}, mode=2)
            continue
        if bits & _native.DEVERR_SPECTRUM_TOO_LONG:
            raise NativeError("cms_modified_cosine_sparse: a spectrum has more than 32767 peaks",
                              _native.CMS_ERR_DEVICE)
        _raise_device_error(bits, "cms_modified_cosine_sparse")
        n = int(count.item())
        if n <= cap:
            return SparseHits(*bufs, n)
        cap = n


def mass_match_matrix(ref_values, q_values, tolerance: float, ppm: bool = False, *, out=None,
                      stream=None):
    """matchms ParentMassMatch / PrecursorMzMatch for all pairs -> uint8 (0/1)
    [n_ref, n_q] on the device.  ref_values / q_values: float64 device
    tensors (parent masses or precursor m/z); ppm selects the tolerance in
    parts per million of the pair's mean."""
    lib = _native.load()
    device = ref_values.device
    s = _stream(device, stream)
    n_r, n_q = int(ref_values.shape[0]), int(q_values.shape[0])
    if ref_values.dtype != torch.float64 or q_values.dtype != torch.float64:
        raise TypeError("mass_match_matrix takes float64 values")
    if out is None:
        out = torch.empty((n_r, n_q), dtype=torch.uint8, device=device)
    rc = lib.cms_mass_match(ptr(ref_values.contiguous()), n_r, ptr(q_values.contiguous()), n_q,
                            float(tolerance), 1 if ppm else 0, ptr(out), int(out.stride(0)),
                            stream_handle(s))
    check(rc, "cms_mass_match")
    return out


def intersect_mz_matrix(ref_mz, ref_off, q_mz, q_off, scaling: float = 1.0, *, out=None,
                        stream=None, check_errors: bool = False):
    """matchms IntersectMz for all pairs -> float64 [n_ref, n_q] on the
    device.  *_mz: float64 peak m/z (sorted within each spectrum), *_off:
    int64 CSR offsets [n + 1], all device tensors."""
    lib = _native.load()
    device = ref_off.device
    s = _stream(device, stream)
    n_r, n_q = int(ref_off.shape[0]) - 1, int(q_off.shape[0]) - 1
    for t, name in ((ref_mz, "ref_mz"), (q_mz, "q_mz")):
        if t.dtype != torch.float64:
            raise TypeError(f"{name} must be float64")
    for t, name in ((ref_off, "ref_off"), (q_off, "q_off")):
        if t.dtype != torch.int64:
            raise TypeError(f"{name} must be int64")
    if out is None:
        out = torch.empty((max(n_r, 0), max(n_q, 0)), dtype=torch.float64, device=device)
    ref_mz, ref_off = ref_mz.contiguous(), ref_off.contiguous()
    q_mz, q_off = q_mz.contiguous(), q_off.contiguous()
    err = torch.zeros(1, dtype=torch.int32, device=device) if check_errors else None
    rc = lib.cms_intersect_mz(ptr(ref_mz), ptr(ref_off), n_r, int(ref_mz.shape[0]), ptr(q_mz),
                              ptr(q_off), n_q, int(q_mz.shape[0]), float(scaling), ptr(out),
                              int(out.stride(0)), ptr(err), stream_handle(s))
    check(rc, "cms_intersect_mz")
    if check_errors:
        s.synchronize()
        bits = int(err.item())
        if bits:
            _raise_device_error(bits, "cms_intersect_mz")
    return out
