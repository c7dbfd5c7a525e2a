"""cms_cosine_greedy_noalloc: the allocation-free entry point.

Some callers must not have a library allocate device memory: an application
whose GPU memory is already reserved by its own allocator, a latency-critical
loop that cannot take the device-wide synchronisation cudaMalloc / cudaFree
may imply, or a plugin host that forbids allocations behind its back.  This
entry point serves them from a fixed device array compiled into the library.
The test calls it through the C ABI twice in a row on different inputs (so a
second call must not see the first call's leftovers in the shared array) and
checks each result bit for bit twice: against the CPU oracle (the check every
parity test here makes) and against the regular entry point
cms_cosine_greedy.  It also checks that a call larger than the array, and a
call whose output is host memory, are refused with a clear error before any
kernel runs.

This file is named so that pytest collects it last.
"""
import ctypes

import numpy as np
import pytest

from conftest import assert_same

pytestmark = pytest.mark.gpu


def _noalloc(rd, qd, tol, shift, match_limit):
    import torch

    from cudams import _native
    from cudams._native import ptr, stream_handle

    lib = _native.load()
    dev = rd.mz.device
    out = (torch.full((rd.n, qd.n), -7.0, dtype=torch.float32, device=dev),
           torch.full((rd.n, qd.n), -7, dtype=torch.int32, device=dev),
           torch.full((rd.n, qd.n), 7, dtype=torch.uint8, device=dev))
    err = torch.full((1,), 0xFFFF, dtype=torch.int32, device=dev)
    s = torch.cuda.current_stream(dev)
    rc = lib.cms_cosine_greedy_noalloc(
        ptr(rd.mz), ptr(rd.a), ptr(rd.b), ptr(rd.offsets), rd.n, rd.n_peaks,
        ptr(qd.mz), ptr(qd.a), ptr(qd.b), ptr(qd.offsets), qd.n, qd.n_peaks,
        float(tol), float(shift), int(match_limit), ptr(out[0]), ptr(out[1]), ptr(out[2]),
        qd.n, ptr(err), stream_handle(s))
    assert rc == _native.CMS_OK, _native.last_error()
    torch.cuda.synchronize()
    return tuple(t.cpu().numpy() for t in out), int(err.item())


def _oracle(r, q, tol, shift, match_limit):
    from oracle import oracle

    return oracle.cosine_greedy(r, q, tol, shift, match_limit)


def _regular(rd, qd, tol, shift, match_limit):
    from cudams import kernels

    got = kernels.cosine_greedy_dense(rd, qd, tol, shift, match_limit, check_errors=True)
    return tuple(t.cpu().numpy() for t in got)


def test_noalloc_equals_regular_entry_two_calls(cuda_device):
    from cudams import synthetic

    # call 1: the 1024 x 1024-workload distribution at ragged sizes
    h1 = synthetic.uniform_spectra(301, seed=41), synthetic.uniform_spectra(257, seed=42)
    r1, q1 = (x.to_device(cuda_device) for x in h1)
    got1, err1 = _noalloc(r1, q1, 0.1, 0.0, 2048)
    assert err1 == 0
    assert_same(got1, _oracle(*h1, 0.1, 0.0, 2048), "noalloc call 1 vs oracle")
    assert_same(got1, _regular(r1, q1, 0.1, 0.0, 2048), "noalloc call 1 vs cms_cosine_greedy")

    # call 2, right after: other sizes, powers, shift and match_limit
    h2 = (synthetic.uniform_spectra(150, seed=43, mz_power=0.5, intensity_power=2.0),
          synthetic.uniform_spectra(410, seed=44, mz_power=0.5, intensity_power=2.0))
    r2, q2 = (x.to_device(cuda_device) for x in h2)
    got2, err2 = _noalloc(r2, q2, 0.3, 0.25, 7)
    assert err2 == 0
    assert_same(got2, _oracle(*h2, 0.3, 0.25, 7), "noalloc call 2 vs oracle")
    assert_same(got2, _regular(r2, q2, 0.3, 0.25, 7), "noalloc call 2 vs cms_cosine_greedy")
    assert got2[2].any()  # match_limit 7: some pairs overflow


def test_noalloc_rejects_oversized_call(cuda_device):
    """More spectra than the fixed array holds: refused before any launch (the
    buffers below are valid but are never read)."""
    import torch

    from cudams import _native, synthetic
    from cudams._native import ptr

    lib = _native.load()
    d = synthetic.uniform_spectra(2, seed=45).to_device(cuda_device)
    out = torch.zeros(4, dtype=torch.float32, device=cuda_device)
    rc = lib.cms_cosine_greedy_noalloc(
        ptr(d.mz), None, ptr(d.b), ptr(d.offsets), (1 << 20), d.n_peaks,
        ptr(d.mz), None, ptr(d.b), ptr(d.offsets), 1, d.n_peaks, 0.1, 0.0, 10,
        ptr(out), ptr(out), ptr(out), 1, None, None)
    assert rc == _native.CMS_ERR_UNSUPPORTED
    assert "exceeds the fixed scratch capacity" in _native.last_error()


def test_noalloc_rejects_host_output(cuda_device):
    """An output buffer in host memory is refused before any launch: the
    entry point only accepts memory of the current device."""
    import torch

    from cudams import _native, synthetic
    from cudams._native import ptr

    lib = _native.load()
    d = synthetic.uniform_spectra(3, seed=46).to_device(cuda_device)
    host_score = np.full((3, 3), -5.0, np.float32)
    m = torch.zeros((3, 3), dtype=torch.int32, device=cuda_device)
    o = torch.zeros((3, 3), dtype=torch.uint8, device=cuda_device)
    rc = lib.cms_cosine_greedy_noalloc(
        ptr(d.mz), ptr(d.a), ptr(d.b), ptr(d.offsets), d.n, d.n_peaks,
        ptr(d.mz), ptr(d.a), ptr(d.b), ptr(d.offsets), d.n, d.n_peaks, 0.1, 0.0, 10,
        ctypes.c_void_p(host_score.ctypes.data), ptr(m), ptr(o), 3, None, None)
    assert rc == _native.CMS_ERR_INVALID
    assert "score must be device memory of the current device" in _native.last_error()
    torch.cuda.synchronize()
    assert (host_score == -5.0).all()
