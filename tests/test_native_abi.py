"""The C ABI library loads on a machine without a GPU and exports every
entry point that include/cudams_b200.h declares (no compute calls)."""
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def declared_functions():
    text = (ROOT / "include" / "cudams_b200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(cms_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_entry_points():
    names = declared_functions()
    for required in ("cms_create", "cms_destroy", "cms_last_error", "cms_cosine_greedy",
                     "cms_cosine_greedy_plain", "cms_cosine_greedy_sparse", "cms_fingerprint"):
        assert required in names


def test_library_exports_every_declared_symbol():
    from cudams import _native

    lib = _native.load()
    for name in declared_functions():
        assert hasattr(lib, name), f"{name} declared but not exported"
        assert name in _native.SIGNATURES, f"{name} has no ctypes signature"
    assert lib.cms_version() >= 100


def test_errors_without_gpu_do_not_crash():
    """Argument validation happens before any CUDA call."""
    import ctypes

    from cudams import _native

    lib = _native.load()
    rc = lib.cms_fingerprint(7, None, None, 1, None, None, 1, 64, 0.0, None, 1, None)
    assert rc == _native.CMS_ERR_INVALID
    assert "unknown measure" in _native.last_error()
    rc = lib.cms_cosine_greedy(None, *([None] * 4), 0, 0, *([None] * 4), 0, 0, 0.1, 0.0, 10,
                               None, None, None, 0, None, None)
    assert rc == _native.CMS_ERR_INVALID
    rc = lib.cms_cosine_greedy_plain(*([None] * 4), 1, *([None] * 4), 1, 0.1, 0.0, 0, 1024,
                                     None, None, None, 1, None)
    assert rc == _native.CMS_ERR_INVALID
    out = ctypes.c_void_p()
    rc = lib.cms_create(ctypes.byref(out), 0)
    assert rc != _native.CMS_OK  # no device in this container, or not sm_100


def test_no_cpu_fallback():
    import torch

    from cudams import _native

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(_native.NativeError):
        _native.require_cuda()


def test_metadata_entry_points_validate_without_gpu():
    """cms_mass_match / cms_intersect_mz reject bad arguments before any CUDA
    call, and empty problems succeed without one."""
    from cudams import _native

    lib = _native.load()
    assert lib.cms_mass_match(None, 4, None, 4, 0.1, 2, None, 4, None) == _native.CMS_ERR_INVALID
    assert "ppm" in _native.last_error()
    assert lib.cms_mass_match(None, 4, None, 8, 0.1, 0, None, 4, None) == _native.CMS_ERR_INVALID
    assert lib.cms_mass_match(None, 4, None, 4, 0.1, 0, None, 4, None) == _native.CMS_ERR_INVALID
    assert "null pointer" in _native.last_error()
    assert lib.cms_mass_match(None, 0, None, 4, 0.1, 0, None, 4, None) == _native.CMS_OK
    rc = lib.cms_intersect_mz(None, None, 3, 10, None, None, 5, 10, 1.0, None, 4, None, None)
    assert rc == _native.CMS_ERR_INVALID  # ld < n_q
    rc = lib.cms_intersect_mz(None, None, 3, 10, None, None, 5, 10, 1.0, None, 5, None, None)
    assert rc == _native.CMS_ERR_INVALID and "null pointer" in _native.last_error()
    assert lib.cms_intersect_mz(None, None, 0, 0, None, None, 5, 0, 1.0, None, 5, None,
                                None) == _native.CMS_OK


def test_pack_mz64():
    import numpy as np

    from conftest import Spectrum
    from cudams.similarity.CudaIntersectMz import pack_mz64

    mz, off = pack_mz64([Spectrum([1.0, 2.0, 2.0], [1, 1, 1]), Spectrum([], []),
                         Spectrum([0.5], [1])])
    assert mz.dtype == np.float64 and off.dtype == np.int64
    np.testing.assert_array_equal(off, [0, 3, 3, 4])
    np.testing.assert_array_equal(mz, [1.0, 2.0, 2.0, 0.5])
