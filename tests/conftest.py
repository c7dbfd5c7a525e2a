"""Shared test setup.

Markers: `gpu` marks every test that needs a B200 (run with -m gpu); all
other tests run on CPU.  The package lives in cosine-similarity_b200/ and the
oracle in oracle/ (test infrastructure).
"""
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
PKG = ROOT / "cosine-similarity_b200"
for p in (str(PKG), str(ROOT)):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = ROOT / "tests" / "golden"
PARAM_KEYS = ["tolerance", "mz_power", "intensity_power", "shift", "match_limit", "n_max_peaks"]


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an NVIDIA B200 (sm_100) and libcudams_b200.so")


def golden_cosine_cases():
    return sorted(p.stem[len("cosine_"):] for p in GOLDEN.glob("cosine_*.npz"))


def golden_fingerprint_cases():
    return sorted(p.stem[len("fingerprint_"):] for p in GOLDEN.glob("fingerprint_*.npz"))


def load_cosine_case(name):
    """(ref PackedSpectra, qry PackedSpectra, params dict, reference outputs)."""
    from cudams.packing import pack_csr

    z = np.load(GOLDEN / f"cosine_{name}.npz")
    params = dict(zip(PARAM_KEYS, z["params"].tolist()))
    params["match_limit"] = int(params["match_limit"])
    params["n_max_peaks"] = int(params["n_max_peaks"])
    pk = lambda m, i, o: pack_csr(m, i, o, params["n_max_peaks"], params["mz_power"],  # noqa
                                  params["intensity_power"])
    ref = pk(z["r_mz"], z["r_int"], z["r_off"])
    qry = pk(z["q_mz"], z["q_int"], z["q_off"])
    return ref, qry, params, (z["score"], z["matches"], z["overflow"])


@pytest.fixture(scope="session")
def cuda_device():
    import torch

    from cudams import _native

    return _native.require_cuda()


class _Peaks:
    def __init__(self, mz, intensities):
        self.mz = np.asarray(mz, dtype=np.float64)
        self.intensities = np.asarray(intensities, dtype=np.float64)

    def __len__(self):
        return self.mz.shape[0]


class Spectrum:
    """Minimal stand-in for matchms.Spectrum (peaks + metadata), as the
    reference's tests build them (tests/builder_Spectrum.py)."""

    def __init__(self, mz, intensities, metadata=None):
        self.peaks = _Peaks(mz, intensities)
        self._peaks = self.peaks
        self.metadata = dict(metadata or {})

    def get(self, key, default=None):
        return self.metadata.get(key, default)


def gpu_dense(ref, qry, p, config=None):
    """Fast path -> host (score, matches, overflow)."""
    from cudams import kernels
    import torch

    dev = torch.device("cuda", torch.cuda.current_device())
    s, m, o = kernels.cosine_greedy_dense(ref.to_device(dev), qry.to_device(dev), p["tolerance"],
                                          p["shift"], p["match_limit"], config=config,
                                          check_errors=True)
    return s.cpu().numpy(), m.cpu().numpy(), o.cpu().numpy()


def gpu_plain(ref, qry, p):
    from cudams import kernels
    import torch

    dev = torch.device("cuda", torch.cuda.current_device())
    s, m, o = kernels.cosine_greedy_plain(ref.to_device(dev), qry.to_device(dev), p["tolerance"],
                                          p["shift"], p["match_limit"], p["n_max_peaks"])
    torch.cuda.synchronize()
    return s.cpu().numpy(), m.cpu().numpy(), o.cpu().numpy()


def assert_same(got, want, what=""):
    """Bit-exact equality of (score, matches, overflow)."""
    s, m, o = got
    ws, wm, wo = want
    np.testing.assert_array_equal(o, wo, err_msg=f"{what}: overflow")
    np.testing.assert_array_equal(m, wm, err_msg=f"{what}: matches")
    np.testing.assert_array_equal(s.view(np.uint32), ws.view(np.uint32), err_msg=f"{what}: score")
