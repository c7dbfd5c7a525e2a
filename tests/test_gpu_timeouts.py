"""The bounded waits between the warps of the pipelined kernels, made to run
out on purpose through the CMS_TEST_STALL hook (one role does nothing; no
fault, trap or endless wait is involved): the kernel stops within its 2 s
limit, the host sees the error bit as NativeError, and the next call on the
same context computes correct results."""
import numpy as np
import pytest

from conftest import assert_same, gpu_dense
from oracle import oracle

pytestmark = pytest.mark.gpu


def test_fingerprint_wait_timeout_is_reported(cuda_device, monkeypatch):
    import torch

    from cudams import _native, kernels, synthetic

    bits = synthetic.fingerprints(300, seed=61)
    t = torch.from_numpy(bits).to(cuda_device)
    monkeypatch.setenv("CMS_TEST_STALL", "mma")
    with pytest.raises(_native.NativeError, match="pipeline timeout"):
        kernels.fingerprint_matrix("jaccard", t, None, t, None, bits.shape[1], np.nan,
                                   check_errors=True)
    monkeypatch.delenv("CMS_TEST_STALL")
    got = kernels.fingerprint_matrix("jaccard", t, None, t, None, bits.shape[1], np.nan,
                                     check_errors=True).cpu().numpy()
    want = oracle.fingerprint("jaccard", bits, None, bits, None, bits.shape[1], np.nan)
    np.testing.assert_array_equal(got.view(np.uint32), want.view(np.uint32))


def test_pair_pipeline_wait_timeout_is_reported(cuda_device, monkeypatch):
    from cudams import _native, synthetic

    ref = synthetic.clustered_spectra(60, seed=62)
    qry = synthetic.clustered_spectra(60, seed=63)
    p = {"tolerance": 0.05, "shift": 0.0, "match_limit": 1024, "n_max_peaks": 2048}
    monkeypatch.setenv("CMS_TEST_STALL", "pair")
    with pytest.raises(_native.NativeError, match="bounded wait"):
        gpu_dense(ref, qry, p, {"mode": 2})
    monkeypatch.delenv("CMS_TEST_STALL")
    want = oracle.cosine_greedy(ref, qry, 0.05, 0.0, 1024)
    assert_same(gpu_dense(ref, qry, p, {"mode": 2}), want, "after the timeout")
