"""Modified cosine (matchms ModifiedCosine) on the GPU vs the oracle's
restatement: scores, match counts and overflow flags bit for bit, through the
indexed join (two sweeps: m/z and neutral-loss indexes), the pair kernel over
the whole matrix, the spill path, the sparse output and the class API."""
import numpy as np
import pytest

from conftest import Spectrum, assert_same
from oracle import oracle

pytestmark = pytest.mark.gpu


def _gpu(ref, rprec, qry, qprec, tol, ml, config=None):
    import torch

    from cudams import kernels

    dev = torch.device("cuda", torch.cuda.current_device())
    got = kernels.modified_cosine_dense(ref.to_device(dev), torch.from_numpy(rprec).to(dev),
                                        qry.to_device(dev), torch.from_numpy(qprec).to(dev),
                                        tol, ml, config=config, check_errors=True)
    return tuple(t.cpu().numpy() for t in got)


CONFIGS = [None, {"mode": 1, "tile_spectra": 32}, {"mode": 1, "tile_spectra": 4096},
           {"mode": 2}]


@pytest.mark.parametrize("config", CONFIGS)
def test_analog_families(cuda_device, config):
    from cudams import synthetic

    r, rp = synthetic.analog_spectra(240, seed=31, family_size=6)
    q, qp = synthetic.analog_spectra(200, seed=32, family_size=5)
    want = oracle.modified_cosine(r, q, rp, qp, 0.05, 2048)
    assert_same(_gpu(r, rp, q, qp, 0.05, 2048, config), want, str(config))
    # the same families against themselves: many shifted matches
    want = oracle.modified_cosine(r, r, rp, rp, 0.05, 2048)
    plain = oracle.cosine_greedy(r, r, 0.05, 0.0, 2048)
    assert (want[0] > plain[0] + 1e-3).sum() > 500
    assert_same(_gpu(r, rp, r, rp, 0.05, 2048, config), want, f"{config} self")


def test_lognormal_shift_window(cuda_device):
    """Heavy-tailed spectra of the batched workload with precursors spread over
    [300, 2000]: the neutral-loss windows see large |m/z - precursor|."""
    from cudams import synthetic

    r = synthetic.lognormal_spectra(700, seed=33)
    q = synthetic.lognormal_spectra(600, seed=34)
    rng = np.random.default_rng(35)
    rp = rng.uniform(300.0, 2000.0, r.n)
    qp = rng.uniform(300.0, 2000.0, q.n)
    qp[::7] = rp[: q.n][::7]  # equal precursors: every match appears twice
    want = oracle.modified_cosine(r, q, rp, qp, 0.01, 4096)
    assert_same(_gpu(r, rp, q, qp, 0.01, 4096), want, "lognormal")


@pytest.mark.parametrize("ml", [1, 5, 24])
def test_match_limit_and_spill(cuda_device, ml):
    """match_limit counted over the concatenated (unshifted, shifted) order:
    overflowed pairs go to the pair kernel and take the first ml candidates."""
    from cudams import synthetic

    r, rp = synthetic.analog_spectra(120, seed=36, family_size=4, median_peaks=120)
    want = oracle.modified_cosine(r, r, rp, rp, 0.05, ml)
    assert want[2].any()
    for cfg in (None, {"mode": 2}):
        assert_same(_gpu(r, rp, r, rp, 0.05, ml, cfg), want, f"ml={ml} {cfg}")


def test_sparse_equals_dense(cuda_device):
    import torch

    from cudams import kernels, synthetic

    r, rp = synthetic.analog_spectra(300, seed=37, family_size=6)
    dense = oracle.modified_cosine(r, r, rp, rp, 0.05, 2048)
    dev = torch.device("cuda", torch.cuda.current_device())
    hits = kernels.modified_cosine_sparse(r.to_device(dev), torch.from_numpy(rp).to(dev),
                                          r.to_device(dev), torch.from_numpy(rp).to(dev), 0.05,
                                          2048, 0.6)
    hr, hq, hs, hm, ho = hits.to_host(sort=True)
    keep = dense[0] >= np.float32(0.6)
    rr, qq = np.nonzero(keep)
    np.testing.assert_array_equal(hr, rr)
    np.testing.assert_array_equal(hq, qq)
    np.testing.assert_array_equal(hs.view(np.uint32), dense[0][keep].view(np.uint32))
    np.testing.assert_array_equal(hm, dense[1][keep])


def test_class_api(cuda_device):
    """CudaModifiedCosine on matchms-like spectra with precursor_mz metadata:
    matrix (numpy, sparse, symmetric), pair, and a missing precursor."""
    from cudams import synthetic
    from cudams.similarity import CudaModifiedCosine

    r, rp = synthetic.analog_spectra(60, seed=38, family_size=5)
    spectra = []
    for i in range(r.n):
        a, b = r.offsets[i], r.offsets[i + 1]
        spectra.append(Spectrum(r.mz[a:b].astype(np.float64), r.b[a:b].astype(np.float64),
                                {"precursor_mz": float(rp[i])}))
    want = oracle.modified_cosine(r, r, rp, rp, 0.05, 2048)
    sim = CudaModifiedCosine(tolerance=0.05)
    got = sim.matrix(spectra, spectra)
    assert_same((got["score"], got["matches"], got["overflow"]), want, "class")
    sym = sim.matrix(spectra, spectra, is_symmetric=True)
    lower = np.tril_indices(r.n, -1)
    ws = want[0].copy()
    ws[lower] = want[0].T[lower]
    np.testing.assert_array_equal(sym["score"].view(np.uint32), ws.view(np.uint32))
    p = sim.pair(spectra[3], spectra[4])
    assert p["score"] == want[0][3, 4] and p["matches"] == want[1][3, 4]
    sp = CudaModifiedCosine(tolerance=0.05, sparse_threshold=0.7).matrix(spectra, spectra,
                                                                          array_type="sparse")
    dense = sp.to_array("sparse_score") if hasattr(sp, "to_array") else None
    if dense is not None:
        np.testing.assert_array_equal(dense >= 0.7, want[0] >= np.float32(0.7))
    bad = Spectrum(np.array([100.0]), np.array([1.0]))  # no precursor
    with pytest.raises(AssertionError, match="Precursor_mz missing"):
        sim.matrix([bad], spectra[:2])


def test_rejects_over_32767_peaks(cuda_device):
    import torch

    from cudams import _native, kernels
    from cudams.packing import pack_csr

    n = 33000
    mz = np.linspace(100.0, 1000.0, n).astype(np.float32)
    big = pack_csr(mz, np.ones(n, np.float32), np.array([0, n], np.int64), None)
    dev = torch.device("cuda", torch.cuda.current_device())
    p = torch.tensor([500.0], dtype=torch.float64, device=dev)
    with pytest.raises(_native.NativeError, match="32767"):
        kernels.modified_cosine_dense(big.to_device(dev), p, big.to_device(dev), p, 0.1, 2048,
                                      check_errors=True)
