"""Host-side packers (no GPU)."""
import numpy as np
import pytest

from conftest import Spectrum


def test_pack_spectra_truncates_and_rounds():
    from cudams.packing import pack_spectra

    s = [Spectrum(np.arange(10) * 100.1 + 50, np.linspace(0.1, 1, 10)),
         None,
         Spectrum([], []),
         Spectrum([75.123456789], [0.3])]
    p = pack_spectra(s, n_max_peaks=4, mz_power=0.0, intensity_power=2.0)
    np.testing.assert_array_equal(p.lengths, [4, 0, 0, 1])
    assert p.mz.dtype == np.float32 and p.a is None
    np.testing.assert_array_equal(p.mz[:4], (np.arange(4) * 100.1 + 50).astype(np.float32))
    want_b = np.linspace(0.1, 1, 10)[:4].astype(np.float32).astype(np.float64) ** 2
    np.testing.assert_array_equal(p.b[:4], want_b)
    assert p.mz[4] == np.float32(75.123456789)


def test_pack_csr_equals_pack_spectra():
    from cudams import synthetic
    from cudams.packing import pack_csr, pack_spectra

    rng = np.random.default_rng(0)
    spectra = []
    for _ in range(50):
        k = int(rng.integers(0, 40))
        spectra.append((np.sort(rng.uniform(50, 900, k)), rng.uniform(0, 1, k)))
    a = pack_spectra(spectra, 17, 1.5, 0.5)
    mz = np.concatenate([m for m, _ in spectra])
    it = np.concatenate([i for _, i in spectra])
    off = np.concatenate([[0], np.cumsum([len(m) for m, _ in spectra])])
    b = pack_csr(mz, it, off, 17, 1.5, 0.5)
    for f in ("mz", "a", "b", "offsets"):
        np.testing.assert_array_equal(getattr(a, f), getattr(b, f))


def test_pack_rejects_unsorted_and_nonfinite():
    from cudams.packing import pack_spectra

    with pytest.raises(ValueError):
        pack_spectra([(np.array([2.0, 1.0]), np.array([1.0, 1.0]))])
    with pytest.raises(ValueError):
        pack_spectra([(np.array([1.0, np.nan]), np.array([1.0, 1.0]))])
    # a descent across a spectrum boundary is fine
    p = pack_spectra([(np.array([5.0, 6.0]), np.ones(2)), (np.array([1.0, 2.0]), np.ones(2))])
    assert p.n == 2
    with pytest.raises(ValueError):
        pack_spectra([(np.arange(70000.0), np.ones(70000))], n_max_peaks=None)


def test_truncate_equals_packing_truncation():
    from cudams import synthetic
    from cudams.packing import pack_csr

    p = synthetic.uniform_spectra(60, seed=2)
    t = p.truncate(37)
    want = pack_csr(p.mz, p.b, p.offsets, 37)
    for f in ("mz", "b", "offsets"):
        np.testing.assert_array_equal(getattr(t, f), getattr(want, f))
    assert p.truncate(5000) is p


def test_subset():
    from cudams import synthetic

    p = synthetic.lognormal_spectra(100, seed=1)
    s = p.subset(10, 20)
    assert s.n == 10
    np.testing.assert_array_equal(s.mz, p.mz[p.offsets[10]:p.offsets[20]])
    assert s.offsets[0] == 0


def test_pack_fingerprints():
    from cudams.packing import pack_fingerprint_matrix, pack_fingerprints

    rng = np.random.default_rng(1)
    fps = [(rng.random(70) < 0.3).astype(int) for _ in range(5)] + [None]
    bits, valid, n = pack_fingerprints(fps)
    assert n == 70 and bits.shape == (6, 3) and bits.dtype == np.uint32
    np.testing.assert_array_equal(valid, [1, 1, 1, 1, 1, 0])
    for i in range(5):
        for k in range(70):
            assert ((bits[i, k // 32] >> (k % 32)) & 1) == fps[i][k]
    assert (bits[5] == 0).all()
    b2, _, _ = pack_fingerprint_matrix(np.stack(fps[:5]))
    np.testing.assert_array_equal(b2, bits[:5])
    with pytest.raises(ValueError):
        pack_fingerprints([np.array([0, 2, 1])])
    with pytest.raises(ValueError):
        pack_fingerprints([np.zeros(5), np.zeros(6)])


def test_synthetic_shapes():
    from cudams import synthetic

    u = synthetic.uniform_spectra(200, seed=3)
    assert u.lengths.min() >= 10 and u.lengths.max() <= 200
    assert u.mz.min() >= 50 and u.mz.max() <= 1000
    ln = synthetic.lognormal_spectra(5000, seed=4)
    assert ln.lengths.min() >= 5 and ln.lengths.max() <= 1000
    assert 50 <= np.median(ln.lengths) <= 70
    # intensities scaled to max 1 per spectrum
    mx = np.maximum.reduceat(ln.b, ln.offsets[:-1])
    np.testing.assert_allclose(mx, 1.0)
    c = synthetic.clustered_spectra(3, seed=5)
    assert c.lengths.min() >= 1000 and c.a is not None
    f = synthetic.fingerprints(100, seed=6)
    dens = np.unpackbits(f.view(np.uint8), axis=1).mean(1)
    assert 0.03 < dens.min() and dens.max() < 0.17


def test_sparse_standin():
    from cudams.sparse import StackedSparseArray

    sp = StackedSparseArray(3, 4)
    data = np.rec.fromarrays([np.array([0.5, 0.9], np.float32), np.array([2, 3], np.int32)],
                             names=["score", "matches"])
    sp.add_sparse_data(np.array([0, 2]), np.array([1, 3]), data, name="sparse")
    a = sp.to_array("sparse_score")
    assert a.shape == (3, 4) and a[0, 1] == np.float32(0.5) and a[2, 3] == np.float32(0.9)
    assert sp.to_array("sparse_matches")[2, 3] == 3
    sp2 = StackedSparseArray(2, 2)
    sp2.add_dense_matrix(np.array([[np.nan, 0], [0.5, 1]], np.float32), "")
    out = sp2.to_array()
    assert np.isnan(out[0, 0]) and out[1, 0] == np.float32(0.5) and out[0, 1] == 0


def test_autotune_sampling_matches_oracle_counts():
    from cudams import autotune, synthetic

    r = synthetic.uniform_spectra(30, seed=7)
    q = synthetic.uniform_spectra(30, seed=8)
    c = autotune.sample_candidates(r, q, 0.1, n_pairs=200, seed=1)
    assert c.shape == (200,) and 0.5 < c.mean() < 6
    stats = autotune.workload_stats(r, q, 0.1)
    cfg = autotune.heuristic_config(stats, q.n)
    assert cfg["mode"] == 1 and 32 <= cfg["tile_spectra"] <= 4096
    dense = autotune.WorkloadStats(500.0, 900.0, 1500.0, 1500.0)
    assert autotune.heuristic_config(dense, 1000)["mode"] == 2


def test_mean_candidates_estimate_matches_exact_mean():
    """The tuner's peak-level estimate of candidates per pair agrees with the
    exact mean over every pair (window counts by the same rule as the kernels)
    within a few percent, for the heavy-tailed benchmark distribution where a
    sample of whole pairs is noisy."""
    import numpy as np

    from cudams import autotune, synthetic

    r = synthetic.lognormal_spectra(400, seed=11)
    q = synthetic.lognormal_spectra(300, seed=12)
    exact = 0
    mq = q.mz.astype(np.float64)
    for i in range(r.n):
        mr = r.mz[r.offsets[i]:r.offsets[i + 1]].astype(np.float64)
        # candidates of reference spectrum i with every query spectrum at once
        for j in range(q.n):
            m = mq[q.offsets[j]:q.offsets[j + 1]]
            exact += int((np.searchsorted(m, mr + 0.01, side="right")
                          - np.searchsorted(m, mr - 0.01, side="left")).sum())
    exact /= r.n * q.n
    est = autotune.mean_candidates(r, q, 0.01)
    assert abs(est - exact) / exact < 0.05, (est, exact)
    # the heuristic turns it into ~CANDIDATES_PER_ITEM candidates per work item
    cfg = autotune.heuristic_config(autotune.WorkloadStats(est, 0.0, 99.0, 99.0), 100_000, 100_000)
    assert abs(cfg["tile_spectra"] * est - autotune.CANDIDATES_PER_ITEM) < 32 * est + 1
