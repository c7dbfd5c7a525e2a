"""The drop-in classes, exercised with the reference's own test cases
(tests/similarity/test_cosine_greedy.py, test_fingerprint_similarity.py)."""
import numpy as np
import pytest

from conftest import Spectrum
from oracle import oracle

pytestmark = pytest.mark.gpu


def compute_expected_score(mz_power, intensity_power, spectrum_1, spectrum_2, matches):
    intensity1 = spectrum_1.peaks.intensities
    mz1 = spectrum_1.peaks.mz
    intensity2 = spectrum_2.peaks.intensities
    mz2 = spectrum_2.peaks.mz
    multiply = ((mz1[matches[0]] ** mz_power) * (intensity1[matches[0]] ** intensity_power)
                * (mz2[matches[1]] ** mz_power) * (intensity2[matches[1]] ** intensity_power))
    denominator = (np.sqrt((((mz1 ** mz_power) * (intensity1 ** intensity_power)) ** 2).sum())
                   * np.sqrt((((mz2 ** mz_power) * (intensity2 ** intensity_power)) ** 2).sum()))
    return multiply.sum() / denominator


PAIR_CASES = [
    [[[np.array([100, 200, 300, 500, 510], dtype="float"), np.array([0.1, 0.2, 1.0, 0.3, 0.4])],
      [np.array([100, 200, 290, 490, 510], dtype="float"), np.array([0.1, 0.2, 1.0, 0.3, 0.4])]],
     0.1, 0.0, 1.0, [[0, 1, 4], [0, 1, 4]]],
    [[[np.array([100, 299, 300, 301, 510], dtype="float"), np.array([0.1, 1.0, 0.2, 0.3, 0.4])],
      [np.array([100, 300, 301, 511], dtype="float"), np.array([0.1, 1.0, 0.3, 0.4])]],
     0.2, 0.0, 1.0, [[0, 2, 3], [0, 1, 2]]],
    [[[np.array([100, 299, 300, 301, 510], dtype="float"), np.array([0.1, 1.0, 0.2, 0.3, 0.4])],
      [np.array([100, 300, 301, 511], dtype="float"), np.array([0.1, 1.0, 0.3, 0.4])]],
     2.0, 0.0, 1.0, [[0, 1, 3, 4], [0, 1, 2, 3]]],
    [[[np.array([100, 200, 300, 500, 510], dtype="float"), np.array([0.1, 0.2, 1.0, 0.3, 0.4])],
      [np.array([100, 200, 290, 490, 510], dtype="float"), np.array([0.1, 0.2, 1.0, 0.3, 0.4])]],
     1.0, 0.5, 2.0, [[0, 1, 4], [0, 1, 4]]],
]


@pytest.mark.parametrize("peaks, tolerance, mz_power, intensity_power, expected_matches",
                         PAIR_CASES)
def test_cosine_greedy_pair(cuda_device, peaks, tolerance, mz_power, intensity_power,
                            expected_matches):
    from cudams.similarity import CudaCosineGreedy

    spectrum_1 = Spectrum(peaks[0][0], peaks[0][1])
    spectrum_2 = Spectrum(peaks[1][0], peaks[1][1])
    cosine_greedy = CudaCosineGreedy(batch_size=8, tolerance=tolerance, mz_power=mz_power,
                                     intensity_power=intensity_power)
    score = cosine_greedy.pair(spectrum_1, spectrum_2)
    expected = compute_expected_score(mz_power, intensity_power, spectrum_1, spectrum_2,
                                      expected_matches)
    assert score["score"] == pytest.approx(expected, 1e-6)
    assert abs(float(score["score"]) - expected) <= 1e-5
    assert score["matches"] == len(expected_matches[0])
    assert score["overflow"] == 0
    assert score.dtype == np.dtype(CudaCosineGreedy.score_datatype)


@pytest.mark.parametrize("symmetric", [True, False])
def test_cosine_greedy_matrix(cuda_device, symmetric):
    from cudams.similarity import CudaCosineGreedy

    spectrum_1 = Spectrum(np.array([100, 200, 300.0]), np.array([0.1, 0.2, 1.0]))
    spectrum_2 = Spectrum(np.array([110, 190, 290.0]), np.array([0.5, 0.2, 1.0]))
    spectrums = [spectrum_1, spectrum_2]
    cosine_greedy = CudaCosineGreedy(batch_size=8)
    # the reference warns that is_symmetric is ignored (CudaCosineGreedy.py:131-132);
    # here it is implemented (upper triangle computed, mirrored), so no warning
    scores = cosine_greedy.matrix(spectrums, spectrums, is_symmetric=symmetric)
    assert scores[0][0][0] == pytest.approx(scores[1][1][0], 0.000001)
    assert scores[0][0]["score"] == pytest.approx(scores[1][1]["score"], 0.000001)
    assert scores[0][1][0] == pytest.approx(scores[1][0][0], 0.000001)
    assert scores[0][1]["score"] == pytest.approx(scores[1][0]["score"], 0.000001)
    assert isinstance(scores, np.recarray) and scores.shape == (2, 2)


def test_matrix_row_blocks_and_truncation(cuda_device):
    """A tiny device budget forces many row blocks; results equal the oracle."""
    from cudams import synthetic
    from cudams.similarity import CudaCosineGreedy

    ref = synthetic.uniform_spectra(150, seed=1)
    qry = synthetic.uniform_spectra(90, seed=2)
    k = CudaCosineGreedy(tolerance=0.1, n_max_peaks=64, match_limit=512, batch_size=1,
                         max_device_bytes=90 * 9 * 17)
    res = k.matrix(ref, qry)
    # the packer truncates to the first 64 peaks; the oracle gets the same spectra
    want = oracle.cosine_greedy(_trunc(ref, 64), _trunc(qry, 64), 0.1, 0.0, 512)
    np.testing.assert_array_equal(res["matches"], want[1])
    np.testing.assert_array_equal(res["overflow"], want[2])
    np.testing.assert_array_equal(res["score"].view(np.uint32), want[0].view(np.uint32))
    assert k.kernel_time > 0


def _trunc(packed, n):
    from cudams.packing import pack_csr

    return pack_csr(packed.mz, packed.b, packed.offsets, n)


def test_cosine_sparse_output(cuda_device):
    from cudams import synthetic
    from cudams.similarity import CudaCosineGreedy

    ref = synthetic.uniform_spectra(120, seed=3)
    qry = synthetic.uniform_spectra(100, seed=4)
    k = CudaCosineGreedy(tolerance=0.1, sparse_threshold=0.15)
    sp = k.matrix(ref, qry, array_type="sparse")
    dense = k.matrix(ref, qry)
    keep = dense["score"] >= 0.15
    score = sp.to_array("sparse_score")
    np.testing.assert_array_equal(score[keep], dense["score"][keep])
    assert (score[~keep] == 0).all()
    np.testing.assert_array_equal(sp.to_array("sparse_matches")[keep], dense["matches"][keep])


def test_fingerprint_pair_calculations(cuda_device):
    from cudams.similarity import CudaFingerprintSimilarity

    f1 = np.array([1, 1, 0, 0, 0, 1, 0, 0, 1, 0, 0, 1, 0, 0, 0, 0])
    f2 = np.array([0, 1, 1, 0, 0, 1, 0, 0, 1, 0, 1, 1, 0, 0, 0, 1])
    s1 = Spectrum([], [], {"fingerprint": f1})
    s2 = Spectrum([], [], {"fingerprint": f2})
    for method, expected in (("cosine", 0.6761234), ("jaccard", 0.5), ("dice", 2 / 3)):
        score = CudaFingerprintSimilarity(similarity_measure=method).pair(s1, s2)
        assert score == pytest.approx(expected, 1e-6)


@pytest.mark.parametrize("test_method", ["cosine", "jaccard", "dice"])
def test_fingerprint_empty_fingerprint(cuda_device, test_method):
    from cudams.similarity import CudaFingerprintSimilarity

    s1 = Spectrum([], [], {"fingerprint": np.zeros(16, int)})
    s2 = Spectrum([], [], {"fingerprint": np.array([0, 1, 1, 0, 0, 1, 0, 0, 1, 0, 1, 1, 0, 0, 0, 1])})
    m = CudaFingerprintSimilarity(similarity_measure=test_method).matrix([s1, s2], [s1, s2])
    assert m == pytest.approx(np.array([[0, 0], [0, 1.0]]), 0.001)


@pytest.mark.parametrize("test_method, expected_score, array_type, set_empty", [
    ("cosine", 0.84515425, "numpy", np.nan),
    ("jaccard", 0.71428571, "sparse", np.nan),
    ("dice", 0.83333333, "numpy", 0),
])
def test_fingerprint_missing(cuda_device, test_method, expected_score, array_type, set_empty):
    from cudams.similarity import CudaFingerprintSimilarity
    from cudams.sparse import StackedSparseArray

    s0 = Spectrum([], [], {})
    s1 = Spectrum([], [], {"fingerprint": np.array([0, 0, 1, 0, 0, 1, 0, 0, 1, 0, 1, 1, 0, 0, 0, 0])})
    s2 = Spectrum([], [], {"fingerprint": np.array([0, 1, 1, 0, 0, 1, 0, 0, 1, 0, 1, 1, 0, 0, 0, 1])})
    sim = CudaFingerprintSimilarity(set_empty_scores=set_empty, similarity_measure=test_method)
    m = sim.matrix([s0, s1, s2], [s0, s1, s2], array_type=array_type)
    expected = np.array([[set_empty, set_empty, set_empty], [set_empty, 1, expected_score],
                         [set_empty, expected_score, 1]])
    if isinstance(m, StackedSparseArray):
        m = m.to_array()
    assert np.allclose(m, expected, equal_nan=True)


def test_fingerprint_errors(cuda_device):
    from cudams.similarity import CudaFingerprintSimilarity

    s0 = Spectrum([], [], {})
    with pytest.raises(AssertionError):
        CudaFingerprintSimilarity().matrix([s0], [s0])
    with pytest.raises(AssertionError):
        CudaFingerprintSimilarity("tanimoto")
    s1 = Spectrum([], [], {"fingerprint": np.array([0, 2, 1])})
    with pytest.raises(ValueError):
        CudaFingerprintSimilarity().matrix([s1], [s1])
    s2 = Spectrum([], [], {"fingerprint": np.array([0, 1, 1])})
    with pytest.raises(NotImplementedError):
        CudaFingerprintSimilarity().matrix([s2], [s2], array_type="dense")
