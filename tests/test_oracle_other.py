"""The restatement of matchms' ParentMassMatch / PrecursorMzMatch /
IntersectMz (oracle/matchms_other_restated.py) on hand-computed cases, and
the plug-in classes' argument checks, which run before any device work."""
import numpy as np
import pytest

from conftest import Spectrum
from oracle import matchms_other_restated as other


def test_mass_match_dalton():
    got = other.mass_match([100.0, 200.0], [100.125, 100.1250001, 99.875, 200.0], 0.125)
    np.testing.assert_array_equal(got, [[True, False, True, False],
                                        [False, False, False, True]])


def test_mass_match_ppm():
    # |500 - 500.001| / 500.0005 * 1e6 = 1.999998...
    assert other.mass_match([500.0], [500.001], 2.0, ppm=True)[0, 0]
    assert not other.mass_match([500.0], [500.001], 1.9, ppm=True)[0, 0]
    assert not other.mass_match([500.0], [float("nan")], 2.0, ppm=True)[0, 0]


def test_intersect_mz_sets():
    a = [np.array([100.0, 200.0, 300.0]), np.array([100.0, 100.0, 200.0]), np.array([])]
    b = [np.array([200.0, 300.0, 400.0]), np.array([100.0]), np.array([])]
    got = other.intersect_mz(a, b)
    want = np.array([[2 / 4, 1 / 3, 0 / 3],    # {100,200,300} vs {200,300,400}, {100}, {}
                     [1 / 4, 1 / 2, 0 / 2],    # {100,200}: repeated values count once
                     [0 / 3, 0 / 1, 0.0]])     # {}: 0 / n, and 0 for an empty union
    np.testing.assert_array_equal(got, want)
    assert other.intersect_mz([np.array([1.0, 2.0])], [np.array([2.0])], scaling=2.0)[0, 0] == 1.0


def test_class_argument_checks():
    from cudams.similarity import CudaIntersectMz, CudaParentMassMatch, CudaPrecursorMzMatch

    with pytest.raises(AssertionError, match="Expected type"):
        CudaPrecursorMzMatch(tolerance_type="Da")
    s1 = Spectrum([100.0], [1.0], {"precursor_mz": 120.0})
    s2 = Spectrum([100.0], [1.0], {})
    with pytest.raises(AssertionError, match="Missing precursor m/z"):
        CudaPrecursorMzMatch().matrix([s1], [s2])
    with pytest.raises(AssertionError, match="Missing parent mass"):
        CudaParentMassMatch().pair(s1, s1)
    with pytest.raises(ValueError, match="not sorted"):
        CudaIntersectMz().matrix([Spectrum([200.0, 100.0], [1.0, 1.0])], [s1])
    assert CudaPrecursorMzMatch(0.5, "ppm").to_dict()["tolerance_type"] == "ppm"
