"""matchms ParentMassMatch / PrecursorMzMatch / IntersectMz on the device
(csrc/metadata_match.cu) against the oracle restatement
(oracle/matchms_other_restated.py): bit-exact."""
import numpy as np
import pytest

from conftest import Spectrum
from oracle import matchms_other_restated as other

pytestmark = pytest.mark.gpu


def _dev():
    import torch

    return torch.device("cuda", torch.cuda.current_device())


def _masses(n, rng):
    v = rng.uniform(100.0, 1000.0, n)
    v[::7] = np.round(v[::7], 1)  # repeated and near-equal values
    return v


@pytest.mark.parametrize("n_q", [512, 517])  # 512: 16-byte row stores; 517: per-byte
@pytest.mark.parametrize("ppm", [False, True])
def test_mass_match_kernel(cuda_device, n_q, ppm):
    import torch

    from cudams import kernels

    rng = np.random.default_rng(n_q + ppm)
    r = _masses(300, rng)
    q = _masses(n_q, rng)
    tol = 20.0 if ppm else 0.125
    # pairs exactly at the tolerance and one float64 step beyond it
    q[0], q[1] = r[0] + 0.125, np.nextafter(r[0] + 0.125, np.inf)
    q[2] = r[1] * (1 + 2e-5)
    r[5] = np.nan
    got = kernels.mass_match_matrix(torch.from_numpy(r).to(_dev()),
                                    torch.from_numpy(q).to(_dev()), tol, ppm).cpu().numpy()
    want = other.mass_match(r, q, tol, ppm)
    np.testing.assert_array_equal(got.astype(bool), want)
    assert set(np.unique(got)) <= {0, 1}
    assert want.any() and not want.all()


def _spectra_mz(n, rng, pool):
    out = []
    for i in range(n):
        k = int(rng.integers(0, 60))
        mz = np.sort(rng.choice(pool, size=k, replace=True))  # repeats on purpose
        out.append(mz)
    out[3] = np.zeros(0)
    out[4] = np.sort(rng.choice(pool, size=5000, replace=True))  # past the shared-memory stage
    return out


def _csr(lists):
    import torch

    off = np.zeros(len(lists) + 1, dtype=np.int64)
    off[1:] = np.cumsum([len(a) for a in lists])
    mz = np.concatenate(lists) if lists else np.zeros(0)
    return (torch.from_numpy(mz.astype(np.float64)).to(_dev()),
            torch.from_numpy(off).to(_dev()))


@pytest.mark.parametrize("scaling", [1.0, 0.3])
def test_intersect_mz_kernel(cuda_device, scaling):
    from cudams import kernels

    rng = np.random.default_rng(7)
    pool = rng.uniform(50.0, 500.0, 400)
    a = _spectra_mz(70, rng, pool)
    b = _spectra_mz(300, rng, pool)
    got = kernels.intersect_mz_matrix(*_csr(a), *_csr(b), scaling,
                                      check_errors=True).cpu().numpy()
    want = other.intersect_mz(a, b, scaling)
    np.testing.assert_array_equal(got.view(np.uint64), want.view(np.uint64))
    assert (want > 0).any() and (want == 0).any()


def test_intersect_mz_bad_offsets(cuda_device):
    import torch

    from cudams import _native, kernels

    mz = torch.arange(10, dtype=torch.float64, device=_dev())
    bad = torch.tensor([0, 6, 3], dtype=torch.int64, device=_dev())  # decreasing
    good = torch.tensor([0, 4], dtype=torch.int64, device=_dev())
    with pytest.raises(_native.NativeError, match="offsets"):
        kernels.intersect_mz_matrix(mz, bad, mz, good, check_errors=True)


def _spectra(n, rng):
    pool = rng.uniform(50.0, 500.0, 200)
    out = []
    for i in range(n):
        mz = np.sort(rng.choice(pool, size=int(rng.integers(1, 30)), replace=False))
        out.append(Spectrum(mz, np.ones_like(mz),
                            {"precursor_mz": float(rng.uniform(300, 310)),
                             "parent_mass": float(np.round(rng.uniform(299, 301), 2))}))
    return out


def test_classes(cuda_device):
    from cudams.similarity import CudaIntersectMz, CudaParentMassMatch, CudaPrecursorMzMatch

    rng = np.random.default_rng(3)
    refs, qrys = _spectra(40, rng), _spectra(57, rng)
    pm = [s.get("parent_mass") for s in refs], [s.get("parent_mass") for s in qrys]
    pz = [s.get("precursor_mz") for s in refs], [s.get("precursor_mz") for s in qrys]
    mzs = [s.peaks.mz for s in refs], [s.peaks.mz for s in qrys]

    got = CudaParentMassMatch(0.5).matrix(refs, qrys)
    assert got.dtype == bool
    np.testing.assert_array_equal(got, other.mass_match(*pm, 0.5))
    np.testing.assert_array_equal(CudaPrecursorMzMatch(2.0).matrix(refs, qrys),
                                  other.mass_match(*pz, 2.0))
    np.testing.assert_array_equal(CudaPrecursorMzMatch(5000.0, "ppm").matrix(refs, qrys),
                                  other.mass_match(*pz, 5000.0, ppm=True))
    ix = CudaIntersectMz(0.5).matrix(refs, qrys)
    np.testing.assert_array_equal(ix.view(np.uint64),
                                  other.intersect_mz(*mzs, 0.5).view(np.uint64))
    assert CudaIntersectMz().pair(refs[0], refs[0]) == 1.0
    assert CudaParentMassMatch(0.0).pair(refs[1], refs[1]) is True

    # sparse output holds exactly the nonzero scores; symmetric equals full
    sp = CudaParentMassMatch(0.5).matrix(refs, qrys, array_type="sparse")
    np.testing.assert_array_equal(sp.to_array().astype(bool), other.mass_match(*pm, 0.5))
    sym = CudaIntersectMz().matrix(refs, refs, is_symmetric=True)
    np.testing.assert_array_equal(sym, sym.T)
    np.testing.assert_array_equal(sym, other.intersect_mz(mzs[0], mzs[0]))
