"""Pinned staging ring: uploads equal their sources, for every size class
(plain path, one chunk, many chunks with a ragged tail) and dtype used."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dtype", [np.float32, np.float64, np.int64, np.uint8])
def test_upload_round_trip(cuda_device, dtype):
    import torch

    from cudams import staging

    chunk = staging.stager(cuda_device).chunk
    for k, nbytes in enumerate((100, staging.MIN_STAGED_BYTES + 8, chunk, 3 * chunk + 24)):
        n = nbytes // np.dtype(dtype).itemsize
        want = (np.random.default_rng(k).random(n) * 1000).astype(dtype)
        x = want.copy()
        d = staging.upload(x, cuda_device)
        x[:] = 0  # the source may change as soon as upload returns
        torch.cuda.synchronize()
        got = d.cpu().numpy()
        assert got.dtype == np.dtype(dtype) and got.shape == (n,)
        np.testing.assert_array_equal(got, want)


def test_packed_spectra_staged_equals_plain(cuda_device):
    """A set large enough to be staged: device arrays equal the host arrays."""
    from cudams import synthetic

    s = synthetic.lognormal_spectra(60000, seed=9)
    assert s.b.nbytes > 4 << 20
    d = s.to_device(cuda_device)
    np.testing.assert_array_equal(d.mz.cpu().numpy(), s.mz)
    np.testing.assert_array_equal(d.b.cpu().numpy(), s.b)
    np.testing.assert_array_equal(d.offsets.cpu().numpy(), s.offsets)
