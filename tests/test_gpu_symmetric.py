"""is_symmetric=True (matchms semantics): only pairs (i, j) with i <= j are
scored, as (references[i], queries[j]), and (j, i) receives the same result.

The reference accepts the flag and ignores it (CudaCosineGreedy.py:131-132);
matchms' BaseSimilarity.matrix computes the upper triangle and mirrors it.
The oracle composes that from its full matrix (oracle.cosine_greedy_symmetric);
every comparison is bit for bit.  The reference and query sets differ in
most cases so that the mirrored lower triangle is not what a full computation
would give, i.e. the tests see whether the lower triangle really is a copy.
"""
import numpy as np
import pytest

from conftest import assert_same, gpu_dense
from oracle import oracle

pytestmark = pytest.mark.gpu

CONFIGS = [{}, {"mode": 2}, {"mode": 1, "tile_spectra": 32}, {"mode": 1, "tile_spectra": 4096},
           {"mode": 1, "tile_spectra": 100}]


def P(tol, ml, shift=0.0):
    return {"tolerance": tol, "shift": shift, "match_limit": ml}


@pytest.mark.parametrize("n", [301, 336, 384])  # 336, 384: 16-aligned rows
def test_dense_symmetric_differs_from_full_and_matches_oracle(cuda_device, n):
    from cudams import synthetic

    ref = synthetic.uniform_spectra(n, seed=61)
    qry = synthetic.uniform_spectra(n, seed=62)
    want = oracle.cosine_greedy_symmetric(ref, qry, 0.1, 0.0, 2048)
    full = oracle.cosine_greedy(ref, qry, 0.1, 0.0, 2048)
    assert (want[0] != full[0]).any()
    for cfg in CONFIGS:
        assert_same(gpu_dense(ref, qry, P(0.1, 2048), dict(cfg, symmetric=1)), want, str(cfg))


def test_dense_symmetric_overflow_and_shift(cuda_device):
    from cudams import synthetic

    ref = synthetic.uniform_spectra(150, seed=63, mz_power=0.5, intensity_power=2.0)
    qry = synthetic.uniform_spectra(150, seed=64, mz_power=0.5, intensity_power=2.0)
    want = oracle.cosine_greedy_symmetric(ref, qry, 0.3, 0.25, 7)
    assert want[2].any()
    for cfg in CONFIGS:
        assert_same(gpu_dense(ref, qry, P(0.3, 7, 0.25), dict(cfg, symmetric=1)), want,
                    str(cfg))


def test_dense_symmetric_self_similarity_spills(cuda_device):
    """One set against itself (the usual symmetric call): diagonal pairs have
    long candidate runs that go to the pair kernel."""
    from cudams import synthetic

    s = synthetic.lognormal_spectra(700, seed=65)
    want = oracle.cosine_greedy_symmetric(s, s, 0.01, 0.0, 4096)
    for cfg in ({}, {"mode": 1, "tile_spectra": 64}, {"mode": 2}):
        got = gpu_dense(s, s, P(0.01, 4096), dict(cfg, symmetric=1))
        assert_same(got, want, str(cfg))
        assert (got[0] == got[0].T).all()


def test_dense_symmetric_rejects_rectangular(cuda_device):
    from cudams import synthetic
    from cudams._native import NativeError

    ref = synthetic.uniform_spectra(20, seed=66)
    qry = synthetic.uniform_spectra(21, seed=67)
    with pytest.raises(NativeError, match="symmetric"):
        gpu_dense(ref, qry, P(0.1, 2048), {"symmetric": 1})


def test_sparse_symmetric(cuda_device):
    import torch

    from cudams import kernels, synthetic

    ref = synthetic.uniform_spectra(260, seed=68)
    qry = synthetic.uniform_spectra(260, seed=69)
    want = oracle.cosine_greedy_symmetric(ref, qry, 0.1, 0.0, 2048)
    thr = float(np.quantile(want[0], 0.9))
    dev = torch.device("cuda", torch.cuda.current_device())
    for cfg in ({}, {"mode": 2}, {"mode": 1, "tile_spectra": 32}):
        hits = kernels.cosine_greedy_sparse(ref.to_device(dev), qry.to_device(dev), 0.1, 0.0,
                                            2048, thr, config=dict(cfg, symmetric=1))
        r, q, sc, mt, ov = hits.to_host(sort=True)
        wr, wq = np.nonzero(want[0] >= thr)  # row-major = sorted by (r, q)
        np.testing.assert_array_equal(r, wr, err_msg=str(cfg))
        np.testing.assert_array_equal(q, wq, err_msg=str(cfg))
        np.testing.assert_array_equal(sc.view(np.uint32), want[0][wr, wq].view(np.uint32))
        np.testing.assert_array_equal(mt, want[1][wr, wq])
        np.testing.assert_array_equal(ov, want[2][wr, wq])


def test_matrix_is_symmetric_numpy_sparse_and_blocked(cuda_device):
    from cudams import synthetic
    from cudams.similarity import CudaCosineGreedy

    ref = synthetic.uniform_spectra(140, seed=70)
    qry = synthetic.uniform_spectra(140, seed=71)
    want = oracle.cosine_greedy_symmetric(ref, qry, 0.1, 0.0, 2048)
    thr = float(np.quantile(want[0], 0.95))
    k = CudaCosineGreedy(tolerance=0.1, sparse_threshold=thr)
    res = k.matrix(ref, qry, is_symmetric=True)
    assert_same((res["score"], res["matches"], res["overflow"]), want, "numpy")

    # a device budget of ~25 rows forces the blocked symmetric path
    kb = CudaCosineGreedy(tolerance=0.1, batch_size=1, max_device_bytes=140 * 9 * 25)
    res = kb.matrix(ref, qry, is_symmetric=True)
    assert_same((res["score"], res["matches"], res["overflow"]), want, "blocked")

    sp = k.matrix(ref, qry, array_type="sparse", is_symmetric=True)
    got = sp.to_array("sparse_score")
    keep = want[0] >= np.float32(thr)
    assert keep.any() and not keep.all()
    np.testing.assert_array_equal(got.view(np.uint32),
                                  np.where(keep, want[0], 0).astype(np.float32).view(np.uint32))
    np.testing.assert_array_equal(sp.to_array("sparse_matches"), np.where(keep, want[1], 0))

    with pytest.raises(ValueError, match="is_symmetric"):
        k.matrix(ref, synthetic.uniform_spectra(139, seed=72), is_symmetric=True)


@pytest.mark.parametrize("cfg", [{}, {"mode": 2}, {"mode": 1, "tile_spectra": 64}])
def test_dense_symmetric_into_stale_pitched_output(cuda_device, cfg):
    """Symmetric dense results written from both sides of the diagonal into
    output buffers with a row pitch above n that hold stale values: every
    pair is written (no stale value survives) and the pitch padding keeps its
    contents."""
    import torch

    from cudams import kernels, synthetic

    dev = cuda_device
    n, ld = 203, 211
    s = synthetic.uniform_spectra(n, seed=44)
    want = oracle.cosine_greedy_symmetric(s, s, 0.1, 0.0, 2048)
    bufs = (torch.full((n, ld), 7.0, dtype=torch.float32, device=dev),
            torch.full((n, ld), 99, dtype=torch.int32, device=dev),
            torch.full((n, ld), 3, dtype=torch.uint8, device=dev))
    sd = s.to_device(dev)
    kernels.cosine_greedy_dense(sd, sd, 0.1, 0.0, 2048, out=tuple(b[:, :n] for b in bufs),
                                config=dict(cfg, symmetric=1), check_errors=True)
    got = tuple(b.cpu().numpy() for b in bufs)
    assert_same(tuple(g[:, :n] for g in got), want, str(cfg))
    assert (got[0][:, n:] == 7.0).all() and (got[1][:, n:] == 99).all()
    assert (got[2][:, n:] == 3).all()
