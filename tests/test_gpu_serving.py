"""Resident library search and the continuous-batching server.

- A library search returns exactly the pairs the dense path scores at or above
  the threshold, with bit-identical values (and those equal the oracle).
- Isolation: every request's result is the same when it runs alone and when
  it runs concurrently with others in the server.
"""
import numpy as np
import pytest

from oracle import oracle

pytestmark = pytest.mark.gpu


def _dense_hits(lib_p, qry_p, tol, ml, thr, shift=0.0):
    from conftest import gpu_dense

    s, m, o = gpu_dense(lib_p, qry_p, {"tolerance": tol, "shift": shift, "match_limit": ml,
                                       "n_max_peaks": 1024})
    keep = s >= thr
    r, q = np.nonzero(keep)
    order = np.lexsort((r, q))
    return r[order], q[order], s[keep][order], m[keep][order], o[keep][order], (s, m, o)


def _threshold(lib_p, qry_p, tol, ml, shift=0.0):
    """A threshold that keeps about the top 10% of the non-zero scores."""
    _, _, _, _, _, (s, _, _) = _dense_hits(lib_p, qry_p, tol, ml, 1.0, shift)
    nz = s[s > 0]
    return float(np.quantile(nz, 0.9)) if nz.size else 0.5


@pytest.mark.parametrize("tol,shift", [(0.1, 0.0), (0.05, 0.0), (0.3, 0.25)])
def test_library_search_equals_dense(cuda_device, tol, shift):
    from cudams import synthetic
    from cudams.serving import SpectrumLibrary

    lib_p = synthetic.uniform_spectra(1500, seed=21)
    qry_p = synthetic.uniform_spectra(333, seed=22)
    thr = _threshold(lib_p, qry_p, tol, 2048, shift)
    lib = SpectrumLibrary(lib_p, tolerance=tol, shift=shift, match_limit=2048)
    try:
        res = lib.search(qry_p, threshold=thr)
    finally:
        lib.close()
    r, q, s, m, o, dense = _dense_hits(lib_p, qry_p, tol, 2048, thr, shift)
    assert res.ref.shape[0] == r.shape[0] > 0
    np.testing.assert_array_equal(res.ref, r)
    np.testing.assert_array_equal(res.query, q)
    np.testing.assert_array_equal(res.score.view(np.uint32), s.view(np.uint32))
    np.testing.assert_array_equal(res.matches, m)
    np.testing.assert_array_equal(res.overflow, o)
    want = oracle.cosine_greedy(lib_p, qry_p, tol, shift, 2048)
    np.testing.assert_array_equal(dense[0].view(np.uint32), want[0].view(np.uint32))


def test_library_search_heavy_tail_and_spills(cuda_device):
    """Heavy-tailed peaks, a query set containing library spectra (long runs go
    to the pair kernel) and a small match_limit (overflowed hits)."""
    from cudams import synthetic
    from cudams.packing import pack_csr
    from cudams.serving import SpectrumLibrary

    lib_p = synthetic.lognormal_spectra(2000, seed=23)
    extra = synthetic.lognormal_spectra(100, seed=24)
    # queries: 100 fresh spectra followed by 50 spectra copied from the library
    copy = lib_p.subset(0, 50)
    mz = np.concatenate([extra.mz, copy.mz])
    it = np.concatenate([extra.b, copy.b])
    off = np.concatenate([extra.offsets, copy.offsets[1:] + extra.offsets[-1]])
    qry_p = pack_csr(mz, it, off, 1024)
    for ml in (4096, 16):
        thr = _threshold(lib_p, qry_p, 0.01, ml)
        lib = SpectrumLibrary(lib_p, tolerance=0.01, match_limit=ml)
        try:
            res = lib.search(qry_p, threshold=thr)
        finally:
            lib.close()
        r, q, s, m, o, _ = _dense_hits(lib_p, qry_p, 0.01, ml, thr)
        np.testing.assert_array_equal(res.ref, r)
        np.testing.assert_array_equal(res.query, q)
        np.testing.assert_array_equal(res.score.view(np.uint32), s.view(np.uint32))
        np.testing.assert_array_equal(res.matches, m)
        np.testing.assert_array_equal(res.overflow, o)
        if ml == 4096:
            # self-matches of the copied spectra are hits with score 1
            for k in range(50):
                sel = (res.query == 100 + k) & (res.ref == k)
                assert sel.sum() == 1 and abs(float(res.score[sel][0]) - 1.0) < 1e-6
        else:
            assert res.overflow.any()  # truncated pairs are reported as overflowed


def test_server_isolation(cuda_device):
    """Each request's hits are identical alone and in the concurrent mix."""
    from cudams import synthetic
    from cudams.serving import Server, SpectrumLibrary

    lib_p = synthetic.lognormal_spectra(20000, seed=25)
    lib = SpectrumLibrary(lib_p, tolerance=0.01, match_limit=4096)
    rng = np.random.default_rng(26)
    sizes = [1, 7, 300, 1000, 64, 2500, 3, 900, 0, 1500, 33, 4096]
    batches = [synthetic.lognormal_spectra(int(k), seed=100 + i) if k else
               synthetic.lognormal_spectra(1, seed=99).subset(0, 0)
               for i, k in enumerate(sizes)]
    try:
        alone = [lib.search(b, threshold=0.01) for b in batches]
        with Server(lib, threshold=0.01, slots=4) as srv:
            futs = [srv.submit(b) for b in batches]
            mixed = [f.result(timeout=600) for f in futs]
            conc = srv.max_concurrent
    finally:
        lib.close()
    for a, b, k in zip(alone, mixed, sizes):
        assert a.n_queries == b.n_queries == k
        assert a.as_set() == b.as_set()
        np.testing.assert_array_equal(a.score.view(np.uint32), b.score.view(np.uint32))
    assert sum(a.ref.shape[0] for a in alone) > 0
    assert conc >= 2  # requests really overlapped
    assert all(b.latency_s > 0 for b in mixed)


def test_server_requests_overlap_on_device(cuda_device):
    """A long low-priority request (12 batches of 1000 queries against a
    60k-spectrum library, tolerance 0.05) is running when a 1000-query request
    arrives; the latter runs on the high-priority stream.  The device
    timestamps of their work items (%globaltimer at each item's start and end,
    tagged by request) show the two executing at the same time: many items of
    the long request run during the short request's span.  Each result is
    also identical to the request's result alone."""
    import time

    from cudams import synthetic
    from cudams.serving import Server, SpectrumLibrary

    lib_p = synthetic.lognormal_spectra(60000, seed=27)
    lib = SpectrumLibrary(lib_p, tolerance=0.05, match_limit=4096)
    big = synthetic.lognormal_spectra(12000, seed=28)
    small = synthetic.lognormal_spectra(1000, seed=29)
    n_tiles = -(-60000 // 1024)
    try:
        alone = [lib.search(b, threshold=0.5) for b in (big, small)]
        with Server(lib, threshold=0.5, slots=2, warmup_queries=1024,
                    trace_capacity=1_000_000) as srv:
            fb = srv.submit(big)
            t0 = time.perf_counter()
            while srv._running == 0 and time.perf_counter() - t0 < 10:
                time.sleep(0.001)
            time.sleep(0.02)  # the long request is on the GPU by now
            fs = srv.submit(small)
            rb, rs = fb.result(timeout=600), fs.result(timeout=600)
    finally:
        lib.close()
    for a, b in zip(alone, (rb, rs)):
        assert a.as_set() == b.as_set()
    assert rb.extra["priority"] == "low" and rs.extra["priority"] == "high"
    tb, ts = rb.extra["trace"], rs.extra["trace"]
    assert tb.shape[0] == 12000 * n_tiles and ts.shape[0] == 1000 * n_tiles  # every item, once
    assert ((tb[:, 0] & 0xFFFFFFFF) == rb.extra["seq"]).all()
    assert ((ts[:, 0] & 0xFFFFFFFF) == rs.extra["seq"]).all()
    s0, s1 = ts[:, 2].min(), ts[:, 3].max()
    b0, b1 = tb[:, 2].min(), tb[:, 3].max()
    assert b0 < s0 and s1 < b1, "the short request ran inside the long one's span"
    # items of the long request executing while the short one executed
    concurrent = ((tb[:, 2] < s1) & (tb[:, 3] > s0)).sum()
    assert concurrent >= 100, concurrent
