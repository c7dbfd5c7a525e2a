"""Greedy cosine on the GPU vs the oracle: bit-exact score, matches, overflow.

The oracle's float64 mode restates matchms CosineGreedy (the reference's
float64 target); its norms and score sums are taken in the same order as the
kernels', so all three outputs are compared bit for bit (which is stricter
than the 1e-5 score tolerance the specification asks for).
"""
import numpy as np
import pytest

from conftest import (assert_same, golden_cosine_cases, gpu_dense, gpu_plain, load_cosine_case)
from oracle import oracle

pytestmark = pytest.mark.gpu

CONFIGS = [None, {"mode": 2}, {"mode": 1, "tile_spectra": 32}, {"mode": 1, "tile_spectra": 4096},
           {"mode": 1, "bucket_width": 0.75}, {"mode": 1, "n_buckets": 1024},
           {"mode": 2, "pair_threads": 512}]


def P(tol, ml, n_max=1024, shift=0.0):
    return {"tolerance": tol, "shift": shift, "match_limit": ml, "n_max_peaks": n_max}


@pytest.mark.parametrize("name", golden_cosine_cases())
def test_fast_vs_oracle_golden(cuda_device, name):
    ref, qry, p, _ = load_cosine_case(name)
    want = oracle.cosine_greedy(ref, qry, p["tolerance"], p["shift"], p["match_limit"])
    for cfg in CONFIGS:
        assert_same(gpu_dense(ref, qry, p, cfg), want, f"{name} {cfg}")


@pytest.mark.parametrize("name", golden_cosine_cases())
def test_plain_vs_oracle_golden(cuda_device, name):
    ref, qry, p, _ = load_cosine_case(name)
    want = oracle.cosine_greedy(ref, qry, p["tolerance"], p["shift"], p["match_limit"])
    assert_same(gpu_plain(ref, qry, p), want, name)


def test_uniform_ragged_tiles(cuda_device):
    """1024x1024-config distribution at ragged sizes (tile edges, partial warps)."""
    from cudams import synthetic

    ref = synthetic.uniform_spectra(301, seed=1)
    qry = synthetic.uniform_spectra(257, seed=2)
    p = P(0.1, 2048)
    want = oracle.cosine_greedy(ref, qry, 0.1, 0.0, 2048)
    for cfg in CONFIGS:
        assert_same(gpu_dense(ref, qry, p, cfg), want, str(cfg))
    assert_same(gpu_plain(ref, qry, p), want, "plain")


def test_lognormal_heavy_tail(cuda_device):
    """100k-config distribution (heavy-tailed peak counts, tol 0.01), 1500 x 1200."""
    from cudams import synthetic

    ref = synthetic.lognormal_spectra(1500, seed=3)
    qry = synthetic.lognormal_spectra(1200, seed=4)
    p = P(0.01, 4096)
    want = oracle.cosine_greedy(ref, qry, 0.01, 0.0, 4096)
    assert_same(gpu_dense(ref, qry, p), want, "auto")
    assert_same(gpu_dense(ref, qry, p, {"mode": 1, "tile_spectra": 4096}), want, "tile4096")


def test_per_class_widths(cuda_device):
    """Per-length-class first sub-range widths (the tuner's per-bucket choice):
    narrow, odd and whole-tile widths for different classes, results
    bit-exact."""
    from cudams import synthetic

    ref = synthetic.lognormal_spectra(900, seed=13)
    qry = synthetic.lognormal_spectra(1100, seed=14)
    p = P(0.01, 4096)
    want = oracle.cosine_greedy(ref, qry, 0.01, 0.0, 4096)
    widths = [0] * 17
    widths[5], widths[6], widths[7], widths[8], widths[9], widths[10] = 32, 1, 96, 1024, 64, 7
    assert_same(gpu_dense(ref, qry, p, {"mode": 1, "tile_spectra": 1024,
                                        "width_by_class": widths}), want, "widths")


def test_measured_tuner_config(cuda_device, tmp_path):
    """Tuner.measure times tiles and per-bucket widths on the device, records
    them, and the chosen config computes the oracle's results."""
    from cudams import autotune, synthetic

    ref = synthetic.lognormal_spectra(3000, seed=15)
    qry = synthetic.lognormal_spectra(2500, seed=16)
    t = autotune.Tuner(str(tmp_path / "tune.json"))
    cfg, report = t.measure(ref, qry, 0.01, 0.0, 4096, device=cuda_device, sample_ref=1000,
                            tiles_per_trial=2)  # a torch.device, as bench.py passes it
    assert cfg["mode"] == 1 and len(cfg["width_by_class"]) == 17
    assert report["trials"] and report["buckets"]
    st = autotune.workload_stats(ref, qry, 0.01)
    assert t.lookup(st, "B200", qry.n, ref.n) == cfg
    want = oracle.cosine_greedy(ref, qry, 0.01, 0.0, 4096)
    assert_same(gpu_dense(ref, qry, P(0.01, 4096), cfg), want, "measured")


def test_clustered_overflow(cuda_device):
    """Overflow-stress distribution: ~all pairs reach match_limit; flags and counts exact."""
    from cudams import synthetic

    ref = synthetic.clustered_spectra(24, seed=5)
    qry = synthetic.clustered_spectra(20, seed=6)
    p = P(0.05, 1024, 2048)
    want = oracle.cosine_greedy(ref, qry, 0.05, 0.0, 1024)
    assert want[2].mean() > 0.9
    assert_same(gpu_dense(ref, qry, p, {"mode": 2}), want, "mode2")
    assert_same(gpu_dense(ref, qry, p, {"mode": 1, "tile_spectra": 32}), want, "mode1")
    assert_same(gpu_plain(ref, qry, p), want, "plain")


@pytest.mark.parametrize("ml, threads", [(512, 64), (1024, 128), (2048, 256), (4096, 512),
                                         (1000, 128), (700, 64)])
def test_pair_kernel_register_sort(cuda_device, ml, threads):
    """The pair kernel sorts in registers when a pair's padded candidate count
    is eight per thread (pairs that fill match_limit with threads = cap / 8),
    and in shared memory otherwise; both bit-exact.  Clustered spectra fill any
    of these limits; a few empty and short spectra give small pairs too."""
    from cudams import synthetic
    from cudams.packing import PackedSpectra

    ref = synthetic.clustered_spectra(18, seed=7, min_peaks=600, max_peaks=1500)
    qry = synthetic.clustered_spectra(14, seed=8, min_peaks=600, max_peaks=1500)
    # append a 3-peak and an empty query so that some pairs are tiny
    mz = np.concatenate([qry.mz, np.array([100.0, 200.0, 300.0], np.float32)])
    b = np.concatenate([qry.b, np.array([1.0, 0.5, 0.25])])
    a = None if qry.a is None else np.concatenate([qry.a, np.ones(3)])
    off = np.concatenate([qry.offsets, [qry.offsets[-1] + 3, qry.offsets[-1] + 3]])
    qry2 = PackedSpectra(mz, a, b, off.astype(np.int64), qry.mz_power, qry.intensity_power,
                         qry.n_max_peaks)
    p = P(0.05, ml, 2048)
    want = oracle.cosine_greedy(ref, qry2, 0.05, 0.0, ml)
    assert want[2].mean() > 0.5
    assert_same(gpu_dense(ref, qry2, p, {"mode": 2, "pair_threads": threads}), want,
                f"ml {ml} threads {threads}")
    assert_same(gpu_dense(ref, qry2, p, {"mode": 2}), want, f"ml {ml} auto threads")


def _block_spectra(n, seed, levels):
    """Spectra of 50 tight groups of 20 peaks (every peak of a group within
    0.01 of the others) with intensities drawn from `levels`: one intensity
    level gives all-equal keys, ordered by generation alone."""
    from cudams.packing import PackedSpectra

    rng = np.random.default_rng(seed)
    centres = 100.0 + 10.0 * np.arange(50)
    mz, b, off = [], [], [0]
    for _ in range(n):
        m = np.sort((np.repeat(centres, 20) + rng.uniform(-0.004, 0.004, 1000)).astype(np.float32))
        mz.append(m)
        b.append(rng.choice(np.asarray(levels, np.float64), m.shape[0]))
        off.append(off[-1] + m.shape[0])
    return PackedSpectra(np.concatenate(mz), None, np.concatenate(b),
                         np.asarray(off, np.int64), 0.0, 1.0, 2048)


@pytest.mark.parametrize("levels", [[1.0], [0.25, 0.5, 1.0], None])
@pytest.mark.parametrize("ml", [1024, 2048])
def test_pair_kernel_equal_keys(cuda_device, levels, ml):
    """Blocks of 20 x 20 candidates per peak group with all-equal keys (the
    order is generation alone), a few intensity levels (many ties broken by
    generation) or distinct keys (None): bit-exact through the whole-matrix
    pair kernel (register and shared-memory sorts) and through spills."""
    lv = levels if levels is not None else list(np.linspace(0.01, 1.0, 997))
    ref = _block_spectra(5, 30 + ml, lv)
    qry = _block_spectra(4, 40 + ml, lv)
    p = P(0.01, ml, 2048)
    want = oracle.cosine_greedy(ref, qry, 0.01, 0.0, ml)
    assert want[2].mean() > 0.5
    assert_same(gpu_dense(ref, qry, p, {"mode": 2}), want, f"mode2 {levels}")
    assert_same(gpu_dense(ref, qry, p, {"mode": 2, "pair_threads": 64}), want, f"64 {levels}")
    assert_same(gpu_dense(ref, qry, p, {"mode": 1, "tile_spectra": 32}), want, f"spill {levels}")


def test_self_similarity_spills(cuda_device):
    """Identical sets: diagonal pairs have one candidate per peak (long runs ->
    pair kernel), off-diagonal pairs few; both paths must agree."""
    from cudams import synthetic

    s = synthetic.uniform_spectra(200, seed=7)
    p = P(0.1, 2048)
    want = oracle.cosine_greedy(s, s, 0.1, 0.0, 2048)
    assert_same(gpu_dense(s, s, p), want, "auto")
    assert_same(gpu_dense(s, s, p, {"mode": 1, "tile_spectra": 4096}), want, "tile4096")
    d = np.diagonal(want[0])
    assert np.allclose(d, 1.0, atol=1e-6)


def test_pool_overflow_split(cuda_device):
    """Wide tolerance: ~50 candidates per pair, so a 4096-query tile overflows
    the 256-entry pool and the join must split the range down to single pairs."""
    from cudams import synthetic

    ref = synthetic.uniform_spectra(64, seed=8)
    qry = synthetic.uniform_spectra(300, seed=9)
    p = P(2.0, 2048)
    want = oracle.cosine_greedy(ref, qry, 2.0, 0.0, 2048)
    assert_same(gpu_dense(ref, qry, p, {"mode": 1, "tile_spectra": 4096}), want, "split")


def test_small_match_limit(cuda_device):
    """match_limit below typical candidate counts: runs >= limit go to the pair kernel."""
    from cudams import synthetic

    ref = synthetic.uniform_spectra(50, seed=10)
    qry = synthetic.uniform_spectra(40, seed=11)
    for ml in (1, 2, 3, 7):
        p = P(0.5, ml)
        want = oracle.cosine_greedy(ref, qry, 0.5, 0.0, ml)
        assert_same(gpu_dense(ref, qry, p), want, f"ml={ml}")
        assert_same(gpu_plain(ref, qry, p), want, f"plain ml={ml}")


def test_edge_spectra(cuda_device):
    """Empty spectra, single peaks, duplicate m/z, exact tolerance edges."""
    from cudams.packing import pack_spectra

    spectra = [
        (np.zeros(0), np.zeros(0)),
        (np.array([100.0]), np.array([1.0])),
        (np.array([100.0, 100.0, 100.0]), np.array([0.5, 1.0, 0.5])),
        (np.array([99.9, 100.1, 100.2]), np.array([1.0, 1.0, 1.0])),
        (np.array([50.0, 1000.0]), np.array([0.0, 1.0])),
    ]
    s = pack_spectra(spectra, 16)
    for tol in (0.0, 0.1, 0.2, 5.0):
        p = P(tol, 64, 16)
        want = oracle.cosine_greedy(s, s, tol, 0.0, 64)
        for cfg in CONFIGS:
            assert_same(gpu_dense(s, s, p, cfg), want, f"tol={tol} {cfg}")
        assert_same(gpu_plain(s, s, p), want, f"plain tol={tol}")


def test_powers_and_shift(cuda_device):
    from cudams import synthetic

    ref = synthetic.uniform_spectra(90, seed=12, mz_power=0.5, intensity_power=2.0)
    qry = synthetic.uniform_spectra(70, seed=13, mz_power=0.5, intensity_power=2.0)
    for shift in (0.0, 0.5, -1.25):
        p = P(0.3, 2048, shift=shift)
        want = oracle.cosine_greedy(ref, qry, 0.3, shift, 2048)
        for cfg in CONFIGS:
            assert_same(gpu_dense(ref, qry, p, cfg), want, f"shift={shift} {cfg}")


def test_long_spectra(cuda_device):
    """Spectra near the 16-bit peak-index limit."""
    from cudams.packing import pack_csr

    rng = np.random.default_rng(14)
    n = [65535, 3000, 7]
    mz = np.concatenate([np.sort(rng.uniform(50, 2000, k)) for k in n])
    it = rng.uniform(0.1, 1.0, mz.shape[0])
    off = np.concatenate([[0], np.cumsum(n)])
    s = pack_csr(mz, it, off, None)
    p = P(0.01, 4096, 65535)
    want = oracle.cosine_greedy(s, s, 0.01, 0.0, 4096)
    assert_same(gpu_dense(s, s, p), want, "auto")
    assert_same(gpu_dense(s, s, p, {"mode": 2}), want, "mode2")


def test_sparse_equals_dense_filtered(cuda_device):
    import torch

    from cudams import kernels, synthetic

    ref = synthetic.uniform_spectra(400, seed=15)
    qry = synthetic.uniform_spectra(350, seed=16)
    want = oracle.cosine_greedy(ref, qry, 0.1, 0.0, 2048)
    dev = torch.device("cuda", torch.cuda.current_device())
    for thr in (0.05, 0.2, 0.6):
        hits = kernels.cosine_greedy_sparse(ref.to_device(dev), qry.to_device(dev), 0.1, 0.0,
                                            2048, thr, capacity=16)  # forces a regrow
        r, q, s, m, o = hits.to_host()
        keep = want[0] >= thr
        rr, qq = np.nonzero(keep)
        np.testing.assert_array_equal(r, rr)
        np.testing.assert_array_equal(q, qq)
        np.testing.assert_array_equal(s.view(np.uint32), want[0][keep].view(np.uint32))
        np.testing.assert_array_equal(m, want[1][keep])
        np.testing.assert_array_equal(o, want[2][keep])


def test_bad_offsets_reported(cuda_device):
    """Non-monotone offsets: the validation kernel stops every later kernel and
    the call raises (no out-of-bounds access)."""
    import torch

    from cudams import kernels, synthetic
    from cudams._native import NativeError
    from cudams.packing import DeviceSpectra

    s = synthetic.uniform_spectra(10, seed=17)
    dev = torch.device("cuda", torch.cuda.current_device())
    d = s.to_device(dev)
    off = d.offsets.clone()
    off[3] = off[5] + 1
    bad = DeviceSpectra(d.mz, d.a, d.b, off, d.n, d.n_peaks)
    with pytest.raises(NativeError):
        kernels.cosine_greedy_dense(bad, d, 0.1, 0.0, 2048, check_errors=True)
    # the context stays usable
    want = oracle.cosine_greedy(s, s, 0.1, 0.0, 2048)
    assert_same(gpu_dense(s, s, P(0.1, 2048)), want, "after error")


def test_large_sampled(cuda_device):
    """12k x 12k heavy-tailed spectra: 40k sampled pairs bit-exact, and a
    second run bit-identical to the first (determinism)."""
    import torch

    from cudams import kernels, synthetic

    ref = synthetic.lognormal_spectra(12000, seed=18)
    qry = synthetic.lognormal_spectra(12000, seed=19)
    dev = torch.device("cuda", torch.cuda.current_device())
    rd, qd = ref.to_device(dev), qry.to_device(dev)
    a = kernels.cosine_greedy_dense(rd, qd, 0.01, 0.0, 4096, check_errors=True)
    a = [t.cpu().numpy() for t in a]
    b = kernels.cosine_greedy_dense(rd, qd, 0.01, 0.0, 4096, check_errors=True)
    b = [t.cpu().numpy() for t in b]
    assert_same(b, a, "determinism")
    rng = np.random.default_rng(0)
    pr = rng.integers(0, ref.n, 40000)
    pq = rng.integers(0, qry.n, 40000)
    # plus every pair that has a candidate in a band of rows
    band = np.nonzero(a[1][:200] != 0)
    pr = np.concatenate([pr, band[0]])
    pq = np.concatenate([pq, band[1]])
    s, m, o = oracle.cosine_greedy_pairs(ref, qry, pr, pq, 0.01, 0.0, 4096)
    np.testing.assert_array_equal(a[2][pr, pq], o)
    np.testing.assert_array_equal(a[1][pr, pq], m)
    np.testing.assert_array_equal(a[0][pr, pq].view(np.uint32), s.view(np.uint32))
