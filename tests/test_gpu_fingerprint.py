"""Fingerprint kernel (tensor-core intersection counts) vs the oracle and the
reference's own float32 formulas: bit-exact.  Every call also checks the
kernel's error word (a pipeline wait that ran out of time)."""
import numpy as np
import pytest

from conftest import GOLDEN, golden_fingerprint_cases
from oracle import oracle

pytestmark = pytest.mark.gpu
MEASURES = ["jaccard", "dice", "cosine"]


def _gpu(measure, rb, rv, qb, qv, n_words, fill):
    import torch

    from cudams import kernels

    dev = torch.device("cuda", torch.cuda.current_device())
    t = lambda x: None if x is None else torch.from_numpy(np.ascontiguousarray(x)).to(dev)  # noqa
    out = kernels.fingerprint_matrix(measure, t(rb), t(rv), t(qb), t(qv), n_words, fill,
                                     check_errors=True)
    return out.cpu().numpy()


def _bits_equal(a, b):
    np.testing.assert_array_equal(a.view(np.uint32), b.view(np.uint32))


@pytest.mark.parametrize("name", golden_fingerprint_cases())
@pytest.mark.parametrize("measure", MEASURES)
def test_golden(cuda_device, name, measure):
    from cudams.packing import pack_fingerprint_matrix

    z = np.load(GOLDEN / f"fingerprint_{name}.npz")
    rb, rv, _ = pack_fingerprint_matrix(z["ref"])
    qb, qv, _ = pack_fingerprint_matrix(z["qry"])
    got = _gpu(measure, rb, rv, qb, qv, rb.shape[1], np.nan)
    _bits_equal(got, oracle.fingerprint(measure, rb, rv, qb, qv, rb.shape[1], np.nan))
    if measure != "cosine":  # cosine: see test_oracle (torch-CPU sqrt quirk)
        _bits_equal(got, z[measure])


@pytest.mark.parametrize("measure", MEASURES)
def test_vs_reference_formula_on_cuda(cuda_device, measure):
    """The reference's own torch expressions (vector_similarity_functions.py
    :42-46, :87-90, :116-118) run in float32 on the same B200: bit-exact."""
    import torch

    from cudams import synthetic
    from cudams.packing import pack_fingerprint_matrix

    rng = np.random.default_rng(1)
    dens_r = rng.uniform(0.05, 0.15, 700)[:, None]
    dens_q = rng.uniform(0.05, 0.15, 513)[:, None]
    R = (rng.random((700, 2048)) < dens_r).astype(np.uint8)
    Q = (rng.random((513, 2048)) < dens_q).astype(np.uint8)
    R[3] = 0
    Q[4] = 0
    dev = torch.device("cuda", torch.cuda.current_device())
    refs = torch.from_numpy(R).to(dev).float()
    ques = torch.from_numpy(Q).to(dev).float()
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    try:
        inter = refs @ ques.T
        if measure == "jaccard":
            union = refs.sum(1, keepdim=True) + ques.sum(1, keepdim=True).T
            union -= inter
            want = inter.div(union).nan_to_num()
        elif measure == "dice":
            union = refs.sum(1, keepdim=True).abs() + ques.sum(1, keepdim=True).abs().T
            want = 2 * inter.div(union).nan_to_num()
        else:
            norm = refs.pow(2).sum(1, keepdim=True) @ ques.pow(2).sum(1, keepdim=True).T
            want = inter.div(norm.sqrt()).nan_to_num(0)
        want = want.cpu().numpy()
    finally:
        torch.backends.cuda.matmul.allow_tf32 = prev
    rb, rv, _ = pack_fingerprint_matrix(R)
    qb, qv, _ = pack_fingerprint_matrix(Q)
    _bits_equal(_gpu(measure, rb, rv, qb, qv, rb.shape[1], np.nan), want)


@pytest.mark.parametrize("n_bits", [1, 31, 32, 100, 2048, 2049, 4096, 32768])
@pytest.mark.parametrize("measure", MEASURES)
def test_sizes_and_masks(cuda_device, n_bits, measure):
    from cudams.packing import pack_fingerprints

    rng = np.random.default_rng(n_bits)
    nr, nq = 131, 257
    fps_r = [(rng.random(n_bits) < 0.3).astype(np.int8) if rng.random() > 0.1 else None
             for _ in range(nr)]
    fps_q = [(rng.random(n_bits) < 0.3).astype(np.int8) if rng.random() > 0.1 else None
             for _ in range(nq)]
    rb, rv, _ = pack_fingerprints(fps_r, n_bits)
    qb, qv, _ = pack_fingerprints(fps_q, n_bits)
    for fill in (np.nan, 0.0, -1.5):
        got = _gpu(measure, rb, rv, qb, qv, rb.shape[1], fill)
        _bits_equal(got, oracle.fingerprint(measure, rb, rv, qb, qv, rb.shape[1], fill))


def test_branch_free_arithmetic_exhaustive(cuda_device):
    """The epilogue's division and square root equal CUDA's IEEE ones, bit
    for bit, over every operand the three measures can produce (and a 2^30
    sample of the large-fingerprint cosine triples)."""
    import ctypes

    import torch

    from cudams import _native

    counts = (ctypes.c_uint64 * 5)()
    with torch.cuda.device(cuda_device):
        _native.check(_native.load().cms_fingerprint_arith_check(counts, None),
                      "cms_fingerprint_arith_check")
    assert list(counts) == [0, 0, 0, 0, 0]


@pytest.mark.parametrize("n_bits", [16384, 32768])
def test_exact_large_counts(cuda_device, n_bits):
    """Nearly full fingerprints: intersection counts up to n_bits, odd ones
    among them, so every bit of a 15-bit count must survive the tensor-core
    accumulation exactly."""
    rng = np.random.default_rng(n_bits + 1)
    words = n_bits // 32
    nr, nq = 40, 300

    def rows(n):
        b = np.full((n, words), 0xFFFFFFFF, dtype=np.uint32)
        for i in range(1, n):  # row 0 stays full
            drop = rng.choice(n_bits, size=int(rng.integers(1, 64)), replace=False)
            np.bitwise_and.at(b[i], drop // 32, ~(np.uint32(1) << (drop % 32).astype(np.uint32)))
        return b

    rb, qb = rows(nr), rows(nq)
    for measure in MEASURES:
        got = _gpu(measure, rb, None, qb, None, words, np.nan)
        _bits_equal(got, oracle.fingerprint(measure, rb, None, qb, None, words, np.nan))
    assert _gpu("jaccard", rb[:1], None, qb[:1], None, words, np.nan)[0, 0] == 1.0


def test_large_symmetric(cuda_device):
    """12k x 12k of the 2048-bit workload against itself: symmetric, diagonal 1,
    and 20k sampled entries equal to the oracle."""
    from cudams import synthetic

    bits = synthetic.fingerprints(12000, seed=3)
    got = _gpu("jaccard", bits, None, bits, None, bits.shape[1], np.nan)
    _bits_equal(got, got.T.copy())
    assert (np.diagonal(got) == 1.0).all()
    rng = np.random.default_rng(0)
    rows = rng.integers(0, 12000, 64)
    want = oracle.fingerprint("jaccard", bits[rows], None, bits, None, bits.shape[1], np.nan)
    _bits_equal(got[rows], want)


@pytest.mark.parametrize("n", [301, 320])  # 320: 16-aligned rows (vector mirror)
@pytest.mark.parametrize("measure", MEASURES)
def test_symmetric(cuda_device, measure, n):
    """is_symmetric=True: (i, j), i <= j, computed as (reference i, query j)
    and mirrored.  For one set against itself this equals the full matrix bit
    for bit; for two sets the lower triangle is the mirrored upper one."""
    import torch

    from cudams import kernels, synthetic

    dev = torch.device("cuda", torch.cuda.current_device())
    t = lambda x: torch.from_numpy(np.ascontiguousarray(x)).to(dev)  # noqa: E731
    n_words = 64   # 3 tile rows/columns of 128, ragged edge
    a = synthetic.fingerprints(n, seed=11)
    b = synthetic.fingerprints(n, seed=12)
    va = np.ones(n, np.uint8)
    vb = np.ones(n, np.uint8)
    va[7] = 0
    vb[130] = 0
    full_aa = oracle.fingerprint(measure, a, va, a, va, n_words, np.nan)
    got = kernels.fingerprint_matrix(measure, t(a), t(va), t(a), t(va), n_words, np.nan,
                                     symmetric=True, check_errors=True).cpu().numpy()
    _bits_equal(got, full_aa)
    # the same arrays on both sides: computed as the full matrix
    ta, tva = t(a), t(va)
    got = kernels.fingerprint_matrix(measure, ta, tva, ta, tva, n_words, np.nan,
                                     symmetric=True, check_errors=True).cpu().numpy()
    _bits_equal(got, full_aa)

    full_ab = oracle.fingerprint(measure, a, va, b, vb, n_words, -1.0)
    lower = np.tril_indices(n, -1)
    want = full_ab.copy()
    want[lower] = full_ab.T[lower]
    assert (want != full_ab).any()
    got = kernels.fingerprint_matrix(measure, t(a), t(va), t(b), t(vb), n_words, -1.0,
                                     symmetric=True, check_errors=True).cpu().numpy()
    _bits_equal(got, want)


def test_symmetric_class_api(cuda_device):
    from conftest import Spectrum
    from cudams.similarity import CudaFingerprintSimilarity

    rng = np.random.default_rng(13)
    fps = [(rng.random(2048) < 0.1).astype(np.uint8) for _ in range(40)]
    spectra = [Spectrum(np.array([100.0]), np.array([1.0]), {"fingerprint": fp}) for fp in fps]
    spectra[5] = Spectrum(np.array([100.0]), np.array([1.0]))  # no fingerprint
    sim = CudaFingerprintSimilarity("jaccard", set_empty_scores=0.5)
    full = sim.matrix(spectra, spectra)
    sym = sim.matrix(spectra, spectra, is_symmetric=True)
    _bits_equal(sym, full)
    with pytest.raises(ValueError, match="is_symmetric"):
        sim.matrix(spectra, spectra[:-1], is_symmetric=True)


@pytest.mark.parametrize("ld", [517, 520, 640])  # 520, 640: tensor-store path; 517: per-lane stores
@pytest.mark.parametrize("measure", MEASURES)
def test_output_pitch(cuda_device, measure, ld):
    """Results land in an output with row pitch ld >= n_q (ragged tiles on both
    sides); the columns between n_q and ld keep their contents."""
    import torch

    from cudams import kernels, synthetic

    dev = torch.device("cuda", torch.cuda.current_device())
    t = lambda x: torch.from_numpy(np.ascontiguousarray(x)).to(dev)  # noqa: E731
    nr, nq, n_words = 300, 517, 64
    a = synthetic.fingerprints(nr, seed=21)
    b = synthetic.fingerprints(nq, seed=22)
    va = np.ones(nr, np.uint8)
    va[299] = 0
    buf = torch.full((nr, ld), 7.0, dtype=torch.float32, device=dev)
    out = buf[:, :nq]
    kernels.fingerprint_matrix(measure, t(a), t(va), t(b), None, n_words, np.nan, out=out,
                               check_errors=True)
    host = buf.cpu().numpy()
    _bits_equal(host[:, :nq], oracle.fingerprint(measure, a, va, b, None, n_words, np.nan))
    assert (host[:, nq:] == 7.0).all()
