"""The CPU oracle, pinned against the reference's own outputs and tests.

- key_mode 1 (the reference kernel's float32 arithmetic) must reproduce the
  reference kernel's match counts and overflow flags exactly on every golden
  case generated from the reference under numba's CUDA simulator
  (tests/golden/make_golden.py), and its scores to float32 rounding.
- key_mode 0 (matchms float64 semantics) must meet the reference's own
  known-answer tests (tests/similarity/test_cosine_greedy.py:27-120) and
  agree with an independent pure-Python restatement of matchms CosineGreedy.
- The fingerprint oracle must equal the reference's torch functions bit for
  bit (tests/golden/fingerprint_*.npz).
"""
import numpy as np
import pytest

from conftest import golden_cosine_cases, golden_fingerprint_cases, load_cosine_case, GOLDEN
from oracle import matchms_restated, oracle


@pytest.mark.parametrize("name", golden_cosine_cases())
def test_oracle_f32_mode_reproduces_reference_kernel(name):
    ref, qry, p, (sc, mt, ov) = load_cosine_case(name)
    s, m, o = oracle.cosine_greedy(ref, qry, p["tolerance"], p["shift"], p["match_limit"],
                                   key_mode=1)
    np.testing.assert_array_equal(o, ov)
    np.testing.assert_array_equal(m, mt)
    # reference norms use float32 atomics in no fixed order: compare to ~1 ulp
    np.testing.assert_allclose(s, sc, rtol=2e-6, atol=1e-7)


@pytest.mark.parametrize("name", golden_cosine_cases())
def test_oracle_f64_mode_close_to_reference_kernel(name):
    """float64 keys may only reorder exact float32 ties; scores stay within 1e-5."""
    ref, qry, p, (sc, mt, ov) = load_cosine_case(name)
    s, m, o = oracle.cosine_greedy(ref, qry, p["tolerance"], p["shift"], p["match_limit"],
                                   key_mode=0)
    np.testing.assert_array_equal(o, ov)
    ok = ov == 0
    if ok.any():
        assert np.abs(s[ok] - sc[ok]).max() <= 1e-5
        assert (m[ok] == mt[ok]).mean() >= 0.99


KNOWN = [
    ([[100, 200, 300, 500, 510], [0.1, 0.2, 1.0, 0.3, 0.4]],
     [[100, 200, 290, 490, 510], [0.1, 0.2, 1.0, 0.3, 0.4]], 0.1, 0.0, 1.0, [[0, 1, 4], [0, 1, 4]]),
    ([[100, 299, 300, 301, 510], [0.1, 1.0, 0.2, 0.3, 0.4]],
     [[100, 300, 301, 511], [0.1, 1.0, 0.3, 0.4]], 0.2, 0.0, 1.0, [[0, 2, 3], [0, 1, 2]]),
    ([[100, 299, 300, 301, 510], [0.1, 1.0, 0.2, 0.3, 0.4]],
     [[100, 300, 301, 511], [0.1, 1.0, 0.3, 0.4]], 2.0, 0.0, 1.0, [[0, 1, 3, 4], [0, 1, 2, 3]]),
    ([[100, 200, 300, 500, 510], [0.1, 0.2, 1.0, 0.3, 0.4]],
     [[100, 200, 290, 490, 510], [0.1, 0.2, 1.0, 0.3, 0.4]], 1.0, 0.5, 2.0, [[0, 1, 4], [0, 1, 4]]),
]


def expected_score(p, q, s1, s2, matches):
    # tests/similarity/test_cosine_greedy.py:9-24
    mz1, i1 = map(np.asarray, s1)
    mz2, i2 = map(np.asarray, s2)
    num = (mz1[matches[0]] ** p * i1[matches[0]] ** q * mz2[matches[1]] ** p
           * i2[matches[1]] ** q).sum()
    den = np.sqrt(((mz1 ** p * i1 ** q) ** 2).sum()) * np.sqrt(((mz2 ** p * i2 ** q) ** 2).sum())
    return num / den


@pytest.mark.parametrize("case", KNOWN)
def test_oracle_known_answers(case):
    from cudams.packing import pack_spectra

    s1, s2, tol, p, q, em = case
    a = pack_spectra([tuple(np.array(x, float) for x in s1)], 1024, p, q)
    b = pack_spectra([tuple(np.array(x, float) for x in s2)], 1024, p, q)
    s, m, o = oracle.cosine_greedy(a, b, tol, 0.0, 2048)
    assert s[0, 0] == pytest.approx(expected_score(p, q, s1, s2, em), rel=1e-6)
    assert m[0, 0] == len(em[0])
    assert o[0, 0] == 0


def _restated(ref, qry, tol, p, q, shift=0.0):
    """matchms restatement on the float32-rounded spectra of a packed set."""
    s = np.zeros((ref.n, qry.n))
    m = np.zeros((ref.n, qry.n), int)
    for i in range(ref.n):
        r0, r1 = ref.offsets[i:i + 2]
        for j in range(qry.n):
            q0, q1 = qry.offsets[j:j + 2]
            ri = ref.b[r0:r1] if q == 1 else np.power(ref.b[r0:r1], 1.0 / q)
            qi = qry.b[q0:q1] if q == 1 else np.power(qry.b[q0:q1], 1.0 / q)
            s[i, j], m[i, j] = matchms_restated.cosine_greedy_pair(
                ref.mz[r0:r1], ri, qry.mz[q0:q1], qi, tol, p, q, shift)
    return s, m


def test_oracle_vs_matchms_restatement_uniform():
    from cudams import synthetic

    R = synthetic.uniform_spectra(30, seed=11)
    Q = synthetic.uniform_spectra(30, seed=12)
    s, m, o = oracle.cosine_greedy(R, Q, 0.1, 0.0, 2048)
    rs, rm = _restated(R, Q, 0.1, 0.0, 1.0)
    np.testing.assert_array_equal(m, rm)
    assert np.abs(s - rs).max() <= 1e-6
    assert not o.any()


def test_oracle_vs_matchms_restatement_ties():
    """Coarse intensity grid: many exactly tied products; tie order decides matches."""
    from cudams.packing import pack_spectra

    rng = np.random.default_rng(5)
    spectra = []
    for _ in range(25):
        k = int(rng.integers(5, 30))
        mz = np.sort(rng.choice(np.arange(100.0, 120.0, 0.25), k, replace=False))
        it = rng.choice(np.array([0.25, 0.5, 1.0]), k)
        spectra.append((mz, it))
    P = pack_spectra(spectra, 1024)
    s, m, o = oracle.cosine_greedy(P, P, 0.3, 0.0, 4096)
    rs, rm = _restated(P, P, 0.3, 0.0, 1.0)
    np.testing.assert_array_equal(m, rm)
    assert np.abs(s - rs).max() <= 1e-6


def test_oracle_pairs_entry_matches_dense():
    from cudams import synthetic

    R = synthetic.lognormal_spectra(25, seed=3)
    Q = synthetic.lognormal_spectra(25, seed=4)
    s, m, o = oracle.cosine_greedy(R, Q, 0.05, 0.0, 4096)
    rr, qq = np.meshgrid(np.arange(25), np.arange(25), indexing="ij")
    ps, pm, po = oracle.cosine_greedy_pairs(R, Q, rr.ravel(), qq.ravel(), 0.05, 0.0, 4096)
    np.testing.assert_array_equal(ps.reshape(25, 25), s)
    np.testing.assert_array_equal(pm.reshape(25, 25), m)


def test_oracle_overflow_rule():
    """Exactly match_limit candidates count as overflow (reference :149)."""
    from cudams.packing import pack_spectra

    s1 = (np.array([100, 200, 300, 500, 510.0]), np.array([0.1, 0.2, 1.0, 0.3, 0.4]))
    P = pack_spectra([s1], 16)
    for limit, ovf, matches in ((5, 1, 5), (6, 0, 5), (3, 1, 3)):
        s, m, o = oracle.cosine_greedy(P, P, 0.1, 0.0, limit)
        assert o[0, 0] == ovf and m[0, 0] == matches


def _fp_case(name):
    z = np.load(GOLDEN / f"fingerprint_{name}.npz")
    return z


@pytest.mark.parametrize("name", golden_fingerprint_cases())
@pytest.mark.parametrize("measure", ["jaccard", "dice", "cosine"])
def test_fingerprint_oracle_bit_exact_vs_reference(name, measure):
    from cudams.packing import pack_fingerprint_matrix

    z = _fp_case(name)
    rb, rv, nb = pack_fingerprint_matrix(z["ref"])
    qb, qv, _ = pack_fingerprint_matrix(z["qry"])
    out = oracle.fingerprint(measure, rb, rv, qb, qv, rb.shape[1], float("nan"))
    ref = z[measure]
    assert out.dtype == np.float32
    if measure != "cosine":
        np.testing.assert_array_equal(out.view(np.uint32), ref.view(np.uint32))
        return
    # The fixtures come from torch on CPU, whose float32 sqrt (AVX-512 build)
    # is not correctly rounded for some inputs; the reference's target, torch
    # on CUDA, and the oracle use IEEE sqrt.  Every difference must be
    # explained by torch-CPU's sqrt of the same a*b.
    import torch

    a = z["ref"].sum(1).astype(np.float32)[:, None]
    b = z["qry"].sum(1).astype(np.float32)[None, :]
    inter = (z["ref"].astype(np.int64) @ z["qry"].T.astype(np.int64)).astype(np.float32)
    ab = (a * b).astype(np.float32)
    t_sqrt = torch.from_numpy(ab).sqrt().numpy()
    quirk = t_sqrt.view(np.uint32) != np.sqrt(ab).view(np.uint32)
    with np.errstate(invalid="ignore", divide="ignore"):
        via_torch = np.nan_to_num(inter / t_sqrt, nan=0.0).astype(np.float32)
    np.testing.assert_array_equal(out[~quirk].view(np.uint32), ref[~quirk].view(np.uint32))
    np.testing.assert_array_equal(via_torch[quirk].view(np.uint32), ref[quirk].view(np.uint32))


def test_modified_cosine_oracle_vs_matchms_restatement():
    """The C restatement of matchms ModifiedCosine against the independent
    pure-Python one (unshifted + precursor-shifted matches, one stable sort,
    one greedy) on analogue families, where shifted matches matter."""
    from cudams import synthetic

    P, prec = synthetic.analog_spectra(24, seed=21, family_size=6)
    s, m, o = oracle.modified_cosine(P, P, prec, prec, 0.05, 1 << 20)
    assert not o.any()
    plain, _, _ = oracle.cosine_greedy(P, P, 0.05, 0.0, 1 << 20)
    assert (s > plain + 1e-3).sum() > 20  # the shifted matches raise many scores
    for i in range(P.n):
        r0, r1 = P.offsets[i:i + 2]
        for j in range(P.n):
            q0, q1 = P.offsets[j:j + 2]
            rs, rm = matchms_restated.modified_cosine_pair(
                P.mz[r0:r1], P.b[r0:r1], P.mz[q0:q1], P.b[q0:q1], prec[i], prec[j], 0.05)
            assert m[i, j] == rm, (i, j)
            assert abs(float(s[i, j]) - rs) <= 1e-6, (i, j)


def test_modified_cosine_oracle_match_limit():
    """Generation stops at match_limit over the concatenated (unshifted, then
    shifted) order and sets overflow; the survivors are a prefix."""
    from cudams import synthetic

    P, prec = synthetic.analog_spectra(16, seed=22, family_size=4)
    full = oracle.modified_cosine(P, P, prec, prec, 0.05, 1 << 20)
    lim = oracle.modified_cosine(P, P, prec, prec, 0.05, 6)
    assert lim[2].any() and not full[2].any()
    ok = lim[2] == 0
    np.testing.assert_array_equal(lim[1][ok], full[1][ok])
    np.testing.assert_array_equal(lim[0][ok], full[0][ok])
    assert (lim[1] <= 6).all()
