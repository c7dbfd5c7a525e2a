"""MGF reader: CSR arrays equal to packing the same spectra one by one."""
import io

import numpy as np

from cudams.mgf import read_mgf
from cudams.packing import pack_spectra

MGF = """\
# a comment line
BEGIN IONS
TITLE=first
PEPMASS=301.5 1000
CHARGE=1+
300.2 5.0
100.1 10.0
200.3 7.5
END IONS

BEGIN IONS
TITLE=empty
END IONS
BEGIN IONS
TITLE=three columns
PEPMASS=150.0
50.5 1.0 "b2"
60.25 2.0
55.0 0.5 annotated
END IONS
"""


def test_small_file_fields_and_order():
    packed, meta = read_mgf(io.StringIO(MGF))
    assert packed.n == 3
    assert [m["title"] for m in meta] == ["first", "empty", "three columns"]
    assert meta[0]["precursor_mz"] == 301.5 and meta[2]["precursor_mz"] == 150.0
    np.testing.assert_array_equal(packed.offsets, [0, 3, 3, 6])
    np.testing.assert_array_equal(packed.mz, np.float32([100.1, 200.3, 300.2, 50.5, 55.0, 60.25]))
    np.testing.assert_array_equal(packed.b, np.float32([10.0, 7.5, 5.0, 1.0, 0.5, 2.0]))
    want = pack_spectra([(np.array([100.1, 200.3, 300.2]), np.array([10.0, 7.5, 5.0])),
                         None,
                         (np.array([50.5, 55.0, 60.25]), np.array([1.0, 0.5, 2.0]))])
    for f in ("mz", "b", "offsets"):
        np.testing.assert_array_equal(getattr(packed, f), getattr(want, f))


def test_round_trip_synthetic_with_truncation_and_powers(tmp_path):
    from cudams import synthetic

    s = synthetic.uniform_spectra(60, seed=21)
    lines = []
    rng = np.random.default_rng(0)
    for i in range(s.n):
        lines.append("BEGIN IONS")
        lines.append(f"TITLE=s{i}")
        mz = s.mz[s.offsets[i]:s.offsets[i + 1]]
        it = s.b[s.offsets[i]:s.offsets[i + 1]]
        for k in rng.permutation(mz.shape[0]):  # peaks in random order in the file
            lines.append(f"{float(mz[k])!r} {float(it[k])!r}")
        lines.append("END IONS")
    path = tmp_path / "synthetic.mgf"
    path.write_text("\n".join(lines) + "\n")
    for n_max, p in ((None, (0.0, 1.0)), (50, (0.5, 2.0))):
        packed, meta = read_mgf(path, n_max_peaks=n_max, mz_power=p[0], intensity_power=p[1])
        want = pack_spectra([(s.mz[s.offsets[i]:s.offsets[i + 1]].astype(np.float64),
                              s.b[s.offsets[i]:s.offsets[i + 1]]) for i in range(s.n)],
                            n_max, p[0], p[1])
        assert len(meta) == s.n and meta[7]["title"] == "s7"
        for f in ("mz", "b", "offsets"):
            np.testing.assert_array_equal(getattr(packed, f), getattr(want, f))
        if p[0]:
            np.testing.assert_array_equal(packed.a, want.a)
