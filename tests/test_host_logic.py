"""Host logic that needs no GPU: the tuner's cache, the benchmark's clock
summary, and the CosineConfig layout the C ABI reads."""
import ctypes
import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]


def test_tuner_cache_round_trip(tmp_path):
    from cudams import autotune

    t = autotune.Tuner(str(tmp_path / "tune.json"))
    st = autotune.WorkloadStats(0.1, 2.0, 99.0, 99.0)
    assert t.lookup(st, "B200", 100_000, 100_000) == autotune.heuristic_config(st, 100_000, 100_000)
    t.record(st, "B200", {"mode": 1, "tile_spectra": 777})
    t2 = autotune.Tuner(str(tmp_path / "tune.json"))           # read back from disk
    assert t2.lookup(st, "B200", 100_000)["tile_spectra"] == 777
    assert t2.lookup(st, "B200", 500)["tile_spectra"] == 500      # capped by the query count
    # a workload in another bucket (10x the candidates) is not served from the cache
    other = autotune.WorkloadStats(1.0, 2.0, 99.0, 99.0)
    assert t2.lookup(other, "B200", 100_000) == autotune.heuristic_config(other, 100_000)
    assert json.loads((tmp_path / "tune.json").read_text())


def _bench():
    sys.path.insert(0, str(ROOT))
    import bench

    return bench


def test_clock_summary_keeps_samples_inside_the_timed_region():
    bench = _bench()
    c = bench.ClockSampler(0)
    row = ("2026/12/04 00:00:00.000, 0, {mhz}, 1965, 700.0, 0x0, {hw}, Not Active, "
           "Not Active, {cap}")
    c.lines = [(1.0, row.format(mhz=800, hw="Not Active", cap="Not Active")),    # warm-up
               (2.0, row.format(mhz=1965, hw="Not Active", cap="Active")),
               (2.5, row.format(mhz=1900, hw="Not Active", cap="Active")),
               (3.0, row.format(mhz=1965, hw="Not Active", cap="Not Active")),
               (9.0, row.format(mhz=600, hw="Active", cap="Not Active"))]        # after
    c.t0, c.t1 = 1.5, 3.5
    s = c.summary()
    assert s["samples"] == 3 and s["sm_mhz"] == 1965 and s["sm_max_mhz"] == 1965
    assert s["reasons"] == ["sw_power_cap"]
    c.t0, c.t1 = 8.5, 9.5
    assert c.summary()["reasons"] == ["hw_slowdown"]
    empty = bench.ClockSampler(0)
    assert empty.summary()["reasons"] == ["unsampled"]


def test_cosine_config_layout_matches_the_header():
    """Field offsets of the ctypes struct follow the C declaration (int32,
    double, int32 x 3, double, int32 with natural alignment)."""
    from cudams._native import CosineConfig

    want = {"tile_spectra": 0, "bucket_width": 8, "n_buckets": 16, "mode": 20,
            "pair_threads": 24, "cand_per_pair": 32, "symmetric": 40, "width_by_class": 44}
    got = {name: getattr(CosineConfig, name).offset for name, _ in CosineConfig._fields_}
    assert got == want
    assert ctypes.sizeof(CosineConfig) == 112
    header = (ROOT / "include" / "cudams_b200.h").read_text()
    body = header[header.index("typedef struct {", header.index("Tuning of the tiled path")):
                  header.index("} cms_cosine_config;")]
    names = [ln.split()[-1].rstrip(";") for ln in body.splitlines()[1:] if ln.strip()]
    assert [n.split("[")[0] for n in names] == list(want)
    assert names[-1] == "width_by_class[17]"


def test_cosine_config_from_dict():
    """Per-class widths (a list, as the tuner's JSON cache holds them) fill the
    17-entry array, zero-padded; other keys map to fields."""
    from cudams._native import CosineConfig

    c = CosineConfig.from_dict({"mode": 1, "tile_spectra": 640, "width_by_class": [0, 0, 32, 64]})
    assert c.mode == 1 and c.tile_spectra == 640
    assert list(c.width_by_class) == [0, 0, 32, 64] + [0] * 13


def test_tuner_records_per_bucket_widths(tmp_path):
    """A measured config (per-bucket widths included) round-trips through the
    on-disk cache and is what lookup returns for that workload's bucket."""
    from cudams import autotune

    t = autotune.Tuner(str(tmp_path / "tune.json"))
    st = autotune.WorkloadStats(0.1, 2.0, 99.0, 99.0)
    cfg = {"mode": 1, "tile_spectra": 1344, "cand_per_pair": 0.1,
           "width_by_class": [0] * 8 + [320, 160] + [0] * 7}
    t.record(st, "B200", cfg)
    got = autotune.Tuner(str(tmp_path / "tune.json")).lookup(st, "B200", 100_000, 100_000)
    assert got == cfg
    key = autotune.Tuner.key(st, "B200")
    assert key.startswith("B200|c") and "|r6|" in key and key.endswith("|q6")


def test_take_selects_spectra():
    from cudams import synthetic

    P = synthetic.lognormal_spectra(50, seed=1)
    idx = [5, 2, 49, 0, 5]
    T = P.take(idx)
    assert T.n == 5
    for k, i in enumerate(idx):
        np.testing.assert_array_equal(T.mz[T.offsets[k]:T.offsets[k + 1]],
                                      P.mz[P.offsets[i]:P.offsets[i + 1]])
        np.testing.assert_array_equal(T.b[T.offsets[k]:T.offsets[k + 1]],
                                      P.b[P.offsets[i]:P.offsets[i + 1]])
