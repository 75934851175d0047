"""bench.py helpers that need no GPU: the algorithmic work per PBS, the
DRAM traffic scaled from the committed ncu summary, and the HBM view with
and without a measured peak."""
import importlib.util
import json
import os

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_flops_per_pbs_matches_the_stated_counts(bench):
    from tfhe_b200.params import CONFIG1, CONFIG2
    # (2L + 2) transforms of 5 d log2 d flops and 8 d (2 2L M + 2 2L) pointwise flops per group
    assert bench.flops_per_pbs(CONFIG2) == 634880 * 371 == 235540480
    assert bench.flops_per_pbs(CONFIG1) == 626688 * 210 == 131604480


def test_traffic_scales_with_the_batch(bench):
    per = bench.read_traffic(1)
    assert per is not None and 600_000 < per < 800_000     # the key once per wave of 296, plus I/O
    assert bench.read_traffic(16384) == pytest.approx(16384 * per, rel=1e-6)


def test_hbm_view_uses_the_measured_peak_or_says_it_falls_back(bench, tmp_path, monkeypatch):
    assert bench.hbm_view(None, 1.0) is None
    monkeypatch.setattr(bench, "ROOT", str(tmp_path))
    v = bench.hbm_view(11_000_000_000, 275.0)
    assert v["peak_gbs"] == 6650.0 and v["peak_source"].startswith("fallback")
    assert v["achieved_gbs"] == pytest.approx(40.0, abs=0.1)
    (tmp_path / "MEASURED_PEAKS.json").write_text(json.dumps({"hbm_gbs": 6453.1}))
    v = bench.hbm_view(11_000_000_000, 275.0)
    assert v["peak_gbs"] == 6453.1 and v["peak_source"].startswith("MEASURED_PEAKS.json")
    assert v["frac"] == pytest.approx(40.0 / 6453.1, abs=1e-4)
