"""
The benchmark's roofline arithmetic (bench.py), on CPU: algorithmic bytes of
the surface stages and the adjoint, DRAM traffic scaled from the captured
per-unit figures, and the peak taken from the measured peaks file or, when it
is absent, the pool's fallback copy bandwidth (named as such).
"""

import importlib.util
import os

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


TOTALS = dict(atoms=1000, nb_entries=30000, bu_entries=500, probes=400, toroids=2000, convex=9000,
              toroidal=8000, concave=7000)
WORK = dict(cms_pairs=10 ** 9, cms_queries=5000, band_pairs=10 ** 9, band_queries=5000, sc_pairs=10 ** 8,
            sc_queries=900)


def test_stage_bytes(bench):
    nb4 = 4 * TOTALS["nb_entries"]
    assert bench.stage_bytes("triples_count", TOTALS) == nb4 + 76 * TOTALS["probes"]
    assert bench.stage_bytes("toroidal_emit", TOTALS) == 8 * TOTALS["toroids"] + nb4 + 62 * TOTALS["toroidal"]
    assert bench.stage_bytes("cms_backward", TOTALS, WORK) == 4 * 5000 + 92 * 2500 + 24 * 1000
    assert bench.stage_bytes("cms_backward", TOTALS) is None          # needs the search's query count
    assert bench.stage_bytes("no_such_stage", TOTALS) is None


def test_traffic_scales_with_units(bench):
    per, unit = bench.TRAFFIC_PER_UNIT["triples_count"]
    assert bench.stage_traffic("triples_count", TOTALS, WORK) == pytest.approx(per * TOTALS[unit])
    assert bench.stage_traffic("attention", TOTALS, WORK) is None


def test_roofline_peak_sources(bench):
    stages = {"triples_count": 10.0, "attention": 1.0}
    r = bench.stage_roofline(stages, WORK, TOTALS, {}, 80.0)
    assert r["kernel"] == "triples_count" and r["bound"] == "hbm"
    assert r["peak"] == bench.FALLBACK_HBM_GBS and "fallback" in r["peak_source"]
    achieved = bench.stage_bytes("triples_count", TOTALS) / 10e-3 / 1e9
    assert r["achieved"] == pytest.approx(achieved) and r["frac"] == pytest.approx(achieved / bench.FALLBACK_HBM_GBS)
    m = bench.stage_roofline(stages, WORK, TOTALS, {"hbm_gbs": 7000.0}, 80.0)
    assert m["peak"] == 7000.0 and "measured" in m["peak_source"]
    # a search stage on top is reported against the FP32 throughput
    n = bench.stage_roofline({"cms_nn": 5.0}, WORK, TOTALS, {}, 80.0)
    assert n["bound"] == "fp32" and n["unit"] == "TFLOP/s"
