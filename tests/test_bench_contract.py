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


def test_search_roofline_uses_evaluated_pairs(bench):
    ev = {"cms_evaluated": 10 ** 8, "cms_rechecks": 5}
    r = bench.stage_roofline({"cms_nn": 5.0}, WORK, TOTALS, {}, 80.0, ev)
    assert r["evaluated_pairs"] == 10 ** 8 and r["fp64_rechecks"] == 5
    assert r["achieved"] == pytest.approx(8.0 * 10 ** 8 / 5e-3 / 1e12)
    assert r["brute_force_equivalent_tflops"] == pytest.approx(8.0 * WORK["cms_pairs"] / 5e-3 / 1e12)
    assert r["frac"] == pytest.approx(r["achieved"] / 80.0)
    rows = bench.stage_rooflines({"cms_nn": 5.0, "triples_count": 10.0, "attention": 5.0}, WORK, TOTALS, {}, 80.0,
                                 ev)
    assert rows["attention"]["bound"] == "latency" and rows["triples_count"]["bound"] == "hbm"
    assert "fp64_pipe_active_pct" in rows["triples_count"]
    assert sum(v["share"] for v in rows.values()) == pytest.approx(1.0)


def test_stratified_sample_spans_sizes_and_ligands(bench):
    import numpy as np
    rng = np.random.default_rng(0)
    sizes = rng.integers(600, 5000, 500)
    ligand = rng.random(500) < 0.05
    pick = bench.stratified_sample(sizes, ligand, 16)
    assert int(np.argmin(sizes)) in pick and int(np.argmax(sizes)) in pick
    assert int(ligand[pick].sum()) >= 2
    assert 14 <= len(pick) <= 16
    assert list(sizes[pick]) == sorted(sizes[pick])


def test_extrapolation_fit(bench):
    import numpy as np
    sizes = np.array([1000, 2000, 4000])
    secs = 1e-6 * sizes ** 1.5
    total, expo = bench._fit_extrapolation(sizes, secs, [1000, 1000, 4000])
    assert expo == pytest.approx(1.5)
    assert total == pytest.approx(2 * 1e-6 * 1000 ** 1.5 + 1e-6 * 4000 ** 1.5)


def test_multi_gpu_self_launch_command(bench, monkeypatch):
    """--gpus N without a launcher re-runs the script under torch.distributed.run with N ranks on 127.0.0.1."""
    import subprocess
    import sys
    seen = {}

    class Done:
        returncode = 0

    def fake_run(cmd, *a, **k):
        seen["cmd"] = cmd
        return Done()

    monkeypatch.setattr(subprocess, "run", fake_run)
    monkeypatch.setattr(sys, "argv", ["bench.py", "--gpus", "4", "--steps", "2"])
    assert bench.self_launch(bench.parse(["--gpus", "4", "--steps", "2"])) == 0
    cmd = seen["cmd"]
    assert cmd[:4] == ["timeout", "-k", "60", "3600"]
    assert "torch.distributed.run" in cmd and "--nproc-per-node=4" in cmd and "127.0.0.1" in cmd
    assert cmd[-4:] == ["--gpus", "4", "--steps", "2"]


def test_global_batch_shards_cover_the_batch(bench):
    """The ranks' shards of one global batch cover every complex once and balance the atoms."""
    import numpy as np
    from cms_cuda import synth
    from cms_cuda.shard import balanced_shards
    nt, nb, lig = synth.batched_sizes(4096 * 4, 2)
    shards = balanced_shards(nt.astype(np.int64) + nb, 4)
    allidx = np.sort(np.concatenate(shards))
    assert np.array_equal(allidx, np.arange(4096 * 4))
    loads = [int((nt[s] + nb[s]).sum()) for s in shards]
    assert max(loads) - min(loads) <= int((nt + nb).max())
    # a shard is generated alone, identical to its complexes in the whole batch
    b = synth.config_batched(64, 2, select=[3, 40])
    full_sizes = synth.batched_sizes(64, 2)
    assert list(np.diff(b.atom_off)) == [int(full_sizes[0][c] + full_sizes[1][c]) for c in (3, 40)]
