#!/usr/bin/env python
"""
Benchmark: batched CMS + SC + gradient throughput (complexes/s) on B200.

Workload: 4096 synthetic complexes per GPU of uneven size (target log-uniform
600-4000 heavy atoms, binder log-uniform 80-1200, ~5 % ligand-like 20-60 atom
binders), seeded; each step runs the whole pipeline on the whole batch --
attention, neighbour lists, pairs/triples, convex/toroidal/concave dots with
burial, CMS of both sides, shape complementarity and the FP64 adjoint of the
target-side CMS -- as one replay of a captured CUDA graph.  Inputs (9 M atoms,
~290 MB of coordinates) are larger than L2, so no flush is needed between
steps.

  value     device time of K graph replays with inputs resident (CUDA events on
            the pipeline's stream), max over ranks, all ranks' complexes
  e2e       the public batch API from pinned host buffers: upload, pipeline,
            per-complex results and gradients back to the host, every step
            (BatchCalculator.run_stream: the copies of neighbouring steps
            overlap the pipeline)
  roofline  the dominant stage against its bound; rooflines: every stage
  plain_gpu one complex per call through the drop-in calculator on the same GPU
            (the reference's usage pattern), for the batched-vs-plain ratio
  single_complex  per-complex latency of the public API on the two plain
            configurations (450 + 1200 and 1800 + 8000 atoms)
  differentiation 512 complexes of 2000 + 500 atoms: CMS + gradient throughput
            and the gradient's error against finite differences and torch
            FP64 autograd of the same fixed-topology formula
  pose_refinement 256 complexes, 200 captured ascent steps
  cpu_baseline    the CPU oracle (NumPy restatement of the reference) on
            stratified samples, all host cores; the one place besides the
            reference arm where this script runs the oracle

--impl reference times the reference's CPU algorithm (the oracle port: the
reference itself is a Python package that cannot be installed on the GPU
box) on all host cores, on bounded samples of the same workload.

--gpus N > 1 without a launcher starts N ranks with torch.distributed.run.
Multi-GPU is replicas only (weak scaling): one global batch of 4096 x N
complexes is split by cost over the ranks, each rank evaluates its share with
no data-path collective, and per-complex results are gathered to rank 0.
"""

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
for _p in (ROOT, os.path.join(ROOT, "cms-cuda_b200")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np

METRIC = "complexes/s CMS+SC(+grad), batched vs plain GPU path, dot counts bit-exact"
UNIT = "complexes/s"
WORKLOAD = ("batched 4096 complexes per GPU: target log-uniform 600-4000, binder log-uniform 80-1200 heavy atoms, "
            "~5% ligand binders of 20-60 atoms; surfaces + CMS (both sides) + SC + d(CMS)/d(xyz) per complex")


def parse(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--batch", type=int, default=4096, help="complexes per GPU")
    ap.add_argument("--seed", type=int, default=2)
    ap.add_argument("--cpu-sample", type=int, default=16, help="complexes of the CPU baseline's stratified sample")
    ap.add_argument("--plain-sample", type=int, default=32)
    ap.add_argument("--no-extras", action="store_true", help="the headline numbers only (profiling runs)")
    ap.add_argument("--refine-steps", type=int, default=200, help="pose-refinement steps of the refinement report")
    ap.add_argument("--refine-batch", type=int, default=256)
    ap.add_argument("--diff-batch", type=int, default=512, help="complexes of the differentiation report (0: skip)")
    return ap.parse_args(argv)


def dist_env():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


def self_launch(args):
    """--gpus N without a launcher: run this script on N ranks (one per GPU) and return their status."""
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    # the ranks' process group times out after 600 s; the launcher as a whole is bounded well above that
    cmd = ["timeout", "-k", "60", "3600", sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           f"--nproc-per-node={args.gpus}", "--master-addr", "127.0.0.1", f"--master-port={port}",
           os.path.abspath(__file__)] + sys.argv[1:]
    return subprocess.run(cmd).returncode


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.QUERY,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.file, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.file.flush()
        self.file.seek(0)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.file.read().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.file.name)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------
# CPU baselines: the oracle (a NumPy restatement of the reference) on the
# host cores.  The oracle is the checker and the baseline here, never the
# product: nothing measured on the GPU goes through it.
# ---------------------------------------------------------------------------
def _oracle_task(task):
    """Worker (spawned process): ('cms_sc' | 'cms' | 'max', inputs) -> (seconds, values)."""
    kind, arrays = task
    from oracle import cms_oracle
    t = time.perf_counter()
    if kind == "max":
        mx, _, _ = cms_oracle.run_max_cms(*arrays)
        out = {"max_cms": float(mx)}
    else:
        r = cms_oracle.run_complex(*arrays, sc=kind == "cms_sc")
        S = r["surface"]
        out = {"cms": float(r["cms"]), "dots": [len(S.dot_arrays[0]["area"]), len(S.dot_arrays[1]["area"])]}
        if kind == "cms_sc":
            out["sc"] = float(r["sc"])
    return time.perf_counter() - t, out


def _pool(cores):
    import multiprocessing as mp
    os.environ.setdefault("OMP_NUM_THREADS", "1")
    return mp.get_context("spawn").Pool(cores)


def stratified_sample(sizes, ligand, k):
    """
    k complexes spread over the whole size range (evenly spaced ranks of the
    size order, smallest and largest included), at least two of them with a
    ligand binder (the smallest and largest such complex replace the nearest
    protein picks).
    """
    order = np.argsort(sizes, kind="stable")
    k = max(2, min(k, len(order)))
    pick = [int(order[int(round(q * (len(order) - 1)))]) for q in np.linspace(0.0, 1.0, k)]
    lig = [int(c) for c in order if ligand[c]]
    for c in (lig[:1] + lig[-1:]) if len(lig) >= 2 else lig:
        if c in pick:
            continue
        # replace the protein pick nearest in size
        prot = [i for i, p in enumerate(pick) if not ligand[p] and i not in (0, len(pick) - 1)]
        if prot:
            j = min(prot, key=lambda i: abs(int(sizes[pick[i]]) - int(sizes[c])))
            pick[j] = c
    return sorted(set(pick), key=lambda c: sizes[c])


def _fit_extrapolation(sample_sizes, sample_secs, all_sizes):
    """Per-complex CPU seconds ~ a * atoms^b (least squares in log space), summed over the whole batch."""
    x, y = np.log(np.asarray(sample_sizes, float)), np.log(np.asarray(sample_secs, float))
    b, a = np.polyfit(x, y, 1)
    pred = np.exp(a) * np.asarray(all_sizes, float) ** b
    return float(pred.sum()), float(b)


def cpu_baseline_batched(batch, k, cores):
    """The oracle on a stratified sample of the batched workload, one complex per core."""
    sizes = np.diff(batch.atom_off)
    idx = stratified_sample(sizes, batch.ligand, k)
    cores = max(1, min(cores, len(idx)))
    with _pool(cores) as pool:
        t0 = time.perf_counter()
        res = pool.map(_oracle_task, [("cms_sc", batch.complex(c)) for c in idx], chunksize=1)
        wall = time.perf_counter() - t0
    secs = [r[0] for r in res]
    total_cpu, expo = _fit_extrapolation(sizes[idx], secs, sizes)
    per_core = len(idx) / sum(secs)
    return {"value": len(idx) / wall, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{len(idx)} complexes of the batch stratified over its whole size range "
                      f"({int(sizes[idx].min())}-{int(sizes[idx].max())} atoms, {int(np.sum(batch.ligand[idx]))} "
                      f"ligand binders), CMS both sides + SC, {cores} processes, {wall:.1f} s wall "
                      f"(the reference has no gradient)",
            "per_core_complexes_per_s": per_core,
            "sample_cpu_seconds": [round(s, 3) for s in secs],
            "workload_extrapolation": {
                "model": f"cpu seconds per complex ~ atoms^{expo:.2f} (fit on the sample)",
                "whole_batch_cpu_seconds": total_cpu,
                "complexes_per_s_per_core": batch.B / total_cpu,
                "complexes_per_s_on_these_cores": cores * batch.B / total_cpu}}


def cpu_baseline_single(cores, large_max=False):
    """The oracle's per-complex times on the two plain configurations (CMS, CMS + SC, max-CMS)."""
    from cms_cuda import synth
    tasks, keys = [], []
    for name, make in (("450+1200", synth.config_plain_small), ("1800+8000", synth.config_plain_large)):
        bx, br, tx, tr = make(0)
        tasks += [("cms", (bx, br, tx, tr)), ("cms_sc", (bx, br, tx, tr))]
        keys += [(name, "cms"), (name, "cms_sc")]
        if name == "450+1200" or large_max:
            tasks.append(("max", (tx, tr)))
            keys.append((name, "max_cms"))
    with _pool(max(1, min(cores, len(tasks)))) as pool:
        res = pool.map(_oracle_task, tasks, chunksize=1)
    out = {}
    for (name, what), (secs, vals) in zip(keys, res):
        out.setdefault(name, {})[f"{what}_s"] = round(secs, 3)
        out[name][f"{what}_value"] = vals.get("max_cms" if what == "max_cms" else "cms")
    if not large_max:
        out["1800+8000"]["max_cms_s"] = None
        out["1800+8000"]["note"] = "max-CMS of the 8000-atom target not timed on the CPU (needs about 40 GB of RAM)"
    return out


def cpu_check_poses(xyz, radius, atom_off, n_binder, complexes, batched_cms, cores):
    """The oracle's CMS of refined final poses (time per pose and agreement with the batched GPU value)."""
    tasks = []
    for c in complexes:
        a0, a1, n = int(atom_off[c]), int(atom_off[c + 1]), int(n_binder[c])
        tasks.append(("cms", (xyz[a0:a0 + n], radius[a0:a0 + n], xyz[a0 + n:a1], radius[a0 + n:a1])))
    with _pool(max(1, min(cores, len(tasks)))) as pool:
        res = pool.map(_oracle_task, tasks, chunksize=1)
    rel = [abs(batched_cms[c] - r[1]["cms"]) / max(1.0, abs(r[1]["cms"])) for c, r in zip(complexes, res)]
    return {"complexes": [int(c) for c in complexes], "oracle_seconds": [round(r[0], 3) for r in res],
            "max_rel_diff_vs_oracle": float(max(rel)), "within_1e-12": bool(max(rel) <= 1e-12)}


def run_reference(args):
    """The reference's CPU algorithm on all host cores, bounded samples of the workload."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    from cms_cuda import synth
    batch = synth.config_batched(args.batch, args.seed)
    cores = os.cpu_count() or 1
    sizes = np.diff(batch.atom_off)
    # per step: one complex per core, rotating through a sample stratified over the whole size range
    pool_idx = stratified_sample(sizes, batch.ligand, max(cores, 16))
    with _pool(cores) as pool:
        def step(s):
            sel = [pool_idx[(s * cores + i) % len(pool_idx)] for i in range(cores)]
            t = time.perf_counter()
            pool.map(_oracle_task, [("cms_sc", batch.complex(c)) for c in sel], chunksize=1)
            return len(sel), time.perf_counter() - t
        for s in range(args.warmup):
            step(s)
        n, secs = 0, 0.0
        for s in range(args.steps):
            a, b = step(args.warmup + s)
            n += a
            secs += b
    value = n / secs
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * secs / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator)",
            "impl": "reference",
            "config": {"workload": WORKLOAD, "sample_per_step": f"{cores} complexes, one per core",
                       "inputs": "the batch is generated by the repository's seeded C generator (libcms_synth.so), "
                                 "outside the timed region"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": f"{cores} complexes per step rotating through {len(pool_idx)} complexes "
                                       f"stratified over the batch's whole size range "
                                       f"({int(np.sum(batch.ligand[pool_idx]))} ligand binders), "
                                       f"CMS both sides + SC (the reference has no gradient)"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# rooflines
# ---------------------------------------------------------------------------
# Algorithmic bytes of the surface stages (HBM-bound by convention): 34 B read
# per atom (xyz 24, radius 8, molecule 1, attention 1), 12 B per neighbour
# entry (id 4 + d2 8), 4 B per buried-partner entry, 62 B per emitted dot
# (coordinates 24, normal 24, area 8, buried 1, type 1, atom 4), 4 B per
# neighbour entry read by a generating unit, 68 B per probe (3 ids 12,
# height 8, centre 24, direction 24), 8 B per toroid pair.  The triple count
# pass also writes each probe to the stash (76 B: the probe and its final
# slot), which the scatter reads back before writing the probe arrays.  The
# CMS adjoint reads 4 B per buried entry (its complex & molecule), and per
# entry of the differentiated side (half the entries) the query and reference
# points 48 B, the area 8 B and the nearest index 4 B, and writes the dot
# adjoint 32 B; it writes 24 B of gradient per atom.
def stage_bytes(name, t, work=None):
    nb4 = 4 * t["nb_entries"]
    nbur = (work or {}).get("cms_queries")
    table = {
        "neighbor_count": 34 * t["atoms"],
        "neighbor_emit": 34 * t["atoms"] + 12 * t["nb_entries"] + 4 * t["bu_entries"],
        "triples_count": nb4 + 76 * t["probes"],
        "triples_emit": (76 + 68) * t["probes"],
        "convex_count": nb4,
        "convex_emit": nb4 + 62 * t["convex"],
        "toroidal_count": 8 * t["toroids"] + nb4,
        "toroidal_emit": 8 * t["toroids"] + nb4 + 62 * t["toroidal"],
        "concave_count": 68 * t["probes"],
        "concave_emit": 68 * t["probes"] + 62 * t["concave"],
        "cms_backward": None if nbur is None else 4 * nbur + (48 + 8 + 4 + 32) * nbur // 2 + 24 * t["atoms"],
    }
    return table.get(name)


# DRAM traffic per unit of work (dram__bytes_read.sum + dram__bytes_write.sum of
# one launch, ncu on the 256-complex batch of this generator, divided by that
# batch's units); scaled by the units of the measured batch
TRAFFIC_PER_UNIT = {
    "neighbor_count": (78.47e6 / 558670, "atoms"),         # per atom
    "neighbor_emit": (163.85e6 / 558670, "atoms"),
    "triples_count": (95.88e6 / 558670, "atoms"),
    "cms_nn": (273.01e6 / 2750610, "cms_queries"),         # per query dot (k_nn_w, 4 queries per lane)
    "sc_band_nn": (251.90e6 / 2750610, "band_queries"),
}

# FP64 pipe utilisation of the FP64-bound stages (sm__pipe_fp64_cycles_active %, ncu --set full on the
# 256-complex batch; the captures under profiles/; stages whose kernels changed since their capture are left out)
FP64_PIPE_PCT = {
    "triples_count": (19.6, "profiles/fp64_count_passes_256_complexes.md"),
    "cms_backward": (19.6, "profiles/k_adj_units_256_complexes.md"),
}
NN_STAGES = {"cms_nn": "cms", "sc_band_nn": "band", "sc_argmin_nn": "sc"}
NN_WORK_KEYS = {"cms": ("cms_pairs", "cms_queries"), "band": ("band_pairs", "band_queries"),
                "sc": ("sc_pairs", "sc_queries")}

# when no measured peaks file is present: an earlier STREAM-style copy on this GPU pool
FALLBACK_HBM_GBS = 6650.0


def stage_traffic(name, totals, work):
    t = TRAFFIC_PER_UNIT.get(name)
    if t is None:
        return None
    per, unit = t
    n = totals.get(unit, work.get(unit))
    return None if n is None else per * n


def _hbm_peak(peaks):
    hbm = peaks.get("hbm_gbs")
    if hbm:
        return float(hbm), "MEASURED_PEAKS.json hbm_gbs (of measured)"
    return FALLBACK_HBM_GBS, "fallback copy bandwidth of this GPU pool, 6.65 TB/s (of fallback)"


def stage_entry(name, ms, work, totals, peaks, fp32_peak, evaluated=None):
    """Roofline of one pipeline stage: a nearest-dot search against the measured FP32 throughput, a surface
    stage (and the adjoint) against the measured HBM bandwidth, anything else as latency."""
    if name in NN_STAGES:
        key = NN_STAGES[name]
        brute = work[NN_WORK_KEYS[key][0]]
        ev = (evaluated or {}).get(f"{key}_evaluated")
        pairs = ev if ev is not None else brute
        achieved = 8.0 * pairs / (ms * 1e-3) / 1e12
        e = {"bound": "fp32", "kernel": f"k_nn ({name})", "ms": ms, "achieved": achieved, "peak": fp32_peak,
             "unit": "TFLOP/s", "frac": achieved / fp32_peak if fp32_peak else None,
             "traffic": stage_traffic(name, totals, work),
             "pairs": "evaluated by the FP32 filter after box culling (counted on the device)" if ev is not None
                      else "full brute force (no evaluated count)",
             "evaluated_pairs": ev, "brute_force_pairs": brute,
             "brute_force_equivalent_tflops": 8.0 * brute / (ms * 1e-3) / 1e12,
             "fp64_rechecks": (evaluated or {}).get(f"{key}_rechecks"),
             "peak_source": "measured FP32 FMA throughput of this GPU (cms_fp32_peak, in this run)"}
        return e
    nbytes = stage_bytes(name, totals, work)
    if nbytes is None:
        return {"bound": "latency", "kernel": name, "ms": ms}
    hbm, source = _hbm_peak(peaks)
    achieved = nbytes / (ms * 1e-3) / 1e9
    e = {"bound": "hbm", "kernel": name, "ms": ms, "achieved": achieved, "peak": hbm, "unit": "GB/s",
         "frac": achieved / hbm, "traffic": stage_traffic(name, totals, work), "algorithmic_bytes": nbytes,
         "peak_source": source}
    if name in FP64_PIPE_PCT:
        e["fp64_pipe_active_pct"], e["fp64_pipe_source"] = FP64_PIPE_PCT[name]
        e["note"] = "FP64 geometry: bound by FP64 issue latency, not HBM"
    return e


def stage_roofline(stages, work, totals, peaks, fp32_peak, evaluated=None):
    """Roofline of the most expensive stage."""
    name = max(stages, key=lambda k: stages[k])
    return stage_entry(name, stages[name], work, totals, peaks, fp32_peak, evaluated)


def stage_rooflines(stages, work, totals, peaks, fp32_peak, evaluated=None):
    step = sum(stages.values())
    out = {}
    for name, ms in stages.items():
        if ms <= 0:
            continue
        e = stage_entry(name, ms, work, totals, peaks, fp32_peak, evaluated)
        e["share"] = ms / step
        out[name] = e
    return out


# ---------------------------------------------------------------------------
# GPU reports beside the headline
# ---------------------------------------------------------------------------
def plain_path(batch, local, totals, sc, grad_dev, sample):
    """
    One complex per call through the drop-in calculator (CMS, SC, gradient;
    the reference's usage pattern), after warming one pooled context on a
    complex of every size class of the sample (so no workspace growth falls
    in the timed calls); per-complex latency with a synchronised clock.
    """
    import torch
    from cms_cuda import MolecularSurfaceCalculator
    idx = list(range(min(sample, batch.B)))
    sizes = np.diff(batch.atom_off)[idx]
    warm = [idx[i] for i in np.argsort(sizes)[np.linspace(0, len(idx) - 1, 4).astype(int)]]
    for c in warm + [idx[int(np.argmax(sizes))]]:
        m = MolecularSurfaceCalculator(local)
        m.add_binder_and_target(*batch.complex(c))
        m.CalcLoaded(); m.CalcLoadedSC(); m.calc_contact_molecular_surface_gradient(True)
        del m
    torch.cuda.synchronize(local)
    lat, match = [], True
    for c in idx:
        t0 = time.perf_counter()
        m = MolecularSurfaceCalculator(local)
        m.add_binder_and_target(*batch.complex(c))
        cms, _ = m.CalcLoaded()
        s = m.CalcLoadedSC()
        g = m.calc_contact_molecular_surface_gradient(True)
        lat.append(time.perf_counter() - t0)
        a0, a1 = int(batch.atom_off[c]), int(batch.atom_off[c + 1])
        match &= (cms == totals[c, 1]) and (s[0] == sc[c, 0]) and bool(np.array_equal(g, grad_dev[a0:a1]))
        del m
    lat = np.array(lat)
    return {"value": len(idx) / lat.sum(), "unit": UNIT, "median_latency_ms": float(1e3 * np.median(lat)),
            "p90_latency_ms": float(1e3 * np.percentile(lat, 90)),
            "sample": f"first {len(idx)} complexes of the batch ({int(sizes.min())}-{int(sizes.max())} atoms, mean "
                      f"{int(sizes.mean())}), one per call (CMS, SC, gradient), after warming the pooled context "
                      f"on every size class",
            "python_trace_hook_active": bool(sys.gettrace() or sys.getprofile()),
            "results_match_batched": bool(match)}


def single_complex(local, repeats=5):
    """Latency of the public API (host arrays in, results on the host) on the two plain configurations."""
    import torch
    from cms_cuda import (calculate_contact_ms, calculate_maximum_possible_contact_ms,
                          calculate_shape_complementarity, synth)
    out = {}
    for name, make in (("450+1200", synth.config_plain_small), ("1800+8000", synth.config_plain_large)):
        bx, br, tx, tr = make(0)
        calls = {"cms": lambda: calculate_contact_ms(bx, br, tx, tr)[0],
                 "sc": lambda: calculate_shape_complementarity(bx, br, tx, tr)[0],
                 "max_cms": lambda: calculate_maximum_possible_contact_ms(tx, tr)[0]}
        row = {"binder_atoms": len(br), "target_atoms": len(tr)}
        for what, f in calls.items():
            f()
            torch.cuda.synchronize(local)
            ts = []
            for _ in range(repeats):
                t0 = time.perf_counter()
                v = f()
                ts.append(time.perf_counter() - t0)
            row[f"{what}_ms"] = round(1e3 * float(np.median(ts)), 3)
            row[f"{what}_value"] = float(v)
        out[name] = row
    return out


def _dir_topology(ctx, B, side=1):
    """What the gradient holds fixed, per complex: dot counts, burial, type, owner, nearest-dot choices."""
    out = []
    for c in range(B):
        info = ctx.info(c)
        t = [(tuple(info.n_dots), info.convex, info.toroidal, info.concave, info.n_probes)]
        pts = []
        for m in (0, 1):
            coor, _, _, bur, typ, atom = ctx.export_dots(c, m, info)
            t.append((bur.tobytes(), typ.tobytes(), atom.tobytes()))
            pts.append(coor[bur.astype(bool)])
        q, r = pts[side], pts[1 - side]
        t.append(ctx.nearest_dots(q, r)[1].tobytes() if len(q) and len(r) else b"")
        out.append(t)
    return out


def differentiation(local, B, steps, warmup, n_check=8, seed=4):
    """
    512 complexes of 2000 + 500 atoms: CMS + d(CMS)/d(xyz) throughput through
    the captured graph, then the gradient of n_check of them against central
    finite differences (1e-5 A steps on directions that keep the topology)
    and against torch FP64 autograd of the fixed-topology formula.
    """
    import torch
    from cms_cuda import _lib, synth
    b = synth.make_batch(np.full(B, 2000), np.full(B, 500), seed)
    ctx = _lib.Context(local)
    ctx.load_batch(b.atom_off, b.n_binder, b.xyz, b.radius)
    ctx.set_backward(True, target_side=True)
    ctx.run_graph()
    for _ in range(warmup):
        ctx.graph_launch()
    ctx.graph_check()
    torch.cuda.synchronize(local)
    t0 = time.perf_counter()
    for _ in range(steps):
        ctx.graph_launch()
    ctx.graph_check()
    secs = (time.perf_counter() - t0) / steps
    del ctx

    # gradient checks on n_check complexes loaded as their own batch
    sub = synth.make_batch(np.full(B, 2000), np.full(B, 500), seed, select=np.arange(n_check))
    X, R, off, nb = sub.xyz, sub.radius, sub.atom_off, sub.n_binder
    ctx = _lib.Context(local)
    ctx.load_batch(off, nb, X, R)
    ctx.generate(all_atoms=False)
    ctx.contact_ms(per_atom=False)
    grad = ctx.contact_ms_backward(True)
    base = _dir_topology(ctx, n_check)
    h = 1e-5
    rng = np.random.default_rng(11)
    fd_err, fd_checked, fd_skipped = [], 0, 0
    for d in range(6):
        V = np.zeros_like(X)
        for c in range(n_check):
            a0, a1 = int(off[c]), int(off[c + 1])
            g = grad[a0:a1].reshape(-1)
            if d < 3:        # the coordinates with the largest gradients, one at a time
                v = np.zeros_like(g)
                v[np.argsort(-np.abs(g))[d]] = 1.0
            else:            # whole-complex random directions
                v = rng.normal(size=g.shape)
                v /= np.linalg.norm(v)
            V[a0:a1] = v.reshape(-1, 3)
        vals, topo = [], []
        for sgn in (1.0, -1.0):
            ctx.load_batch(off, nb, X + sgn * h * V, R)
            ctx.generate(all_atoms=False)
            vals.append(ctx.contact_ms(per_atom=False)[1][:, 1])
            topo.append(_dir_topology(ctx, n_check))
        for c in range(n_check):
            if topo[0][c] != base[c] or topo[1][c] != base[c]:
                fd_skipped += 1
                continue
            a0, a1 = int(off[c]), int(off[c + 1])
            fd = (vals[0][c] - vals[1][c]) / (2 * h)
            an = float((grad[a0:a1] * V[a0:a1]).sum())
            fd_err.append(abs(fd - an) / max(1.0, abs(an)))
            fd_checked += 1

    # torch FP64 autograd of the same fixed-topology formula (test infrastructure: tests/torch_cms_formula.py)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import torch_cms_formula as F
    ctx.load_batch(off, nb, X, R)
    ctx.generate(all_atoms=False)
    ctx.contact_ms(per_atom=False)
    ag_err = []
    for c in range(n_check):
        a0, a1 = int(off[c]), int(off[c + 1])
        topo = F.topology(ctx, c, nearest=ctx.nearest_dots)
        Xt = torch.tensor(X[a0:a1], dtype=torch.float64, requires_grad=True)
        F.contact_ms(Xt, R[a0:a1], 1.7, 0.5, topo, 1).backward()
        ref = Xt.grad.numpy()
        ag_err.append(float(np.abs(ref - grad[a0:a1]).max() / max(1.0, np.abs(ref).max())))
    return {"complexes": B, "atoms_per_complex": "2000 + 500", "complexes_per_s": B / secs,
            "ms_per_step": 1e3 * secs,
            "step": "surfaces + CMS both sides + SC + d(target CMS)/d(xyz), one graph replay",
            "gradient_checked_complexes": n_check,
            "max_rel_err_fd": float(max(fd_err)) if fd_err else None,
            "fd_checks": fd_checked, "fd_directions_changing_topology": fd_skipped,
            "max_rel_err_autograd": float(max(ag_err)),
            "rel_err_definition": "fd: |FD - g.v| / max(1, |g.v|), central differences with 1e-5 A steps on "
                                  "directions keeping counts, burial, owners and nearest-dot choices; autograd: "
                                  "max |g - g_torch| / max(1, max |g_torch|) per complex"}


def pose_refinement(args, device):
    """
    Rigid-body refinement of a batch of perturbed complexes (random rotations
    up to 15 degrees and shifts up to 2 A from contact): CMS gain, steps/s,
    and the final poses evaluated afresh (batched, and per complex through
    the plain calculator).
    """
    from cms_cuda import MolecularSurfaceCalculator, synth, _lib
    from cms_cuda.refine import perturb_binders, refine_poses
    b = synth.config_refine(args.refine_batch, 5)
    x0 = perturb_binders(b.xyz, b.atom_off, b.n_binder, max_deg=15.0, max_shift=2.0, seed=17)
    res = refine_poses(b.atom_off, b.n_binder, x0, b.radius, steps=args.refine_steps, device=device)
    final = res.history[-1]
    ctx = _lib.Context(device)
    ctx.load_batch(b.atom_off, b.n_binder, res.xyz, b.radius)
    ctx.generate(all_atoms=False)
    _, tot = ctx.contact_ms(per_atom=False)
    diffs = []
    for c in range(min(16, b.B)):
        a0, a1, n = int(b.atom_off[c]), int(b.atom_off[c + 1]), int(b.n_binder[c])
        m = MolecularSurfaceCalculator(device)
        m.add_binder_and_target(res.xyz[a0:a0 + n], b.radius[a0:a0 + n], res.xyz[a0 + n:a1], b.radius[a0 + n:a1])
        diffs.append(abs(m.CalcLoaded()[0] - tot[c, 1]))
    report = {"complexes": int(b.B), "atoms": int(b.N), "steps": res.steps, "steps_per_s": res.steps_per_s,
              "complex_steps_per_s": res.steps_per_s * b.B,
              "cms_start_mean": float(res.initial.mean()), "cms_final_mean": float(final.mean()),
              "cms_best_mean": float(res.best.mean()), "cms_gain_mean": float((final - res.initial).mean()),
              "complexes_improved": int((final > res.initial).sum()),
              "final_pose_plain_vs_batched_max_abs_diff": float(max(diffs)) if diffs else None,
              "start": "random rotation <= 15 deg about the binder centroid and shift <= 2 A from contact",
              "step": "clipped gradient ascent, <= 0.05 A and <= 0.5 deg per step"}
    return report, (res.xyz, b.radius, b.atom_off, b.n_binder, tot[:, 1])


# ---------------------------------------------------------------------------
# our implementation
# ---------------------------------------------------------------------------
def rank_batch(per_gpu, seed, rank, world):
    """
    This rank's share of one global batch of per_gpu * world complexes, split
    by cost (atoms) over the ranks: (global size, global indices, the batch of
    those complexes, each identical to its copy in the whole batch).
    """
    from cms_cuda import synth
    from cms_cuda.shard import balanced_shards
    B_global = per_gpu * world
    if world == 1:
        batch = synth.config_batched(B_global, seed)
        return B_global, np.arange(batch.B), batch
    nt, nb, _ = synth.batched_sizes(B_global, seed)
    mine = balanced_shards(nt.astype(np.int64) + nb, world)[rank]
    return B_global, mine, synth.config_batched(B_global, seed, select=mine)


def run_ours(args):
    import torch
    import torch.distributed as dist
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=dev)
    from cms_cuda import _lib
    from cms_cuda.shard import gather_per_complex, max_over_ranks

    B_global, mine, batch = rank_batch(args.batch, args.seed, rank, world)
    B, N = batch.B, batch.N
    # pinned host inputs for the end-to-end path
    xyz_h = torch.from_numpy(batch.xyz).pin_memory()
    rad_h = torch.from_numpy(batch.radius).pin_memory()
    xyz_np, rad_np = xyz_h.numpy(), rad_h.numpy()

    stream = torch.cuda.Stream(device=dev)
    ctx = _lib.Context(local, stream=stream.cuda_stream)
    ctx.load_batch(batch.atom_off, batch.n_binder, xyz_np, rad_np)
    ctx.set_backward(True, target_side=True)         # each step: surfaces, CMS, SC and d(CMS)/d(xyz)
    ctx.run_graph()                                  # sizes the workspace, captures, replays once
    infos = [ctx.info(c) for c in range(B)]
    statuses = [i.status for i in infos]
    surf = {"atoms": N, "nb_entries": sum(i.nb_entries for i in infos), "bu_entries": sum(i.bu_entries for i in infos),
            "probes": sum(i.n_probes for i in infos), "toroids": sum(i.n_toroid for i in infos),
            "convex": sum(i.convex for i in infos), "toroidal": sum(i.toroidal for i in infos),
            "concave": sum(i.concave for i in infos)}
    work = ctx.nn_work()
    launches = ctx.kernel_launches()
    tv, tms = ctx.nn_variants()
    autotune = {stage: {"shape": _lib.NN_VARIANT_NAMES[tv[k]],
                        "ms": {_lib.NN_VARIANT_NAMES[v]: round(float(tms[k, v]), 3) for v in range(4)}}
                for k, stage in enumerate(("cms_nn", "sc_band_nn", "sc_argmin_nn"))}
    sv, sms = ctx.surface_variants()
    for k, stage in enumerate(_lib.SURFACE_STAGES):
        names = _lib.SURFACE_VARIANT_NAMES[stage.split("_")[0]]
        autotune[stage] = {"shape": names[sv[k]],
                           "ms": {names[v]: round(float(sms[k, v]), 3) for v in range(_lib.SURFACE_VARIANTS)}}
    free_b, total_b = torch.cuda.mem_get_info(dev)
    device_gb = (total_b - free_b) / 1e9             # whole GPU in use while the context holds its workspace

    # ---- device throughput: graph replays with inputs resident -------------
    for _ in range(args.warmup):
        ctx.graph_launch()
    stream.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    clk = ClockSampler(local)
    clk.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        ctx.graph_launch()
    e1.record(stream)
    e1.synchronize()
    clocks = clk.stop()
    ms = e0.elapsed_time(e1) / args.steps
    ctx.graph_check()
    torch.cuda.synchronize(dev)
    ms_max = max_over_ranks(ms)                      # the job is as fast as its slowest replica
    if world > 1:
        dist.barrier()
    value = B_global / (ms_max * 1e-3)
    _, totals = ctx.contact_ms(per_atom=False)
    sc, _ = ctx.shape_complementarity()
    grad_dev = ctx.grad_xyz()
    # per-complex results of every rank, in global order on rank 0
    gathered = gather_per_complex(np.stack([totals[:, 1], sc[:, 0]], 1), mine, B_global)

    extras = {}
    if rank == 0 and world == 1 and not args.no_extras:
        stages = ctx.profile_stages()
        fp32 = ctx.fp32_peak()
        evaluated = ctx.nn_evaluated()
        peaks = {}
        pk = os.path.join(ROOT, "MEASURED_PEAKS.json")
        if os.path.exists(pk):
            with open(pk) as f:
                peaks = json.load(f)
        extras["roofline"] = stage_roofline(stages, work, surf, peaks, fp32, evaluated)
        extras["rooflines"] = stage_rooflines(stages, work, surf, peaks, fp32, evaluated)
        extras["surface_totals"] = surf
        extras["device_memory_gb"] = round(device_gb, 1)
        extras["stages_ms"] = {k: round(v, 3) for k, v in stages.items()}
        extras["nn_work"] = {**work, **evaluated}
    del ctx
    torch.cuda.synchronize(dev)

    # ---- end to end through the public batch API ---------------------------
    # BatchCalculator.run_stream: every step uploads its coordinates and radii from pinned host memory and
    # reads its results and gradient back to pinned host memory; the copies of neighbouring steps overlap
    # the pipeline (a copy stream), as a service evaluating a stream of batches would run
    from cms_cuda.batch import BatchCalculator
    bc = BatchCalculator(local)
    grad_h = [torch.empty((xyz_np.shape[0], 3), dtype=torch.float64).pin_memory().numpy() for _ in range(2)]
    step_in = (batch.atom_off, batch.n_binder, xyz_np, rad_np)
    bc.load(*step_in)
    bc.run(graph=True, grad=True)
    bc.run_stream([step_in] * max(args.warmup, 1), [grad_h[k % 2] for k in range(max(args.warmup, 1))])
    h0, d0 = bc.ctx.transfer_bytes()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    res = bc.run_stream([step_in] * args.steps, [grad_h[k % 2] for k in range(args.steps)])
    e2e_s = (time.perf_counter() - t0) / args.steps
    h1, d1 = bc.ctx.transfer_bytes()
    r = res[-1]
    same = bool(np.array_equal(r.cms, totals[:, 1]) and np.array_equal(r.sc, sc[:, 0]) and
                np.array_equal(r.grad, grad_dev))
    del bc
    e2e = {"value": B_global / max_over_ranks(e2e_s), "unit": UNIT,
           "h2d_bytes_per_step": (h1 - h0) // args.steps + xyz_np.nbytes + rad_np.nbytes,
           "d2h_bytes_per_step": (d1 - d0) // args.steps + grad_h[0].nbytes,
           "api": "BatchCalculator.run_stream (uploads and gradient downloads of neighbouring steps overlap the "
                  "pipeline on a copy stream)",
           "results_match_device_run": same}

    if rank == 0 and world == 1 and not args.no_extras:
        cores = os.cpu_count() or 1
        extras["plain_gpu"] = plain_path(batch, local, totals, sc, grad_dev, args.plain_sample)
        extras["batched_vs_plain"] = value / extras["plain_gpu"]["value"]
        extras["single_complex"] = single_complex(local)
        if args.diff_batch > 0:
            extras["differentiation"] = differentiation(local, args.diff_batch, max(3, args.steps // 2),
                                                        args.warmup)
        poses = None
        if args.refine_steps > 0:
            extras["pose_refinement"], poses = pose_refinement(args, local)
        # CPU legs (the oracle, on the host cores)
        extras["cpu_baseline"] = cpu_baseline_batched(batch, args.cpu_sample, cores)
        ram_gb = os.sysconf("SC_PAGE_SIZE") * os.sysconf("SC_PHYS_PAGES") / 1e9
        cpu_single = cpu_baseline_single(cores, large_max=ram_gb >= 96)
        for name, row in cpu_single.items():
            extras["single_complex"][name]["oracle_cpu"] = row
        if poses is not None:
            xyz_f, rad_f, off_f, nb_f, cms_f = poses
            extras["pose_refinement"]["final_pose_oracle_check"] = cpu_check_poses(
                xyz_f, rad_f, off_f, nb_f, list(range(min(4, len(nb_f)))), cms_f, cores)

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_max, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator, complexes of random residues)",
                "config": {"workload": WORKLOAD, "complexes": B_global, "complexes_per_gpu": args.batch,
                           "atoms_rank0": N,
                           "parallelism": f"replicas x{world}: one global batch split by cost over the GPUs, "
                                          f"no data-path collective",
                           "l2": "inputs larger than L2 (9M atoms), no flush",
                           "nn_search": "FP32 filter + FP64 recheck over every pair not excluded by a proven "
                                        "box-distance bound",
                           "grad": "included: d(target-side CMS)/d(xyz) of binder and target atoms, FP64 adjoint "
                                   "with the dot topology fixed, in every step"},
                "e2e": e2e, "gpu_launches": launches * args.steps, "clocks": clocks, "autotune": autotune,
                "complex_status_nonzero": int(sum(1 for s in statuses if s)),
                "gathered_complexes": int(np.isfinite(gathered).all(axis=1).sum()) if gathered is not None else None}
        line.update(extras)
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        sys.exit(self_launch(args))
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
