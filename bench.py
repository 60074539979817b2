#!/usr/bin/env python
"""
Benchmark: batched CMS + SC throughput (complexes/s) on B200.

Workload: 4096 synthetic complexes of uneven size (target log-uniform
600-4000 heavy atoms, binder log-uniform 80-1200, ~5 % ligand-like 20-60 atom
binders), seeded; each step runs the whole pipeline on the whole batch --
attention, neighbour lists, pairs/triples, convex/toroidal/concave dots with
burial, CMS of both sides and shape complementarity -- as one replay of a
captured CUDA graph.  Inputs (9 M atoms, ~290 MB of coordinates) are larger
than L2, so no explicit flush is needed between steps.

  value     device time of K graph replays with inputs resident (CUDA events on
            the pipeline's stream), max over ranks, all ranks' complexes
  e2e       the public batch API from pinned host buffers: upload, pipeline,
            per-complex results back to the host, every step
  plain_gpu one complex per call through the drop-in calculator (the reference's
            usage pattern) on the same GPU, for the batched-vs-plain ratio
  cpu_baseline  the CPU oracle (NumPy restatement of the reference) on a
            bounded sample, one core
  roofline  the dominant pipeline stage against its bound

--impl reference times the reference's CPU algorithm (the oracle port: the
reference itself is a Python package that cannot be installed on the GPU
box) on all host cores, on bounded samples of the same workload.

Multi-GPU (torchrun): weak scaling, each rank evaluates its own batch of
independent complexes; the only collective is the max of the step time.
"""

import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
for _p in (ROOT, os.path.join(ROOT, "cms-cuda_b200")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np

METRIC = "complexes/s CMS+SC(+grad), batched vs plain GPU path, dot counts bit-exact"
UNIT = "complexes/s"
WORKLOAD = ("batched 4096 complexes: target log-uniform 600-4000, binder log-uniform 80-1200 heavy atoms, "
            "~5% ligand binders of 20-60 atoms; surfaces + CMS (both sides) + SC per complex")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--batch", type=int, default=4096)
    ap.add_argument("--seed", type=int, default=2)
    ap.add_argument("--cpu-sample", type=int, default=2)
    ap.add_argument("--plain-sample", type=int, default=32)
    ap.add_argument("--no-extras", action="store_true", help="skip plain / CPU baselines (profiling runs)")
    ap.add_argument("--refine-steps", type=int, default=200, help="pose-refinement steps of the refinement report")
    ap.add_argument("--refine-batch", type=int, default=256)
    return ap.parse_args()


def dist_env():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


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
# CPU baselines (the oracle is the checker / baseline, never the product)
# ---------------------------------------------------------------------------
def _oracle_one(args):
    bx, br, tx, tr = args
    from oracle import cms_oracle
    t = time.perf_counter()
    out = cms_oracle.run_complex(bx, br, tx, tr, sc=True)
    return time.perf_counter() - t, out["cms"]


def sample_indices(batch, k, seed):
    """k complexes spread over the batch's size distribution (deterministic)."""
    sizes = np.diff(batch.atom_off)
    order = np.argsort(sizes, kind="stable")
    pos = np.linspace(0.2, 0.8, k) if k > 1 else np.array([0.5])
    return [int(order[int(p * (len(order) - 1))]) for p in pos]


def cpu_baseline_single(batch, k):
    idx = sample_indices(batch, k, 0)
    tot = 0.0
    for c in idx:
        dt, _ = _oracle_one(batch.complex(c))
        tot += dt
    atoms = int(np.mean([batch.atom_off[c + 1] - batch.atom_off[c] for c in idx]))
    return {"value": len(idx) / tot, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"{len(idx)} complexes of the batch (sizes at the 20-80th percentile, mean {atoms} atoms), "
                      f"CMS both sides + SC, one process, {tot:.1f} s (the reference has no gradient)"}


def run_reference(args):
    """The reference's CPU algorithm on all host cores, bounded samples of the workload."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    import multiprocessing as mp
    from cms_cuda import synth
    batch = synth.config_batched(args.batch, args.seed)
    cores = os.cpu_count() or 1
    # per step: one complex per core, rotating through a fixed sample of mid-sized complexes
    pool_idx = sample_indices(batch, max(cores, 8), 0)
    ctx = mp.get_context("spawn")
    os.environ.setdefault("OMP_NUM_THREADS", "1")
    with ctx.Pool(cores) as pool:
        def step(s):
            sel = [pool_idx[(s * cores + i) % len(pool_idx)] for i in range(cores)]
            t = time.perf_counter()
            pool.map(_oracle_one, [batch.complex(c) for c in sel])
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
            "config": {"workload": WORKLOAD, "sample_per_step": f"{cores} complexes, one per core"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": f"{cores} mid-sized complexes of the batch per step, CMS both sides + SC"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# our implementation
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
    "toroidal_emit": (365.19e6 / 5021616, "toroidal"),     # per toroidal dot
    "toroidal_count": (45.53e6 / 558670, "atoms"),         # per atom
    "triples_count": (105.68e6 / 558670, "atoms"),         # per atom
    "triples_emit": (19.46e6 / 558670, "atoms"),           # the probe scatter
    "cms_nn": (104.73e6 / 2750610, "cms_queries"),         # per query dot
    "sc_band_nn": (405.62e6 / 2750610, "band_queries"),
}


def stage_traffic(name, totals, work):
    t = TRAFFIC_PER_UNIT.get(name)
    if t is None:
        return None
    per, unit = t
    n = totals.get(unit, work.get(unit))
    return None if n is None else per * n


# when no measured peaks file is present: an earlier STREAM-style copy on this GPU pool
FALLBACK_HBM_GBS = 6650.0


def stage_roofline(stages, work, totals, peaks, fp32_peak):
    """Roofline of the most expensive stage: the nearest-dot search against the
    measured FP32 throughput (8 FLOP per pair), a surface stage against the
    measured HBM bandwidth (algorithmic bytes above)."""
    nn = {"cms_nn": work["cms_pairs"], "sc_band_nn": work["band_pairs"], "sc_argmin_nn": work["sc_pairs"]}
    name = max(stages, key=lambda k: stages[k])
    ms = stages[name]
    if name in nn:
        achieved = 8.0 * nn[name] / (ms * 1e-3) / 1e12
        return {"bound": "fp32", "kernel": f"k_nn ({name})", "achieved": achieved, "peak": fp32_peak,
                "unit": "TFLOP/s", "frac": achieved / fp32_peak, "traffic": stage_traffic(name, totals, work), "ms": ms,
                "peak_source": "measured FP32 FMA throughput of this GPU (cms_fp32_peak, in this run)"}
    hbm = peaks.get("hbm_gbs")
    source = "MEASURED_PEAKS.json hbm_gbs (of measured)"
    if not hbm:
        hbm, source = FALLBACK_HBM_GBS, "fallback copy bandwidth of this GPU pool, 6.65 TB/s (of fallback)"
    nbytes = stage_bytes(name, totals, work)
    achieved = nbytes / (ms * 1e-3) / 1e9 if nbytes is not None else None
    return {"bound": "hbm", "kernel": name, "achieved": achieved, "peak": hbm, "unit": "GB/s",
            "frac": (achieved / hbm) if achieved is not None else None,
            "traffic": stage_traffic(name, totals, work), "ms": ms,
            "algorithmic_bytes": nbytes,
            "peak_source": source,
            "note": "FP64 geometry: the stage is bound by FP64 issue latency, not HBM (ncu summaries under profiles/)"}


def pose_refinement(args, device):
    """
    Rigid-body refinement of a batch of perturbed complexes (random rotations
    up to 15 degrees and shifts up to 2 A from contact): CMS gain, steps/s, and
    the final poses' CMS from a fresh plain (one complex per call) evaluation.
    """
    from cms_cuda import MolecularSurfaceCalculator, synth
    from cms_cuda.refine import perturb_binders, refine_poses
    b = synth.config_refine(args.refine_batch, 5)
    x0 = perturb_binders(b.xyz, b.atom_off, b.n_binder, max_deg=15.0, max_shift=2.0, seed=17)
    res = refine_poses(b.atom_off, b.n_binder, x0, b.radius, steps=args.refine_steps, device=device)
    final = res.history[-1]
    # plain FP64 evaluation of the final poses (a sample of complexes)
    from cms_cuda import _lib
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
    return {"complexes": int(b.B), "atoms": int(b.N), "steps": res.steps, "steps_per_s": res.steps_per_s,
            "complex_steps_per_s": res.steps_per_s * b.B,
            "cms_start_mean": float(res.initial.mean()), "cms_final_mean": float(final.mean()),
            "cms_best_mean": float(res.best.mean()), "cms_gain_mean": float((final - res.initial).mean()),
            "complexes_improved": int((final > res.initial).sum()),
            "final_pose_plain_vs_batched_max_abs_diff": float(max(diffs)) if diffs else None,
            "start": "random rotation <= 15 deg about the binder centroid and shift <= 2 A from contact",
            "step": "clipped gradient ascent, <= 0.05 A and <= 0.5 deg per step"}


def run_ours(args):
    import torch
    import torch.distributed as dist
    rank, world, local = dist_env()
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    from cms_cuda import _lib, synth, MolecularSurfaceCalculator
    from cms_cuda.shard import max_over_ranks

    batch = synth.config_batched(args.batch, args.seed + 1000 * rank)
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
    value = world * B / (ms_max * 1e-3)
    _, totals = ctx.contact_ms(per_atom=False)
    sc, _ = ctx.shape_complementarity()
    grad_dev = ctx.grad_xyz()

    extras = {}
    if rank == 0 and world == 1 and not args.no_extras:
        stages = ctx.profile_stages()
        fp32 = ctx.fp32_peak()
        peaks = {}
        pk = os.path.join(ROOT, "MEASURED_PEAKS.json")
        if os.path.exists(pk):
            peaks = json.load(open(pk))
        extras["roofline"] = stage_roofline(stages, work, surf, peaks, fp32)
        extras["surface_totals"] = surf
        extras["device_memory_gb"] = round(device_gb, 1)
        extras["stages_ms"] = {k: round(v, 3) for k, v in stages.items()}
        extras["nn_work"] = work
    del ctx
    torch.cuda.synchronize(dev)

    # ---- end to end through the public batch API ---------------------------
    from cms_cuda.batch import BatchCalculator
    bc = BatchCalculator(local)
    grad_h = torch.empty((xyz_np.shape[0], 3), dtype=torch.float64).pin_memory().numpy()
    bc.load(batch.atom_off, batch.n_binder, xyz_np, rad_np)
    r = bc.run(graph=True, grad=True, grad_out=grad_h)
    for _ in range(args.warmup):
        bc.load(batch.atom_off, batch.n_binder, xyz_np, rad_np)
        r = bc.run(graph=True, grad=True, grad_out=grad_h)
    h0, d0 = bc.ctx.transfer_bytes()
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        bc.load(batch.atom_off, batch.n_binder, xyz_np, rad_np)
        r = bc.run(graph=True, grad=True, grad_out=grad_h)
    e2e_s = (time.perf_counter() - t0) / args.steps
    h1, d1 = bc.ctx.transfer_bytes()
    same = bool(np.array_equal(r.cms, totals[:, 1]) and np.array_equal(r.sc, sc[:, 0]) and
                np.array_equal(r.grad, grad_dev))
    del bc
    e2e = {"value": world * B / max_over_ranks(e2e_s), "unit": UNIT,
           "h2d_bytes_per_step": (h1 - h0) // args.steps, "d2h_bytes_per_step": (d1 - d0) // args.steps,
           "results_match_device_run": same}

    if rank == 0 and world == 1 and not args.no_extras:
        # plain GPU path: one complex per call through the drop-in calculator
        idx = list(range(min(args.plain_sample, B)))
        for c in idx[:2]:
            m = MolecularSurfaceCalculator(local)
            m.add_binder_and_target(*batch.complex(c))
            m.CalcLoaded(); m.CalcLoadedSC(); m.calc_contact_molecular_surface_gradient(True)
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        plain_match = True
        for c in idx:
            m = MolecularSurfaceCalculator(local)
            m.add_binder_and_target(*batch.complex(c))
            cms, _ = m.CalcLoaded()
            s = m.CalcLoadedSC()
            g = m.calc_contact_molecular_surface_gradient(True)
            a0, a1 = int(batch.atom_off[c]), int(batch.atom_off[c + 1])
            plain_match &= (cms == totals[c, 1]) and (s[0] == sc[c, 0]) and bool(np.array_equal(g, grad_dev[a0:a1]))
        plain = len(idx) / (time.perf_counter() - t0)
        extras["plain_gpu"] = {"value": plain, "unit": UNIT,
                               "sample": f"first {len(idx)} complexes, one per call (CMS, SC, gradient)",
                               "results_match_batched": bool(plain_match)}
        extras["batched_vs_plain"] = value / plain
        extras["cpu_baseline"] = cpu_baseline_single(batch, args.cpu_sample)
        if args.refine_steps > 0:
            extras["pose_refinement"] = pose_refinement(args, local)

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_max, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator, complexes of random residues)",
                "config": {"workload": WORKLOAD, "complexes_per_gpu": B, "atoms_per_gpu": N,
                           "parallelism": f"replicas x{world} (independent complexes per GPU)",
                           "l2": "inputs larger than L2 (9M atoms), no flush",
                           "nn_search": "FP32 filter + FP64 recheck over every pair not excluded by a proven box-distance bound",
                           "grad": "included: d(target-side CMS)/d(xyz) of binder and target atoms, FP64 adjoint "
                                   "with the dot topology fixed, in every step"},
                "e2e": e2e, "gpu_launches": launches * args.steps, "clocks": clocks, "autotune": autotune,
                "complex_status_nonzero": int(sum(1 for s in statuses if s))}
        line.update(extras)
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
