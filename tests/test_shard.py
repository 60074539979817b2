"""
Host logic of the multi-GPU replica path (cms_cuda.shard), on CPU: the
cost-balanced split of a batch and the two collectives (max of step times,
gather of per-complex outputs) over a world of two gloo ranks.
"""

import os
import socket

import numpy as np
import pytest


def test_balanced_shards_cover_and_balance():
    from cms_cuda.shard import balanced_shards
    rng = np.random.default_rng(3)
    costs = np.exp(rng.uniform(np.log(700), np.log(5200), 257))
    for world in (1, 2, 3, 8):
        shards = balanced_shards(costs, world)
        allidx = np.concatenate(shards)
        assert len(allidx) == len(costs) and len(np.unique(allidx)) == len(costs)
        loads = np.array([costs[s].sum() for s in shards])
        assert loads.max() - loads.min() <= costs.max()
        assert all(np.all(np.diff(s) > 0) for s in shards)
    assert [s.tolist() for s in balanced_shards(costs, 3)] == [s.tolist() for s in balanced_shards(costs, 3)]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, costs, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        from cms_cuda.shard import gather_per_complex, max_over_ranks, shard_for_rank
        idx = shard_for_rank(costs, rank, world)
        vals = np.stack([idx * 2.0, idx * 3.0], 1)          # per-complex outputs of this rank
        out = gather_per_complex(vals, idx, len(costs))
        t = max_over_ranks(0.25 + rank)
        q.put((rank, t, None if out is None else out.tolist()))
    finally:
        dist.destroy_process_group()


def test_two_rank_collectives_gloo():
    import torch.multiprocessing as mp
    costs = np.arange(1, 40, dtype=np.float64) ** 1.3
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, costs, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    assert [r[1] for r in res] == [1.25, 1.25]
    assert res[1][2] is None
    out = np.array(res[0][2])
    n = len(costs)
    assert np.array_equal(out, np.stack([np.arange(n) * 2.0, np.arange(n) * 3.0], 1))


def _bench_worker(rank, world, port, q):
    """One rank of the benchmark's multi-GPU plan on CPU: its shard of one global batch, then the gather."""
    import datetime
    import importlib.util
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
        spec = importlib.util.spec_from_file_location("bench_rank", os.path.join(root, "bench.py"))
        bench = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(bench)
        from cms_cuda.shard import gather_per_complex, max_over_ranks
        B_global, mine, batch = bench.rank_batch(24, 2, rank, world)
        sizes = np.diff(batch.atom_off).astype(np.float64)
        first = np.array([batch.xyz[int(batch.atom_off[c])][0] for c in range(batch.B)])
        out = gather_per_complex(np.stack([sizes, first], 1), mine, B_global)
        t = max_over_ranks(float(batch.N))
        q.put((rank, B_global, len(mine), t, None if out is None else out.tolist()))
    finally:
        dist.destroy_process_group()


def test_two_rank_benchmark_plan_gloo():
    """
    The benchmark's N > 1 path on two gloo ranks: each rank generates only its
    cost-balanced share of one global batch (48 complexes), the shares cover
    the batch once, and the gather returns every complex's size and first
    coordinate in global order, equal to the single-process batch.
    """
    import torch.multiprocessing as mp
    from cms_cuda import synth
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_bench_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [48, 48] and res[0][2] + res[1][2] == 48
    assert res[0][3] == res[1][3]                   # the max over ranks is shared
    whole = synth.config_batched(48, 2)
    out = np.array(res[0][4])
    assert np.array_equal(out[:, 0], np.diff(whole.atom_off).astype(np.float64))
    assert np.array_equal(out[:, 1], whole.xyz[whole.atom_off[:-1], 0])
