"""
Replicas over several GPUs: one process per GPU, complexes split between the
processes, no exchange during the computation.

Complexes are independent, so a batch shards by complex: each rank evaluates
its own share through its own context and the only collectives are the
bookkeeping ones here -- the slowest rank's time (a job is as fast as its
slowest replica) and one gather of per-complex outputs to rank 0.  The
reference runs one complex per calculator (cms-cuda/_api.py:41-133) and has no
multi-GPU path.
"""

import numpy as np


def balanced_shards(costs, world):
    """
    Split complexes into `world` shards of similar total cost (longest
    processing time first: the next most expensive complex goes to the least
    loaded shard, ties to the lower rank).  Returns one sorted index array per
    rank; deterministic for given costs.
    """
    costs = np.asarray(costs, dtype=np.float64)
    if world < 1:
        raise ValueError("world must be >= 1")
    order = np.lexsort((np.arange(len(costs)), -costs))
    load = np.zeros(world)
    owner = np.empty(len(costs), np.int64)
    for i in order:
        r = int(np.argmin(load))
        owner[i] = r
        load[r] += costs[i]
    return [np.nonzero(owner == r)[0] for r in range(world)]


def shard_for_rank(costs, rank, world):
    return balanced_shards(costs, world)[rank]


def _device_for(dist):
    import torch
    return torch.device("cuda", torch.cuda.current_device()) if dist.get_backend() == "nccl" else torch.device("cpu")


def max_over_ranks(value):
    """The largest of every rank's `value` (e.g. a step time), on every rank."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=_device_for(dist))
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_per_complex(local_values, local_indices, n_total):
    """
    Rank 0 receives the per-complex rows of every rank in global complex
    order (other ranks receive None).  local_values: array whose first axis
    matches local_indices.
    """
    import torch.distributed as dist
    local_values = np.asarray(local_values)
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        out = np.empty((n_total,) + local_values.shape[1:], local_values.dtype)
        out[np.asarray(local_indices)] = local_values
        return out
    parts = [None] * dist.get_world_size()
    dist.all_gather_object(parts, (np.asarray(local_indices), local_values))
    if dist.get_rank() != 0:
        return None
    out = np.empty((n_total,) + local_values.shape[1:], local_values.dtype)
    for idx, vals in parts:
        out[idx] = vals
    return out
