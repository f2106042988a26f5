"""Instances over ranks: one process per GPU, each solving its own share of independent CG2D instances.

Ensemble members (and LLC90 / LLC270 instances in one batch) are independent solves, so a batch is partitioned
across ranks with no collective inside the solve; the reference's own tile-sharded single solve was slower on
4 GPUs than on 1 (docs/VALIDATION.md:57), so one solve is never split. The collectives used are host-side
bookkeeping after the solves: the max of the ranks' device times (the job's time) and the gathering of per-instance
diagnostics.
"""

import numpy as np


def estimated_work(points, iterations=None):
    """Work estimate of each instance: interior points x expected iterations (iterations default to 1)."""
    points = np.asarray(points, dtype=np.float64)
    it = np.ones_like(points) if iterations is None else np.asarray(iterations, dtype=np.float64)
    return points * it


def shard_instances(work, world, rank):
    """Indices of the instances rank `rank` of `world` solves: greedy largest-first assignment to the least loaded
    rank (ties to the lowest rank), so that per-rank work differs by at most one instance's. Every instance goes
    to exactly one rank; the result is sorted."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} of {world}")
    work = np.asarray(work, dtype=np.float64)
    load = np.zeros(world)
    owner = np.empty(len(work), dtype=np.int64)
    for i in sorted(range(len(work)), key=lambda i: (-work[i], i)):
        r = int(np.argmin(load))
        owner[i] = r
        load[r] += work[i]
    return [i for i in range(len(work)) if owner[i] == rank]


def max_over_ranks(value, device=None):
    """The largest of the ranks' values (a job is as slow as its slowest rank); the value itself without a process
    group."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_records(records):
    """Every rank's list of per-instance records, concatenated in rank order (plain list without a process group)."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return list(records)
    out = [None] * dist.get_world_size()
    dist.all_gather_object(out, list(records))
    return [r for part in out for r in part]
