"""Multi-GPU plumbing of the B200 path: one process per GPU, no data-path collective.

A single log-likelihood evaluation is one dependent Cholesky DAG and does not
shard at these sizes, so several GPUs run independent replicas (the bench) or
independent problems (many regional likelihoods, serving requests).  The only
cross-rank traffic is scalars: the slowest rank's device time, and the
per-problem results gathered at the end.  Works with any torch.distributed
backend (NCCL on GPUs, gloo on CPU for the tests).
"""
from __future__ import annotations

import heapq


def max_over_ranks(value: float, dist=None, device: str = "cpu") -> float:
    """The maximum of `value` over all ranks (the job's time is its slowest rank's)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def shard_by_cost(sizes, world: int) -> list[list[int]]:
    """Partition problem indices over `world` ranks, greedily by n^3 cost (largest first).

    Deterministic: every rank computes the same partition from the same sizes.
    """
    if world <= 0:
        raise ValueError("world must be positive")
    order = sorted(range(len(sizes)), key=lambda i: (-float(sizes[i]) ** 3, i))
    heap = [(0.0, r) for r in range(world)]
    shards: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        shards[r].append(i)
        heapq.heappush(heap, (load + float(sizes[i]) ** 3, r))
    for s in shards:
        s.sort()
    return shards


def gather_results(local: dict, dist=None) -> dict:
    """Union of every rank's {problem index: result} (scalars only cross ranks)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return dict(local)
    parts = [None] * dist.get_world_size()
    dist.all_gather_object(parts, dict(local))
    out: dict = {}
    for p in parts:
        out.update(p)
    return out


def replica_rate(units_per_rank: float, local_seconds: float, dist=None, device: str = "cpu") -> float:
    """Whole-job throughput: units of all ranks / the slowest rank's time."""
    world = dist.get_world_size() if dist is not None and dist.is_initialized() else 1
    return world * units_per_rank / max_over_ranks(local_seconds, dist, device)
