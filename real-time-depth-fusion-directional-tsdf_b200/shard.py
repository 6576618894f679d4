"""Host logic for running independent scans on several GPUs.

A single scene does not shard: a ray's first crossing can lie anywhere in
the volume, so N GPUs run N replicas.  Batched workloads -- many independent
scans -- shard by scan with no exchange on the data path: each rank fuses
its own scans, and the only collectives are a barrier around the timed
region, the maximum of the per-rank times, and an end-of-run gather of
per-rank statistics.  These helpers are backend-agnostic (gloo on CPU for the
tests, NCCL over NVLink on GPUs).
"""
from __future__ import annotations


def partition(work: list[float], world: int) -> list[list[int]]:
    """Greedy longest-processing-time assignment of items (by their work,
    e.g. frames x pixels) to `world` ranks: items in decreasing work order,
    each to the least-loaded rank (lowest rank on ties).  Deterministic, so
    every rank computes the same assignment without communicating; the
    heaviest rank carries at most the mean load plus the largest item."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(work)), key=lambda i: (-work[i], i))
    load = [0.0] * world
    parts: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += work[i]
    for p in parts:
        p.sort()
    return parts


def _device_for(dist):
    return "cuda" if dist.get_backend() == "nccl" else "cpu"


def max_over_ranks(value: float, dist=None) -> float:
    """The maximum of `value` over all ranks (the job's time is its slowest
    rank's); the value itself without a process group."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=_device_for(dist))
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, dist=None) -> float:
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=_device_for(dist))
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def gather_stats(stats: dict, dist=None) -> list[dict]:
    """Every rank's `stats` dict, in rank order (end-of-run only)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return [stats]
    out: list = [None] * dist.get_world_size()
    dist.all_gather_object(out, stats)
    return out
