"""Host logic for running the path on several GPUs as independent replicas.

The SpMV path does not shard inside one product here: each GPU (one process
per GPU) owns whole matrices. This module holds the pieces that need more
than one rank: a size-balanced assignment of matrices to ranks, the
max-over-ranks device time, and the whole-job throughput of a weak-scaling
run. torch.distributed is only plumbing (NCCL on GPUs, gloo on CPU tests);
no data-path collective is involved.
"""
from __future__ import annotations

from typing import Sequence


def assign_to_ranks(sizes: Sequence[int], world: int) -> list[list[int]]:
    """Greedy longest-processing-time assignment of matrix indices to ranks
    (largest first, each to the least-loaded rank; ties to the lower rank).
    Deterministic, so every rank computes the same map without talking."""
    order = sorted(range(len(sizes)), key=lambda i: (-int(sizes[i]), i))
    load = [0] * world
    out: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        out[r].append(i)
        load[r] += int(sizes[i])
    for lst in out:
        lst.sort()
    return out


def owner_of(assignment: list[list[int]]) -> dict[int, int]:
    """matrix index -> owning rank."""
    return {i: r for r, lst in enumerate(assignment) for i in lst}


def max_over_ranks(value: float, device=None) -> float:
    """Max of a per-rank scalar (e.g. elapsed device ms) over the default
    process group; identity when not distributed."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, device=None) -> float:
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def weak_scaling_gbs(bytes_per_rank: float, steps: int, max_ms: float, world: int) -> float:
    """Whole-job GB/s when every rank moves bytes_per_rank per step and the
    slowest rank took max_ms for `steps` steps."""
    return world * bytes_per_rank * steps / (max_ms / 1e3) / 1e9
