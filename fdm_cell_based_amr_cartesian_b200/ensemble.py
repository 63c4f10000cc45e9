"""Placement of independent solver instances on ranks (one process per GPU)
and the max-over-ranks timing of the benchmark.

Instances of the ensemble configuration are independent AMR problems, so
they shard without any exchange: each rank owns whole instances, balanced by
estimated leaf count (longest-processing-time greedy), and the only
collective is the reduction of one timing scalar."""
from __future__ import annotations

import heapq

import torch
import torch.distributed as dist


def partition(weights, world: int):
    """Owner rank of each instance: heaviest first to the least loaded rank.
    Deterministic (ties by index), so every rank computes the same map."""
    order = sorted(range(len(weights)), key=lambda i: (-weights[i], i))
    heap = [(0.0, r) for r in range(world)]
    owner = [0] * len(weights)
    for i in order:
        load, r = heapq.heappop(heap)
        owner[i] = r
        heapq.heappush(heap, (load + float(weights[i]), r))
    return owner


def max_over_ranks(value: float, device=None) -> float:
    """Max of a per-rank scalar (elapsed ms) over the process group."""
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, device=None) -> float:
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
