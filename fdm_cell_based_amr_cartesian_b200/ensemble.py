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


# ------------------------------------------------- the ensemble workload
# Bands (distance from the split lines) refined to levels 1..5 in the
# statically refined meshes of the ensemble members: a member with maximum
# level L refines the first L bands.  Each band is at least two cells of the
# finer level narrower than the previous one, so the meshes keep the 2:1
# balance.
ENSEMBLE_BANDS = (0.2, 0.15, 0.1, 0.05, 0.025)
ENSEMBLE_SEEDS = tuple(range(1000, 1064))
# Background grid of the members.  At 128^2 a level-5 member has a finest
# spacing of 1/4096, where the reference's hanging-node least squares (in
# absolute coordinates) loses its digits: on a band-refined level-5 mesh the
# parent WLS values overshoot the data range by up to 4x and the state turns
# NaN within one step, in the CPU restatement as on the GPU.  At 64^2 the
# finest spacing is 1/2048, that of the four-quadrant problem at 128^2 with 4
# levels.
ENSEMBLE_BASE = 64


def ensemble_configs(seeds=ENSEMBLE_SEEDS, base: int = ENSEMBLE_BASE):
    """Random four-quadrant problems (rho, p ~ U[0.1,2], u, v ~ U[-1,1]) with
    the maximum level drawn from U{2..5}, one per seed."""
    from . import params as P
    return [P.random_riemann4(s, base=base) for s in seeds]


def ensemble_meshes(cfgs):
    """(keys, prim) of every member: the band-refined mesh of its level and
    the quadrant initial state.  Meshes and quadrant maps are shared by the
    members of one level; the state of a member is its four quadrant states
    picked by the map (the same values as solver.initial_state)."""
    import numpy as np

    from . import solver as S
    cache = {}
    out = []
    for cfg in cfgs:
        L = int(cfg.params.lvl_amr)
        if L not in cache:
            keys = S.distance_refined_keys(cfg, [("x", 0.5), ("y", 0.5)], list(ENSEMBLE_BANDS[:L]))
            cx, cy = S.node_centers(cfg, keys)
            icp = cfg.ic_params
            east, north = cx > icp[0], cy > icp[1]
            q = np.where(north, np.where(east, 0, 1), np.where(east, 3, 2))
            cache[L] = (keys, q)
        keys, q = cache[L]
        st = np.asarray(cfg.ic_params[2:18], dtype=np.float64).reshape(4, 4)
        out.append((keys, st[q]))
    return out
