"""Independent units across GPUs: one process per GPU, no data-path collective.

The step itself does not shard (a 256^3 field stays on one GPU); what spreads
over GPUs are independent units -- ensemble members, UPO guesses, gradient
directions -- as the reference's drivers spread independent jobs over MPI
ranks (3D_NavierStokes/src/main.F90:32-40).  Units are dealt out by cost,
largest first, to the rank with the least work so far (greedy list
scheduling), which every rank computes identically from the same list, so no
message is exchanged to agree on the split.  The only collectives are the
timing reduction (max over ranks) and the final gather of small per-unit
results, both on the host side of the process group.
"""
from __future__ import annotations

import heapq
from typing import Sequence


def shard(costs: Sequence[float], world: int) -> list[list[int]]:
    """Assign unit i (cost costs[i]) to a rank; returns the unit indices of every
    rank, each list in increasing order.  Deterministic: ties go to the lower
    rank, equal costs keep their input order."""
    if world < 1:
        raise ValueError("world size must be positive")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    heap = [(0.0, r) for r in range(world)]
    out: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + float(costs[i]), r))
    return [sorted(u) for u in out]


def cost2d(n: int, steps: int = 1) -> float:
    """relative cost of a 2D instance: N^2 log2 N per step"""
    return float(n * n * (n.bit_length() - 1) * steps)


def max_over_ranks(seconds: float, dist=None, device=None) -> float:
    """the slowest rank's time (the whole job's time when ranks run at once)"""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(seconds)
    import torch
    t = torch.tensor([float(seconds)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, dist=None, device=None) -> float:
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
