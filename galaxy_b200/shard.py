"""Placement of independent simulations on the GPUs of one node, one process
per GPU.  Batched and served simulations never exchange data, so each rank
advances its own share with the batched engine and only host-side results
(particle-steps, timings, per-request latencies) are gathered; nothing
crosses NVLink on the data path.  A single simulation is not partitioned
(that needs a global sort and a locally-essential-tree exchange): it runs as
a replica.

The plan is a pure function of the sizes, so every rank computes the same
plan without communication.
"""
from __future__ import annotations

import math
from typing import Callable, Sequence


def work_estimate(n: int, steps: int = 1) -> float:
    """Relative cost of one simulation: the build is ~N and the traversal
    ~N log N per step."""
    return float(n) * max(math.log2(max(n, 2)), 1.0) * max(steps, 1)


def plan_shards(sizes: Sequence[int], world: int, steps: Sequence[int] | None = None,
                footprint: Callable[[int], int] | None = None,
                budget_bytes: int | None = None) -> list[list[int]]:
    """Longest-processing-time placement: simulations in decreasing estimated
    work (index order among equals) each go to the rank with the least work so
    far that still has room in its HBM budget.  Returns the simulation indices
    of every rank, each list in increasing index order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    steps = list(steps) if steps is not None else [1] * len(sizes)
    order = sorted(range(len(sizes)), key=lambda i: (-work_estimate(sizes[i], steps[i]), i))
    load = [0.0] * world
    used = [0] * world
    shards: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        need = footprint(i) if footprint else 0
        ranks = sorted(range(world), key=lambda r: (load[r], r))
        for r in ranks:
            if budget_bytes is None or used[r] + need <= budget_bytes:
                break
        else:
            raise MemoryError(f"simulation {i} ({need} bytes) fits no rank's budget")
        shards[r].append(i)
        load[r] += work_estimate(sizes[i], steps[i])
        used[r] += need
    return [sorted(s) for s in shards]


def _reduce(pg, value: float, op, device: str | None) -> float:
    import torch
    if device is None:  # NCCL reduces device tensors, gloo host tensors
        device = "cuda" if pg.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=op)
    return float(t.item())


def max_over_ranks(pg, value: float, device: str | None = None) -> float:
    """The maximum of `value` over all ranks (device times are reported as
    the slowest rank's); `pg` is torch.distributed or None for one rank."""
    return float(value) if pg is None else _reduce(pg, value, pg.ReduceOp.MAX, device)


def sum_over_ranks(pg, value: float, device: str | None = None) -> float:
    return float(value) if pg is None else _reduce(pg, value, pg.ReduceOp.SUM, device)


def gather_to_all(pg, obj) -> list:
    """Every rank's `obj`, in rank order, on every rank."""
    if pg is None:
        return [obj]
    out = [None] * pg.get_world_size()
    pg.all_gather_object(out, obj)
    return out
