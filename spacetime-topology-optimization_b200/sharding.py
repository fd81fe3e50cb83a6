"""Sharding independent space-time problems over ranks (one process per GPU).

The solve path has no exchange step: stage rows, load cases and whole problems are
independent units.  Units are given to ranks whole, balanced by their estimated cost
(elements x stage rows, the work of the batched solves), and each rank solves its own
with ``spacetime.objective_and_gradient_many``; nothing crosses ranks during a solve.
``gather`` (optional) collects every rank's results afterwards, for callers that want
the full list on every rank.
"""

from __future__ import annotations

import heapq
from typing import Callable, Sequence

import torch
from torch import Tensor


def unit_cost(x: Tensor, n_stage: int) -> float:
    """Estimated work of one problem: its elements times its rows (heat + stages)."""
    return float(x.numel()) * (n_stage + 1)


def partition(costs: Sequence[float], world: int) -> list[list[int]]:
    """Indices of the units of each rank: longest-processing-time-first onto the least
    loaded rank (ties to the lower rank), each rank's list in increasing index order.
    Deterministic, so every rank computes the same partition without communicating."""
    if world <= 0:
        raise ValueError("world must be positive")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    heap = [(0.0, r) for r in range(world)]
    parts: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + float(costs[i]), r))
    return [sorted(p) for p in parts]


def rank_seed(seed: int, rank: int) -> int:
    """The seed of a rank's own synthetic problem (distinct units per rank)."""
    return int(seed) + 7919 * int(rank)


def _dist():
    import torch.distributed as dist

    return dist


def world_and_rank(group=None) -> tuple[int, int]:
    dist = _dist()
    if not (dist.is_available() and dist.is_initialized()):
        return 1, 0
    return dist.get_world_size(group), dist.get_rank(group)


def max_over_ranks(value: float, group=None, device=None) -> float:
    """The maximum of a per-rank time over the ranks (all_reduce MAX)."""
    world, _ = world_and_rank(group)
    if world == 1:
        return float(value)
    dist = _dist()
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def objective_and_gradient_sharded(xs: Sequence[Tensor], ws: Sequence[Tensor], n_stages: Sequence[int], *,
                                   group=None, solve: Callable | None = None, **kw):
    """This rank's share of the problems ``(xs[i], ws[i], n_stages[i])``: returns
    ``(indices, outputs)`` with ``outputs[j]`` the result of problem ``indices[j]``.
    ``solve`` defaults to ``spacetime.objective_and_gradient_many`` (keyword arguments
    are passed on)."""
    if not (len(xs) == len(ws) == len(n_stages)):
        raise ValueError("xs, ws and n_stages must have the same length")
    world, rank = world_and_rank(group)
    mine = partition([unit_cost(x, n) for x, n in zip(xs, n_stages)], world)[rank]
    if solve is None:
        from . import spacetime

        solve = spacetime.objective_and_gradient_many
    if not mine:
        return [], []
    outs = solve([xs[i] for i in mine], [ws[i] for i in mine], [int(n_stages[i]) for i in mine], **kw)
    return mine, list(outs)


def gather(indices: Sequence[int], values: Sequence[Tensor], n: int, group=None) -> list[Tensor]:
    """Every rank's ``(indices, values)`` into one list of ``n`` tensors on every rank
    (host copies, through ``all_gather_object``)."""
    world, _ = world_and_rank(group)
    local = [(int(i), v.detach().cpu()) for i, v in zip(indices, values)]
    if world == 1:
        pieces = [local]
    else:
        pieces = [None] * world
        _dist().all_gather_object(pieces, local, group=group)
    out: list = [None] * n
    for piece in pieces:
        for i, v in piece:
            out[i] = v
    missing = [i for i, v in enumerate(out) if v is None]
    if missing:
        raise RuntimeError(f"no rank returned units {missing[:8]}")
    return out


__all__ = ["unit_cost", "partition", "rank_seed", "world_and_rank", "max_over_ranks",
           "objective_and_gradient_sharded", "gather"]
