"""Spreading the space-time work over ranks (one process per GPU).

The solve path has no exchange step inside a solve: stage rows, load cases and whole
problems are independent units.

* Independent problems (``objective_and_gradient_sharded``): given to ranks whole,
  balanced by their estimated cost (elements x stage rows, the work of the batched
  solves); each rank solves its own with ``spacetime.objective_and_gradient_many``;
  ``gather`` (optional) collects the results afterwards.
* One objective split over ranks (``objective_and_gradient_split``): the reference's
  unit is the stage stack of one objective (sttopt/compliance.py:228-242, one batched
  solve over the stage rows).  Rank 0 solves the heat time field and broadcasts tPhys
  (one NCCL broadcast of ``nel`` doubles); every rank solves its share of the stages and
  their adjoints; rank 0 also runs the heat adjoint; one all-reduce (sum) of the
  gradient and the stage compliances combines them.  Every rank takes the same two
  collectives in the same order.  Peers' data only arrives through these collectives,
  into local buffers.
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


def stage_partition(n_stage: int, world: int, heat_cost: float = 1.0) -> list[list[int]]:
    """The stages of each rank when one objective is split: stages have equal cost (one
    grid, one row each); rank 0 starts loaded with ``heat_cost`` stage-equivalents (the
    heat solve and its adjoint), and each stage goes to the least loaded rank (ties to the
    lower rank).  Deterministic; each list ascending."""
    if world <= 0:
        raise ValueError("world must be positive")
    load = [float(heat_cost)] + [0.0] * (world - 1)
    parts: list[list[int]] = [[] for _ in range(world)]
    for s in range(n_stage):
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(s)
        load[r] += 1.0
    return parts


def objective_and_gradient_split(xPhys: Tensor, w: Tensor, *, n_stage: int = 16, group=None,
                                 solve: Callable | None = None, heat_cost: float = 1.0, **kw) -> dict:
    """One space-time objective and its gradient with the stages spread over the ranks of
    ``group``; every rank returns the whole result (``objective``, ``c_s`` of all stages,
    ``J_t``, ``tPhys``, ``gradient``) and ``stages``, its own share.

    ``solve(x, w, n_stage=, stages=, tphys=, publish=, **kw)`` computes a rank's share: the
    given stages' compliances and gradient terms, the heat solve (calling ``publish(tPhys)``
    as soon as it exists) and the heat adjoint when ``tphys`` is None, else the given time
    field.  It defaults to ``spacetime.objective_and_gradient_part``."""
    world, rank = world_and_rank(group)
    mine = stage_partition(n_stage, world, heat_cost)[rank]
    if solve is None:
        from . import spacetime

        solve = spacetime.objective_and_gradient_part
    if world == 1:
        part = solve(xPhys, w, n_stage=n_stage, stages=mine, tphys=None, publish=None, **kw)
        return dict(part, stages=mine)
    dist = _dist()
    src = dist.get_global_rank(group, 0) if group is not None else 0
    if rank == 0:
        part = solve(xPhys, w, n_stage=n_stage, stages=mine, tphys=None,
                     publish=lambda t: dist.broadcast(t.reshape(-1).contiguous(), src=src, group=group), **kw)
    else:
        tphys = torch.empty(xPhys.numel(), dtype=torch.float64, device=xPhys.device)
        dist.broadcast(tphys, src=src, group=group)
        part = solve(xPhys, w, n_stage=n_stage, stages=mine, tphys=tphys.reshape(xPhys.shape), publish=None, **kw)
    nel = xPhys.numel()
    buf = torch.zeros(nel + n_stage, dtype=torch.float64, device=xPhys.device)
    buf[:nel] = part["gradient"].reshape(-1).to(torch.float64)
    if mine:
        buf[nel + torch.tensor(mine, device=xPhys.device)] = part["c_s"].to(torch.float64)
    dist.all_reduce(buf, group=group)
    c_s = buf[nel:]
    tPhys = part["tPhys"].reshape(xPhys.shape)
    J_t = (w.to(torch.float64) * tPhys).sum()
    return dict(objective=c_s.sum() + J_t, c_s=c_s, J_t=J_t, tPhys=tPhys,
                gradient=buf[:nel].reshape(xPhys.shape), stages=mine)


__all__ = ["unit_cost", "partition", "rank_seed", "world_and_rank", "max_over_ranks",
           "objective_and_gradient_sharded", "gather", "stage_partition", "objective_and_gradient_split"]
