"""Sharding one ensemble of lens realizations across ranks (one rank per GPU).

The members are independent problems, so the ensemble splits across GPUs with no collective in
the data path: every rank draws the same member list, keeps the members assigned to it, advances
them in its own batched launches (ewg.Ensemble), and the results meet once at the end (a gather
of per-member reports, and of the fields when the caller asks for them).

Assignment: greedy longest-processing-time on an estimated cost per member,
    cost = cells x expected BiCGStab iterations,  expected iterations ~ n (the cube edge in cells)
    x sqrt(dt / 250 s),
the per-step work of a member with an ILU(0)-preconditioned Krylov solve whose iteration count
grows with the grid's diameter and with the time step. Members are taken in decreasing cost and
each goes to the rank with the least assigned cost (ties: lowest rank), which bounds the
heaviest rank's cost by the mean plus the largest member's cost. The assignment is a pure
function of the member list and the rank count, so every rank computes the same one.
"""
from __future__ import annotations

import math

import numpy as np


def member_cost(n_cells: int, dt: float) -> float:
    """Estimated work of one implicit step of a cube member of n_cells cells at step size dt."""
    edge = round(n_cells ** (1.0 / 3.0))
    return float(n_cells) * edge * math.sqrt(dt / 250.0)


def assign_members(costs, world: int) -> list[list[int]]:
    """Greedy cost balance: members[r] lists the member indices of rank r, each in ascending order."""
    if world < 1:
        raise ValueError("world must be at least 1")
    order = sorted(range(len(costs)), key=lambda m: (-costs[m], m))
    load = [0.0] * world
    members: list[list[int]] = [[] for _ in range(world)]
    for m in order:
        r = min(range(world), key=lambda q: (load[q], q))
        members[r].append(m)
        load[r] += costs[m]
    return [sorted(ms) for ms in members]


def rank_loads(costs, members) -> list[float]:
    return [float(sum(costs[m] for m in ms)) for ms in members]


def gather_results(dist, rank: int, world: int, mine: dict, dst: int = 0):
    """Collect {member index: result} from every rank on rank dst (None elsewhere). dist is
    torch.distributed with an initialised process group, or None for a single process."""
    if dist is None or world == 1:
        return dict(mine)
    out = [None] * world if rank == dst else None
    dist.gather_object(mine, out, dst=dst)
    if rank != dst:
        return None
    merged = {}
    for part in out:
        merged.update(part)
    return merged


def imbalance(costs, members) -> float:
    """Heaviest rank's cost over the mean rank cost (1 = perfectly balanced)."""
    loads = rank_loads(costs, members)
    mean = float(np.mean(loads)) if loads else 0.0
    return max(loads) / mean if mean > 0 else 1.0
