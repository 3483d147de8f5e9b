"""Assignment of independent solve units to GPUs.

The path shards only as independent units (the x and y systems of one
netlist, the netlists of a batch): no exchange happens during a solve, so a
multi-GPU run is an assignment problem. Units go to ranks longest-first onto
the least-loaded rank (LPT), which is deterministic for equal inputs, so
every rank computes the same assignment without communicating.
"""
from __future__ import annotations

from typing import Sequence


def lpt_assign(costs: Sequence[float], world: int) -> list:
    """Returns, per rank, the unit indices it owns (ascending)."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    load = [0.0] * world
    owned = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        owned[r].append(i)
        load[r] += float(costs[i])
    return [sorted(o) for o in owned]


def makespan(costs: Sequence[float], owned: list) -> float:
    return max((sum(float(costs[i]) for i in o) for o in owned), default=0.0)


def rank_design_seed(rank: int, base: int = 1) -> int:
    """Seed of the netlist a rank solves in the weak-scaling bench."""
    return base + rank
