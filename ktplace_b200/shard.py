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


class ShardPlan:
    """LPT plan of independent solve units over `world` ranks, with the host
    layout of their results: unit u owns entries offsets[u]:offsets[u+1] of
    one host buffer of `total` entries (the x then y solution of a netlist,
    say), so the ranks write disjoint slices and nothing is exchanged during
    the solve. The units of one netlist are independent because the x and y
    systems of the reference's solve never read each other
    (simpl_lss.cc:274-284), and netlists of a batch share nothing at all.
    """

    def __init__(self, sizes: Sequence[int], costs: Sequence[float] = None, world: int = 1):
        import numpy as np
        self.sizes = [int(s) for s in sizes]
        if any(s < 0 for s in self.sizes):
            raise ValueError("negative unit size")
        self.costs = [float(c) for c in (costs if costs is not None else self.sizes)]
        if len(self.costs) != len(self.sizes):
            raise ValueError("one cost per unit")
        self.world = int(world)
        self.owned = lpt_assign(self.costs, self.world)
        self.offsets = np.concatenate([[0], np.cumsum(self.sizes, dtype=np.int64)])

    @property
    def total(self) -> int:
        return int(self.offsets[-1])

    def share(self, rank: int) -> list:
        if not 0 <= rank < self.world:
            raise ValueError("rank out of range")
        return list(self.owned[rank])

    def slice(self, unit: int) -> slice:
        return slice(int(self.offsets[unit]), int(self.offsets[unit + 1]))

    def makespan(self) -> float:
        return makespan(self.costs, self.owned)


def run_share(plan: ShardPlan, rank: int, solve_units, out) -> list:
    """One rank's part of a sharded solve: `solve_units(units)` solves the
    rank's units (plan.share(rank), largest first is not required) and returns
    one host vector per unit in that order; each is written into its slice of
    `out`, the host buffer of all units (plan.total entries). Returns the
    units solved."""
    units = plan.share(rank)
    if not units:
        return units
    vecs = solve_units(units)
    if len(vecs) != len(units):
        raise RuntimeError(f"solver returned {len(vecs)} results for {len(units)} units")
    for u, v in zip(units, vecs):
        sl = plan.slice(u)
        if len(v) != sl.stop - sl.start:
            raise RuntimeError(f"unit {u}: {len(v)} entries for a slice of {sl.stop - sl.start}")
        out[sl] = v
    return units


def gather_to_root(plan: ShardPlan, rank: int, out, group=None):
    """Assembles every rank's slices of `out` on rank 0 through
    torch.distributed (object gather; host data, after the solve) and returns
    the full buffer there, None on the other ranks."""
    import numpy as np
    import torch.distributed as dist
    mine = {u: np.asarray(out[plan.slice(u)]).copy() for u in plan.share(rank)}
    parts = [None] * plan.world if rank == 0 else None
    dist.gather_object(mine, parts, dst=0, group=group)
    if rank != 0:
        return None
    full = np.zeros(plan.total, dtype=np.asarray(out).dtype)
    seen = set()
    for p in parts:
        for u, v in p.items():
            if u in seen:
                raise RuntimeError(f"unit {u} solved twice")
            seen.add(u)
            full[plan.slice(u)] = v
    if len(seen) != len(plan.sizes):
        raise RuntimeError(f"{len(plan.sizes) - len(seen)} units were not solved")
    return full


class BatchShardSolver:
    """The GPU solver of one rank's share of a batch of netlists: each owned
    netlist's x and y B2B systems are built on this rank's GPU and loaded into
    one Batch, which is autotuned once (cluster shape, then the pairs sent
    to the whole GPU, then the size split) and solved by graph replay. `make_unit(u)` returns
    (netlist, x, y, anchor_x, anchor_y, alpha) for netlist u; a unit's host
    result is its x solution followed by its y solution.
    """

    def __init__(self, make_unit, device: int = 0, tol: float = 1e-6, max_iter: int = 100000,
                 precision: int = 1, inner_tol: float = 1e-3, autotune: bool = True,
                 stream: int = 0):
        self.make_unit = make_unit
        self.device = device
        self.tol, self.max_iter = tol, max_iter
        self.precision, self.inner_tol = precision, inner_tol
        self.autotune = autotune
        self.stream = stream
        self.batch = None
        self.units = []
        self.rows = []
        self.shape = None
        self.split = None
        self.offload = None

    def load(self, units) -> None:
        """Builds and loads the systems of `units` (once)."""
        from .gpu import Context, Batch
        self.close()
        self.batch = Batch(self.device)
        if self.stream:
            self.batch.set_stream(self.stream)
        self.units, self.rows = list(units), []
        with Context(self.device) as ctx:
            for u in self.units:
                nl, x, y, ax, ay, alpha = self.make_unit(u)
                fx, fy = nl.floors()
                ctx.upload_netlist(nl)
                ctx.build_b2b(x, y, alpha, ax, ay, fx, fy)
                self.batch.add_from_context(ctx, x, y)
                self.rows.append(nl.num_movable)
        if self.autotune:
            c, t, _ = self.batch.autotune(self.tol, precision=self.precision,
                                          inner_tol=self.inner_tol, probe_iter=40)
            self.shape = (c, t)
            self.offload, _, _ = self.batch.autotune_offload(
                self.tol, precision=self.precision, inner_tol=self.inner_tol,
                max_iter=self.max_iter)
            self.split, _, _ = self.batch.autotune_split(self.tol, precision=self.precision,
                                                         inner_tol=self.inner_tol,
                                                         max_iter=self.max_iter)

    def solve(self, reset: bool = True) -> None:
        """Enqueues the solve of every loaded system (from its start vector
        when `reset`)."""
        if reset:
            self.batch.reset_x()
        self.batch.solve(self.tol, self.max_iter, precision=self.precision,
                         inner_tol=self.inner_tol)

    def results(self) -> list:
        import numpy as np
        res = self.batch.results()
        bad = [r for r in res if r["status"] != 0]
        if bad:
            raise RuntimeError(f"{len(bad)} systems of the share did not converge")
        out = []
        for k, n in enumerate(self.rows):
            out.append(np.concatenate([self.batch.get_x(2 * k, n), self.batch.get_x(2 * k + 1, n)]))
        return out

    def __call__(self, units) -> list:
        if self.batch is None or list(units) != self.units:
            self.load(units)
        self.solve()
        return self.results()

    def close(self):
        if self.batch is not None:
            self.batch.close()
            self.batch = None
