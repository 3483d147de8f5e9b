"""The reference's SimPL solve interface, backed by the B200 path.

Mirrors, name for name, the types and calls of globalPlacer/simpl/simpl_lss.h
so code written against the reference reads the same:

  SparseSystem         simpl_lss.h:38-58 (rowPtr/col/val/diag/rhs, multiply)
  Residuals            simpl_lss.h:60-63
  LinearSystems        simpl_lss.h:68-84 (buildB2B)
  solveBothAxes        simpl_lss.h:86-88
  getHpwl, getOccupancy, getOverflow
                       simplPlacer::Impl, simpl_placer.cc:256-297
  SimplOptions         the legalizer's options, simpl_options.h:24-26
  LookAheadLegalizer   simpl_lal.h:18-60 (legalize), built as
                       simplPlacer::Impl::lookAheadLegalize does
                       (simpl_placer.cc:299-310)
  GlobalLoop           the B2B rounds of getInitialPlacement and the loop of
                       getGlobalPlacement (simpl_placer.cc:406-448, 463-539):
                       look-ahead legalization of the lower bound, B2B build
                       anchored at the legalized (upper-bound) positions,
                       warm-started solve, on device-resident data

All arithmetic runs in the CUDA library through the C ABI; nothing here
computes a result on the CPU. A SparseSystem produced by buildB2B remembers
the context whose device copy it mirrors, so solveBothAxes reuses that copy
instead of uploading the CSR again (any other system is uploaded).
"""
from __future__ import annotations

import dataclasses
from typing import Callable, Optional

import numpy as np

from .gpu import Context
from .grid import BinGrid, FreeSpace


@dataclasses.dataclass
class SparseSystem:
    rowPtr: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros(1, np.int64))
    col: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros(0, np.int32))
    val: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros(0))
    diag: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros(0))
    rhs: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros(0))
    _ctx: Optional[Context] = dataclasses.field(default=None, repr=False)
    _gen: int = dataclasses.field(default=-1, repr=False)
    _axis: int = dataclasses.field(default=-1, repr=False)

    def size(self) -> int:
        return int(self.diag.shape[0])

    def as_dict(self) -> dict:
        return dict(row_ptr=self.rowPtr, col=self.col, val=self.val, diag=self.diag,
                    rhs=self.rhs)


@dataclasses.dataclass
class Residuals:
    x: float = 0.0
    y: float = 0.0


IterateObserver = Callable[[int, Residuals, bool], None]


class LinearSystems:
    """simpl_lss.h:68-84. ``context`` is the GPU context holding the netlist."""

    def __init__(self, netlist, sysX: SparseSystem, sysY: SparseSystem, floorX: float,
                 floorY: float, context: Context):
        self.netlist = netlist
        self.sysX = sysX
        self.sysY = sysY
        self.floorX = floorX
        self.floorY = floorY
        self.ctx = context
        if context.nl is not netlist:
            context.upload_netlist(netlist)

    def buildB2B(self, x, y, alpha: float, anchorX, anchorY):
        """LinearSystems::buildB2B (simpl_lss.cc:11-114)."""
        ax = anchorX if alpha > 0.0 else None
        ay = anchorY if alpha > 0.0 else None
        self.ctx.build_b2b(x, y, alpha, ax, ay, self.floorX, self.floorY)
        gen = getattr(self.ctx, "_gen", 0) + 1
        self.ctx._gen = gen
        for axis, s in enumerate((self.sysX, self.sysY)):
            d = self.ctx.system(axis)
            s.rowPtr, s.col, s.val, s.diag, s.rhs = (d["row_ptr"], d["col"], d["val"],
                                                     d["diag"], d["rhs"])
            s._ctx, s._gen, s._axis = self.ctx, gen, axis


def _on_device(ctx: Context, s: SparseSystem, axis: int) -> bool:
    return s._ctx is ctx and s._axis == axis and s._gen == getattr(ctx, "_gen", -2)


def solveBothAxes(sysX: SparseSystem, x: np.ndarray, sysY: SparseSystem, y: np.ndarray,
                  tolerance: float, maxIterations: int,
                  observe: Optional[IterateObserver] = None,
                  context: Optional[Context] = None) -> Residuals:
    """solveBothAxes (simpl_lss.cc:203-290): x and y are updated in place.

    The observer is called once per loop iteration with that iteration's
    residuals, after the device solve returns (the residual history is
    recorded on the device)."""
    ctx = context or sysX._ctx or sysY._ctx
    if ctx is None:
        raise ValueError("solveBothAxes needs a Context (or systems built by one)")
    if sysX.size() != sysY.size():
        raise ValueError("x and y systems differ in size")
    for axis, s in enumerate((sysX, sysY)):
        if not _on_device(ctx, s, axis):
            ctx.upload_system(axis, s.as_dict())
    for axis, s in enumerate((sysX, sysY)):
        s._ctx, s._axis = ctx, axis
        s._gen = getattr(ctx, "_gen", 0)
    cap = int(min(maxIterations, 1 << 20)) if observe else 0
    r = ctx.solve(x, y, tolerance, maxIterations, hist_cap=cap)
    x[...] = r["x"]
    y[...] = r["y"]
    if observe:
        k = r["iters"]
        for it in range(1, k + 1):
            last = it == k and r["live"] == 0
            observe(it, Residuals(float(r["hist_x"][it - 1]), float(r["hist_y"][it - 1])), last)
    return Residuals(r["resid"][0], r["resid"][1])


def getHpwl(context: Context, x, y) -> float:
    """simplPlacer::Impl::getHpwl (simpl_placer.cc:256-275)."""
    return context.hpwl(x, y)


def getOccupancy(context: Context, grid: BinGrid, x, y) -> np.ndarray:
    """simplPlacer::Impl::getOccupancy (simpl_placer.cc:282-289)."""
    if getattr(context, "grid", None) is not grid:
        context.set_grid(grid)
    occ, _ = context.occupancy(x, y, want_map=True)
    return occ


def getOverflowOf(context: Context, grid: BinGrid, x, y) -> float:
    """getOverflow(getOccupancy(x, y)) (simpl_placer.cc:291-297) in one pass."""
    if getattr(context, "grid", None) is not grid:
        context.set_grid(grid)
    _, ov = context.occupancy(x, y, want_map=False)
    return ov


@dataclasses.dataclass
class SimplOptions:
    """The look-ahead legalizer's fields of SimplOptions (simpl_options.h:24-26)."""
    maxLevel: int = 20
    minCellsToSplit: int = 4
    stripeAreaFraction: float = 0.1


@dataclasses.dataclass
class LookAheadLegalizer:
    """LookAheadLegalizer (simpl_lal.h:18-60) on the GPU. The cell widths,
    heights and areas are those of the netlist uploaded to ``context``;
    ``freeSpace`` carries the rows, obstacles and die (grid.build_free_space);
    ``densityLimit`` is the grid's. ``legalize`` updates x and y in place, as
    the reference's does (ktg_lal: bit-identical positions)."""
    context: Context
    grid: BinGrid
    freeSpace: FreeSpace
    opts: SimplOptions = dataclasses.field(default_factory=SimplOptions)

    def legalize(self, x: np.ndarray, y: np.ndarray) -> None:
        ctx = self.context
        if getattr(ctx, "grid", None) is not self.grid:
            ctx.set_grid(self.grid)
        if getattr(ctx, "_fs_obj", None) is not self.freeSpace:
            ctx.set_free_space(self.freeSpace)
            ctx._fs_obj = self.freeSpace
        nx, ny = ctx.lal(x, y, self.opts.maxLevel, self.opts.minCellsToSplit,
                         self.opts.stripeAreaFraction)
        x[...] = nx
        y[...] = ny



def alpha_linear(it: int, iters: int = 30, first: float = 0.01, last: float = 1.0) -> float:
    """Anchor weight rising linearly from `first` to `last` over `iters`
    global iterations (the schedule of the mixed-precision study; the
    reference's own default is alphaBase * (1 + it), simpl_placer.cc:513)."""
    return first + (last - first) * min(it, iters - 1) / max(iters - 1, 1)


@dataclasses.dataclass
class GlobalIterate:
    """State of one global iteration, taken right after its B2B build (the
    context then holds that iteration's systems): the lower-bound positions
    the systems were built at (the solve's warm start), the legalized
    upper-bound positions that anchor them, and the anchor weight."""
    it: int
    alpha: float
    x: np.ndarray
    y: np.ndarray
    ux: np.ndarray
    uy: np.ndarray


class GlobalLoop:
    """SimPL's global placement loop on the GPU path (simpl_placer.cc:463-539).

    Every iteration: upper = lookAheadLegalize(lower) (ktg_lal), then
    buildB2B(lower, alpha, upper) (ktg_build_b2b) and the warm-started solve
    of lower (``solve``, by default the FP64 Jacobi-PCG of ktg_solve). The
    initial placement is SimPL's B2B initial rounds with no anchor
    (initialRounds with init_net b2b, simpl_placer.cc:406-448: buildB2B with
    alpha 0 and a solve per round). ``iterations`` yields a GlobalIterate
    after each build, before the solve, so a caller can solve or inspect the
    same systems another way; ``solve`` then advances the lower bound.
    Convergence checks and refinement are the caller's (the iteration count
    is fixed)."""

    def __init__(self, context: Context, netlist, grid: BinGrid, free_space: FreeSpace,
                 tol: float = 1e-6, max_iter: int = 100000, opts: Optional[SimplOptions] = None):
        self.ctx = context
        self.nl = netlist
        if context.nl is not netlist:
            context.upload_netlist(netlist)
        self.fx, self.fy = netlist.floors()
        self.lal = LookAheadLegalizer(context, grid, free_space, opts or SimplOptions())
        self.tol = tol
        self.max_iter = max_iter

    def solve(self, x, y):
        r = self.ctx.solve(x, y, self.tol, self.max_iter)
        return r["x"], r["y"]

    def initial_rounds(self, x, y, rounds: int = 5):
        x, y = np.array(x, dtype=np.float64), np.array(y, dtype=np.float64)
        for _ in range(rounds):
            self.ctx.build_b2b(x, y, 0.0, None, None, self.fx, self.fy)
            x, y = self.solve(x, y)
        return x, y

    def iterations(self, x, y, iters: int, alpha=alpha_linear, solve=None):
        """Yields GlobalIterate k = 0 .. iters-1; between yields the lower
        bound is solved with ``solve(x, y) -> (x, y)`` (default: FP64)."""
        solve = solve or self.solve
        x, y = np.array(x, dtype=np.float64), np.array(y, dtype=np.float64)
        for it in range(iters):
            ux, uy = x.copy(), y.copy()
            self.lal.legalize(ux, uy)
            a = float(alpha(it))
            self.ctx.build_b2b(x, y, a, ux, uy, self.fx, self.fy)
            yield GlobalIterate(it, a, x.copy(), y.copy(), ux, uy)
            x, y = solve(x, y)
