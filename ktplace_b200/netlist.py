"""SimPL's flattened netlist as device-ready structure-of-arrays.

Mirrors ``ktplace::simpl::Netlist`` (globalPlacer/simpl/simpl_lss.h:27-36) and
the way ``collectCells`` / ``collectNets`` build it (globalPlacer/simpl/
simpl_dm.cc:16-85):

* movable vertices get consecutive variable ids in vertex order; fixed and
  terminal vertices map to no variable (-1 here, ``noVar`` there);
* each net's pins are stable-sorted by cell id and a cell's second and later
  pins on the same net are dropped, keeping the first pin's offset;
* ``pin_start``/``pin_net``/``pin_q`` list, per movable cell, its (net, pin
  index) pairs in ascending net order.

Also carries what the density reduction needs (width, height, area of the
movable cells, obstacles and rows for the bin grid).
"""
from __future__ import annotations

import dataclasses

import numpy as np

from .synth import RawDesign


@dataclasses.dataclass
class Netlist:
    num_vertices: int
    num_movable: int
    mov_vertex: np.ndarray      # [n] i32
    var_of_vertex: np.ndarray   # [V] i32, -1 = fixed
    fixed_x: np.ndarray         # [V] f64
    fixed_y: np.ndarray         # [V] f64
    net_start: np.ndarray       # [N+1] i64
    pin_cell: np.ndarray        # [P] i32
    off_x: np.ndarray           # [P] f64, lower-left relative
    off_y: np.ndarray           # [P] f64
    net_weight: np.ndarray      # [N] f64
    pin_start: np.ndarray       # [n+1] i64
    pin_net: np.ndarray         # [Pm] i32
    pin_q: np.ndarray           # [Pm] i32
    width: np.ndarray           # [n] f64 (movable cells)
    height: np.ndarray          # [n] f64
    obstacles: np.ndarray       # [K,4] f64 (lx, ly, ux, uy) of fixed cells with area
    rows: np.ndarray            # [R,5] f64 (coordinate, height, pitch, xlo, xhi)
    die: tuple                  # (lx, ly, ux, uy)

    @property
    def num_nets(self) -> int:
        return int(self.net_start.shape[0] - 1)

    @property
    def num_pins(self) -> int:
        return int(self.net_start[-1])

    @property
    def area(self) -> np.ndarray:
        return self.width * self.height

    def floors(self) -> tuple:
        """Minimum B2B edge lengths: mean movable width and height
        (simplPlacer::Impl::collect, simpl_placer.cc:169-179)."""
        n = self.num_movable
        if n == 0:
            return 1.0, 1.0
        # Sequential accumulation in index order, as std::accumulate does.
        fx = 0.0
        for v in self.width.tolist():
            fx += v
        fy = 0.0
        for v in self.height.tolist():
            fy += v
        return fx / n, fy / n


def flatten(d: RawDesign, kraftwerk2: bool = False) -> Netlist:
    """Flatten a raw design the way SimPL's buildSimplDM does.

    kraftwerk2=True keeps every pin in its listed order instead, duplicates
    of a cell within a net included, as Kraftwerk2's collectNets does
    (globalPlacer/kraftwerk2/kraftwerk2_dm.cc:34-54)."""
    V = d.num_vertices
    movable = ~d.fixed
    mov_vertex = np.nonzero(movable)[0].astype(np.int32)
    n = int(mov_vertex.shape[0])
    var = np.full(V, -1, dtype=np.int32)
    var[mov_vertex] = np.arange(n, dtype=np.int32)

    N = d.num_nets
    deg_raw = np.diff(d.net_start)
    net_of = np.repeat(np.arange(N, dtype=np.int64), deg_raw)
    P_raw = int(d.net_start[-1])
    # Stable sort by cell id within each net (lexsort keys: last is primary).
    if kraftwerk2:
        sel = np.arange(P_raw)
    else:
        order = np.lexsort((np.arange(P_raw), d.pin_cell, net_of))
        cells_sorted = d.pin_cell[order]
        nets_sorted = net_of[order]
        keep = np.ones(P_raw, dtype=bool)
        keep[1:] = ~((nets_sorted[1:] == nets_sorted[:-1]) &
                     (cells_sorted[1:] == cells_sorted[:-1]))
        sel = order[keep]
    pin_cell = d.pin_cell[sel].astype(np.int32)
    pin_net_all = net_of[sel]
    # Lower-left relative offsets, as bookshelfToKTAdaptor.cc:430 forms them.
    off_x = d.pin_fox[sel] + 0.5 * d.width[d.pin_cell[sel]]
    off_y = d.pin_foy[sel] + 0.5 * d.height[d.pin_cell[sel]]
    deg = np.bincount(pin_net_all, minlength=N)
    net_start = np.zeros(N + 1, dtype=np.int64)
    np.cumsum(deg, out=net_start[1:])
    q_all = np.arange(pin_cell.shape[0], dtype=np.int64) - net_start[pin_net_all]

    pv = var[pin_cell]
    mov_pins = np.nonzero(pv >= 0)[0]
    # Stable by variable: keeps ascending (net, q) order within a cell.
    o2 = np.argsort(pv[mov_pins], kind="stable")
    mp = mov_pins[o2]
    pin_net = pin_net_all[mp].astype(np.int32)
    pin_q = q_all[mp].astype(np.int32)
    counts = np.bincount(pv[mov_pins], minlength=n)
    pin_start = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(counts, out=pin_start[1:])

    fx = d.fixed
    obst_mask = fx & (d.width > 0) & (d.height > 0)
    obstacles = np.stack([d.x[obst_mask], d.y[obst_mask],
                          d.x[obst_mask] + d.width[obst_mask],
                          d.y[obst_mask] + d.height[obst_mask]], axis=1) if obst_mask.any() \
        else np.zeros((0, 4))
    R = d.num_rows
    rows = np.stack([np.arange(R) * d.row_height, np.full(R, d.row_height),
                     np.full(R, d.site_width), np.zeros(R),
                     np.full(R, d.sites_per_row * d.site_width)], axis=1).astype(np.float64)
    return Netlist(
        num_vertices=V, num_movable=n, mov_vertex=mov_vertex, var_of_vertex=var,
        fixed_x=d.x.astype(np.float64).copy(), fixed_y=d.y.astype(np.float64).copy(),
        net_start=net_start, pin_cell=pin_cell, off_x=off_x, off_y=off_y,
        net_weight=d.net_weight.astype(np.float64).copy(), pin_start=pin_start,
        pin_net=pin_net, pin_q=pin_q, width=d.width[mov_vertex].astype(np.float64),
        height=d.height[mov_vertex].astype(np.float64), obstacles=obstacles, rows=rows,
        die=d.die)
