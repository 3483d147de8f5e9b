"""SimPL's density bin grid, built on the host once per grid size.

Restates, for the host side of the GPU path, how simplPlacer::Impl::buildGrid
(globalPlacer/simpl/simpl_placer.cc:190-224) derives the free row area of each
bin: rows are cut by the fixed obstacles (FreeSpace::build, simpl_grid.h:
145-177), every free span is deposited into the bins it overlaps
(BinGrid::deposit, simpl_grid.h:108-123), slivers under 1e-3 of the smallest
site are zeroed, and the total is a sequential sum. The arithmetic follows the
reference's expression order so the result is bit-identical; the GPU uploads
it once (ktg_set_grid) and only the occupancy is recomputed per iteration.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np


@dataclasses.dataclass
class BinGrid:
    origin_x: float
    origin_y: float
    dx: float
    dy: float
    nx: int
    ny: int
    avail: np.ndarray      # [ny*nx], bin (ix, iy) at iy*nx+ix
    total_avail: float
    density_limit: float = 1.0

    @property
    def size(self) -> int:
        return self.nx * self.ny


def _min(a, b):
    return b if b < a else a


def _max(a, b):
    return b if a < b else a


def _clamp_index(f: float, n: int) -> int:
    hi = float(n) - 1e-9
    c = 0.0 if f < 0.0 else (hi if hi < f else f)
    return int(c)


def default_bins_per_axis(num_movable: int) -> int:
    """getDefaultBinsPerAxis (simpl_placer.cc:181-188) with no override."""
    v = math.sqrt(float(max(num_movable, 1)) / 51.0)
    return int(min(max(v, 16.0), 256.0))


def free_spans(rows: np.ndarray, obstacles: np.ndarray, subrows=None):
    """FreeSpace::build: per row (sorted by bottom edge) the free x spans.

    A row's spans are its subrows' x intervals (buildGrid, simpl_placer.cc:
    199-212) when `subrows` ([S, 3]: row index, x start, x end, as the
    Bookshelf reader returns them) is given, else the row's one span
    (xlo, xhi)."""
    out = []
    smallest = math.inf
    raw = []
    per_row = None
    if subrows is not None and len(subrows):
        per_row = {}
        for sr in np.asarray(subrows, np.float64).reshape(-1, 3):
            per_row.setdefault(int(sr[0]), []).append((float(sr[1]), float(sr[2])))
    for ri, r in enumerate(rows):
        coord, height, pitch, xlo, xhi = (float(v) for v in r)
        if not (height > 0.0) or not (pitch > 0.0):
            continue
        smallest = min(smallest, pitch * height)
        spans = [(xlo, xhi)] if per_row is None else per_row.get(ri, [])
        raw.append((coord, coord + height, spans))
    raw.sort(key=lambda t: t[0])  # stable
    for y0, y1, spans in raw:
        cuts = sorted((float(o[0]), float(o[2])) for o in obstacles
                      if o[3] > y0 and o[1] < y1)
        spans = sorted(spans)
        opened = []
        for s0, s1 in spans:
            a = s0
            for c0, c1 in cuts:
                if c1 <= a or c0 >= s1:
                    continue
                if c0 > a:
                    opened.append((a, c0))
                a = _max(a, c1)
            if s1 > a:
                opened.append((a, s1))
        out.append((y0, y1, opened))
    return out, smallest


@dataclasses.dataclass
class FreeSpace:
    """FreeSpace (simpl_grid.h:130-177) flattened for ktg_set_free_space:
    row r spans y in row_y[r] and holds spans[row_span[r]:row_span[r+1]]."""
    row_y: np.ndarray       # [R, 2] y start, y end (sorted by y start)
    row_span: np.ndarray    # [R + 1] int64
    spans: np.ndarray       # [S, 2] x start, x end
    obstacles: np.ndarray   # [K, 4] lx ly ux uy
    die: tuple


def build_free_space(nl) -> FreeSpace:
    """The free space LookAheadLegalizer works in: the design's rows cut by its
    obstacles (free_spans), the same obstacles and the die."""
    rows, _ = free_spans(nl.rows, nl.obstacles, getattr(nl, "subrows", None))
    row_y = np.array([(r[0], r[1]) for r in rows], np.float64).reshape(-1, 2)
    counts = np.array([len(r[2]) for r in rows], np.int64)
    row_span = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    spans = np.array([sp for r in rows for sp in r[2]], np.float64).reshape(-1, 2)
    obst = np.asarray(nl.obstacles, np.float64).reshape(-1, 4)
    return FreeSpace(row_y=row_y, row_span=row_span, spans=spans, obstacles=obst,
                     die=tuple(float(v) for v in nl.die))


def build_grid(nl, per_axis: int, density_limit: float = 1.0) -> BinGrid:
    lx, ly, ux, uy = nl.die
    nx = ny = int(per_axis)
    dx = _max(ux - lx, 1e-9) / float(per_axis)
    dy = _max(uy - ly, 1e-9) / float(per_axis)
    avail = np.zeros(nx * ny)
    rows, smallest = free_spans(nl.rows, nl.obstacles, getattr(nl, "subrows", None))

    def col(x):
        return _clamp_index((x - lx) / dx, nx)

    def row(y):
        return _clamp_index((y - ly) / dy, ny)

    for y0, y1, spans in rows:
        for a, b in spans:
            if not (b > a) or not (y1 > y0):
                continue
            ix0, ix1 = col(a), col(b)
            ixs = np.arange(ix0, ix1 + 1, dtype=np.float64)
            e0 = lx + ixs * dx
            e1 = lx + (ixs + 1.0) * dx
            ox = np.where(e1 < b, e1, b) - np.where(a < e0, e0, a)
            for iy in range(row(y0), row(y1) + 1):
                ey0 = ly + float(iy) * dy
                ey1 = ly + float(iy + 1) * dy
                oy = _min(y1, ey1) - _max(y0, ey0)
                if not (oy > 0.0):
                    continue
                m = ox > 0.0
                idx = iy * nx + np.arange(ix0, ix1 + 1)[m]
                avail[idx] += (1.0 * ox[m]) * oy
    sliver = 1e-3 * smallest if smallest < math.inf else 0.0
    avail[avail < sliver] = 0.0
    total = 0.0
    for v in avail.tolist():
        total += v
    return BinGrid(origin_x=lx, origin_y=ly, dx=dx, dy=dy, nx=nx, ny=ny, avail=avail,
                   total_avail=total, density_limit=min(max(density_limit, 0.05), 1.0))
