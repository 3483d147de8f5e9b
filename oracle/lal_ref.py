"""Reference restatement of SimPL's look-ahead legalization (test infrastructure only).

Pure Python over IEEE doubles, following the reference's operation order so
that its results are bit-identical to LookAheadLegalizer::legalize
(globalPlacer/simpl/simpl_lal.cc:43-372) with the BinGrid and FreeSpace of
globalPlacer/simpl/simpl_grid.h. It is the checker for the GPU legalizer
(ktplace_b200/csrc/ktg_lal.cu) and is itself pinned against the compiled
reference (oracle/_ref, RefDesign.lal) in tests/test_lal_oracle.py. Meant for
small designs (it is a plain Python loop).

Inputs: width/height/area of the movable cells, the bin grid (origin, dx, dy,
nx, ny, avail), the FreeSpace rows (sorted by bottom edge, spans already cut
by the obstacles), the obstacles, the die, densityLimit and the options
maxLevel, minCellsToSplit, stripeAreaFraction.
"""
from __future__ import annotations

import bisect
import math

INF = float("inf")
DBL_MAX = 1.7976931348623157e308


def smax(a, b):  # std::max
    return b if a < b else a


def smin(a, b):  # std::min
    return b if b < a else a


def clamp(v, lo, hi):  # std::clamp
    return lo if v < lo else (hi if hi < v else v)


class Profile:
    """AxisProfile (simpl_grid.h:29-65)."""

    def __init__(self, lo):
        self.edges = [lo]
        self.prefix = [0.0]

    def extend(self, to, area):
        if to > self.edges[-1]:
            self.edges.append(to)
            self.prefix.append(self.prefix[-1] + area)

    def total(self):
        return self.prefix[-1]

    def before(self, c):
        e = self.edges
        if c <= e[0]:
            return 0.0
        if c >= e[-1]:
            return self.total()
        k = bisect.bisect_right(e, c) - 1
        f = (c - e[k]) / (e[k + 1] - e[k])
        return self.prefix[k] + f * (self.prefix[k + 1] - self.prefix[k])

    def between(self, a, b):
        return self.before(b) - self.before(a)

    def coordinate_at(self, target):
        if target <= 0.0:
            return self.edges[0]
        if target >= self.total():
            return self.edges[-1]
        k = bisect.bisect_left(self.prefix, target)
        step = self.prefix[k] - self.prefix[k - 1]
        f = (target - self.prefix[k - 1]) / step if step > 0.0 else 1.0
        return self.edges[k - 1] + f * (self.edges[k] - self.edges[k - 1])


class LAL:
    def __init__(self, width, height, grid, rows, obstacles, die, density_limit=1.0,
                 max_level=20, min_cells=4, stripe_fraction=0.1):
        self.w = [float(v) for v in width]
        self.h = [float(v) for v in height]
        self.area = [a * b for a, b in zip(self.w, self.h)]
        g = grid
        self.ox, self.oy, self.dx, self.dy = float(g["origin"][0]), float(g["origin"][1]), \
            float(g["dx"]), float(g["dy"])
        self.nx, self.ny = int(g["nx"]), int(g["ny"])
        self.avail = [float(v) for v in g["avail"]]
        # rows: list of (y0, y1, [(x0, x1), ...]) sorted by y0
        self.rows = rows
        self.row_end = [r[1] for r in rows]
        self.obst = [tuple(float(v) for v in o) for o in obstacles]
        self.die = tuple(float(v) for v in die)
        self.limit = float(density_limit)
        self.max_level = max_level
        self.min_cells = min_cells
        self.frac = stripe_fraction

    # ---- grid ---------------------------------------------------------------
    def clamp_index(self, f, n):
        return int(clamp(f, 0.0, float(n) - 1e-9))

    def bin_of(self, cx, cy):
        ix = self.clamp_index((cx - self.ox) / self.dx, self.nx)
        iy = self.clamp_index((cy - self.oy) / self.dy, self.ny)
        return iy * self.nx + ix

    def edge(self, vertical, t):
        return self.ox + float(t) * self.dx if vertical else self.oy + float(t) * self.dy

    def box_of(self, r):
        x0, x1, y0, y1 = r
        return (self.edge(True, x0), self.edge(False, y0), self.edge(True, x1 + 1),
                self.edge(False, y1 + 1))

    def rect_sum(self, field, r):
        x0, x1, y0, y1 = r
        t = 0.0
        for iy in range(y0, y1 + 1):
            for ix in range(x0, x1 + 1):
                t += field[iy * self.nx + ix]
        return t

    def density(self, occ, r):
        cells = self.rect_sum(occ, r)
        room = self.rect_sum(self.avail, r)
        if room > 0.0:
            return cells / room
        return INF if cells > 0.0 else 0.0

    def centre(self, pos, i, vertical):
        return pos[i] + 0.5 * (self.w[i] if vertical else self.h[i])

    # ---- free space -------------------------------------------------------------
    def profile(self, box, vertical):
        lx, ly, ux, uy = box
        first = bisect.bisect_right(self.row_end, ly)  # first row with ly < y.end
        lo, hi = (lx, ux) if vertical else (ly, uy)
        out = Profile(lo)
        if vertical:
            steps = []
            r = first
            while r < len(self.rows) and self.rows[r][0] < uy:
                y0, y1, spans = self.rows[r]
                h = smin(uy, y1) - smax(ly, y0)
                for s0, s1 in spans:
                    a = smax(s0, lo)
                    z = smin(s1, hi)
                    if h > 0.0 and z > a:
                        steps.append((a, h))
                        steps.append((z, -h))
                r += 1
            steps.sort()
            height = 0.0
            for at, dh in steps:
                out.extend(at, height * (at - out.edges[-1]))
                height += dh
        else:
            r = first
            while r < len(self.rows) and self.rows[r][0] < uy:
                y0, y1, spans = self.rows[r]
                a = smax(lo, y0)
                z = smin(hi, y1)
                if z > a:
                    out.extend(a, 0.0)
                    length = 0.0
                    for s0, s1 in spans:
                        length += smax(0.0, smin(ux, s1) - smax(lx, s0))
                    out.extend(z, length * (z - a))
                r += 1
        out.extend(hi, 0.0)
        if len(out.edges) == 1:
            out.edges.append(hi)
            out.prefix.append(0.0)
        return out

    # ---- clusters ---------------------------------------------------------------
    def clusters(self, occ):
        nx, ny = self.nx, self.ny
        over = [1 if occ[k] > self.limit * self.avail[k] else 0 for k in range(nx * ny)]
        regions = []
        for seed in range(nx * ny):
            if not over[seed]:
                continue
            over[seed] = 0
            frontier = [seed]
            r = [seed % nx, seed % nx, seed // nx, seed // nx]
            while frontier:
                k = frontier.pop()
                ix, iy = k % nx, k // nx
                r = [min(r[0], ix), max(r[1], ix), min(r[2], iy), max(r[3], iy)]
                for sx, sy in ((1, 0), (-1, 0), (0, 1), (0, -1)):
                    px, py = ix + sx, iy + sy
                    if px < 0 or py < 0 or px >= nx or py >= ny:
                        continue
                    kk = py * nx + px
                    if over[kk]:
                        over[kk] = 0
                        frontier.append(kk)
            regions.append(tuple(r))
        return regions

    def grown(self, r, occ):
        x0, x1, y0, y1 = r
        while self.density(occ, (x0, x1, y0, y1)) > self.limit:
            wider = [(x0 - 1 if x0 > 0 else x0, x1, y0, y1),
                     (x0, x1 + 1 if x1 + 1 < self.nx else x1, y0, y1),
                     (x0, x1, y0 - 1 if y0 > 0 else y0, y1),
                     (x0, x1, y0, y1 + 1 if y1 + 1 < self.ny else y1)]
            bins = (x1 - x0 + 1) * (y1 - y0 + 1)
            best, best_d = None, INF
            for w in wider:
                if (w[1] - w[0] + 1) * (w[3] - w[2] + 1) == bins:
                    continue
                d = self.density(occ, w)
                if best is None or d < best_d:
                    best, best_d = w, d
            if best is None:
                break
            x0, x1, y0, y1 = best
        return (x0, x1, y0, y1)

    # ---- bisection ----------------------------------------------------------------
    def stripes(self, box, vertical, cell_area, region_room):
        lx, ly, ux, uy = box
        lo, hi = (lx, ux) if vertical else (ly, uy)
        room = self.profile(box, vertical)
        cuts = [lo, hi]
        for o in self.obst:
            if o[2] <= lx or o[0] >= ux or o[3] <= ly or o[1] >= uy:
                continue
            for e in ((o[0], o[2]) if vertical else (o[1], o[3])):
                if e > lo and e < hi:
                    cuts.append(e)
        cuts.sort()
        uniq = []
        for c in cuts:
            if not uniq or uniq[-1] != c:
                uniq.append(c)
        cuts = uniq
        limit = self.frac * (region_room if region_room > 0.0 else room.total())
        fill = smin(self.limit, cell_area / room.total()) if room.total() > 0.0 else self.limit
        s = 0
        while s + 1 < len(cuts):
            a, b = cuts[s], cuts[s + 1]
            here = room.between(a, b)
            mid = room.coordinate_at(room.before(a) + 0.5 * here)
            if here > limit and mid > a and mid < b:
                cuts.insert(s + 1, mid)
            else:
                s += 1
        return [[cuts[s], cuts[s + 1], fill * room.between(cuts[s], cuts[s + 1]), 0.0, []]
                for s in range(len(cuts) - 1)]

    def nonlinear_scale(self, cells, box, vertical, cutline, below, pos, region_room):
        if not cells:
            return
        cell_area = 0.0
        for i in cells:
            cell_area += self.area[i]
        strips = self.stripes(box, vertical, cell_area, region_room)

        def from_cut(c):
            return cutline - c if below else c - cutline

        strips.sort(key=lambda st: -from_cut(0.5 * (st[0] + st[1])))  # stable, descending
        order = sorted(cells, key=lambda i: (-from_cut(self.centre(pos, i, vertical)), i))
        s = 0
        for i in order:
            while s + 1 < len(strips) and strips[s][3] >= strips[s][2]:
                s += 1
            strips[s][4].append(i)
            strips[s][3] += self.area[i]
        for st in strips:
            if not st[4]:
                continue
            lo, hi = DBL_MAX, -DBL_MAX
            for i in st[4]:
                c = self.centre(pos, i, vertical)
                lo = smin(lo, c)
                hi = smax(hi, c)
            for i in st[4]:
                t = (self.centre(pos, i, vertical) - lo) / (hi - lo) if hi > lo else 0.5
                size = self.w[i] if vertical else self.h[i]
                c = st[0] + t * (st[1] - st[0])
                pos[i] = clamp(c - 0.5 * size, st[0], smax(st[0], st[1] - size))

    def legalize_block(self, box, level, vertical, cells, region_room, x, y):
        stack = [(box, level, vertical, cells)]
        while stack:
            box, level, vertical, cells = stack.pop()
            if level >= self.max_level or len(cells) <= self.min_cells:
                continue
            pos = x if vertical else y
            cells = sorted(cells, key=lambda i: (self.centre(pos, i, vertical), i))
            cell_area = 0.0
            for i in cells:
                cell_area += self.area[i]
            m, low_area = 0, 0.0
            while m + 1 < len(cells) and (m == 0 or low_area < 0.5 * cell_area):
                low_area += self.area[cells[m]]
                m += 1
            low, high = cells[:m], cells[m:]
            lx, ly, ux, uy = box
            lo, hi = (lx, ux) if vertical else (ly, uy)
            room = self.profile(box, vertical)
            share = low_area / cell_area if cell_area > 0.0 else 0.5
            cut = room.coordinate_at(share * room.total()) if room.total() > 0.0 \
                else lo + share * (hi - lo)
            low_box = (lx, ly, cut, uy) if vertical else (lx, ly, ux, cut)
            high_box = (cut, ly, ux, uy) if vertical else (lx, cut, ux, uy)
            self.nonlinear_scale(low, low_box, vertical, cut, True, pos, region_room)
            self.nonlinear_scale(high, high_box, vertical, cut, False, pos, region_room)
            stack.append((high_box, level + 1, not vertical, high))
            stack.append((low_box, level + 1, not vertical, low))

    # ---- top level -------------------------------------------------------------------
    def legalize(self, x, y):
        x, y = [float(v) for v in x], [float(v) for v in y]
        n = len(x)
        binof = [self.bin_of(self.centre(x, i, True), self.centre(y, i, False)) for i in range(n)]
        occ = [0.0] * (self.nx * self.ny)
        for i in range(n):
            occ[binof[i]] += self.area[i]

        def reach(r):
            return (r[0] - 1 if r[0] > 0 else 0, min(r[1] + 1, self.nx - 1),
                    r[2] - 1 if r[2] > 0 else 0, min(r[3] + 1, self.ny - 1))

        def touches(a, b):
            return a[0] <= b[1] and b[0] <= a[1] and a[2] <= b[3] and b[2] <= a[3]

        batch = []

        def run_batch():
            for bins, _ in batch:
                cells = [i for i in range(n)
                         if bins[0] <= binof[i] % self.nx <= bins[1]
                         and bins[2] <= binof[i] // self.nx <= bins[3]]
                room = self.rect_sum(self.avail, bins)
                self.legalize_block(self.box_of(bins), 1, True, cells, room, x, y)
                for i in cells:
                    k = self.bin_of(self.centre(x, i, True), self.centre(y, i, False))
                    if k != binof[i]:
                        occ[binof[i]] -= self.area[i]
                        occ[k] += self.area[i]
                        binof[i] = k
            batch.clear()

        for cluster in self.clusters(occ):
            bins = self.grown(cluster, occ)
            if any(touches(t[1], reach(bins)) for t in batch):
                run_batch()
                bins = self.grown(cluster, occ)
            batch.append((bins, reach(bins)))
        run_batch()
        lx, ly, ux, uy = self.die
        for i in range(n):
            x[i] = clamp(x[i], lx, smax(lx, ux - self.w[i]))
            y[i] = clamp(y[i], ly, smax(ly, uy - self.h[i]))
        return x, y


def free_rows(rows, row_span, spans):
    """FreeSpace rows in the form LAL takes, from RefDesign.free_space()."""
    out = []
    for r in range(rows.shape[0]):
        sp = [(float(spans[s, 0]), float(spans[s, 1])) for s in range(row_span[r], row_span[r + 1])]
        out.append((float(rows[r, 0]), float(rows[r, 1]), sp))
    return out
