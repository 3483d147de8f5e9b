"""Seeded synthetic standard-cell netlists in the shape of KTPlace's benchmarks.

The generator stands in for the public Bookshelf suites (ISPD-2005 adaptec1 and
friends) that the reference is run on: no benchmark file is read or reproduced,
only their published shapes (cell/net/pin counts, one-row standard cells,
fixed macros and boundary pads) are imitated with seeded random draws.

A design is produced as flat numpy arrays and can be written out as a Bookshelf
directory (.aux/.nodes/.nets/.pl/.scl) that the reference's own reader
(adaptor/bookshelfToKTAdaptor.cc) accepts, so the oracle build and the GPU path
consume the same netlist.

Geometry conventions follow the reference reader:
  * .nets pin offsets are centre-relative; the reader stores
    ``offset + 0.5 * size`` (lower-left relative), bookshelfToKTAdaptor.cc:430.
  * terminals are fixed (bookshelfToKTAdaptor.cc:286-291).
"""
from __future__ import annotations

import dataclasses
import math
import os
from typing import Optional

import numpy as np

ROW_HEIGHT = 12.0
SITE_WIDTH = 1.0


@dataclasses.dataclass
class SynthSpec:
    """Parameters of one synthetic design."""

    num_movable: int
    num_nets: int
    num_pads: int
    num_rows: int
    utilization: float = 0.7
    num_macros: int = 0
    macro_rows: tuple = (10, 60)
    macro_sites: tuple = (20, 200)
    width_sites: tuple = (1, 8)
    degree_min: int = 2
    degree_max: int = 50
    degree_exponent: float = 2.5
    seed: int = 0
    name: str = "synth"


@dataclasses.dataclass
class RawDesign:
    """Unflattened design, in Bookshelf order (movable cells, macros, pads)."""

    name: str
    width: np.ndarray        # [V] f64
    height: np.ndarray       # [V] f64
    x: np.ndarray            # [V] f64 lower-left (fixed cells; 0 for movable)
    y: np.ndarray            # [V] f64
    fixed: np.ndarray        # [V] bool
    net_start: np.ndarray    # [N+1] i64, pins of net n in file order
    pin_cell: np.ndarray     # [Pf] i64
    pin_fox: np.ndarray      # [Pf] f64 centre-relative offsets as written in .nets
    pin_foy: np.ndarray      # [Pf] f64
    net_weight: np.ndarray   # [N] f64
    num_rows: int
    sites_per_row: int
    row_height: float = ROW_HEIGHT
    site_width: float = SITE_WIDTH

    @property
    def num_vertices(self) -> int:
        return int(self.width.shape[0])

    @property
    def num_nets(self) -> int:
        return int(self.net_start.shape[0] - 1)

    @property
    def die(self):
        """Placement die box (lx, ly, ux, uy): rows unioned with fixed cells.

        Mirrors the result of getPlacementDieBox (datamodel/kt_die.cc:45-104)
        for designs whose pads and macros lie inside the row area, which is how
        this generator places them.
        """
        lx, ly = 0.0, 0.0
        ux = self.sites_per_row * self.site_width
        uy = self.num_rows * self.row_height
        fx = self.fixed
        if fx.any():
            lx = min(lx, float(self.x[fx].min()))
            ly = min(ly, float(self.y[fx].min()))
            ux = max(ux, float((self.x[fx] + np.maximum(self.width[fx], 1.0)).max()))
            uy = max(uy, float((self.y[fx] + np.maximum(self.height[fx], 1.0)).max()))
        return (lx, ly, ux, uy)


def degree_pmf(dmin: int, dmax: int, exponent: float) -> tuple:
    d = np.arange(dmin, dmax + 1, dtype=np.float64)
    p = d ** (-exponent)
    p /= p.sum()
    return d.astype(np.int64), p


def mean_degree(dmin: int = 2, dmax: int = 50, exponent: float = 2.5) -> float:
    d, p = degree_pmf(dmin, dmax, exponent)
    return float((d * p).sum())


def exponent_for_mean(target: float, dmin: int = 2, dmax: int = 50) -> float:
    """Power-law exponent whose truncated mean degree equals ``target``."""
    lo, hi = 1.0, 6.0
    for _ in range(80):
        mid = 0.5 * (lo + hi)
        if mean_degree(dmin, dmax, mid) > target:
            lo = mid
        else:
            hi = mid
    return 0.5 * (lo + hi)


def _place_macros(rng, n_macros, rows, sites, macro_rows, macro_sites):
    """Non-overlapping macros at uniform positions (rejection sampling on a
    row x site occupancy bitmap, largest first). Returns arrays in row/site
    units: (r0, s0, nr, ns)."""
    nr = rng.integers(macro_rows[0], macro_rows[1] + 1, size=n_macros)
    ns = rng.integers(macro_sites[0], macro_sites[1] + 1, size=n_macros)
    order = np.argsort(-(nr * ns), kind="stable")
    occ = np.zeros((rows, sites), dtype=bool)
    r0 = np.zeros(n_macros, dtype=np.int64)
    s0 = np.zeros(n_macros, dtype=np.int64)
    for k in order:
        h, w = int(nr[k]), int(ns[k])
        h = min(h, rows)
        w = min(w, sites)
        placed = False
        for _ in range(4000):
            rr = int(rng.integers(0, rows - h + 1))
            ss = int(rng.integers(0, sites - w + 1))
            if not occ[rr:rr + h, ss:ss + w].any():
                placed = True
                break
        if not placed:
            # Shrink until a free slot is found: keeps the count exact even
            # when random sequential packing jams.
            while not placed and (h > 1 or w > 1):
                h = max(1, h // 2)
                w = max(1, w // 2)
                for _ in range(4000):
                    rr = int(rng.integers(0, rows - h + 1))
                    ss = int(rng.integers(0, sites - w + 1))
                    if not occ[rr:rr + h, ss:ss + w].any():
                        placed = True
                        break
        occ[rr:rr + h, ss:ss + w] = True
        r0[k], s0[k], nr[k], ns[k] = rr, ss, h, w
    return r0, s0, nr.astype(np.int64), ns.astype(np.int64)


def generate(spec: SynthSpec) -> RawDesign:
    """Build a seeded synthetic design.

    Sites per row are derived from the stated utilisation, defined as movable
    area / (row area - macro area); the row count is kept as given.
    """
    rng = np.random.default_rng(spec.seed)
    n = spec.num_movable
    wsites = rng.integers(spec.width_sites[0], spec.width_sites[1] + 1, size=n)
    mov_w = wsites.astype(np.float64) * SITE_WIDTH
    mov_h = np.full(n, ROW_HEIGHT)
    mov_area_sites = float(wsites.sum())  # in site x row units

    m_nr = rng.integers(spec.macro_rows[0], spec.macro_rows[1] + 1, size=spec.num_macros)
    m_ns = rng.integers(spec.macro_sites[0], spec.macro_sites[1] + 1, size=spec.num_macros)
    macro_area = float((m_nr * m_ns).sum())
    total = mov_area_sites / spec.utilization + macro_area
    sites = int(math.ceil(total / spec.num_rows))
    sites = max(sites, spec.width_sites[1] * 4)

    r0, s0, nr, ns = _place_macros(rng, spec.num_macros, spec.num_rows, sites,
                                   spec.macro_rows, spec.macro_sites)
    mac_x = s0.astype(np.float64) * SITE_WIDTH
    mac_y = r0.astype(np.float64) * ROW_HEIGHT
    mac_w = ns.astype(np.float64) * SITE_WIDTH
    mac_h = nr.astype(np.float64) * ROW_HEIGHT

    # Pads: zero-size terminals evenly spaced on the die boundary (inside the
    # row area so the placement die stays the row box).
    W = sites * SITE_WIDTH
    H = spec.num_rows * ROW_HEIGHT
    per = 2.0 * (W + H)
    t = (np.arange(spec.num_pads, dtype=np.float64) + 0.5) * per / max(spec.num_pads, 1)
    pad_x = np.empty(spec.num_pads)
    pad_y = np.empty(spec.num_pads)
    for i, s in enumerate(t):
        if s < W:
            pad_x[i], pad_y[i] = s, 0.0
        elif s < W + H:
            pad_x[i], pad_y[i] = W - 1.0, s - W
        elif s < 2 * W + H:
            pad_x[i], pad_y[i] = W - (s - W - H), H - 1.0
        else:
            pad_x[i], pad_y[i] = 0.0, H - (s - 2 * W - H)
    pad_x = np.floor(np.clip(pad_x, 0.0, W - 1.0))
    pad_y = np.floor(np.clip(pad_y, 0.0, H - 1.0))

    V = n + spec.num_macros + spec.num_pads
    width = np.concatenate([mov_w, mac_w, np.zeros(spec.num_pads)])
    height = np.concatenate([mov_h, mac_h, np.zeros(spec.num_pads)])
    x = np.concatenate([np.zeros(n), mac_x, pad_x])
    y = np.concatenate([np.zeros(n), mac_y, pad_y])
    fixed = np.concatenate([np.zeros(n, bool), np.ones(spec.num_macros + spec.num_pads, bool)])

    # Nets: power-law degree, distinct cells drawn uniformly from all vertices.
    dvals, p = degree_pmf(spec.degree_min, spec.degree_max, spec.degree_exponent)
    deg = rng.choice(dvals, size=spec.num_nets, p=p)
    deg = np.minimum(deg, V)
    net_start = np.zeros(spec.num_nets + 1, dtype=np.int64)
    np.cumsum(deg, out=net_start[1:])
    P = int(net_start[-1])
    pin_cell = rng.integers(0, V, size=P)
    # Resample duplicates inside a net until every net has distinct cells.
    net_of_pin = np.repeat(np.arange(spec.num_nets), deg)
    for _ in range(64):
        key = net_of_pin * V + pin_cell
        order = np.argsort(key, kind="stable")
        ks = key[order]
        dup = np.zeros(P, bool)
        dup[order[1:]] = ks[1:] == ks[:-1]
        nd = int(dup.sum())
        if nd == 0:
            break
        pin_cell[dup] = rng.integers(0, V, size=nd)
    # Centre-relative pin offsets, uniform inside the cell.
    u = rng.random(P)
    v = rng.random(P)
    pin_fox = (u - 0.5) * width[pin_cell]
    pin_foy = (v - 0.5) * height[pin_cell]
    return RawDesign(
        name=spec.name, width=width, height=height, x=x, y=y, fixed=fixed,
        net_start=net_start, pin_cell=pin_cell.astype(np.int64),
        pin_fox=pin_fox, pin_foy=pin_foy,
        net_weight=np.ones(spec.num_nets), num_rows=spec.num_rows, sites_per_row=sites)


# --- the configurations the hot path is measured and checked on -------------

def spec_small(seed: int = 0) -> SynthSpec:
    """12,000 movable cells, 13,000 nets, 200 pads, 120 rows at 70% density."""
    return SynthSpec(num_movable=12_000, num_nets=13_000, num_pads=200, num_rows=120,
                     utilization=0.7, seed=seed, name=f"synth12k_s{seed}")


def spec_adaptec1_like(seed: int = 1) -> SynthSpec:
    """211k movable cells, 221k nets, 550 macros, 1,000 pads, 890 rows at 60%."""
    return SynthSpec(num_movable=211_000, num_nets=221_000, num_pads=1_000, num_rows=890,
                     utilization=0.6, num_macros=550, seed=seed, name=f"synth211k_s{seed}")


def spec_batch_member(k: int, seed_base: int = 1000) -> SynthSpec:
    """Netlist k of the 64-design batch: log-uniform 5k-200k cells, mean
    degree 3.5, 65% density."""
    rng = np.random.default_rng(seed_base + k)
    cells = int(round(math.exp(rng.uniform(math.log(5_000), math.log(200_000)))))
    nets = int(round(cells * 13 / 12))
    rows = max(20, int(round(120 * math.sqrt(cells / 12_000))))
    pads = max(50, int(round(200 * math.sqrt(cells / 12_000))))
    return SynthSpec(num_movable=cells, num_nets=nets, num_pads=pads, num_rows=rows,
                     utilization=0.65, degree_exponent=exponent_for_mean(3.5),
                     seed=seed_base + k, name=f"synthbatch{k}")


def spec_2m(seed: int = 4) -> SynthSpec:
    """2.2M movable cells, 2.25M nets, 8,000 macros at 60% density."""
    rows = 2_900
    return SynthSpec(num_movable=2_200_000, num_nets=2_250_000, num_pads=4_000,
                     num_rows=rows, utilization=0.6, num_macros=8_000, seed=seed,
                     name=f"synth2m_s{seed}")


def spec_tiny(seed: int = 0, cells: int = 300, nets: int = 330, pads: int = 16,
              rows: int = 12, macros: int = 0) -> SynthSpec:
    return SynthSpec(num_movable=cells, num_nets=nets, num_pads=pads, num_rows=rows,
                     utilization=0.7, num_macros=macros, macro_rows=(2, 4),
                     macro_sites=(4, 12), seed=seed, name=f"tiny{cells}_s{seed}")


# --- Bookshelf output ----------------------------------------------------------

def _names(d: RawDesign, n_movable: int):
    names = []
    for v in range(d.num_vertices):
        names.append(f"o{v}" if v < n_movable else f"t{v}")
    return names


def write_bookshelf(d: RawDesign, directory: str) -> str:
    """Write ``d`` as a Bookshelf design directory named after ``d.name``.

    Floating-point values are written with ``repr`` so that they read back
    bit-exactly through ``std::stod``.
    """
    os.makedirs(directory, exist_ok=True)
    base = os.path.join(directory, d.name)
    V = d.num_vertices
    n_mov = int((~d.fixed).sum())
    assert not d.fixed[:n_mov].any(), "movable cells must come first"
    names = _names(d, n_mov)
    with open(base + ".aux", "w") as f:
        f.write(f"RowBasedPlacement : {d.name}.nodes {d.name}.nets {d.name}.wts "
                f"{d.name}.pl {d.name}.scl\n")
    with open(base + ".nodes", "w") as f:
        f.write("UCLA nodes 1.0\n\n")
        f.write(f"NumNodes : {V}\nNumTerminals : {V - n_mov}\n")
        lines = []
        for v in range(V):
            t = " terminal" if d.fixed[v] else ""
            lines.append(f"{names[v]} {repr(float(d.width[v]))} {repr(float(d.height[v]))}{t}\n")
        f.writelines(lines)
    with open(base + ".nets", "w") as f:
        f.write("UCLA nets 1.0\n\n")
        f.write(f"NumNets : {d.num_nets}\nNumPins : {int(d.net_start[-1])}\n")
        lines = []
        ns = d.net_start
        for n in range(d.num_nets):
            a, b = int(ns[n]), int(ns[n + 1])
            lines.append(f"NetDegree : {b - a} n{n}\n")
            for p in range(a, b):
                lines.append(f"\t{names[int(d.pin_cell[p])]} I : "
                             f"{repr(float(d.pin_fox[p]))} {repr(float(d.pin_foy[p]))}\n")
        f.writelines(lines)
    with open(base + ".wts", "w") as f:
        f.write("UCLA wts 1.0\n\n")
    with open(base + ".pl", "w") as f:
        f.write("UCLA pl 1.0\n\n")
        lines = []
        for v in range(V):
            fx = " /FIXED" if d.fixed[v] else ""
            lines.append(f"{names[v]} {repr(float(d.x[v]))} {repr(float(d.y[v]))} : N{fx}\n")
        f.writelines(lines)
    with open(base + ".scl", "w") as f:
        f.write("UCLA scl 1.0\n\n")
        f.write(f"NumRows : {d.num_rows}\n\n")
        for r in range(d.num_rows):
            f.write("CoreRow Horizontal\n")
            f.write(f"  Coordinate : {repr(float(r * d.row_height))}\n")
            f.write(f"  Height : {repr(float(d.row_height))}\n")
            f.write(f"  Sitewidth : {repr(float(d.site_width))}\n")
            f.write(f"  Sitespacing : {repr(float(d.site_width))}\n")
            f.write("  Siteorient : 1\n  Sitesymmetry : 1\n")
            f.write(f"  SubrowOrigin : 0 NumSites : {d.sites_per_row}\n")
            f.write("End\n")
    return directory


# --- positions for one SimPL iteration -----------------------------------------

def seed_positions(d: RawDesign, n_movable: int, seed: int):
    """Uniform random lower-left positions of the movable cells inside the die
    (the same law as SimPL's seedUniform, simpl_placer.cc:226-237, drawn from
    numpy's PCG64 instead of mt19937_64)."""
    rng = np.random.default_rng(seed)
    lx, ly, ux, uy = d.die
    w = d.width[:n_movable]
    h = d.height[:n_movable]
    x = lx + rng.random(n_movable) * np.maximum((ux - lx) - w, 0.0)
    y = ly + rng.random(n_movable) * np.maximum((uy - ly) - h, 0.0)
    return x, y
