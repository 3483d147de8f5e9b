"""Parity cases shared by the golden-vector generator and the tests.

Each case is a seeded synthetic design plus the inputs of one SimPL
iteration (positions, anchors, alpha). ``edge_design`` is hand-built to hit the
corner cases of the path: one-pin nets, all-fixed nets, a cell listed twice on
a net, coincident pins (lo == hi), ties for the extreme pin, a net wider than
a warp, non-unit weights, an isolated cell and a macro.
"""
import numpy as np

from ktplace_b200 import synth
from ktplace_b200.synth import RawDesign, ROW_HEIGHT

TOL = 1e-6
MAX_ITER = 1000


def edge_design() -> RawDesign:
    rng = np.random.default_rng(7)
    n_mov, n_pad = 40, 6
    width = np.concatenate([rng.integers(1, 9, n_mov).astype(float), [4.0], np.zeros(n_pad)])
    height = np.concatenate([np.full(n_mov, ROW_HEIGHT), [24.0], np.zeros(n_pad)])
    V = n_mov + 1 + n_pad
    x = np.zeros(V)
    y = np.zeros(V)
    x[n_mov], y[n_mov] = 20.0, 12.0                       # macro
    pads = n_mov + 1 + np.arange(n_pad)
    x[pads] = [0.0, 59.0, 30.0, 0.0, 59.0, 10.0]
    y[pads] = [0.0, 0.0, 47.0, 30.0, 40.0, 47.0]
    fixed = np.zeros(V, bool)
    fixed[n_mov:] = True
    nets = []
    w = []
    nets.append([0, 1]); w.append(1.0)                     # 2-pin
    nets.append([2]); w.append(1.0)                        # 1-pin
    nets.append([pads[0], pads[1]]); w.append(1.0)         # all fixed
    nets.append([3, 4, 3, 5]); w.append(1.0)               # cell 3 twice
    nets.append([10, 11]); w.append(1.0)                   # coincident pins
    nets.append([12, 13, 14]); w.append(1.0)               # ties for the minimum
    big = list(range(5, 35)) + list(pads) + [n_mov] + [36, 37, 38]
    nets.append(big); w.append(1.0)                        # 40 pins
    nets.append([15, 16, pads[2]]); w.append(2.5)
    nets.append([17, 18, 19, 20]); w.append(0.5)
    nets.append([21, n_mov, 22]); w.append(1.0)            # macro pin
    nets.append([23, 24, 25, 26, 27, 28]); w.append(1.0)
    nets.append([29, 30]); w.append(1.0)
    nets.append([31, 32, 33, pads[3], pads[4]]); w.append(1.0)
    nets.append([34, 0, 1, 2]); w.append(1.0)
    nets.append([]); w.append(1.0)                          # empty net
    # cell 39 is on no net at all
    net_start = np.zeros(len(nets) + 1, np.int64)
    np.cumsum([len(a) for a in nets], out=net_start[1:])
    pin_cell = np.array([c for a in nets for c in a], np.int64)
    fox = (rng.random(pin_cell.shape[0]) - 0.5) * width[pin_cell]
    foy = (rng.random(pin_cell.shape[0]) - 0.5) * height[pin_cell]
    # coincident net: identical offsets on both cells (positions set equal below)
    k = net_start[4]
    fox[k + 1], foy[k + 1] = fox[k], foy[k]
    width[11] = width[10]
    fox[k + 1] = fox[k]
    # tie net: cells 12 and 13 end up with the same pin coordinate (positions below)
    k = net_start[5]
    fox[k + 1], foy[k + 1] = fox[k], foy[k]
    width[13] = width[12]
    return RawDesign(name="edge", width=width, height=height, x=x, y=y, fixed=fixed,
                     net_start=net_start, pin_cell=pin_cell, pin_fox=fox, pin_foy=foy,
                     net_weight=np.array(w), num_rows=4, sites_per_row=60)


def edge_positions(raw, nl, seed):
    x, y = synth.seed_positions(raw, nl.num_movable, seed)
    x[11], y[11] = x[10], y[10]
    x[13], y[13] = x[12], y[12]
    return x, y


CASES = {
    "tiny_macros": dict(spec=lambda: synth.spec_tiny(seed=0, cells=300, nets=330, pads=16,
                                                     rows=12, macros=3),
                        pos_seed=11, anchor_seed=12, alpha=0.2, grid=16),
    "edge_alpha0": dict(raw=edge_design, pos_seed=3, anchor_seed=4, alpha=0.0, grid=8),
    "edge_alpha": dict(raw=edge_design, pos_seed=3, anchor_seed=4, alpha=0.3, grid=8),
    "small12k": dict(spec=lambda: synth.spec_small(seed=0), pos_seed=21, anchor_seed=22,
                     alpha=0.2, grid=32),
}


def build_case(name):
    """Returns (raw, netlist, x, y, ax, ay, alpha, grid_bins) for a case."""
    from ktplace_b200 import netlist
    c = CASES[name]
    raw = c["raw"]() if "raw" in c else synth.generate(c["spec"]())
    nl = netlist.flatten(raw)
    if "raw" in c:
        x, y = edge_positions(raw, nl, c["pos_seed"])
        ax, ay = synth.seed_positions(raw, nl.num_movable, c["anchor_seed"])
    else:
        x, y = synth.seed_positions(raw, nl.num_movable, c["pos_seed"])
        ax, ay = synth.seed_positions(raw, nl.num_movable, c["anchor_seed"])
    return raw, nl, x, y, ax, ay, c["alpha"], c["grid"]


def digest(a: np.ndarray) -> str:
    import hashlib
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def netlist_digest(nl) -> str:
    parts = [nl.mov_vertex.astype(np.int32), nl.var_of_vertex.astype(np.int32),
             nl.net_start.astype(np.int64), nl.pin_cell.astype(np.int32), nl.off_x, nl.off_y,
             nl.net_weight, nl.pin_start.astype(np.int64), nl.pin_net.astype(np.int32),
             nl.pin_q.astype(np.int32), nl.fixed_x, nl.fixed_y, nl.width, nl.height]
    return digest(np.concatenate([np.frombuffer(np.ascontiguousarray(p).tobytes(), np.uint8)
                                  for p in parts]))
