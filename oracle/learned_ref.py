"""Float64 reference of the learned preconditioner (test infrastructure only).

The checker for the GPU kernels in ktplace_b200/csrc/ktg_learned.cu: same
features, same network, same loss, with analytic gradients (themselves
checked by finite differences in tests/test_learned_oracle.py).

Preconditioner (SPD by construction, on A's sparsity pattern):
    M = D^-1/2 (I + S) D^-1/2,   D = diag(A)
    s_e = t_e * |a_e| / sqrt(d_i d_j)                 for entry e = (i, j) of A
    t_e = clamp(tanh(phi_e), -0.999, 0.999),  phi_e = <p_i, p_j> / 4
|S| <= 0.999 B entrywise with B = D^-1/2 |A_off| D^-1/2, and rho(B) <= 1 for the
diagonally dominant M-matrices SimPL builds, so rho(S) < 1 and I + S is SPD;
t = 1 everywhere would be the first-order Neumann preconditioner.

Network over the cell-net bipartite graph (mean aggregation), hidden 64:
    h0 = relu(x W_in + b_in)                                    x: 8 features/cell
    for l in 0..2:
        m_k = mean over movable cells c of net k of h[c]
        e_k = relu(m_k Wa_l + ba_l)
        g_c = mean over nets k of cell c of e_k
        h   = relu(h Wb_l + g Wc_l + bb_l)
    p = h P                                                      P: 64 x 16
Loss over K Rademacher probes v:  L = mean_k ||M A v_k - v_k||^2 / n.

Learned coarse vector (the two-level aggregation preconditioner's z): the
same trunk on features of the netlist alone (topo_features), then per system
    u_i = (p_i, c_i, l_i),  c_i = sum_j |a_ij| / a_ii,  l_i = log a_ii - mean log a
    z_i = softplus(relu(u_i Wh + bh) . wz + bz)
and the projection loss of test vectors e_t on z in the A-inner product
    L = mean_t (1 - (z^T A e_t)^2 / ((z^T A z)(e_t^T A e_t))).
"""
from __future__ import annotations

import numpy as np

HID = 64
PROJ = 16
NFEAT = 8
LAYERS = 3

PARAM_SHAPES = [("W_in", (NFEAT, HID)), ("b_in", (HID,))]
for _l in range(LAYERS):
    PARAM_SHAPES += [(f"Wa{_l}", (HID, HID)), (f"ba{_l}", (HID,)), (f"Wb{_l}", (HID, HID)),
                     (f"Wc{_l}", (HID, HID)), (f"bb{_l}", (HID,))]
PARAM_SHAPES += [("P", (HID, PROJ))]
HEAD_IN = PROJ + 2
HEAD_H = 16
PARAM_SHAPES += [("Wh", (HEAD_IN, HEAD_H)), ("bh", (HEAD_H,)), ("wz", (HEAD_H,)), ("bz", (1,))]


def num_params() -> int:
    return int(sum(np.prod(s) for _, s in PARAM_SHAPES))


def unflatten(flat: np.ndarray) -> dict:
    out, o = {}, 0
    for name, shape in PARAM_SHAPES:
        k = int(np.prod(shape))
        out[name] = flat[o:o + k].reshape(shape)
        o += k
    return out


def flatten(params: dict) -> np.ndarray:
    return np.concatenate([params[n].reshape(-1) for n, _ in PARAM_SHAPES])


def rows_of(s):
    n = s["diag"].shape[0]
    return np.repeat(np.arange(n), np.diff(s["row_ptr"]).astype(np.int64))


def features(s, nl) -> np.ndarray:
    """Per-cell features of one axis system (see the module docstring)."""
    n = s["diag"].shape[0]
    d = s["diag"]
    rows = rows_of(s)
    absa = np.abs(s["val"])
    rowabs = np.bincount(rows, weights=absa, minlength=n)
    rowmax = np.zeros(n)
    np.maximum.at(rowmax, rows, absa)
    rownnz = np.diff(s["row_ptr"]).astype(np.float64)
    npins = np.diff(nl.pin_start).astype(np.float64)
    logd = np.log(d)
    x = np.zeros((n, NFEAT))
    x[:, 0] = 1.0
    x[:, 1] = logd - logd.mean()
    x[:, 2] = (d - rowabs) / d
    x[:, 3] = rownnz / 16.0
    x[:, 4] = npins / 8.0
    x[:, 5] = rowabs / d
    x[:, 6] = rowmax / d
    x[:, 7] = np.log1p(rownnz) / 4.0
    return x


class Graph:
    """Mean-aggregation operators of the cell-net bipartite graph."""

    def __init__(self, nl):
        n = nl.num_movable
        N = nl.num_nets
        pv = nl.var_of_vertex[nl.pin_cell]
        net_of_pin = np.repeat(np.arange(N), np.diff(nl.net_start))
        mov = pv >= 0
        self.mc = pv[mov].astype(np.int64)           # movable pin -> cell
        self.mn = net_of_pin[mov].astype(np.int64)   # movable pin -> net
        self.net_cnt = np.bincount(self.mn, minlength=N).astype(np.float64)
        self.cell_cnt = np.bincount(self.mc, minlength=n).astype(np.float64)
        self.n, self.N = n, N

    def cells_to_nets(self, h):
        m = np.zeros((self.N, h.shape[1]))
        np.add.at(m, self.mn, h[self.mc])
        return m / np.maximum(self.net_cnt, 1.0)[:, None]

    def nets_to_cells(self, e):
        g = np.zeros((self.n, e.shape[1]))
        np.add.at(g, self.mc, e[self.mn])
        return g / np.maximum(self.cell_cnt, 1.0)[:, None]

    def cells_to_nets_T(self, dm):
        dh = np.zeros((self.n, dm.shape[1]))
        np.add.at(dh, self.mc, (dm / np.maximum(self.net_cnt, 1.0)[:, None])[self.mn])
        return dh

    def nets_to_cells_T(self, dg):
        de = np.zeros((self.N, dg.shape[1]))
        np.add.at(de, self.mn, (dg / np.maximum(self.cell_cnt, 1.0)[:, None])[self.mc])
        return de


def relu(z):
    return np.maximum(z, 0.0)


def forward(params, x, graph: Graph):
    cache = {"x": x}
    z = x @ params["W_in"] + params["b_in"]
    h = relu(z)
    cache["z_in"] = z
    cache["h0"] = h
    for l in range(LAYERS):
        m = graph.cells_to_nets(h)
        za = m @ params[f"Wa{l}"] + params[f"ba{l}"]
        e = relu(za)
        g = graph.nets_to_cells(e)
        zb = h @ params[f"Wb{l}"] + g @ params[f"Wc{l}"] + params[f"bb{l}"]
        cache[f"m{l}"], cache[f"za{l}"], cache[f"e{l}"], cache[f"g{l}"] = m, za, e, g
        cache[f"zb{l}"] = zb
        h = relu(zb)
        cache[f"h{l + 1}"] = h
    p = h @ params["P"]
    cache["p"] = p
    return p, cache


TMAX = 0.999


def entry_values(s, p):
    """phi, t, c and s for every stored entry of A."""
    rows = rows_of(s)
    cols = s["col"].astype(np.int64)
    d = s["diag"]
    phi = np.einsum("ij,ij->i", p[rows], p[cols]) / 4.0
    t = np.clip(np.tanh(phi), -TMAX, TMAX)
    c = np.abs(s["val"]) / np.sqrt(d[rows] * d[cols])
    return rows, cols, phi, t, c, t * c


def apply_m(s, svals, u):
    """M u = u / d + D^-1/2 S D^-1/2 u."""
    rows = rows_of(s)
    cols = s["col"].astype(np.int64)
    dis = 1.0 / np.sqrt(s["diag"])
    v = dis * u
    su = np.bincount(rows, weights=svals * v[cols], minlength=u.shape[0])
    return u / s["diag"] + dis * su


def spmv(s, v):
    rows = rows_of(s)
    return s["diag"] * v + np.bincount(rows, weights=s["val"] * v[s["col"].astype(np.int64)],
                                       minlength=v.shape[0])


def probes(n: int, k: int, seed: int) -> np.ndarray:
    """Rademacher probes shared with the GPU (hash of seed, probe, row)."""
    i = np.arange(n, dtype=np.uint64)
    out = np.empty((k, n))
    for j in range(k):
        h = (i * np.uint64(0x9E3779B97F4A7C15)) ^ np.uint64((seed * 0x632BE59BD9B4E019 +
                                                               j * 0xD1B54A32D192ED03)
                                                              & 0xFFFFFFFFFFFFFFFF)
        h ^= h >> np.uint64(31)
        h *= np.uint64(0xBF58476D1CE4E5B9)
        h ^= h >> np.uint64(29)
        out[j] = np.where((h >> np.uint64(17)) & np.uint64(1), 1.0, -1.0)
    return out


def loss_and_grad(params, s, nl, k: int = 4, seed: int = 0, graph: Graph | None = None):
    graph = graph or Graph(nl)
    x = features(s, nl)
    p, cache = forward(params, x, graph)
    rows, cols, phi, t, c, sv = entry_values(s, p)
    n = s["diag"].shape[0]
    d = s["diag"]
    dis = 1.0 / np.sqrt(d)
    V = probes(n, k, seed)
    L = 0.0
    ds = np.zeros_like(sv)
    for j in range(k):
        v = V[j]
        u = spmv(s, v)
        q = apply_m(s, sv, u)
        e = q - v
        L += float(e @ e) / (k * n)
        gq = 2.0 * e / (k * n)
        ds += gq[rows] * dis[rows] * dis[cols] * u[cols]
    dphi = ds * c * np.where(np.abs(np.tanh(phi)) < TMAX, 1.0 - t * t, 0.0)
    # symmetric use of p: d phi_e / d p_i = p_j / 4 and d / d p_j = p_i / 4
    dp = np.zeros_like(p)
    np.add.at(dp, rows, dphi[:, None] * p[cols] / 4.0)
    np.add.at(dp, cols, dphi[:, None] * p[rows] / 4.0)
    grads = {name: np.zeros(shape) for name, shape in PARAM_SHAPES}
    trunk_backward(params, cache, graph, dp, grads)
    return L, grads, sv


def trunk_backward(params, cache, graph, dp, grads):
    """Accumulates the trunk's parameter gradients from dL/dp."""
    x = cache["x"]
    h = cache[f"h{LAYERS}"]
    grads["P"] = h.T @ dp
    dh = dp @ params["P"].T
    for l in reversed(range(LAYERS)):
        dzb = dh * (cache[f"zb{l}"] > 0)
        hin = cache[f"h{l}"]
        grads[f"Wb{l}"] = hin.T @ dzb
        grads[f"Wc{l}"] = cache[f"g{l}"].T @ dzb
        grads[f"bb{l}"] = dzb.sum(0)
        dh_prev = dzb @ params[f"Wb{l}"].T
        dg = dzb @ params[f"Wc{l}"].T
        de = graph.nets_to_cells_T(dg)
        dza = de * (cache[f"za{l}"] > 0)
        grads[f"Wa{l}"] = cache[f"m{l}"].T @ dza
        grads[f"ba{l}"] = dza.sum(0)
        dm = dza @ params[f"Wa{l}"].T
        dh = dh_prev + graph.cells_to_nets_T(dm)
    dzin = dh * (cache["z_in"] > 0)
    grads["W_in"] = x.T @ dzin
    grads["b_in"] = dzin.sum(0)


def topo_features(nl) -> np.ndarray:
    """Per-cell features of the netlist alone (no positions): 1, pins/8,
    mean over the cell's nets of (movable pins - 1)/8, of fixed pins/4, share
    of its nets with a fixed pin, mean 1/(degree - 1), log(area)/8,
    log1p(pins)/2."""
    n = nl.num_movable
    N = nl.num_nets
    deg = np.diff(nl.net_start).astype(np.float64)
    pv = nl.var_of_vertex[nl.pin_cell]
    net_of_pin = np.repeat(np.arange(N), np.diff(nl.net_start))
    mov = np.bincount(net_of_pin[pv >= 0], minlength=N).astype(np.float64)
    cell = np.repeat(np.arange(n), np.diff(nl.pin_start))
    k = np.diff(nl.pin_start).astype(np.float64)
    nets = nl.pin_net.astype(np.int64)
    inv = np.where(k > 0, 1.0 / np.maximum(k, 1.0), 0.0)
    smov = np.bincount(cell, weights=mov[nets] - 1.0, minlength=n)
    sfix = np.bincount(cell, weights=deg[nets] - mov[nets], minlength=n)
    anyfix = np.bincount(cell, weights=(deg[nets] > mov[nets]).astype(np.float64), minlength=n)
    sinv = np.bincount(cell, weights=np.where(deg[nets] >= 2, 1.0 / np.maximum(deg[nets] - 1, 1),
                                              0.0), minlength=n)
    area = nl.width * nl.height
    x = np.zeros((n, NFEAT))
    x[:, 0] = 1.0
    x[:, 1] = k / 8.0
    x[:, 2] = smov * inv / 8.0
    x[:, 3] = sfix * inv / 4.0
    x[:, 4] = anyfix * inv
    x[:, 5] = sinv * inv
    x[:, 6] = np.where(area > 0, np.log(np.maximum(area, 1e-300)) / 8.0, 0.0)
    x[:, 7] = np.log1p(k) / 2.0
    return x


def softplus(o):
    return np.where(o > 20.0, o, np.log1p(np.exp(np.minimum(o, 20.0))))


def coarse_head(params, p, s):
    """z and the head's intermediates for one axis system."""
    rows = rows_of(s)
    n = s["diag"].shape[0]
    d = s["diag"]
    c = np.bincount(rows, weights=np.abs(s["val"]), minlength=n) / d
    logd = np.log(d)
    u = np.concatenate([p, c[:, None], (logd - logd.mean())[:, None]], axis=1)
    zh = u @ params["Wh"] + params["bh"]
    hh = relu(zh)
    o = hh @ params["wz"] + params["bz"][0]
    return softplus(o), dict(u=u, zh=zh, hh=hh, o=o)


def coarse_loss_and_grad(params, s, nl, E, graph: Graph | None = None):
    """Projection loss of the test vectors E [T, n] on the predicted coarse
    vector of system s, and its analytic parameter gradients."""
    graph = graph or Graph(nl)
    x = topo_features(nl)
    p, cache = forward(params, x, graph)
    z, hc = coarse_head(params, p, s)
    E = np.atleast_2d(E)
    T = E.shape[0]
    az = spmv(s, z)
    q = float(z @ az)
    A_e = np.stack([spmv(s, e) for e in E])
    pt = A_e @ z
    St = np.einsum("ij,ij->i", E, A_e)
    L = float(np.mean(1.0 - pt * pt / (q * St)))
    dz = np.zeros_like(z)
    for t in range(T):
        dz += -2.0 * pt[t] * A_e[t] / (T * q * St[t]) + 2.0 * pt[t] ** 2 * az / (T * q * q * St[t])
    sig = np.where(hc["o"] > 20.0, 1.0, 1.0 / (1.0 + np.exp(-np.minimum(hc["o"], 20.0))))
    do = dz * sig
    grads = {name: np.zeros(shape) for name, shape in PARAM_SHAPES}
    grads["wz"] = hc["hh"].T @ do
    grads["bz"] = np.array([do.sum()])
    dzh = np.outer(do, params["wz"]) * (hc["zh"] > 0)
    grads["Wh"] = hc["u"].T @ dzh
    grads["bh"] = dzh.sum(0)
    dp = (dzh @ params["Wh"].T)[:, :PROJ]
    trunk_backward(params, cache, graph, dp, grads)
    return L, grads, z


def init_params(seed: int = 0) -> dict:
    rng = np.random.default_rng(seed)
    out = {}
    for name, shape in PARAM_SHAPES:
        if name.startswith("b") or len(shape) == 1:
            out[name] = np.zeros(shape)
        else:
            fan = shape[0] + shape[1]
            scale = np.sqrt(2.0 / fan) * (0.05 if name == "P" else 1.0)
            out[name] = rng.standard_normal(shape) * scale
    out["wz"] = rng.standard_normal(HEAD_H) * np.sqrt(2.0 / (HEAD_H + 1)) * 0.1
    out["bz"] = np.array([0.5413248546129181])
    return out
