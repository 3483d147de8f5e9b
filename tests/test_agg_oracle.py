"""The aggregation preconditioner's reference (oracle/agg_ref.py) on its own:
valid aggregates and layout, exact block inverses, and fewer PCG iterations
than Jacobi on the same systems. CPU only."""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import oracle  # noqa: E402
from oracle import agg_ref  # noqa: E402
from cases import build_case  # noqa: E402


def port_systems(name):
    raw, nl, x, y, ax, ay, alpha, _ = build_case(name)
    fx, fy = nl.floors()
    port = oracle.PortNetlist(nl)
    sx = port.b2b_axis(True, x, fx, alpha, ax)
    sy = port.b2b_axis(False, y, fy, alpha, ay)
    return nl, x, y, sx, sy


def dense_block(s, rows):
    """A restricted to `rows` (per-axis indices), duplicates summed."""
    k = len(rows)
    where = {int(r): q for q, r in enumerate(rows)}
    B = np.zeros((k, k))
    for m, i in enumerate(rows):
        B[m, m] += s["diag"][i]
        for e in range(int(s["row_ptr"][i]), int(s["row_ptr"][i + 1])):
            q = where.get(int(s["col"][e]))
            if q is not None:
                B[m, q] += s["val"][e]
    return B


@pytest.mark.parametrize("name", ["tiny_macros", "edge_alpha"])
def test_aggregates_layout_and_inverses(name, port_built):
    nl, x, y, sx, sy = port_systems(name)
    n = sx["diag"].shape[0]
    ag = agg_ref.aggregate(sx, sy)
    order, newpos, size, start = ag["order"], ag["newpos"], ag["size"], ag["start"]
    assert sorted(order.tolist()) == list(range(2 * n))
    assert np.array_equal(order[newpos], np.arange(2 * n))
    assert size.min() >= 1 and size.max() <= agg_ref.AGG_MAX
    assert start[-1] == 2 * n
    # every x row before every y row; no aggregate crosses the axes
    assert np.all(order[:n] < n) and np.all(order[n:] >= n)
    minv, meta = agg_ref.block_inverses(sx, sy, ag)
    for J in range(size.shape[0]):
        first, k = int(start[J]), int(size[J])
        axis = 1 if first >= n else 0
        s = sy if axis else sx
        rows = order[first:first + k] - axis * n
        B = dense_block(s, rows)
        Minv = minv[first:first + k, :k]
        assert np.allclose(Minv @ B, np.eye(k), atol=1e-9), J
        assert np.all(minv[first:first + k, k:] == 0.0)
        assert np.all(meta[first:first + k] == (first - axis * n) * agg_ref.AGG_MAX + k - 1)


def test_aggregation_cuts_iterations(port_built):
    """Jacobi-PCG vs aggregation-PCG from the same start on small12k."""
    import scipy.sparse as sp
    nl, x, y, sx, sy = port_systems("small12k")
    n = sx["diag"].shape[0]
    ag = agg_ref.aggregate(sx, sy)
    minv, meta = agg_ref.block_inverses(sx, sy, ag)
    order = ag["order"]
    for axis, s, x0 in ((0, sx, x), (1, sy, y)):
        rows = np.repeat(np.arange(n), np.diff(s["row_ptr"]))
        A = (sp.csr_matrix((s["val"], (rows, s["col"])), shape=(n, n)) + sp.diags(s["diag"])).tocsr()
        b = s["rhs"]
        o = order[axis * n:(axis + 1) * n] - axis * n

        def agg_m(r):
            rp = np.zeros(2 * n)
            rp[axis * n:(axis + 1) * n] = r[o]
            u = agg_ref.apply(minv, meta, rp)[axis * n:(axis + 1) * n]
            out = np.empty(n)
            out[o] = u
            return out

        def pcg(m):
            xx = x0.copy()
            r = b - A @ xx
            z = m(r)
            p = z.copy()
            rz = r @ z
            nb = np.linalg.norm(b)
            for k in range(2000):
                if np.linalg.norm(r) / nb <= 1e-6:
                    return k
                Ap = A @ p
                a = rz / (p @ Ap)
                xx += a * p
                r -= a * Ap
                z = m(r)
                rz2 = r @ z
                p = z + rz2 / rz * p
                rz = rz2
            return 2000

        it_j = pcg(lambda r: r / s["diag"])
        it_a = pcg(agg_m)
        assert it_a * 2 < it_j, (axis, it_j, it_a)
