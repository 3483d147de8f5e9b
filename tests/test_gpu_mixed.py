"""Mixed precision (FP32 inner Jacobi-PCG inside FP64 iterative refinement)
against the FP64 oracle.

Bar: the true FP64 relative residual ||b - A x|| / ||b|| (recomputed here on
the host from the oracle's CSR) meets the tolerance, the solution is within
1e-4 relative of the FP64 oracle solution, and its HPWL within 0.1%.
"""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import oracle  # noqa: E402
from cases import build_case, TOL, MAX_ITER  # noqa: E402

pytestmark = pytest.mark.gpu

SOL_RTOL = 1e-4
HPWL_RTOL = 1e-3


def true_resid(s, x):
    n = s["diag"].shape[0]
    rows = np.repeat(np.arange(n), np.diff(s["row_ptr"]))
    ax = s["diag"] * x
    np.add.at(ax, rows, s["val"] * x[s["col"]])
    b = s["rhs"]
    nb = np.linalg.norm(b)
    return np.linalg.norm(b - ax) / nb if nb > 0 else 0.0


@pytest.mark.parametrize("name", ["tiny_macros", "edge_alpha", "small12k"])
@pytest.mark.parametrize("inner_tol", [1e-2, 1e-3])
def test_mixed_matches_fp64(name, inner_tol, gpu_ctx, port_built):
    raw, nl, x, y, ax, ay, alpha, _ = build_case(name)
    gpu_ctx.upload_netlist(nl)
    fx, fy = nl.floors()
    gpu_ctx.build_b2b(x, y, alpha, ax, ay, fx, fy)
    sx, sy = gpu_ctx.system(0), gpu_ctx.system(1)
    ref = oracle.port_solve_both(sx, x, sy, y, TOL, MAX_ITER)
    r = gpu_ctx.solve_mixed(x, y, TOL, inner_tol=inner_tol, hist_cap=64)
    assert true_resid(sx, r["x"]) <= TOL * 1.0001
    assert true_resid(sy, r["y"]) <= TOL * 1.0001
    for k in ("x", "y"):
        err = np.linalg.norm(r[k] - ref[k]) / np.linalg.norm(ref[k])
        assert err <= SOL_RTOL, (k, err)
    port = oracle.PortNetlist(nl)
    h_ref = port.hpwl(ref["x"], ref["y"])
    h_mix = port.hpwl(r["x"], r["y"])
    assert abs(h_mix - h_ref) <= HPWL_RTOL * h_ref
    # the reported residual is the true one
    assert abs(r["resid"][0] - true_resid(sx, r["x"])) <= 1e-3 * max(r["resid"][0], 1e-12)


def test_mixed_stall_falls_back_to_fp64(gpu_ctx):
    """An inner tolerance of 0.999 stops each correction solve after about one
    iteration, which cannot halve the residual per round: the solve must
    still reach the tolerance through the FP64 fallback."""
    raw, nl, x, y, ax, ay, alpha, _ = build_case("tiny_macros")
    gpu_ctx.upload_netlist(nl)
    fx, fy = nl.floors()
    gpu_ctx.build_b2b(x, y, alpha, ax, ay, fx, fy)
    sx = gpu_ctx.system(0)
    r = gpu_ctx.solve_mixed(x, y, TOL, inner_tol=0.999, max_outer=3)
    assert r["fp64_iters"][0] > 0 or r["fp64_iters"][1] > 0
    assert true_resid(sx, r["x"]) <= 10 * TOL
