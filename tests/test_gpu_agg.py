"""Aggregation preconditioner on the GPU (ktg_set_option(ctx, "precond", 2)).

Bars: the aggregates and the row order are bit-identical to the reference
restatement (oracle/agg_ref.py) on the same systems; the block inverses agree
with it to FP32 rounding (|diff| <= 2e-6 x the row's largest entry); the
mixed solve with it meets the FP64 tolerance on the true residual, lands
within 1e-4 relative of the FP64 oracle solution and 0.1% of its HPWL, and
needs at most half the inner iterations of the Jacobi mixed solve.
"""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import oracle  # noqa: E402
from oracle import agg_ref  # noqa: E402
from cases import build_case, TOL, MAX_ITER  # noqa: E402
from test_gpu_mixed import true_resid  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.fixture
def agg_ctx(gpu_ctx):
    gpu_ctx.set_option("precond", 2)
    yield gpu_ctx
    gpu_ctx.set_option("precond", 0)


@pytest.mark.parametrize("name", ["tiny_macros", "edge_alpha", "small12k"])
def test_aggregates_match_oracle(name, agg_ctx):
    raw, nl, x, y, ax, ay, alpha, _ = build_case(name)
    agg_ctx.upload_netlist(nl)
    fx, fy = nl.floors()
    agg_ctx.build_b2b(x, y, alpha, ax, ay, fx, fy)
    sx, sy = agg_ctx.system(0), agg_ctx.system(1)
    g = agg_ctx.aggregates()
    ag = agg_ref.aggregate(sx, sy)
    minv, meta = agg_ref.block_inverses(sx, sy, ag)
    assert np.array_equal(g["order"], ag["order"])
    assert np.array_equal(g["meta"], meta)
    scale = np.abs(minv).max(axis=1, keepdims=True)
    assert np.all(np.abs(g["minv"] - minv) <= 2e-6 * scale)


@pytest.mark.parametrize("name", ["tiny_macros", "edge_alpha", "small12k"])
@pytest.mark.parametrize("inner_tol", [1e-2, 1e-3])
def test_agg_mixed_matches_fp64(name, inner_tol, agg_ctx, port_built):
    raw, nl, x, y, ax, ay, alpha, _ = build_case(name)
    agg_ctx.upload_netlist(nl)
    fx, fy = nl.floors()
    agg_ctx.build_b2b(x, y, alpha, ax, ay, fx, fy)
    sx, sy = agg_ctx.system(0), agg_ctx.system(1)
    ref = oracle.port_solve_both(sx, x, sy, y, TOL, MAX_ITER)
    r = agg_ctx.solve_mixed(x, y, TOL, inner_tol=inner_tol)
    assert r["fp64_iters"] == (0, 0)
    assert true_resid(sx, r["x"]) <= TOL * 1.0001
    assert true_resid(sy, r["y"]) <= TOL * 1.0001
    for k in ("x", "y"):
        err = np.linalg.norm(r[k] - ref[k]) / np.linalg.norm(ref[k])
        assert err <= 1e-4, (k, err)
    port = oracle.PortNetlist(nl)
    h_ref = port.hpwl(ref["x"], ref["y"])
    assert abs(port.hpwl(r["x"], r["y"]) - h_ref) <= 1e-3 * h_ref
    agg_ctx.set_option("precond", 0)
    j = agg_ctx.solve_mixed(x, y, TOL, inner_tol=inner_tol)
    agg_ctx.set_option("precond", 2)
    if name == "small12k":
        for a in range(2):
            assert 2 * r["inner"][a] <= j["inner"][a], (r["inner"], j["inner"])


def test_agg_rebuilt_after_new_build(agg_ctx):
    """A new B2B build invalidates the aggregates: solves of two different
    systems in a row each meet the tolerance on their own system."""
    raw, nl, x, y, ax, ay, alpha, _ = build_case("small12k")
    agg_ctx.upload_netlist(nl)
    fx, fy = nl.floors()
    rng = np.random.default_rng(5)
    for k in range(2):
        xs = x + rng.normal(0, 3.0, x.shape) * k
        agg_ctx.build_b2b(xs, y, alpha, ax, ay, fx, fy)
        sx = agg_ctx.system(0)
        g = agg_ctx.aggregates()
        ag = agg_ref.aggregate(sx, agg_ctx.system(1))
        assert np.array_equal(g["order"], ag["order"])
        r = agg_ctx.solve_mixed(xs, y, TOL)
        assert true_resid(sx, r["x"]) <= TOL * 1.0001


def test_agg_large_uses_global_slices(agg_ctx):
    """520k cells: the per-block slices no longer fit in shared memory and the
    solve keeps them in global memory; checked against the FP64 GPU solve."""
    from ktplace_b200 import synth, netlist
    spec = synth.SynthSpec(num_movable=520_000, num_nets=545_000, num_pads=1_500, num_rows=1_400,
                           utilization=0.6, num_macros=800, seed=3, name="synth520k")
    raw = synth.generate(spec)
    nl = netlist.flatten(raw)
    x, y = synth.seed_positions(raw, nl.num_movable, 11)
    ax, ay = synth.seed_positions(raw, nl.num_movable, 12)
    fx, fy = nl.floors()
    agg_ctx.upload_netlist(nl)
    agg_ctx.build_b2b(x, y, 0.2, ax, ay, fx, fy)
    sx, sy = agg_ctx.system(0), agg_ctx.system(1)
    r = agg_ctx.solve_mixed(x, y, TOL)
    assert true_resid(sx, r["x"]) <= TOL * 1.0001
    assert true_resid(sy, r["y"]) <= TOL * 1.0001
    agg_ctx.set_option("precond", 0)
    j = agg_ctx.solve_mixed(x, y, TOL)
    f = agg_ctx.solve(x, y, TOL, MAX_ITER)
    agg_ctx.set_option("precond", 2)
    assert true_resid(sx, j["x"]) <= TOL * 1.0001
    for k in ("x", "y"):
        assert np.linalg.norm(r[k] - f[k]) / np.linalg.norm(f[k]) <= 1e-4
