"""Kraftwerk2's system build and CG on the GPU against the reference's own
code (Kraftwerk2Placer::Impl::buildSystem and solve, compiled into
oracle/_ref by oracle/ref_kraftwerk2.cc).

Bars: the CSR (row pointers, columns, values), diag and rhs of both axes are
bit-identical, with and without the right-hand side and after the
move-weight adjustment; the GPU solve lands within 1e-9 relative of the
reference's solve. Nets keep Kraftwerk2's raw pin lists (edge_alpha lists a
cell twice on one net)."""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import oracle  # noqa: E402
from cases import build_case  # noqa: E402
from ktplace_b200 import netlist  # noqa: E402

pytestmark = pytest.mark.gpu

CASES = ["tiny_macros", "edge_alpha", "small12k"]


def kw2_netlist(name):
    raw, _, x, y, ax, ay, alpha, _ = build_case(name)
    return netlist.flatten(raw, kraftwerk2=True), x, y


def same(a, b):
    return np.array_equal(np.asarray(a), np.asarray(b))


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("with_rhs", [True, False])
def test_build_bit_exact(name, with_rhs, gpu_ctx):
    if not oracle.ref_available():
        pytest.skip("reference library not built")
    nl, x, y = kw2_netlist(name)
    fx, fy = nl.floors()
    ref = oracle.Kraftwerk2Ref(nl)
    gpu_ctx.upload_netlist(nl)
    gpu_ctx.build_kraftwerk2(x, y, with_rhs, fx, fy)
    for axis in (0, 1):
        r = ref.build(x, y, axis == 0, with_rhs, fx, fy)
        g = gpu_ctx.system(axis)
        assert same(g["row_ptr"], r["row_ptr"]), axis
        m = int(r["row_ptr"][-1])
        assert same(g["col"][:m], r["col"]) and same(g["val"][:m], r["val"]), axis
        assert same(g["diag"], r["diag"]) and same(g["rhs"], r["rhs"]), axis


@pytest.mark.parametrize("name", CASES)
def test_adjust_and_solve(name, gpu_ctx):
    """The force step of Kraftwerk2Placer::Impl::place (kraftwerk2_placer.cc:
    710-731): build without rhs, diag += moveWeight, rhs = -moveWeight *
    toward, solve for the move from zero; and the initial placement step
    (build with rhs, diag floor 1e-12, solve from x)."""
    if not oracle.ref_available():
        pytest.skip("reference library not built")
    nl, x, y = kw2_netlist(name)
    n = nl.num_movable
    fx, fy = nl.floors()
    rng = np.random.default_rng(3)
    mw = rng.uniform(0.1, 2.0, n)
    tx, ty = rng.normal(0, 1.0, n), rng.normal(0, 1.0, n)
    ref = oracle.Kraftwerk2Ref(nl)
    gpu_ctx.upload_netlist(nl)
    tol, max_iter = 1e-5, 150
    # force step
    gpu_ctx.build_kraftwerk2(x, y, False, fx, fy)
    gpu_ctx.kraftwerk2_adjust(mw, tx, ty, 0.0)
    zero = np.zeros(n)
    g = gpu_ctx.solve(zero, zero, tol, max_iter)
    for axis, t in ((0, tx), (1, ty)):
        r = ref.build(x, y, axis == 0, False, fx, fy)
        diag, rhs = r["diag"] + mw, -mw * t
        gs = gpu_ctx.system(axis)
        assert same(gs["diag"], diag) and same(gs["rhs"], rhs), axis
        ref.set_diag_rhs(diag, rhs)
        d = ref.solve(zero, tol, max_iter)
        got = g["x"] if axis == 0 else g["y"]
        assert np.linalg.norm(got - d) <= 1e-9 * max(np.linalg.norm(d), 1e-30), axis
    # initial placement step
    gpu_ctx.build_kraftwerk2(x, y, True, fx, fy)
    gpu_ctx.kraftwerk2_adjust(None, None, None, 1e-12)
    g = gpu_ctx.solve(x, y, tol, max_iter)
    for axis, p0 in ((0, x), (1, y)):
        r = ref.build(x, y, axis == 0, True, fx, fy)
        diag = np.maximum(r["diag"], 1e-12)
        assert same(gpu_ctx.system(axis)["diag"], diag), axis
        ref.set_diag_rhs(diag, r["rhs"])
        s = ref.solve(p0, tol, max_iter)
        got = g["x"] if axis == 0 else g["y"]
        assert np.linalg.norm(got - s) <= 1e-9 * np.linalg.norm(s), axis
