"""PCG in the reference's summation order (ktg_set_option "pcg_form" 2).

With form 2 every dot product is summed as getDeterministicSum does
(simpl_parallel.h:35-51: chunks of 4,096 elements left to right, then the
chunk sums in order) and every other operation already rounds as the
reference's, so the bar is bit-identity with the reference's solveBothAxes:
solutions, iteration counts, per-iterate residual histories and final
residuals. Checked against the golden fixtures (made by the compiled
reference) and, at 211k cells, against the reference run live."""
import json
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import oracle  # noqa: E402
from cases import CASES, TOL, MAX_ITER, build_case  # noqa: E402
from ktplace_b200 import netlist, synth  # noqa: E402

pytestmark = pytest.mark.gpu
GOLD = json.load(open(os.path.join(HERE, "golden", "golden.json")))


@pytest.fixture
def exact_form(gpu_ctx):
    gpu_ctx.set_option("pcg_form", 2)
    yield gpu_ctx
    gpu_ctx.set_option("pcg_form", -1)


@pytest.mark.parametrize("name", list(CASES))
def test_exact_pcg_bit_identical_to_golden(name, exact_form):
    ctx = exact_form
    g = np.load(os.path.join(HERE, "golden", f"{name}.npz"))
    meta = GOLD[name]
    raw, nl, x, y, ax, ay, alpha, _ = build_case(name)
    ctx.upload_netlist(nl)
    fx, fy = nl.floors()
    ctx.build_b2b(x, y, alpha, ax if alpha > 0 else None, ay if alpha > 0 else None, fx, fy)
    r = ctx.solve(x, y, TOL, MAX_ITER, hist_cap=MAX_ITER)
    assert r["iters"] == meta["iters"]
    assert np.array_equal(r["x"], g["x"]) and np.array_equal(r["y"], g["y"])
    k = r["iters"]
    assert np.array_equal(r["hist_x"][:k], g["hist_x"][:k])
    assert np.array_equal(r["hist_y"][:k], g["hist_y"][:k])
    assert r["resid"][0] == g["resid"][0] and r["resid"][1] == g["resid"][1]


@pytest.mark.parametrize("max_iter", [3, 60])
def test_exact_pcg_matches_live_reference_211k(max_iter, exact_form):
    """The 211k-cell workload from its seed positions with anchors: capped at
    3 iterations, at SimPL's 60, bit-identical to the reference's solve."""
    if not oracle.ref_available():
        pytest.skip("reference library not built")
    ctx = exact_form
    raw = synth.generate(synth.spec_adaptec1_like(1))
    nl = netlist.flatten(raw)
    x, y = synth.seed_positions(raw, nl.num_movable, 101)
    ax, ay = synth.seed_positions(raw, nl.num_movable, 201)
    ref = oracle.RefDesign.from_netlist(nl)
    ref.build_b2b(x, y, 0.2, ax, ay)
    rr = ref.solve(x, y, 1e-6, max_iter, hist_cap=max_iter)
    ctx.upload_netlist(nl)
    fx, fy = nl.floors()
    ctx.build_b2b(x, y, 0.2, ax, ay, fx, fy)
    r = ctx.solve(x, y, 1e-6, max_iter, hist_cap=max_iter)
    assert r["iters"] == rr["iters"]
    assert np.array_equal(r["x"], rr["x"]) and np.array_equal(r["y"], rr["y"])
    k = r["iters"]
    assert np.array_equal(r["hist_x"][:k], rr["hist_x"][:k])
    assert np.array_equal(r["hist_y"][:k], rr["hist_y"][:k])


def test_default_form_matches_live_reference_211k(gpu_ctx):
    """The library's default solve (pcg_form 3, the fastest) on the 211k-cell
    bench workload, run to full convergence (rtol 1e-6, no iteration cap),
    against the reference's solveBothAxes run live on the same system: same
    iteration count within one, solutions within 1e-9 relative, final
    residuals within the tolerance; the step's HPWL and overflow match the
    reference's."""
    if not oracle.ref_available():
        pytest.skip("reference library not built")
    from ktplace_b200 import grid as kgrid
    raw = synth.generate(synth.spec_adaptec1_like(1))
    nl = netlist.flatten(raw)
    x, y = synth.seed_positions(raw, nl.num_movable, 101)
    ax, ay = synth.seed_positions(raw, nl.num_movable, 201)
    ref = oracle.RefDesign.from_netlist(nl)
    ref.build_b2b(x, y, 0.2, ax, ay)
    rr = ref.solve(x, y, 1e-6, 100000)
    gpu_ctx.upload_netlist(nl)
    fx, fy = nl.floors()
    gpu_ctx.build_b2b(x, y, 0.2, ax, ay, fx, fy)
    r = gpu_ctx.solve(x, y, 1e-6, 100000)
    assert abs(r["iters"] - rr["iters"]) <= 1, (r["iters"], rr["iters"])
    for k in ("x", "y"):
        err = np.linalg.norm(r[k] - rr[k]) / np.linalg.norm(rr[k])
        assert err <= 1e-9, (k, err)
    assert max(r["resid"]) <= 1e-6
    h_ref = ref.hpwl(rr["x"], rr["y"])
    assert abs(gpu_ctx.hpwl(r["x"], r["y"]) - h_ref) <= 1e-6 * h_ref
    ref.grid(512, 1.0)
    _, ov_ref = ref.occupancy_map(rr["x"], rr["y"], 512 * 512)
    gpu_ctx.set_grid(kgrid.build_grid(nl, 512, 1.0))
    _, ov = gpu_ctx.occupancy(r["x"], r["y"], want_map=False)
    assert abs(ov - ov_ref) <= 1e-4
