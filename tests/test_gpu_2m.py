"""The largest configuration: 2.2M movable cells, 2.25M nets, 8,000 macros
(the seeded generator's 2.2M design), against the reference's own code.

Bars as for the smaller designs: B2B systems bit-identical; the solve in the
reference's summation order (pcg_form 2) bit-identical, the default form
within 1e-9; HPWL within 1e-12 and the occupancy map bit-identical; the
look-ahead legalization of the solved positions bit-identical. The solves are
capped at 20 iterations to keep the reference's side short."""
import os
import resource

import numpy as np
import pytest

import oracle
from ktplace_b200 import grid, netlist, synth

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not oracle.ref_available(), reason="reference library not built")]

ITERS = 20


@pytest.fixture(scope="module")
def design():
    try:  # the reference legalizer's recursion wants a large stack
        resource.setrlimit(resource.RLIMIT_STACK, (resource.RLIM_INFINITY, resource.RLIM_INFINITY))
    except (ValueError, OSError):
        pass
    oracle.set_ref_threads(os.cpu_count() or 1)
    raw = synth.generate(synth.spec_2m(4))
    nl = netlist.flatten(raw)
    x, y = synth.seed_positions(raw, nl.num_movable, 104)
    ax, ay = synth.seed_positions(raw, nl.num_movable, 204)
    ref = oracle.RefDesign.from_netlist(nl)
    return nl, x, y, ax, ay, ref


@pytest.fixture(scope="module")
def built(design, gpu_ctx):
    nl, x, y, ax, ay, ref = design
    gpu_ctx.set_option("pcg_form", -1)
    gpu_ctx.upload_netlist(nl)
    fx, fy = nl.floors()
    gpu_ctx.build_b2b(x, y, 0.2, ax, ay, fx, fy)
    ref.build_b2b(x, y, 0.2, ax, ay)
    return gpu_ctx


def test_b2b_2m_bit_identical(design, built):
    nl, x, y, ax, ay, ref = design
    for axis in (0, 1):
        g, r = built.system(axis), ref.system(axis)
        assert np.array_equal(g["row_ptr"].astype(np.int64), r["row_ptr"].astype(np.int64)), axis
        m = int(r["row_ptr"][-1])
        assert np.array_equal(g["col"][:m].astype(np.int64), r["col"].astype(np.int64)), axis
        for k in ("val",):
            assert np.array_equal(g[k][:m], r[k]), (axis, k)
        for k in ("diag", "rhs"):
            assert np.array_equal(g[k], r[k]), (axis, k)


def test_pcg_2m(design, built):
    nl, x, y, ax, ay, ref = design
    rr = ref.solve(x, y, 1e-6, ITERS, hist_cap=ITERS)
    try:
        built.set_option("pcg_form", 2)
        e = built.solve(x, y, 1e-6, ITERS, hist_cap=ITERS)
    finally:
        built.set_option("pcg_form", -1)
    assert e["iters"] == rr["iters"]
    assert np.array_equal(e["x"], rr["x"]) and np.array_equal(e["y"], rr["y"])
    assert np.array_equal(e["hist_x"][:ITERS], rr["hist_x"][:ITERS])
    d = built.solve(x, y, 1e-6, ITERS)
    for k in ("x", "y"):
        err = np.linalg.norm(d[k] - rr[k]) / np.linalg.norm(rr[k])
        assert err <= 1e-9, (k, err)


def test_hpwl_density_and_legalization_2m(design, built):
    nl, x, y, ax, ay, ref = design
    rr = ref.solve(x, y, 1e-6, ITERS)
    px, py = rr["x"], rr["y"]
    h = built.hpwl(px, py)
    hr = ref.hpwl(px, py)
    assert abs(h - hr) <= 1e-12 * abs(hr)
    bins = grid.default_bins_per_axis(nl.num_movable)
    g = grid.build_grid(nl, bins, 1.0)
    built.set_grid(g)
    occ, _ = built.occupancy(px, py)
    ref.grid(bins, 1.0)
    rocc, _ = ref.occupancy_map(px, py, bins * bins)
    assert np.array_equal(occ, rocc)
    built.set_free_space(grid.build_free_space(nl))
    gx, gy = built.lal(px, py)
    lx, ly = ref.lal(px, py)
    assert np.array_equal(gx, lx) and np.array_equal(gy, ly)
    assert np.mean(gx != px) > 0.1


@pytest.mark.parametrize("precond", [0, 2, 1])
def test_mixed_solves_2m(precond, design, built):
    """Mixed precision at 2.2M cells (FP32 PCG inside FP64 refinement) with
    the Jacobi, aggregation and learned preconditioners: true residual at the
    tolerance and HPWL within 0.1% of the FP64 solve's."""
    nl, x, y, ax, ay, ref = design
    ctx = built
    d = ctx.solve(x, y, 1e-6, 100000)
    h64 = ctx.hpwl(d["x"], d["y"])
    learned = None
    try:
        if precond == 1:
            from ktplace_b200.learned import Learned
            w = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                             "ktplace_b200", "weights", "learned_precond.npy")
            if not os.path.exists(w):
                pytest.skip("no trained weights")
            learned = Learned(0)
            learned.load(w)
            learned.prepare(ctx)
        ctx.set_option("precond", precond)
        m = ctx.solve_mixed(x, y, 1e-6, 1e-3)
    finally:
        ctx.set_option("precond", 0)
        if learned is not None:
            learned.close()
    assert max(m["resid"]) <= 1e-6
    h = ctx.hpwl(m["x"], m["y"])
    assert abs(h - h64) <= 1e-3 * h64
