"""The C++ drop-ins (ktplace_b200/dropin/simpl_lss_b200.cc and
simpl_lal_b200.cc) inside the reference's own, unmodified SimPL code.

oracle/_ref/libktref_gpu.so is the reference's SimPL compiled from its sources
with the drop-ins linked in place of simpl_lss.o and simpl_lal.o;
oracle/_ref/libktref.so is the same code with the reference's objects. The
reference interface (LinearSystems::buildB2B, solveBothAxes,
LookAheadLegalizer::legalize) must give the same systems, solutions and
positions, and a whole SimPL run must land on the same placement.
"""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import oracle  # noqa: E402
from cases import build_case, TOL, MAX_ITER  # noqa: E402

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not (oracle.ref_available("gpu") and oracle.ref_available()),
                                 reason="oracle/_ref drop-in build not present")]


@pytest.mark.parametrize("name", ["tiny_macros", "edge_alpha", "small12k"])
def test_dropin_interface_matches_reference(name):
    raw, nl, x, y, ax, ay, alpha, _ = build_case(name)
    cpu = oracle.RefDesign.from_netlist(nl, "cpu")
    gpu = oracle.RefDesign.from_netlist(nl, "gpu")
    a = ax if alpha > 0 else None
    b = ay if alpha > 0 else None
    cpu.build_b2b(x, y, alpha, a, b)
    gpu.build_b2b(x, y, alpha, a, b)
    for axis in (0, 1):
        s, t = cpu.system(axis), gpu.system(axis)
        for k in ("row_ptr", "col", "val", "diag", "rhs"):
            assert np.array_equal(s[k], t[k]), (axis, k)
    r = cpu.solve(x, y, TOL, MAX_ITER, hist_cap=MAX_ITER)
    g = gpu.solve(x, y, TOL, MAX_ITER, hist_cap=MAX_ITER)
    assert g["iters"] == r["iters"]
    for k in ("x", "y"):
        assert np.linalg.norm(g[k] - r[k]) <= 1e-9 * np.linalg.norm(r[k])
    for k in ("hist_x", "hist_y"):
        assert np.linalg.norm(g[k] - r[k]) <= 1e-6 * np.linalg.norm(r[k])


def test_star_systems_solve_on_gpu():
    raw, nl, x, y, *_ = build_case("tiny_macros")
    cpu = oracle.RefDesign.from_netlist(nl, "cpu")
    gpu = oracle.RefDesign.from_netlist(nl, "gpu")
    assert cpu.build_star() == gpu.build_star()
    for axis in (0, 1):
        s, t = cpu.system(axis), gpu.system(axis)
        for k in ("row_ptr", "col", "val", "diag", "rhs"):
            assert np.array_equal(s[k], t[k]), (axis, k)
    size = cpu.system(0)["diag"].shape[0]
    ext = np.concatenate([x, np.full(size - x.shape[0], x.mean())])
    eyt = np.concatenate([y, np.full(size - y.shape[0], y.mean())])
    r = cpu.solve(ext, eyt, 1e-6, 1000)
    g = gpu.solve(ext, eyt, 1e-6, 1000)
    assert g["iters"] == r["iters"]
    assert np.linalg.norm(g["x"] - r["x"]) <= 1e-9 * np.linalg.norm(r["x"])


def test_full_simpl_run_matches_reference():
    """Whole SimPL flow (star init, B2B rounds, LAL, refinement) with both
    drop-ins: the solve sums in the reference's order (the drop-in's default)
    and the legalizer is exact, so the final placement is the CPU run's, bit
    for bit."""
    import resource
    try:  # the reference legalizer's recursion wants a large stack
        resource.setrlimit(resource.RLIMIT_STACK, (resource.RLIM_INFINITY, resource.RLIM_INFINITY))
    except (ValueError, OSError):
        pass
    raw, nl, *_ = build_case("small12k")
    cpu = oracle.RefDesign.from_netlist(nl, "cpu")
    gpu = oracle.RefDesign.from_netlist(nl, "gpu")
    cx, cy = cpu.run_simpl()
    gx, gy = gpu.run_simpl()
    assert np.array_equal(cx, gx) and np.array_equal(cy, gy)
    hc, hg = cpu.hpwl(cx, cy), cpu.hpwl(gx, gy)
    assert abs(hg - hc) <= 5e-3 * hc, (hg, hc)
    nb = 64 * 64
    cpu.grid(64, 1.0)
    _, oc = cpu.occupancy_map(cx, cy, nb)
    _, og = cpu.occupancy_map(gx, gy, nb)
    assert abs(og - oc) <= 0.05


def test_gpu_star_build_bit_exact(gpu_ctx):
    """ktg_build_star against the reference's buildStar: same size, same CSR,
    values, diagonal and right-hand sides, bit for bit."""
    for name in ("tiny_macros", "edge_alpha", "small12k"):
        raw, nl, *_ = build_case(name)
        cpu = oracle.RefDesign.from_netlist(nl, "cpu")
        size = cpu.build_star()
        gpu_ctx.upload_netlist(nl)
        assert gpu_ctx.build_star() == size
        for axis in (0, 1):
            s, t = cpu.system(axis), gpu_ctx.system(axis)
            for k in ("row_ptr", "col", "val", "diag", "rhs"):
                assert np.array_equal(s[k].astype(np.float64), t[k].astype(np.float64)), (name, axis, k)


@pytest.mark.parametrize("name,start", [("tiny_macros", "solved"), ("small12k", "solved"),
                                        ("small12k", "packed")])
def test_dropin_legalizer_matches_reference(name, start):
    """simpl_lal_b200.cc in place of simpl_lal.o: the reference's own
    simplPlacer::Impl::lookAheadLegalize, called on the same grid and
    positions, gives bit-identical positions through the GPU legalizer."""
    import resource
    try:  # the reference legalizer's recursion wants a large stack
        resource.setrlimit(resource.RLIMIT_STACK, (resource.RLIM_INFINITY, resource.RLIM_INFINITY))
    except (ValueError, OSError):
        pass
    raw, nl, x, y, ax, ay, alpha, bins = build_case(name)
    cpu = oracle.RefDesign.from_netlist(nl, "cpu")
    gpu = oracle.RefDesign.from_netlist(nl, "gpu")
    if start == "solved":
        cpu.build_b2b(x, y, alpha, ax if alpha > 0 else None, ay if alpha > 0 else None)
        r = cpu.solve(x, y, TOL, MAX_ITER)
        px, py = r["x"], r["y"]
    else:
        rng = np.random.default_rng(3)
        lx, ly, ux, uy = nl.die
        px = 0.5 * (lx + ux) + 0.03 * (ux - lx) * rng.standard_normal(nl.num_movable)
        py = 0.5 * (ly + uy) + 0.03 * (uy - ly) * rng.standard_normal(nl.num_movable)
    cpu.grid(bins, 1.0)
    gpu.grid(bins, 1.0)
    cx, cy = cpu.lal(px, py)
    gx, gy = gpu.lal(px, py)
    assert np.array_equal(cx, gx) and np.array_equal(cy, gy)
    assert np.mean(cx != px) > 0.1


def test_full_simpl_run_211k_identical():
    """The same at 211k cells (the bench netlist, 550 macros): the reference's
    SimPL with both drop-ins ends on the CPU run's placement, bit for bit."""
    import resource
    try:
        resource.setrlimit(resource.RLIMIT_STACK, (resource.RLIM_INFINITY, resource.RLIM_INFINITY))
    except (ValueError, OSError):
        pass
    from ktplace_b200 import netlist, synth
    nl = netlist.flatten(synth.generate(synth.spec_adaptec1_like(seed=1)))
    threads = os.cpu_count() or 1
    oracle.set_ref_threads(threads, "cpu")
    oracle.set_ref_threads(threads, "gpu")
    cx, cy = oracle.RefDesign.from_netlist(nl, "cpu").run_simpl()
    gx, gy = oracle.RefDesign.from_netlist(nl, "gpu").run_simpl()
    assert np.array_equal(cx, gx) and np.array_equal(cy, gy)


@pytest.mark.parametrize("name", ["tiny_macros", "small12k"])
def test_dropin_hooks_hpwl_occupancy_bit_exact(name):
    """The reference's simplPlacer::Impl::getHpwl and getOccupancy
    (simpl_placer.cc:256-289) with their bodies routed to the GPU hooks
    (simpl_hooks_b200.h; the drop-in library's simpl_placer.cc is the
    reference's with those two bodies replaced by oracle/hooks/
    apply_hooks.py): the same HPWL, summed in the reference's order, and the
    same occupancy map and overflow, bit for bit, on grids of 16 to 512 bins
    per axis."""
    raw, nl, x, y, ax, ay, alpha, bins = build_case(name)
    cpu = oracle.RefDesign.from_netlist(nl, "cpu")
    gpu = oracle.RefDesign.from_netlist(nl, "gpu")
    rng = np.random.default_rng(11)
    lx, ly, ux, uy = nl.die
    for k in range(2):
        px = x if k == 0 else lx + rng.random(nl.num_movable) * (ux - lx - nl.width)
        py = y if k == 0 else ly + rng.random(nl.num_movable) * (uy - ly - nl.height)
        assert gpu.hpwl(px, py) == cpu.hpwl(px, py)
        for per_axis in (16, 512):
            cpu.grid(per_axis, 1.0)
            gpu.grid(per_axis, 1.0)
            oc, vc = cpu.occupancy_map(px, py, per_axis * per_axis)
            og, vg = gpu.occupancy_map(px, py, per_axis * per_axis)
            assert np.array_equal(oc, og) and vc == vg, (name, k, per_axis)
