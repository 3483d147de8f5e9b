"""GPU parity: the CUDA path through the C ABI against the oracle.

Bar (from the reference's determinism contract and the hot-path spec):
  * bound pins and B2B CSR (row_ptr, col, val, diag, rhs): bit-exact;
  * PCG: same iteration count, residual history within 1e-6 relative per
    iterate, solution within 1e-9 relative (only summation order differs);
  * HPWL: within 1e-12 relative (per-net terms are exact; the sum is a tree);
  * occupancy map: bit-exact (64-bit fixed point, integer areas);
    overflow within 1e-12 relative.
"""
import json
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

from cases import CASES, TOL, MAX_ITER, build_case, digest  # noqa: E402

pytestmark = pytest.mark.gpu
GOLD = json.load(open(os.path.join(HERE, "golden", "golden.json")))

SOL_RTOL = 1e-9
HIST_RTOL = 1e-6
HPWL_RTOL = 1e-12
OVF_RTOL = 1e-12


def gold(name):
    return np.load(os.path.join(HERE, "golden", f"{name}.npz")), GOLD[name]


def rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    den = max(np.linalg.norm(b), 1e-300)
    return float(np.linalg.norm(a - b) / den)


@pytest.mark.parametrize("name", list(CASES))
def test_b2b_bit_exact(name, gpu_ctx):
    g, meta = gold(name)
    raw, nl, x, y, ax, ay, alpha, _ = build_case(name)
    gpu_ctx.upload_netlist(nl)
    fx, fy = nl.floors()
    gpu_ctx.build_b2b(x, y, alpha, ax if alpha > 0 else None, ay if alpha > 0 else None, fx, fy)
    for axis in (0, 1):
        s = gpu_ctx.system(axis)
        lo, hi = gpu_ctx.bound_pins(axis)
        got = dict(row_ptr=s["row_ptr"].astype(np.int64), col=s["col"].astype(np.int32),
                   val=s["val"], diag=s["diag"], rhs=s["rhs"], lo=lo, hi=hi)
        for k, a in got.items():
            assert digest(a) == meta[f"sha_{k}_{axis}"], (name, axis, k)
    assert abs(gpu_ctx.build_hpwl() - meta["hpwl_in"]) <= HPWL_RTOL * abs(meta["hpwl_in"])


@pytest.mark.parametrize("name", list(CASES))
def test_pcg_matches_reference(name, gpu_ctx):
    g, meta = gold(name)
    raw, nl, x, y, ax, ay, alpha, _ = build_case(name)
    gpu_ctx.upload_netlist(nl)
    fx, fy = nl.floors()
    gpu_ctx.build_b2b(x, y, alpha, ax if alpha > 0 else None, ay if alpha > 0 else None, fx, fy)
    r = gpu_ctx.solve(x, y, TOL, MAX_ITER, hist_cap=MAX_ITER)
    assert r["iters"] == meta["iters"]
    assert rel(r["hist_x"], g["hist_x"]) <= HIST_RTOL
    assert rel(r["hist_y"], g["hist_y"]) <= HIST_RTOL
    assert rel(r["x"], g["x"]) <= SOL_RTOL, rel(r["x"], g["x"])
    assert rel(r["y"], g["y"]) <= SOL_RTOL, rel(r["y"], g["y"])
    # Final residuals: relative to the tolerance when a system converges
    # below it in one step (then both sides sit at round-off level).
    for a in (0, 1):
        assert abs(r["resid"][a] - g["resid"][a]) <= HIST_RTOL * max(g["resid"][a], TOL)


@pytest.mark.parametrize("name", ["tiny_macros", "edge_alpha", "small12k"])
@pytest.mark.parametrize("form", [0, 1, 2, 3])
def test_pcg_forms_and_spmv_shapes(name, form, gpu_ctx):
    """Every solve form against the reference, in every SpMV shape. Warp tiles
    (32) and one thread per row (1) add each row's terms in the same order;
    they differ only in which thread's partial of a dot product a row lands
    in, so their solves agree to rounding in forms 0, 1 and 3, and are
    bit-identical in form 2 (the reference's summation order), which equals
    the reference's solution bit for bit."""
    g, meta = gold(name)
    raw, nl, x, y, ax, ay, alpha, _ = build_case(name)
    gpu_ctx.upload_netlist(nl)
    fx, fy = nl.floors()
    gpu_ctx.build_b2b(x, y, alpha, ax if alpha > 0 else None, ay if alpha > 0 else None, fx, fy)
    got = {}
    try:
        gpu_ctx.set_option("pcg_form", form)
        for lanes in (32, 1, 4):
            gpu_ctx.set_option("pcg_lanes", lanes)
            r = gpu_ctx.solve(x, y, TOL, MAX_ITER, hist_cap=MAX_ITER)
            assert r["iters"] == meta["iters"], (form, lanes)
            assert rel(r["hist_x"], g["hist_x"]) <= HIST_RTOL, (form, lanes)
            assert rel(r["x"], g["x"]) <= SOL_RTOL, (form, lanes)
            assert rel(r["y"], g["y"]) <= SOL_RTOL, (form, lanes)
            got[lanes] = r
    finally:
        gpu_ctx.set_option("pcg_form", -1)
        gpu_ctx.set_option("pcg_lanes", 0)
    for k in ("x", "y", "hist_x", "hist_y"):
        if form == 2:
            assert np.array_equal(got[32][k], got[1][k]), (form, k)
        else:
            assert rel(got[32][k], got[1][k]) <= 1e-12, (form, k)
    if form == 2:
        for lanes in (32, 1):
            assert np.array_equal(got[lanes]["x"], g["x"]) and np.array_equal(got[lanes]["y"], g["y"])


def _multiply_order(s, v):
    """SparseSystem::multiply's order (simpl_lss.h:49-57) in numpy: diag * v
    first, then each row's entries in storage order."""
    rp = s["row_ptr"].astype(np.int64)
    col, val = s["col"].astype(np.int64), s["val"]
    want = s["diag"] * v
    lens = np.diff(rp)
    for k in range(int(lens.max()) if len(lens) else 0):
        rows = np.nonzero(lens > k)[0]
        e = rp[rows] + k
        want[rows] = want[rows] + val[e] * v[col[e]]
    return want


@pytest.mark.parametrize("cells", [12_000, 1_000_000])
def test_spmv_device_mode_bit_exact(cells, gpu_ctx):
    """ktg_spmv on device pointers: one wave of blocks at 12k rows, more
    blocks than SMs at 1M rows; bit-identical to the reference's row sums and
    to the host-pointer call. Overlapping in and out are refused."""
    import torch
    from ktplace_b200 import synth, netlist
    spec = synth.spec_small(0) if cells == 12_000 else synth.SynthSpec(
        num_movable=cells, num_nets=int(cells * 1.05), num_pads=1_200, num_rows=1_900,
        utilization=0.6, num_macros=600, seed=9, name="synth1m")
    raw = synth.generate(spec)
    nl = netlist.flatten(raw)
    x, y = synth.seed_positions(raw, nl.num_movable, 21)
    ax, ay = synth.seed_positions(raw, nl.num_movable, 22)
    fx, fy = nl.floors()
    gpu_ctx.upload_netlist(nl)
    gpu_ctx.build_b2b(x, y, 0.2, ax, ay, fx, fy)
    rng = np.random.default_rng(6)
    for axis in (0, 1):
        s = gpu_ctx.system(axis)
        v = rng.standard_normal(len(s["diag"]))
        want = _multiply_order(s, v)
        dv = torch.tensor(v, device="cuda:0")
        dout = torch.empty_like(dv)
        gpu_ctx.spmv_dev(axis, dv, dout)
        torch.cuda.synchronize()
        assert np.array_equal(dout.cpu().numpy(), want), (cells, axis)
        assert np.array_equal(gpu_ctx.spmv(axis, v), want), (cells, axis)
        with pytest.raises(Exception):
            gpu_ctx.spmv_dev(axis, dv, dv)


@pytest.mark.parametrize("name", list(CASES))
def test_spmv_bit_exact(name, gpu_ctx):
    """ktg_spmv against SparseSystem::multiply's order (simpl_lss.h:49-57):
    diag * v first, then the row's entries in storage order."""
    raw, nl, x, y, ax, ay, alpha, _ = build_case(name)
    gpu_ctx.upload_netlist(nl)
    fx, fy = nl.floors()
    gpu_ctx.build_b2b(x, y, alpha, ax if alpha > 0 else None, ay if alpha > 0 else None, fx, fy)
    rng = np.random.default_rng(5)
    for axis in (0, 1):
        s = gpu_ctx.system(axis)
        v = rng.standard_normal(len(s["diag"]))
        assert np.array_equal(gpu_ctx.spmv(axis, v), _multiply_order(s, v)), (name, axis)


@pytest.mark.parametrize("name", list(CASES))
def test_hpwl_and_density(name, gpu_ctx):
    from ktplace_b200 import grid as kgrid
    g, meta = gold(name)
    raw, nl, *_ , gbins = build_case(name)
    gpu_ctx.upload_netlist(nl)
    h = gpu_ctx.hpwl(g["x"], g["y"])
    assert abs(h - meta["hpwl_out"]) <= HPWL_RTOL * abs(meta["hpwl_out"])
    bg = kgrid.build_grid(nl, gbins, 1.0)
    gpu_ctx.set_grid(bg)
    occ, ov = gpu_ctx.occupancy(g["x"], g["y"])
    assert digest(occ) == meta["sha_occ"]
    assert abs(ov - meta["overflow"]) <= OVF_RTOL * max(abs(meta["overflow"]), 1e-300)


def test_solve_is_deterministic(gpu_ctx):
    raw, nl, x, y, ax, ay, alpha, _ = build_case("small12k")
    gpu_ctx.upload_netlist(nl)
    fx, fy = nl.floors()
    gpu_ctx.build_b2b(x, y, alpha, ax, ay, fx, fy)
    a = gpu_ctx.solve(x, y, TOL, MAX_ITER)
    b = gpu_ctx.solve(x, y, TOL, MAX_ITER)
    assert np.array_equal(a["x"], b["x"]) and np.array_equal(a["y"], b["y"])


def test_max_iter_and_zero_iterations(gpu_ctx):
    raw, nl, x, y, ax, ay, alpha, _ = build_case("tiny_macros")
    gpu_ctx.upload_netlist(nl)
    fx, fy = nl.floors()
    gpu_ctx.build_b2b(x, y, alpha, ax, ay, fx, fy)
    r0 = gpu_ctx.solve(x, y, TOL, 0)
    assert r0["iters"] == 0 and np.array_equal(r0["x"], x)
    r3 = gpu_ctx.solve(x, y, TOL, 3, hist_cap=8)
    assert r3["iters"] == 3 and r3["iters_x"] == 3 and r3["live"] == 3


def test_errors_are_reported(gpu_ctx):
    from ktplace_b200._lib import KtgError
    from ktplace_b200.gpu import Context
    c = Context(0)
    with pytest.raises(KtgError):
        c.build_b2b(np.zeros(3), np.zeros(3), 0.0)  # no netlist yet
    raw, nl, *_ = build_case("tiny_macros")
    bad = type(nl)(**{**nl.__dict__})
    bad.pin_cell = nl.pin_cell.copy()
    bad.pin_cell[5] = nl.num_vertices + 7
    with pytest.raises(KtgError):
        c.upload_netlist(bad)
    c.close()
