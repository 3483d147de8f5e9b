"""Two-level aggregation preconditioner: block Jacobi over the aggregates plus
an additive coarse correction z (z^T A z)^-1 z^T r (option "coarse").

Bars:
  - the coarse vector, A z and 1 / (z^T A z) agree with a float64 numpy
    restatement on the downloaded system (FP32 rounding of z and A z);
  - every mixed solve meets the FP64 tolerance on the true residual and lands
    within 1e-4 relative of the FP64 GPU solve, with HPWL within 0.1%;
  - on systems of a SimPL run (the GPU global loop on the 12k design), the
    constant coarse vector needs fewer inner iterations than none.
"""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

from cases import build_case, TOL, MAX_ITER  # noqa: E402
from test_gpu_mixed import true_resid  # noqa: E402

pytestmark = pytest.mark.gpu

SOL_RTOL = 1e-4
HPWL_RTOL = 1e-3


def _csr_apply(s, v):
    n = s["diag"].shape[0]
    rows = np.repeat(np.arange(n), np.diff(s["row_ptr"]))
    out = s["diag"] * v
    np.add.at(out, rows, s["val"] * v[s["col"]])
    return out


def _coarse_numpy(ctx, mode):
    """z, A z (combined natural order) and 1 / (z^T A z) per axis, float64."""
    zs, azs, einv = [], [], []
    for axis in (0, 1):
        s = ctx.system(axis)
        n = s["diag"].shape[0]
        if mode == 1:
            z = np.ones(n)
        else:
            rows = np.repeat(np.arange(n), np.diff(s["row_ptr"]))
            z = np.bincount(rows, weights=np.abs(s["val"]), minlength=n) / s["diag"]
        z = z.astype(np.float32).astype(np.float64)
        az = _csr_apply(s, z)
        e = float(z @ az)
        zs.append(z)
        azs.append(az)
        einv.append(1.0 / e if e > 0 else 0.0)
    return np.concatenate(zs), np.concatenate(azs), np.array(einv)


@pytest.fixture
def coarse_ctx(gpu_ctx):
    gpu_ctx.set_option("precond", 2)
    yield gpu_ctx
    gpu_ctx.set_option("coarse", 0)
    gpu_ctx.set_option("precond", 0)


def simpl_systems(ctx, iters, init_rounds=3):
    """Yields the GlobalIterates of a short GPU SimPL run on the 12k design."""
    from ktplace_b200 import grid as kgrid
    from ktplace_b200 import simpl
    raw, nl, x, y, *_ = build_case("small12k")
    ctx.upload_netlist(nl)
    g = kgrid.build_grid(nl, kgrid.default_bins_per_axis(nl.num_movable), 1.0)
    loop = simpl.GlobalLoop(ctx, nl, g, kgrid.build_free_space(nl), tol=TOL, max_iter=MAX_ITER)
    x, y = loop.initial_rounds(x, y, init_rounds)
    for state in loop.iterations(x, y, iters):
        yield nl, state


@pytest.mark.parametrize("mode", [1, 2])
@pytest.mark.parametrize("name", ["tiny_macros", "edge_alpha", "small12k"])
def test_coarse_vector_matches_numpy(name, mode, coarse_ctx):
    raw, nl, x, y, ax, ay, alpha, _ = build_case(name)
    coarse_ctx.upload_netlist(nl)
    fx, fy = nl.floors()
    coarse_ctx.build_b2b(x, y, alpha, ax, ay, fx, fy)
    coarse_ctx.set_option("coarse", mode)
    got = coarse_ctx.coarse()
    order = coarse_ctx.aggregates()["order"]
    z, az, einv = _coarse_numpy(coarse_ctx, mode)
    assert np.array_equal(got["z"].astype(np.float64), z[order])
    scale = np.abs(az).max()
    assert np.all(np.abs(got["az"] - az[order]) <= 2e-7 * np.abs(az[order]) + 1e-12 * scale)
    for a in range(2):
        assert abs(got["einv"][a] - einv[a]) <= 1e-9 * abs(einv[a])


@pytest.mark.parametrize("mode", [0, 1, 2])
@pytest.mark.parametrize("name", ["tiny_macros", "edge_alpha", "small12k"])
def test_coarse_solve_matches_fp64(name, mode, coarse_ctx):
    raw, nl, x, y, ax, ay, alpha, _ = build_case(name)
    coarse_ctx.upload_netlist(nl)
    fx, fy = nl.floors()
    coarse_ctx.build_b2b(x, y, alpha, ax, ay, fx, fy)
    sx, sy = coarse_ctx.system(0), coarse_ctx.system(1)
    f = coarse_ctx.solve(x, y, TOL, MAX_ITER)
    coarse_ctx.set_option("coarse", mode)
    r = coarse_ctx.solve_mixed(x, y, TOL)
    assert r["fp64_iters"] == (0, 0)
    assert true_resid(sx, r["x"]) <= TOL * 1.0001
    assert true_resid(sy, r["y"]) <= TOL * 1.0001
    for k in ("x", "y"):
        assert np.linalg.norm(r[k] - f[k]) / np.linalg.norm(f[k]) <= SOL_RTOL
    hf, hr = coarse_ctx.hpwl(f["x"], f["y"]), coarse_ctx.hpwl(r["x"], r["y"])
    assert abs(hr - hf) <= HPWL_RTOL * hf


def test_coarse_on_simpl_systems(coarse_ctx):
    """Systems of a SimPL run: both coarse vectors meet the tolerance, agree
    with FP64, and the constant one saves inner iterations over none."""
    saved = 0
    for nl, st in simpl_systems(coarse_ctx, 6):
        if st.it not in (1, 5):
            continue
        sx, sy = coarse_ctx.system(0), coarse_ctx.system(1)
        f = coarse_ctx.solve(st.x, st.y, TOL, MAX_ITER)
        inner = {}
        for mode in (0, 1, 2):
            coarse_ctx.set_option("coarse", mode)
            r = coarse_ctx.solve_mixed(st.x, st.y, TOL)
            assert true_resid(sx, r["x"]) <= TOL * 1.0001
            assert true_resid(sy, r["y"]) <= TOL * 1.0001
            for k in ("x", "y"):
                assert np.linalg.norm(r[k] - f[k]) / np.linalg.norm(f[k]) <= SOL_RTOL
            inner[mode] = sum(r["inner"])
        coarse_ctx.set_option("coarse", 0)
        assert inner[1] < inner[0], inner
        saved += inner[0] - inner[1]
    assert saved > 0


def test_agg_reuse_on_simpl_systems(gpu_ctx):
    """agg_reuse: along a SimPL run the aggregates of a full build serve the
    next builds (only the values are taken afresh). Every solve still meets
    the FP64 tolerance on the true residual and agrees with the FP64 solve,
    and the inner iterations stay within a third of the fresh builds'."""
    from ktplace_b200.gpu import Context
    fresh, reused = 0, 0
    with Context(0) as other:
        other.set_option("precond", 2)
        other.set_option("coarse", 2)
        other.set_option("agg_reuse", 3)
        gpu_ctx.set_option("precond", 2)
        gpu_ctx.set_option("coarse", 2)
        try:
            for nl, st in simpl_systems(gpu_ctx, 8):
                if other.nl is not nl:
                    other.upload_netlist(nl)
                fx, fy = nl.floors()
                other.build_b2b(st.x, st.y, st.alpha, st.ux, st.uy, fx, fy)
                sx, sy = other.system(0), other.system(1)
                r = other.solve_mixed(st.x, st.y, TOL)
                f = gpu_ctx.solve_mixed(st.x, st.y, TOL)
                assert true_resid(sx, r["x"]) <= TOL * 1.0001
                assert true_resid(sy, r["y"]) <= TOL * 1.0001
                for k in ("x", "y"):
                    assert np.linalg.norm(r[k] - f[k]) / np.linalg.norm(f[k]) <= SOL_RTOL
                fresh += sum(f["inner"])
                reused += sum(r["inner"])
        finally:
            gpu_ctx.set_option("coarse", 0)
            gpu_ctx.set_option("precond", 0)
    assert reused <= 1.34 * fresh, (reused, fresh)


def test_trained_coarse_vector_beats_network_off():
    """The committed trained coarse-vector network against the same solver
    with the network switched off (the aggregation preconditioner with no
    coarse vector), along a SimPL run of a held-out 60k-cell design: the
    learned vector (prepared per build) needs fewer inner iterations and
    less device time (CUDA events, per-netlist set-up untimed), and every
    solve meets the FP64 tolerance on the true residual."""
    import torch
    from ktplace_b200 import grid as kgrid
    from ktplace_b200 import simpl
    from ktplace_b200.gpu import Context
    from ktplace_b200.learned import Learned
    from ktplace_b200.train_precond import coarse_design, COARSE_OUT
    from ktplace_b200._lib import MixedInfo
    import ctypes
    nl, x0, y0, _ = coarse_design(1, 60_000, 4242)  # seed outside the training set
    dev = torch.device("cuda:0")
    stream = torch.cuda.Stream(device=dev)
    learned = Learned(0)
    learned.load(COARSE_OUT)
    ctxs = {}
    for name, coarse in (("off", 0), ("learned", 3)):
        c = Context(0)
        c.set_stream(stream.cuda_stream)
        c.upload_netlist(nl)
        c.set_option("precond", 2)
        c.set_option("coarse", coarse)
        c.set_option("agg_reuse", 4)
        ctxs[name] = c
    loop_ctx = Context(0)
    try:
        loop_ctx.upload_netlist(nl)
        g = kgrid.build_grid(nl, kgrid.default_bins_per_axis(nl.num_movable), 1.0)
        loop = simpl.GlobalLoop(loop_ctx, nl, g, kgrid.build_free_space(nl), tol=TOL,
                                max_iter=MAX_ITER)
        x, y = loop.initial_rounds(x0, y0, 3)
        fx, fy = nl.floors()
        for c in ctxs.values():  # untimed: buffers, and the per-netlist trunk
            c.build_b2b(x, y, 0.0, None, None, fx, fy)
            learned.prepare_coarse(c)
            c.solve_mixed(x, y, TOL)
        ms = {k: 0.0 for k in ctxs}
        inner = {k: 0 for k in ctxs}
        with torch.cuda.stream(stream):
            dx = torch.zeros(nl.num_movable, dtype=torch.float64, device=dev)
            dy = torch.zeros_like(dx)
            minfo = torch.zeros(ctypes.sizeof(MixedInfo), dtype=torch.uint8, device=dev)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        for st in loop.iterations(x, y, 10):
            for name, c in ctxs.items():
                c.build_b2b(st.x, st.y, st.alpha, st.ux, st.uy, fx, fy)
                with torch.cuda.stream(stream):
                    dx.copy_(torch.from_numpy(st.x))
                    dy.copy_(torch.from_numpy(st.y))
                torch.cuda.synchronize(dev)
                with torch.cuda.stream(stream):
                    e0.record(stream)
                    if name == "learned":
                        learned.prepare_coarse(c)
                    c.solve_mixed_dev(dx, dy, TOL, 1e-3, MAX_ITER, 50, minfo)
                    e1.record(stream)
                e1.synchronize()
                if st.it > 0:  # the run's first build makes the aggregates afresh in both
                    ms[name] += e0.elapsed_time(e1)
                mi = MixedInfo.from_buffer_copy(bytes(minfo.cpu().numpy()))
                inner[name] += int(mi.inner_x) + int(mi.inner_y)
                sx, sy = c.system(0), c.system(1)
                assert true_resid(sx, dx.cpu().numpy()) <= TOL * 1.0001
                assert true_resid(sy, dy.cpu().numpy()) <= TOL * 1.0001
        assert inner["learned"] < inner["off"], inner
        assert ms["learned"] < ms["off"], (ms, inner)
    finally:
        for c in ctxs.values():
            c.close()
        loop_ctx.close()
        learned.close()
