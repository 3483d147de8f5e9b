"""Learned preconditioner on the GPU.

* Gradients of the hand-written training kernels against the float64 CPU
  oracle (oracle/learned_ref.py) on the same parameters: FP32 CUDA-core path
  within 2e-3 relative, BF16 tensor-core path within 3e-2 of the FP32 path.
* M keeps the solve exact: the learned-preconditioned mixed solve meets the
  true FP64 residual.
* What training buys: after training on SimPL-style systems of a few small
  netlists, held-out systems need fewer PCG iterations than with Jacobi.
"""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import oracle  # noqa: E402
from oracle import learned_ref as lr  # noqa: E402
from cases import build_case, TOL  # noqa: E402

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


@pytest.fixture(scope="module")
def tiny(port_built):
    raw, nl, x, y, ax, ay, alpha, _ = build_case("tiny_macros")
    return raw, nl, x, y, ax, ay, alpha


def test_gradients_match_cpu_oracle(tiny, gpu_ctx):
    from ktplace_b200.learned import Learned
    raw, nl, x, y, ax, ay, alpha = tiny
    gpu_ctx.upload_netlist(nl)
    fx, fy = nl.floors()
    gpu_ctx.build_b2b(x, y, alpha, ax, ay, fx, fy)
    params = lr.init_params(7)
    params["P"] *= 20.0
    flat = lr.flatten(params).astype(np.float32)
    learned = Learned(0, seed=1)
    learned.set_params(flat)
    learned.set_option("probes", 3)
    learned.set_option("tensor_cores", 0)
    s = gpu_ctx.system(0)
    p32 = lr.unflatten(flat.astype(np.float64))
    L_ref, g_ref, _ = lr.loss_and_grad(p32, s, nl, k=3, seed=11)
    L_gpu, g_gpu = learned.loss_grad(gpu_ctx, 0, seed=11)
    assert abs(L_gpu - L_ref) <= 1e-4 * abs(L_ref)
    gr = lr.flatten(g_ref)
    assert rel(g_gpu.astype(np.float64), gr) <= 2e-3
    for name, shape in lr.PARAM_SHAPES:
        a = lr.unflatten(g_gpu.astype(np.float64))[name]
        b = g_ref[name]
        if np.linalg.norm(b) > 1e-6 * np.linalg.norm(gr):
            assert rel(a, b) <= 1e-2, name
    learned.set_option("tensor_cores", 1)
    L_tc, g_tc = learned.loss_grad(gpu_ctx, 0, seed=11)
    assert abs(L_tc - L_gpu) <= 3e-2 * abs(L_gpu)
    assert rel(g_tc, g_gpu) <= 3e-2
    learned.close()


def test_tcgen05_dense_layers_match_mma_sync(tiny, gpu_ctx):
    """The tcgen05 dense layers (BF16 operands, FP32 accumulator in tensor
    memory) against the warp-level mma.sync layers on the same BF16 weights:
    forward, transposed and masked backward layers through the loss and its
    gradient. One CTA walking all 128-row tiles (mbarrier phases alternating,
    accumulator reused) gives the same bits as one CTA per tile."""
    from ktplace_b200.learned import Learned
    raw, nl, x, y, ax, ay, alpha = tiny
    gpu_ctx.upload_netlist(nl)
    fx, fy = nl.floors()
    gpu_ctx.build_b2b(x, y, alpha, ax, ay, fx, fy)
    params = lr.init_params(5)
    params["P"] *= 20.0
    learned = Learned(0, seed=2)
    learned.set_params(lr.flatten(params).astype(np.float32))
    learned.set_option("probes", 2)
    out = {}
    for mode, ctas in ((1, 0), (2, 0), (2, 1), (0, 0)):
        learned.set_option("tensor_cores", mode)
        learned.set_option("tc_ctas", ctas)
        out[(mode, ctas)] = learned.loss_grad(gpu_ctx, 0, seed=5)
    L2, g2 = out[(2, 0)]
    L2b, g2b = out[(2, 1)]
    L1, g1 = out[(1, 0)]
    L0, g0 = out[(0, 0)]
    assert nl.num_movable > 128 and nl.num_movable % 128  # several tiles, the last partial
    assert L2b == L2 and np.array_equal(g2b, g2)
    assert np.isfinite(L2) and np.all(np.isfinite(g2))
    # same BF16 products, FP32 sums in another order
    assert abs(L2 - L1) <= 1e-4 * abs(L1)
    assert rel(g2, g1) <= 1e-3
    assert abs(L2 - L0) <= 3e-2 * abs(L0)
    assert rel(g2, g0) <= 3e-2
    learned.close()


def test_learned_preconditioner_solves_exactly(tiny, gpu_ctx):
    from ktplace_b200.learned import Learned
    raw, nl, x, y, ax, ay, alpha = tiny
    gpu_ctx.upload_netlist(nl)
    fx, fy = nl.floors()
    gpu_ctx.build_b2b(x, y, alpha, ax, ay, fx, fy)
    params = lr.init_params(3)
    params["P"] *= 30.0
    learned = Learned(0)
    learned.set_params(lr.flatten(params).astype(np.float32))
    learned.prepare(gpu_ctx)
    gpu_ctx.set_option("precond", 1)
    r = gpu_ctx.solve_mixed(x, y, TOL, 1e-3)
    gpu_ctx.set_option("precond", 0)
    sx = gpu_ctx.system(0)
    n = sx["diag"].shape[0]
    rows = np.repeat(np.arange(n), np.diff(sx["row_ptr"]))
    axv = sx["diag"] * r["x"]
    np.add.at(axv, rows, sx["val"] * r["x"][sx["col"]])
    assert np.linalg.norm(sx["rhs"] - axv) / np.linalg.norm(sx["rhs"]) <= TOL * 1.0001
    learned.close()


def test_training_reduces_iterations(gpu_ctx):
    from ktplace_b200 import synth, netlist
    from ktplace_b200.learned import Learned, train, compare_solvers
    designs = []
    for k in range(4):
        raw = synth.generate(synth.spec_tiny(seed=60 + k, cells=3000, nets=3300, pads=60, rows=40))
        nl = netlist.flatten(raw)
        x0, y0 = synth.seed_positions(raw, nl.num_movable, 5 + k)
        designs.append((nl, x0, y0))
    learned = Learned(0, seed=2)
    learned.set_option("lr", 3e-3)
    losses = train(learned, designs[:3], iters=6, epochs=3, ctx=gpu_ctx)
    assert np.mean(losses[-6:]) < np.mean(losses[:6])
    nl, x0, y0 = designs[3]
    gpu_ctx.upload_netlist(nl)
    rows = compare_solvers(learned, gpu_ctx, nl, x0, y0, iters=6)
    jac = sum(sum(r["jacobi"]["inner"]) for r in rows)
    lrn = sum(sum(r["learned"]["inner"]) for r in rows)
    for r in rows:
        assert max(r["learned"]["resid"]) <= TOL * 1.0001
    assert lrn < jac, (lrn, jac)
    learned.close()


def test_coarse_gradients_match_cpu_oracle(tiny, gpu_ctx):
    """Learned coarse vector: the GPU's projection loss and parameter
    gradient (trunk on topology features, head, loss, all hand-written
    kernels, FP32 CUDA-core path) against the float64 oracle."""
    from ktplace_b200.learned import Learned
    raw, nl, x, y, ax, ay, alpha = tiny
    gpu_ctx.upload_netlist(nl)
    fx, fy = nl.floors()
    gpu_ctx.build_b2b(x, y, alpha, ax, ay, fx, fy)
    params = lr.init_params(5)
    params["P"] *= 20.0
    params["wz"] *= 10.0
    flat = lr.flatten(params).astype(np.float32)
    learned = Learned(0, seed=1)
    learned.set_params(flat)
    learned.set_option("tensor_cores", 0)
    E = np.random.default_rng(3).standard_normal((2, nl.num_movable))
    p32 = lr.unflatten(flat.astype(np.float64))
    for axis in (0, 1):
        s = gpu_ctx.system(axis)
        L_ref, g_ref, _ = lr.coarse_loss_and_grad(p32, s, nl, E)
        L_gpu, g_gpu = learned.coarse_loss_grad(gpu_ctx, axis, E)
        assert abs(L_gpu - L_ref) <= 1e-4 * abs(L_ref), (L_gpu, L_ref)
        gr = lr.flatten(g_ref)
        assert rel(g_gpu.astype(np.float64), gr) <= 2e-3
        for name, shape in lr.PARAM_SHAPES:
            a = lr.unflatten(g_gpu.astype(np.float64))[name]
            b = g_ref[name]
            if np.linalg.norm(b) > 1e-4 * np.linalg.norm(gr):
                assert rel(a, b) <= 1e-2, (axis, name, rel(a, b))
    learned.close()


def test_prepared_coarse_vector_matches_oracle(tiny, gpu_ctx):
    """ktg_learned_prepare_coarse's z for both axes (permuted into the
    aggregation order) against the oracle's head on the same parameters."""
    from ktplace_b200.learned import Learned
    raw, nl, x, y, ax, ay, alpha = tiny
    gpu_ctx.upload_netlist(nl)
    fx, fy = nl.floors()
    gpu_ctx.build_b2b(x, y, alpha, ax, ay, fx, fy)
    params = lr.init_params(6)
    params["P"] *= 20.0
    params["wz"] *= 10.0
    flat = lr.flatten(params).astype(np.float32)
    learned = Learned(0, seed=1)
    learned.set_params(flat)
    learned.set_option("tensor_cores", 0)
    p32 = lr.unflatten(flat.astype(np.float64))
    p, _ = lr.forward(p32, lr.topo_features(nl), lr.Graph(nl))
    want = np.concatenate([lr.coarse_head(p32, p, gpu_ctx.system(a))[0] for a in (0, 1)])
    gpu_ctx.set_option("precond", 2)
    try:
        learned.prepare_coarse(gpu_ctx)
        gpu_ctx.set_option("coarse", 3)
        got = gpu_ctx.coarse()
        order = gpu_ctx.aggregates()["order"]
        assert rel(got["z"].astype(np.float64), want[order]) <= 1e-4
        r = gpu_ctx.solve_mixed(x, y, TOL)
        sx = gpu_ctx.system(0)
        assert true_resid_of(sx, r["x"]) <= TOL * 1.0001
        # the trunk embedding stays with each context: alternating two
        # contexts of the same netlist reruns only the per-system head
        from ktplace_b200.gpu import Context
        with Context(0) as other:
            other.upload_netlist(nl)
            other.build_b2b(x, y, alpha, ax, ay, fx, fy)
            other.set_option("precond", 2)
            learned.prepare_coarse(other)  # trunk for the second context
            k0 = learned.launches
            learned.prepare_coarse(gpu_ctx)
            learned.prepare_coarse(other)
            assert learned.launches - k0 <= 2 * 4, learned.launches - k0
            other.set_option("coarse", 3)
            assert rel(other.coarse()["z"].astype(np.float64), want[order]) <= 1e-4
        assert rel(gpu_ctx.coarse()["z"].astype(np.float64), want[order]) <= 1e-4
    finally:
        gpu_ctx.set_option("coarse", 0)
        gpu_ctx.set_option("precond", 0)
        learned.close()


def true_resid_of(s, v):
    n = s["diag"].shape[0]
    rows = np.repeat(np.arange(n), np.diff(s["row_ptr"]))
    av = s["diag"] * v
    np.add.at(av, rows, s["val"] * v[s["col"]])
    return np.linalg.norm(s["rhs"] - av) / np.linalg.norm(s["rhs"])
