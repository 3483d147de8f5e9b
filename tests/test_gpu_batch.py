"""Batched cluster solver against the oracle.

FP64: every system of a batch of uneven sizes (a 12k-cell design's systems
next to tiny and corner-case ones) matches the oracle's PCG: same iteration
count, solution within 1e-9 relative. Mixed: every system meets the
tolerance on its true FP64 residual. Also: each cluster shape gives the same
FP64 answer, the autotuner picks a launchable shape, results carry
latencies, and repeated graph replays are identical.
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


def true_resid(s, x):
    n = s["diag"].shape[0]
    rows = np.repeat(np.arange(n), np.diff(s["row_ptr"]))
    ax = s["diag"] * x
    np.add.at(ax, rows, s["val"] * x[s["col"]])
    nb = np.linalg.norm(s["rhs"])
    return np.linalg.norm(s["rhs"] - ax) / nb if nb > 0 else 0.0


@pytest.fixture(scope="module")
def systems(port_built):
    out = []
    for name in ("small12k", "tiny_macros", "edge_alpha", "edge_alpha0"):
        raw, nl, x, y, ax, ay, alpha, _ = build_case(name)
        port = oracle.PortNetlist(nl)
        fx, fy = nl.floors()
        sx = port.b2b_axis(True, x, fx, alpha, ax if alpha > 0 else None)
        sy = port.b2b_axis(False, y, fy, alpha, ay if alpha > 0 else None)
        out += [(sx, x), (sy, y)]
    return out


def make_batch(systems):
    from ktplace_b200.gpu import Batch
    b = Batch(0)
    ids = [b.add_system(s, x0) for s, x0 in systems]
    return b, ids


@pytest.mark.parametrize("cluster,threads", [(2, 256), (8, 512), (16, 1024)])
def test_batch_fp64_matches_oracle(systems, cluster, threads):
    b, ids = make_batch(systems)
    b.set_shape(cluster, threads)
    b.solve(TOL, MAX_ITER, precision=0)
    res = b.results()
    for (s, x0), sid in zip(systems, ids):
        ref = oracle.port_pcg_axis(s, x0, TOL, MAX_ITER)
        got = b.get_x(sid, s["diag"].shape[0])
        assert res[sid]["status"] == 0
        assert res[sid]["iters"] == ref["iters"], (sid, res[sid], ref["iters"])
        assert np.linalg.norm(got - ref["x"]) <= 1e-9 * np.linalg.norm(ref["x"])
        assert res[sid]["latency_ns"] > 0
    b.close()


def test_batch_mixed_meets_true_residual(systems):
    b, ids = make_batch(systems)
    b.solve(TOL, MAX_ITER, precision=1, inner_tol=1e-3)
    res = b.results()
    for (s, x0), sid in zip(systems, ids):
        got = b.get_x(sid, s["diag"].shape[0])
        assert res[sid]["status"] == 0, res[sid]
        assert true_resid(s, got) <= TOL * 1.0001
    b.close()


def test_batch_autotune_and_replay(systems):
    b, ids = make_batch(systems)
    c, t, ms = b.autotune(TOL, precision=0, probe_iter=20)
    assert c in (2, 4, 8, 16) and t in (256, 512, 1024) and ms > 0
    b.solve(TOL, MAX_ITER, precision=0)
    first = [b.get_x(i, s["diag"].shape[0]).copy() for (s, _), i in zip(systems, ids)]
    b.reset_x()
    b.solve(TOL, MAX_ITER, precision=0)
    for (s, _), i, a in zip(systems, ids, first):
        assert np.array_equal(b.get_x(i, s["diag"].shape[0]), a)
    b.close()


@pytest.mark.parametrize("cluster,threads,clusters", [(16, 1024, 1), (8, 1024, 2), (16, 512, 2)])
def test_batch_size_split_matches_oracle(systems, cluster, threads, clusters):
    """The 12k-cell design's two systems go to the large class; every system
    still matches the oracle's PCG exactly as without the split."""
    b, ids = make_batch(systems)
    b.set_shape(4, 256)
    rows = sorted((s["diag"].shape[0] for s, _ in systems), reverse=True)
    b.set_split(rows[1], cluster, threads, clusters)
    sp = b.split()
    assert sp["num_large"] == sum(r >= rows[1] for r in rows) and sp["cluster"] == cluster
    launches = b.launches
    b.solve(TOL, MAX_ITER, precision=0)
    assert b.launches - launches == 2
    res = b.results()
    for (s, x0), sid in zip(systems, ids):
        ref = oracle.port_pcg_axis(s, x0, TOL, MAX_ITER)
        got = b.get_x(sid, s["diag"].shape[0])
        assert res[sid]["status"] == 0
        assert res[sid]["iters"] == ref["iters"], (sid, res[sid], ref["iters"])
        assert np.linalg.norm(got - ref["x"]) <= 1e-9 * np.linalg.norm(ref["x"])
    # mixed precision through the split, then switching the split off again
    b.reset_x()
    b.solve(TOL, MAX_ITER, precision=1, inner_tol=1e-3)
    res = b.results()
    for (s, _), sid in zip(systems, ids):
        assert res[sid]["status"] == 0 and true_resid(s, b.get_x(sid, s["diag"].shape[0])) <= TOL * 1.0001
    b.set_split(0)
    assert b.split()["num_large"] == 0
    b.reset_x()
    b.solve(TOL, MAX_ITER, precision=0)
    assert all(r["status"] == 0 for r in b.results())
    b.close()


def test_batch_all_large_and_autotune_split(systems):
    b, ids = make_batch(systems)
    b.set_split(1, 8, 512, 4)  # every system in the large class: one launch
    launches = b.launches
    b.solve(TOL, MAX_ITER, precision=0)
    assert b.launches - launches == 1
    assert all(r["status"] == 0 for r in b.results())
    b.set_split(0)
    sp, base, best = b.autotune_split(TOL, precision=0, max_iter=MAX_ITER)
    assert base > 0 and 0 < best <= base
    assert sp["rows"] == 0 or sp["num_large"] >= 1
    b.solve(TOL, MAX_ITER, precision=0)
    for (s, x0), sid in zip(systems, ids):
        ref = oracle.port_pcg_axis(s, x0, TOL, MAX_ITER)
        assert np.linalg.norm(b.get_x(sid, s["diag"].shape[0]) - ref["x"]) <= 1e-9 * np.linalg.norm(ref["x"])
    b.close()


def test_sharded_batch_product_path(port_built):
    """shard.ShardPlan + shard.run_share with the GPU share solver: the two
    shares of a world-2 plan solved one after the other on this GPU (they
    never wait on each other), assembled and checked against the oracle."""
    from ktplace_b200 import shard
    names = ("small12k", "tiny_macros", "edge_alpha", "edge_alpha0")
    cases = {}

    def make_unit(u):
        if u not in cases:
            raw, nl, x, y, ax, ay, alpha, _ = build_case(names[u])
            cases[u] = (nl, x, y, ax, ay, alpha)
        return cases[u]

    sizes = [2 * make_unit(u)[0].num_movable for u in range(len(names))]
    plan = shard.ShardPlan(sizes, sizes, world=2)
    out = np.full(plan.total, np.nan)
    for rank in range(2):
        solver = shard.BatchShardSolver(make_unit, device=0, tol=TOL, max_iter=MAX_ITER,
                                        precision=0, autotune=rank == 0)
        assert sorted(shard.run_share(plan, rank, solver, out)) == sorted(plan.share(rank))
        solver.close()
    assert not np.isnan(out).any()
    for u in range(len(names)):
        nl, x, y, ax, ay, alpha = make_unit(u)
        port = oracle.PortNetlist(nl)
        fx, fy = nl.floors()
        n = nl.num_movable
        got = out[plan.slice(u)]
        for axis, (pos, fl, anc) in enumerate(((x, fx, ax), (y, fy, ay))):
            s = port.b2b_axis(axis == 0, pos, fl, alpha, anc if alpha > 0 else None)
            ref = oracle.port_pcg_axis(s, pos, TOL, MAX_ITER)["x"]
            mine = got[axis * n:(axis + 1) * n]
            assert np.linalg.norm(mine - ref) <= 1e-9 * np.linalg.norm(ref), (names[u], axis)


@pytest.mark.parametrize("rows", [1, "big"])
def test_batch_offload_matches_oracle(systems, rows):
    """Pairs of consecutive equal-size systems at or above the threshold go to
    the whole-GPU path (an internal context), the rest to the cluster
    launches; FP64: every system matches the oracle's PCG (iterations and
    solution), mixed (aggregation, coarse vector): every system meets the
    tolerance on its true residual."""
    b, ids = make_batch(systems)
    sizes = [s["diag"].shape[0] for s, _ in systems]
    thr = 1 if rows == 1 else max(sizes)
    b.set_offload(thr, precond=2, coarse=2)
    off = b.offload()
    want_pairs = sum(1 for k in range(0, len(sizes) - 1, 2)
                     if sizes[k] >= thr and sizes[k + 1] == sizes[k])
    assert off["pairs"] == want_pairs >= 1
    b.solve(TOL, MAX_ITER, precision=0)
    res = b.results()
    for (s, x0), sid in zip(systems, ids):
        ref = oracle.port_pcg_axis(s, x0, TOL, MAX_ITER)
        got = b.get_x(sid, s["diag"].shape[0])
        assert res[sid]["status"] == 0, (sid, res[sid])
        assert res[sid]["iters"] == ref["iters"], (sid, res[sid], ref["iters"])
        assert np.linalg.norm(got - ref["x"]) <= 1e-9 * np.linalg.norm(ref["x"])
    for rep in range(2):  # the second solve reloads the pairs' systems afresh
        b.reset_x()
        b.solve(TOL, MAX_ITER, precision=1, inner_tol=1e-3)
        res = b.results()
        for (s, _), sid in zip(systems, ids):
            got = b.get_x(sid, s["diag"].shape[0])
            assert res[sid]["status"] == 0, (sid, res[sid])
            assert true_resid(s, got) <= TOL * 1.0001
            assert res[sid]["latency_ns"] > 0
    b.close()


def offloaded_ids(sizes, thr):
    """Systems the whole-GPU path takes at threshold thr: equal-size
    consecutive pairs of >= thr rows, paired from the front."""
    out, k = set(), 0
    while k + 1 < len(sizes):
        if sizes[k] >= thr and sizes[k + 1] == sizes[k]:
            out |= {k, k + 1}
            k += 2
        else:
            k += 1
    return out


def test_batch_split_counts_queued_systems(systems):
    """With pairs on the whole GPU the size split covers only the systems left
    in the queues (its count and the autotuner's thresholds); with every
    system offloaded the autotuner keeps no split. Every system still meets
    the tolerance on its true residual."""
    b, ids = make_batch(systems)
    sizes = [s["diag"].shape[0] for s, _ in systems]
    thr = max(sizes)
    b.set_offload(thr, precond=2, coarse=0)
    off = offloaded_ids(sizes, thr)
    assert b.offload()["pairs"] == len(off) // 2 >= 1
    b.set_split(1, 8, 512, 1)
    assert b.split()["num_large"] == len(sizes) - len(off)
    b.set_split(0)
    sp, base, best = b.autotune_split(TOL, precision=1, inner_tol=1e-3, max_iter=MAX_ITER)
    assert 0 < best <= base
    queued = [n for k, n in enumerate(sizes) if k not in off]
    assert sp["rows"] == 0 or (sp["rows"] in queued and sp["num_large"] >= 1)
    b.solve(TOL, MAX_ITER, precision=1, inner_tol=1e-3)
    for (s, _), r, sid in zip(systems, b.results(), ids):
        assert r["status"] == 0 and true_resid(s, b.get_x(sid, s["diag"].shape[0])) <= TOL * 1.0001
    if len(offloaded_ids(sizes, 1)) == len(sizes):
        b.set_offload(1, precond=2, coarse=0)
        sp, base, best = b.autotune_split(TOL, precision=1, inner_tol=1e-3, max_iter=MAX_ITER)
        assert sp["rows"] == 0 and base == 0.0 and best == 0.0
        b.solve(TOL, MAX_ITER, precision=1, inner_tol=1e-3)
        for (s, _), r, sid in zip(systems, b.results(), ids):
            assert r["status"] == 0
    b.close()


def test_batch_autotune_offload(systems):
    b, ids = make_batch(systems)
    off, base, best = b.autotune_offload(TOL, precision=1, inner_tol=1e-3, max_iter=MAX_ITER)
    assert base > 0 and 0 < best <= base
    assert off["rows"] == 0 or off["pairs"] >= 1
    b.solve(TOL, MAX_ITER, precision=1, inner_tol=1e-3)
    for (s, _), r, sid in zip(systems, b.results(), ids):
        assert r["status"] == 0 and true_resid(s, b.get_x(sid, s["diag"].shape[0])) <= TOL * 1.0001
    b.close()


def test_upload_second_axis_larger_keeps_first(systems):
    """Installing the y system when it needs more entries than the context
    holds keeps the x system installed just before (the arrays grow with
    their contents), so the solve matches the oracle on both axes."""
    from ktplace_b200.gpu import Context
    (sx, x0), (sy, y0) = systems[0], systems[1]
    small, large = (sx, sy) if len(sx["val"]) <= len(sy["val"]) else (sy, sx)
    s0, s1 = (small, large)
    v0, v1 = (x0, y0) if s0 is sx else (y0, x0)
    with Context(0) as c:
        c.upload_system(0, s0)
        c.upload_system(1, s1)
        r = c.solve(v0, v1, TOL, MAX_ITER)
    for s, v, got in ((s0, v0, r["x"]), (s1, v1, r["y"])):
        ref = oracle.port_pcg_axis(s, v, TOL, MAX_ITER)
        assert np.linalg.norm(got - ref["x"]) <= 1e-9 * np.linalg.norm(ref["x"])
