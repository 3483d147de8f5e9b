"""The config-2 report (bench.py --simpl-report) on a small design: 30 SimPL
global iterations with the anchor weight rising linearly from 0.01 to 1.0
and the anchors at the look-ahead-legalized positions; at every iteration
every mixed variant (Jacobi, aggregation with and without a coarse vector
and structure reuse, the learned coarse vector) meets the FP64 tolerance on
its true residual and ends within 0.1% of the FP64 solve's HPWL."""
import os
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(HERE, "golden"))

from cases import build_case, TOL  # noqa: E402

pytestmark = pytest.mark.gpu


def test_simpl_report_every_iteration_within_bounds():
    import torch
    sys.path.insert(0, ROOT)
    import bench
    raw, nl, x, y, ax, ay, alpha, _ = build_case("small12k")
    dev = torch.device("cuda:0")
    stream = torch.cuda.Stream(device=dev)
    learned = bench.load_coarse_network(dev)
    assert learned is not None, "the committed coarse-vector weights are missing"
    try:
        rep = bench.simpl_report(torch, dev, stream, nl, x, y, 30, learned=learned)
    finally:
        learned.close()
    rows = rep["iterations"]
    assert len(rows) == 30
    assert abs(rows[0]["alpha"] - 0.01) < 1e-12 and abs(rows[-1]["alpha"] - 1.0) < 1e-12
    names = [v[0] for v in bench.SIMPL_VARIANTS]
    for r in rows:
        assert r["fp64_jacobi"]["resid"][0] <= TOL and r["fp64_jacobi"]["resid"][1] <= TOL
        for nm in names[1:]:
            v = r[nm]
            assert max(v["true_resid"]) <= TOL * 1.0001, (r["it"], nm, v["true_resid"])
            assert abs(v["hpwl_rel_vs_fp64"]) <= 1e-3, (r["it"], nm, v["hpwl_rel_vs_fp64"])
    s = rep["summary"]
    assert s["fp32_aggregation"]["iters_mean"] < s["fp32_jacobi"]["iters_mean"]
    assert s["fp32_learned"]["iters_mean"] < s["fp32_aggregation"]["iters_mean"]
