"""Generates the golden vectors in this directory from the reference itself.

Runs the reference's own SimPL code (oracle/_ref/libktref.so, compiled from
the reference sources by oracle/Makefile) on every case of cases.py and stores
its outputs: bound pins, the B2B CSR of both axes, the PCG solution and
residual history, HPWL before and after the solve, the bin grid, the
occupancy map and the overflow. Small arrays are stored whole; the larger
case stores SHA-256 digests of the exact arrays plus the solution.

    python tests/golden/make_golden.py        (needs oracle/_ref built)
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

import oracle  # noqa: E402
from cases import CASES, TOL, MAX_ITER, build_case, digest, netlist_digest  # noqa: E402


def ref_outputs(name):
    raw, nl, x, y, ax, ay, alpha, gbins = build_case(name)
    ref = oracle.RefDesign.from_netlist(nl)
    fx, fy = ref.floors()
    hpwl_in = ref.hpwl(x, y)
    ref.build_b2b(x, y, alpha, ax if alpha > 0 else None, ay if alpha > 0 else None)
    sx, sy = ref.system(0), ref.system(1)
    # Bound pins: the reference keeps them local to buildB2BAxis; the C
    # restatement (pinned bit-exactly against the reference CSR below) gives them.
    port = oracle.PortNetlist(nl)
    bx = port.b2b_axis(True, x, fx, alpha, ax)
    by = port.b2b_axis(False, y, fy, alpha, ay)
    for s, b in ((sx, bx), (sy, by)):
        for k in ("row_ptr", "col", "val", "diag", "rhs"):
            assert np.array_equal(s[k].astype(np.float64), b[k].astype(np.float64)), k
    r = ref.solve(x, y, TOL, MAX_ITER, hist_cap=MAX_ITER)
    hpwl_out = ref.hpwl(r["x"], r["y"])
    g = ref.grid(gbins, 1.0)
    occ, ov = ref.occupancy_map(r["x"], r["y"], g["nx"] * g["ny"])
    out = dict(
        netlist_digest=netlist_digest(nl), floors=np.array([fx, fy]), hpwl_in=hpwl_in,
        hpwl_out=hpwl_out, x=r["x"], y=r["y"], resid=np.array(r["resid"]), iters=r["iters"],
        hist_x=r["hist_x"], hist_y=r["hist_y"], grid_info=np.array(
            [g["origin"][0], g["origin"][1], g["dx"], g["dy"], g["nx"], g["ny"],
             g["total_avail"]]), overflow=ov)
    small = nl.num_movable <= 1000
    for axis, s, b in ((0, sx, bx), (1, sy, by)):
        arrs = dict(row_ptr=s["row_ptr"].astype(np.int64), col=s["col"].astype(np.int32),
                    val=s["val"], diag=s["diag"], rhs=s["rhs"], lo=b["lo"], hi=b["hi"])
        for k, a in arrs.items():
            if small:
                out[f"{k}_{axis}"] = a
            out[f"sha_{k}_{axis}"] = digest(a)
    if small:
        out["avail"] = g["avail"]
        out["occ"] = occ
    out["sha_avail"] = digest(g["avail"])
    out["sha_occ"] = digest(occ)
    return out


def main():
    meta = {}
    for name in CASES:
        out = ref_outputs(name)
        arrays = {k: v for k, v in out.items() if isinstance(v, np.ndarray)}
        scalars = {k: v for k, v in out.items() if not isinstance(v, np.ndarray)}
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **arrays)
        meta[name] = {k: (float(v) if isinstance(v, (float, np.floating)) else v)
                      for k, v in scalars.items()}
        print(name, "iters", out["iters"], "hpwl", out["hpwl_in"], "->", out["hpwl_out"])
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(meta, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
