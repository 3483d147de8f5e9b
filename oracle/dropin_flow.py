"""Whole SimPL flows of the reference with and without the B200 drop-ins
(test infrastructure: it drives the reference's own SimPL, compiled into
oracle/_ref, through oracle.RefDesign.run_simpl).

    python -m oracle.dropin_flow [--cells 211000] [--threads N]

Runs, each in a fresh process (the drop-ins read their settings from the
environment when they create their GPU context): the reference on the CPU;
the reference with libktref_gpu.so's drop-ins (B2B build, solve, HPWL and
occupancy hooks, look-ahead legalizer) at their bit-exact defaults; and the
same with the fast settings (KTPLACE_B200_PCG_FORM=3: the library's default
solve, KTPLACE_B200_HOST_CSR=0: no CSR copy back to the host). Prints one
JSON line: wall seconds and final HPWL per run, and whether each GPU run's
placement is bit-identical to the CPU run's."""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)

CHILD = r"""
import json, os, sys, time, resource
import numpy as np
sys.path.insert(0, sys.argv[1])
try:
    resource.setrlimit(resource.RLIMIT_STACK, (resource.RLIM_INFINITY, resource.RLIM_INFINITY))
except (ValueError, OSError):
    pass
import oracle
from ktplace_b200 import netlist, synth
variant, cells, threads, out = sys.argv[2], int(sys.argv[3]), int(sys.argv[4]), sys.argv[5]
spec = synth.spec_adaptec1_like(seed=1) if cells == 211000 else synth.SynthSpec(
    num_movable=cells, num_nets=int(cells * 1.05), num_pads=1000, num_rows=int(890 * (cells / 211000) ** 0.5),
    utilization=0.6, num_macros=int(550 * cells / 211000), seed=1, name="flow")
nl = netlist.flatten(synth.generate(spec))
oracle.set_ref_threads(threads, variant)
d = oracle.RefDesign.from_netlist(nl, variant)
t0 = time.perf_counter()
x, y = d.run_simpl()
t = time.perf_counter() - t0
np.save(out, np.concatenate([x, y]))
print(json.dumps({"seconds": t, "hpwl": oracle.RefDesign.from_netlist(nl, "cpu").hpwl(x, y)}))
"""


def run(variant: str, env_extra: dict, cells: int, threads: int, out: str) -> dict:
    env = dict(os.environ, **env_extra)
    r = subprocess.run([sys.executable, "-c", CHILD, ROOT, variant, str(cells), str(threads), out],
                       capture_output=True, text=True, env=env, timeout=3600)
    if r.returncode != 0:
        raise RuntimeError(r.stderr[-3000:])
    return json.loads(r.stdout.strip().splitlines()[-1])


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--cells", type=int, default=211000)
    ap.add_argument("--threads", type=int, default=os.cpu_count() or 1)
    ap.add_argument("--tmp", default=os.path.join(ROOT, "oracle", "_ref"))
    args = ap.parse_args(argv)
    os.makedirs(args.tmp, exist_ok=True)
    res = {"cells": args.cells, "threads": args.threads}
    runs = (("cpu", "cpu", {}),
            ("gpu_dropins_exact", "gpu", {}),
            ("gpu_dropins_fast", "gpu", {"KTPLACE_B200_PCG_FORM": "3",
                                          "KTPLACE_B200_HOST_CSR": "0"}))
    place = {}
    for name, variant, env in runs:
        out = os.path.join(args.tmp, f"flow_{name}.npy")
        res[name] = run(variant, env, args.cells, args.threads, out)
        place[name] = np.load(out)
    for name in ("gpu_dropins_exact", "gpu_dropins_fast"):
        res[name]["bit_identical_to_cpu"] = bool(np.array_equal(place[name], place["cpu"]))
        res[name]["hpwl_rel_vs_cpu"] = (res[name]["hpwl"] - res["cpu"]["hpwl"]) / res["cpu"]["hpwl"]
        res[name]["speedup_vs_cpu"] = res["cpu"]["seconds"] / res[name]["seconds"]
    print(json.dumps(res))
    return 0


if __name__ == "__main__":
    sys.exit(main())
