"""Benchmark of the SimPL quadratic-solve hot path on B200.

One step = one SimPL global iteration of the path on a 211k-cell synthetic
netlist shaped like ISPD-2005 adaptec1 (211,000 movable cells, 221,000 nets,
550 macros, 1,000 pads, 890 rows):
  B2B assembly of the x and y systems (alpha 0.2, anchors given),
  FP64 Jacobi-PCG of both systems from the warm start to rtol 1e-6,
  HPWL of the solution, and its 512x512 density map + scaled overflow.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

`value` is device time per step with inputs resident in HBM (CUDA events on
the launching stream, L2 flushed between steps). `e2e` runs the same step
through the C ABI in host-pointer mode from pinned host buffers, copies
included. `--impl reference` times the reference's own CPU code (compiled
from its sources into oracle/_ref) on the same workload with all host cores.
With N > 1 (torchrun), every rank solves its own netlist (weak scaling, no
data-path collective); timings are the max over ranks.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "GP CG solve ms/iter @210k cells: learned+FP32 PCG vs plain FP64 PCG, equal HPWL"
UNIT = "ms/iter"
ALPHA = 0.2
TOL = 1e-6
MAX_ITER = 100000
GRID = 512
MIXED_INNER_TOL = 1e-3
WORKLOAD = ("simpl-global-iteration on synth211k (adaptec1-shaped): B2B build x+y (alpha 0.2), "
            "FP64 Jacobi-PCG x+y warm-start to rtol 1e-6, HPWL, 512x512 density+overflow")
# The reference's own results for this workload (its CPU code, the --impl
# reference arm: HPWL and scaled overflow of the step's solution); the GPU
# arm's step is checked against them: HPWL within 1e-6 relative (the solve's
# summation order differs, solutions agree to about 1e-9), overflow within
# 1e-4 (a cell centre may land in a neighbouring bin).
REFERENCE_RESULT = {"hpwl": 322413208.70273274, "overflow": 0.46628111185456594}


def config_of(nl) -> dict:
    """The workload's config, printed identically by both arms."""
    return {"workload": WORKLOAD, "cells": nl.num_movable, "nets": nl.num_nets,
            "pins": nl.num_pins, "grid": GRID}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=60)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-sample-steps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batch", action="store_true",
                    help="skip the batched-solve leg (64 netlists, 128 systems)")
    ap.add_argument("--profile-batch", action="store_true",
                    help="run the batched-solve workload once for an ncu capture")
    ap.add_argument("--profile-batch-full", action="store_true",
                    help="the 64-netlist batched solve once, with the whole-GPU threshold and "
                         "shape the autotuners pick on B200 (44,725 rows; 4 x 1024 clusters), "
                         "for an ncu launch list")
    ap.add_argument("--profile-pcg", type=int, default=0, metavar="CELLS",
                    help="only one B2B build and FP64 solve of a synthetic design with CELLS "
                         "movable cells (scaled from the 211k design), timed, with its "
                         "algorithmic bytes per second (the PCG capture workload past L2)")
    ap.add_argument("--profile-spmv", type=int, default=0, metavar="CELLS",
                    help="only the standalone SpMV (ktg_spmv) on the scaled design of "
                         "--profile-pcg, timed, with its algorithmic bytes per second (the "
                         "SpMV capture workload past L2)")
    ap.add_argument("--config4", action="store_true",
                    help="only the solve comparison (FP64, FP32 with Jacobi / learned / "
                         "aggregation) on the 2.2M-cell design; prints one JSON line")
    ap.add_argument("--profile-lal", action="store_true",
                    help="run only the look-ahead legalization of the step's solved positions "
                         "twice (the legalizer's capture workload)")
    ap.add_argument("--profile-agg", action="store_true",
                    help="build the 211k systems twice, each followed by a mixed solve with "
                         "the aggregation preconditioner (set-up included), for ncu captures")
    ap.add_argument("--simpl-report", type=int, default=0, metavar="ITERS",
                    help="only the mixed-precision study on the systems of ITERS SimPL global "
                         "iterations of the 211k design (prints one JSON line)")
    ap.add_argument("--coarse-weights", default=None, metavar="NPY",
                    help="weights of the learned coarse vector for the SimPL study (default: "
                         "the committed ktplace_b200/weights/learned_coarse.npy)")
    ap.add_argument("--no-simpl-report", action="store_true",
                    help="skip the 30-iteration SimPL study in the default run")
    ap.add_argument("--profile-dense", action="store_true",
                    help="only the learned network's forward pass (ktg_learned_prepare: "
                         "features, the 3-layer message-passing trunk, the head) on the 211k "
                         "design with each dense-layer engine (tcgen05, mma.sync, FP32 cores); "
                         "prints one JSON line")
    ap.add_argument("--profile-once", action="store_true",
                    help="run the workload once (build, FP64 and mixed solves, HPWL, "
                         "density) for an ncu capture; prints no bench line")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def make_workload(seed: int):
    from ktplace_b200 import synth, netlist
    raw = synth.generate(synth.spec_adaptec1_like(seed))
    nl = netlist.flatten(raw)
    x, y = synth.seed_positions(raw, nl.num_movable, 100 + seed)
    ax, ay = synth.seed_positions(raw, nl.num_movable, 200 + seed)
    return raw, nl, x, y, ax, ay


def cpu_model() -> str:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


# ---- CPU: the reference's own code --------------------------------------------

def reference_steps(nl, x, y, ax, ay, steps: int, threads: int):
    """Runs `steps` SimPL iterations of the path with the reference's code;
    returns per-step seconds and the last step's results."""
    import oracle
    used = oracle.set_ref_threads(threads)
    ref = oracle.RefDesign.from_netlist(nl)
    ref.grid(GRID, 1.0)
    out = []
    res = None
    for _ in range(steps):
        t0 = time.perf_counter()
        ref.build_b2b(x, y, ALPHA, ax, ay)
        r = ref.solve(x, y, TOL, MAX_ITER)
        h = ref.hpwl(r["x"], r["y"])
        occ, ov = ref.occupancy_map(r["x"], r["y"], GRID * GRID)
        out.append(time.perf_counter() - t0)
        res = dict(iters=r["iters"], hpwl=h, overflow=ov)
    return out, res, used


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    import oracle
    if not oracle.ref_available():
        print(json.dumps({"impl": "reference",
                          "unavailable": "oracle/_ref/libktref.so was not built"}))
        return 0
    raw, nl, x, y, ax, ay = make_workload(1)
    threads = os.cpu_count() or 1
    reference_steps(nl, x, y, ax, ay, max(1, min(args.warmup, 1)), threads)
    times, res, used = reference_steps(nl, x, y, ax, ay, args.steps, threads)
    ms = 1000.0 * statistics.mean(times)
    line = {
        "impl": "reference", "metric": METRIC, "value": ms, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded generator, adaptec1 shape)",
        "config": config_of(nl),
        "workload_detail": {"cg_iters": res["iters"]},
        "cpu_baseline": {"value": ms, "unit": UNIT, "cores": used, "kind": "reference",
                         "sample": f"{args.steps} full steps on {cpu_model()}"},
        "e2e": {"value": ms, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "result": {"hpwl": res["hpwl"], "overflow": res["overflow"]},
    }
    print(json.dumps(line))
    return 0


# ---- GPU ------------------------------------------------------------------------

class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        import tempfile
        self.path = os.path.join(tempfile.mkdtemp(prefix="ktg_clocks_"), f"rank{index}.csv")

    def start(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=self.fh, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.fh.close()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [t.strip() for t in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax),
                "samples": len(sm), "reasons": sorted(reasons)}


def pcg_bytes(n: int, m: int, iters: int) -> float:
    """Algorithmic bytes of one axis's PCG: start pass + iters iterations.
    Iteration: val f64 + col i32 per entry, row_ptr, 14 n-vector passes (SpMV
    reads diag and p and writes Ap; update reads x, p, r, Ap, diag and writes
    x, r, z; direction reads z, p and writes p). Start: one SpMV on x plus
    reading diag, x, rhs and writing r, z, p."""
    it = 12.0 * m + 4.0 * (n + 1) + 8.0 * n * 14
    start = 12.0 * m + 4.0 * (n + 1) + 8.0 * n * 6
    return start + iters * it


def spmv_bytes(n: int, m: int) -> float:
    """Algorithmic bytes of one A v: the CSR (4 B column + 8 B value per
    entry, 4 B per row pointer), one 8-byte gather of v per entry, and v, diag
    and the result per row."""
    return 12.0 * m + 4.0 * (n + 1) + 8.0 * m + 24.0 * n


# DRAM bytes (read + write) per launch of the dominant kernel on this
# workload, from an ncu capture of bench.py --profile-once (dram__bytes_read.sum +
# dram__bytes_write.sum of the k_pcg launch).
NCU_TRAFFIC_BYTES = {"k_pcg": 100.221184e6 + 14.856192e6}


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def run_ours(args):
    import torch
    rank, world, local = dist_env()
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = torch.device(f"cuda:{local}")
    torch.cuda.set_device(dev)
    from ktplace_b200.gpu import Context
    from ktplace_b200 import grid as kgrid
    from ktplace_b200._lib import SolveInfo

    raw, nl, x, y, ax, ay = make_workload(1 + rank)
    fx, fy = nl.floors()
    bg = kgrid.build_grid(nl, GRID, 1.0)
    ctx = Context(local)
    ctx.upload_netlist(nl)
    ctx.set_grid(bg)
    stream = torch.cuda.Stream(device=dev)
    ctx.set_stream(stream.cuda_stream)
    n = nl.num_movable
    with torch.cuda.stream(stream):
        dx = torch.tensor(x, device=dev)
        dy = torch.tensor(y, device=dev)
        dax = torch.tensor(ax, device=dev)
        day = torch.tensor(ay, device=dev)
        wx = torch.empty_like(dx)
        wy = torch.empty_like(dy)
        info = torch.zeros(ctypes.sizeof(SolveInfo), dtype=torch.uint8, device=dev)
        scal = torch.zeros(4, dtype=torch.float64, device=dev)
        occ = torch.zeros(GRID * GRID, dtype=torch.float64, device=dev)
        flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MiB > L2

    ev_solve = [torch.cuda.Event(enable_timing=True) for _ in range(2)]

    def step(timed_solve=None):
        ctx.build_b2b_dev(dx, dy, ALPHA, dax, day, fx, fy)
        wx.copy_(dx)
        wy.copy_(dy)
        if timed_solve is not None:
            timed_solve[0].record(stream)
        ctx.solve_dev(wx, wy, TOL, MAX_ITER, info)
        if timed_solve is not None:
            timed_solve[1].record(stream)
        ctx.hpwl_dev(wx, wy, scal[0:1])
        ctx.occupancy_dev(wx, wy, occ, scal[1:2])

    with torch.cuda.stream(stream):
        for _ in range(max(args.warmup, 3)):
            step()
    torch.cuda.synchronize(dev)

    # ---- timed: device-resident inputs ------------------------------------
    clocks = ClockSampler(local)
    clocks.start()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    s_starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    s_ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    launches0 = ctx.launches
    if dist:
        dist.barrier()
    torch.cuda.synchronize(dev)
    with torch.cuda.stream(stream):
        for k in range(args.steps):
            flush.zero_()
            starts[k].record(stream)
            step((s_starts[k], s_ends[k]))
            ends[k].record(stream)
    torch.cuda.synchronize(dev)
    if dist:
        dist.barrier()
    launches = ctx.launches - launches0
    clk = clocks.stop()
    step_ms = [starts[k].elapsed_time(ends[k]) for k in range(args.steps)]
    solve_ms = [s_starts[k].elapsed_time(s_ends[k]) for k in range(args.steps)]
    total_ms = float(sum(step_ms))
    inf = SolveInfo.from_buffer_copy(bytes(info.cpu().numpy()))
    result = {"hpwl": float(scal[0].item()), "overflow": float(scal[1].item())}
    hrel = (result["hpwl"] - REFERENCE_RESULT["hpwl"]) / REFERENCE_RESULT["hpwl"]
    oabs = result["overflow"] - REFERENCE_RESULT["overflow"]
    result_check = {"hpwl_rel": hrel, "overflow_abs": oabs,
                    "ok": bool(abs(hrel) <= 1e-6 and abs(oabs) <= 1e-4) if rank == 0 and
                    nl.num_movable == 211000 else None}
    sx_n, sx_m = ctx.system_info(0)
    _, sy_m = ctx.system_info(1)

    variants = solve_variants(torch, dev, stream, ctx, dx, dy, dax, day, fx, fy, wx, wy, info, scal,
                              flush, max(args.steps // 2, 3))
    learned_step = learned_step_leg(torch, dev, stream, ctx, x, y, ax, ay, dx, dy, dax, day, fx, fy,
                                    wx, wy, scal, occ, flush, max(args.steps // 2, 3),
                                    result["hpwl"])

    # ---- e2e: host buffers through the C ABI, copies included --------------
    pinned = [torch.tensor(a).pin_memory() for a in (x, y, ax, ay, x, y)]
    hx, hy, hax, hay, px, py = (t.numpy() for t in pinned)
    e2e_ms = []
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    for k in range(max(1, args.steps // 2) + 1):
        px[...] = hx  # fresh warm start for every step, outside the timed region
        py[...] = hy
        with torch.cuda.stream(stream):
            flush.zero_()
        torch.cuda.synchronize(dev)
        e0.record(stream)
        ctx.build_b2b(hx, hy, ALPHA, hax, hay, fx, fy)
        ctx.solve(px, py, TOL, MAX_ITER, inplace=True)
        ctx.hpwl(px, py)
        ctx.occupancy(px, py, want_map=True)
        e1.record(stream)
        e1.synchronize()
        if k > 0:
            e2e_ms.append(e0.elapsed_time(e1))
    h2d = 8 * n * (4 + 2 + 2 + 2)
    d2h = 8 * n * 2 + 8 * GRID * GRID + 8 * 3 + ctypes.sizeof(SolveInfo)

    kw2_line = None
    if world == 1:
        kw2_line = kraftwerk2_leg(torch, dev, stream, raw, max(3, args.steps // 10),
                                  cpu=not args.no_cpu_baseline)

    bs_line = None
    if world == 1:
        bs_line = bookshelf_leg(raw, cpu=not args.no_cpu_baseline)

    lal_line = None
    if world == 1:
        lal_line = lal_leg(torch, dev, stream, nl, wx.cpu().numpy(), wy.cpu().numpy(),
                           max(3, args.steps // 10), cpu=not args.no_cpu_baseline)

    simpl_line = None
    if world == 1 and not args.no_simpl_report:
        coarse_net = load_coarse_network(dev)
        simpl_line = simpl_report(torch, dev, stream, nl, x, y, 30, learned=coarse_net)
        if coarse_net is not None:
            coarse_net.close()

    batch_line = None
    if not args.no_batch:  # every rank takes the same steps (barriers, the max reduction)
        batch_line = run_batch_leg(torch, dev, stream, max(3, args.steps // 10), rank, world,
                                   dist)

    # ---- max over ranks --------------------------------------------------------
    vals = torch.tensor([total_ms, float(np.mean(e2e_ms)) * args.steps], dtype=torch.float64,
                        device=dev)
    if dist:
        dist.all_reduce(vals, op=dist.ReduceOp.MAX)
    total_max, e2e_total_max = float(vals[0]), float(vals[1])
    value = total_max / (args.steps * world)
    e2e_value = e2e_total_max / (args.steps * world)

    line = None
    if rank == 0:
        peak, peak_kind = measured_peak()
        solve_med = statistics.median(solve_ms)
        byts = pcg_bytes(sx_n, sx_m, inf.iters_x) + pcg_bytes(sx_n, sy_m, inf.iters_y)
        achieved = byts / (solve_med * 1e-3) / 1e9
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            import oracle
            if oracle.ref_available():
                threads = os.cpu_count() or 1
                t, res, used = reference_steps(nl, x, y, ax, ay, args.cpu_sample_steps, threads)
                cpu = {"value": 1000.0 * statistics.mean(t), "unit": UNIT, "cores": used,
                       "kind": "reference",
                       "sample": f"{args.cpu_sample_steps} full steps of the same workload "
                                 f"(oracle/_ref, OpenMP on {cpu_model()})",
                       "cg_iters": res["iters"]}
                t1, _, used1 = reference_steps(nl, x, y, ax, ay, 1, 1)
                cpu["single_thread"] = {"value": 1000.0 * t1[0], "unit": UNIT, "cores": used1,
                                        "sample": "1 full step of the same workload, 1 thread"}
                oracle.set_ref_threads(threads)
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": value * world,
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded generator, adaptec1 shape; 256 MiB L2 flush between steps)",
            "config": config_of(nl),
            "workload_detail": {"nnz_x": sx_m, "nnz_y": sy_m, "cg_iters": int(inf.iters),
                                "l2": "flushed between steps",
                                "parallelism": f"replicas x{world} (independent netlists)"},
            "result": result,
            "result_vs_reference": result_check,
            "breakdown": {"solve_ms": solve_med, "solve_ms_per_cg_iter": solve_med / inf.iters,
                          "other_ms": statistics.median(step_ms) - solve_med},
            "solve_variants": variants,
            "learned_step": learned_step,
            "roofline": {"kernel": "k_pcg<1, 32, 0, 1> (persistent cooperative PCG, x+y, "
                                   "warp-tile SpMV, two grid barriers per iteration)",
                         "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind,
                         "traffic": NCU_TRAFFIC_BYTES["k_pcg"], "algorithmic_bytes": byts,
                         "note": "working set is L2-resident: traffic << algorithmic bytes",
                         "limiter": "L1TEX data pipe: 57% of peak over the whole solve in the ncu "
                                    "capture (random 8-byte gathers, one LSU wavefront each); "
                                    "L2 39%, DRAM 0.2% (ncu of bench.py --profile-once)"},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "gpu_launches": launches,
            "simpl_report": simpl_line,
            "batch": batch_line,
            "kraftwerk2": kw2_line,
            "bookshelf": bs_line,
            "lal": lal_line,
            "clocks": clk,
        }
        print(json.dumps(line))
    ctx.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def solve_variants(torch, dev, stream, ctx, dx, dy, dax, day, fx, fy, wx, wy, info, scal, flush,
                   reps: int) -> dict:
    """The x+y solve of the same systems to the same true residual (rtol
    1e-6) by each method, per-system set-up included (aggregation build,
    network inference), B2B build excluded: plain FP64 Jacobi-PCG (the
    drop-in), and FP32 PCG inside FP64 refinement with Jacobi, the learned
    preconditioner and the aggregation preconditioner. Reports the median
    device ms, iterations and the HPWL of the solution relative to FP64.
    fp32_learned is the two-level aggregation solve with the learned coarse
    vector (the network's per-system head runs inside the timed region; its
    per-netlist embedding is computed once, in the untimed first repetition,
    like the netlist upload); fp32_learned_spai the learned sparse
    approximate inverse on A's pattern."""
    from ktplace_b200._lib import MixedInfo, SolveInfo
    from ktplace_b200.learned import Learned
    coarse_net = load_coarse_network(dev)
    minfo = torch.zeros(ctypes.sizeof(MixedInfo), dtype=torch.uint8, device=dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    weights = os.path.join(ROOT, "ktplace_b200", "weights", "learned_precond.npy")
    learned = None
    if os.path.exists(weights):
        learned = Learned(dev.index or 0)
        learned.load(weights)
    out = {}
    hpwl_ref = None
    for name, pre, coarse in (("fp64_jacobi", None, 0), ("fp32_jacobi", 0, 0),
                              ("fp32_learned_spai", 1, 0), ("fp32_aggregation", 2, 0),
                              ("fp32_aggregation_coarse_const", 2, 1),
                              ("fp32_aggregation_coarse_coupling", 2, 2),
                              ("fp32_learned", 2, 3)):
        if (pre == 1 and learned is None) or (coarse == 3 and coarse_net is None):
            continue
        if pre is not None:
            ctx.set_option("precond", pre)
            ctx.set_option("coarse", coarse)
        ms = []
        host_ms = 0.0
        for k in range(reps + 1):
            with torch.cuda.stream(stream):
                ctx.build_b2b_dev(dx, dy, ALPHA, dax, day, fx, fy)
                wx.copy_(dx)
                wy.copy_(dy)
                flush.zero_()
            torch.cuda.synchronize(dev)
            host_ms = 0.0
            if pre == 1:
                t0 = time.perf_counter()
                learned.prepare(ctx)  # synchronous: network inference for x and y
                host_ms = 1000.0 * (time.perf_counter() - t0)
            with torch.cuda.stream(stream):
                e0.record(stream)
                if coarse == 3:
                    coarse_net.prepare_coarse_dev(ctx)  # enqueued on ctx's stream
                if pre is None:
                    ctx.solve_dev(wx, wy, TOL, MAX_ITER, info)
                else:
                    ctx.solve_mixed_dev(wx, wy, TOL, MIXED_INNER_TOL, MAX_ITER, 50, minfo)
                e1.record(stream)
                ctx.hpwl_dev(wx, wy, scal[2:3])
            e1.synchronize()
            if k > 0:
                ms.append(e0.elapsed_time(e1) + host_ms)
        h = float(scal[2].item())
        if pre is None:
            inf = SolveInfo.from_buffer_copy(bytes(info.cpu().numpy()))
            hpwl_ref = h
            row = {"ms": statistics.median(ms), "iters": [int(inf.iters_x), int(inf.iters_y)],
                   "true_resid": [inf.resid_x, inf.resid_y]}
        else:
            mi = MixedInfo.from_buffer_copy(bytes(minfo.cpu().numpy()))
            row = {"ms": statistics.median(ms), "iters": [int(mi.inner_x), int(mi.inner_y)],
                   "outer_rounds": [int(mi.outer_x), int(mi.outer_y)],
                   "true_resid": [mi.resid_x, mi.resid_y],
                   "fp64_fallback_iters": [int(mi.fp64_iters_x), int(mi.fp64_iters_y)]}
            if pre == 1:
                row["inference_ms_host_timed"] = host_ms
        row["hpwl_rel_vs_fp64"] = (h - hpwl_ref) / hpwl_ref if hpwl_ref else 0.0
        out[name] = row
    ctx.set_option("precond", 0)
    ctx.set_option("coarse", 0)
    if learned is not None:
        learned.close()
    if coarse_net is not None:
        coarse_net.close()
    base = out["fp64_jacobi"]["ms"]
    for row in out.values():
        row["speedup_vs_fp64"] = base / row["ms"]
    return out


def learned_step_leg(torch, dev, stream, ctx, x, y, ax, ay, dx, dy, dax, day, fx, fy, wx, wy,
                     scal, occ, flush, steps: int, hpwl_fp64: float) -> dict:
    """The bench step with the learned+FP32 solve in place of FP64 PCG: B2B
    build, the two-level aggregation-preconditioned FP32 PCG in FP64
    refinement with the learned coarse vector (the network's per-system head
    inside the timed region, its per-netlist trunk once before it, like the
    netlist upload) to the same true residual, HPWL, 512x512 density.
    `ms`: device-resident inputs, CUDA events, L2 flushed between steps;
    `e2e_ms`: the same calls through the C ABI from pinned host buffers
    (copies included)."""
    from ktplace_b200._lib import MixedInfo
    net = load_coarse_network(dev)
    if net is None:
        return None
    minfo = torch.zeros(ctypes.sizeof(MixedInfo), dtype=torch.uint8, device=dev)
    ctx.set_option("precond", 2)
    ctx.set_option("coarse", 3)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    ms, e2e = [], []
    try:
        for k in range(steps + 1):
            with torch.cuda.stream(stream):
                flush.zero_()
                e0.record(stream)
                ctx.build_b2b_dev(dx, dy, ALPHA, dax, day, fx, fy)
                wx.copy_(dx)
                wy.copy_(dy)
                net.prepare_coarse_dev(ctx)
                ctx.solve_mixed_dev(wx, wy, TOL, MIXED_INNER_TOL, MAX_ITER, 50, minfo)
                ctx.hpwl_dev(wx, wy, scal[2:3])
                ctx.occupancy_dev(wx, wy, occ, scal[3:4])
                e1.record(stream)
            e1.synchronize()
            if k > 0:
                ms.append(e0.elapsed_time(e1))
        hpwl = float(scal[2].item())
        overflow = float(scal[3].item())
        mi = MixedInfo.from_buffer_copy(bytes(minfo.cpu().numpy()))
        pinned = [torch.tensor(a).pin_memory() for a in (x, y, ax, ay, x, y)]
        hx, hy, hax, hay, px, py = (t.numpy() for t in pinned)
        for k in range(steps + 1):
            px[...] = hx
            py[...] = hy
            with torch.cuda.stream(stream):
                flush.zero_()
            torch.cuda.synchronize(dev)
            e0.record(stream)
            ctx.build_b2b(hx, hy, ALPHA, hax, hay, fx, fy)
            net.prepare_coarse(ctx)
            ctx.solve_mixed(px, py, TOL, MIXED_INNER_TOL, inplace=True)
            ctx.hpwl(px, py)
            ctx.occupancy(px, py, want_map=True)
            e1.record(stream)
            e1.synchronize()
            if k > 0:
                e2e.append(e0.elapsed_time(e1))
    finally:
        ctx.set_option("precond", 0)
        ctx.set_option("coarse", 0)
        net.close()
    return {"workload": "the bench step with the learned-coarse-vector two-level aggregation FP32 "
                        "PCG in FP64 refinement (to true rtol 1e-6) in place of FP64 PCG",
            "ms": statistics.median(ms), "e2e_ms": statistics.median(e2e),
            "inner_iters": [int(mi.inner_x), int(mi.inner_y)],
            "true_resid": [mi.resid_x, mi.resid_y],
            "hpwl": hpwl, "overflow": overflow,
            "hpwl_rel_vs_fp64_step": (hpwl - hpwl_fp64) / hpwl_fp64}


# (name, precond, coarse vector, agg_reuse): agg_reuse > 0 keeps an
# aggregate structure across the run's builds, so that variant solves on a
# context of its own whose aggregation history is only its own
SIMPL_VARIANTS = (("fp64_jacobi", None, 0, 0), ("fp32_jacobi", 0, 0, 0),
                  ("fp32_aggregation", 2, 0, 0), ("fp32_aggregation_coarse_const", 2, 1, 0),
                  ("fp32_aggregation_coarse_coupling", 2, 2, 0),
                  ("fp32_learned", 2, 3, 0),
                  ("fp32_aggregation_reuse", 2, 0, 4),
                  ("fp32_aggregation_coarse_const_reuse", 2, 1, 4),
                  ("fp32_aggregation_coarse_coupling_reuse", 2, 2, 4),
                  ("fp32_learned_reuse", 2, 3, 4))


def simpl_report(torch, dev, stream, nl, x0, y0, iters: int = 30, init_rounds: int = 5,
                 variants=SIMPL_VARIANTS, learned=None) -> dict:
    """The mixed-precision study on real SimPL systems: SimPL's B2B initial
    rounds, then `iters` global iterations (simpl_placer.cc:463-539) on the
    GPU path with the anchors at the look-ahead-legalized positions (ktg_lal)
    and the anchor weight rising linearly from 0.01 to 1.0. Every iteration's
    x+y systems are solved by each variant from the same warm start to the
    same true residual (rtol 1e-6): FP64 Jacobi-PCG (the drop-in), and FP32
    PCG in FP64 refinement with Jacobi, aggregation block Jacobi, and
    aggregation with a coarse vector (constant, coupling share, learned).
    Per variant and iteration: device ms (CUDA events, L2 flushed, set-up
    such as the aggregates included, the B2B build excluded), iterations,
    the true FP64 relative residual, the solution's difference from the FP64
    solve and its HPWL relative to FP64's. The loop continues from the FP64
    solution, so every variant sees the same systems."""
    from ktplace_b200 import grid as kgrid
    from ktplace_b200 import simpl
    from ktplace_b200._lib import MixedInfo, SolveInfo
    from ktplace_b200.gpu import Context
    def new_ctx():
        c = Context(dev.index or 0)
        c.set_stream(stream.cuda_stream)
        c.upload_netlist(nl)
        return c

    ctx = new_ctx()
    # every agg_reuse variant keeps its own context: the reused structure is
    # the one its own previous builds left
    vctxs = {name: (new_ctx() if reuse else ctx) for name, _, _, reuse in variants}
    g = kgrid.build_grid(nl, kgrid.default_bins_per_axis(nl.num_movable), 1.0)
    loop = simpl.GlobalLoop(ctx, nl, g, kgrid.build_free_space(nl), tol=TOL, max_iter=MAX_ITER)
    with torch.cuda.stream(stream):
        dx = torch.zeros(nl.num_movable, dtype=torch.float64, device=dev)
        dy = torch.zeros_like(dx)
        info = torch.zeros(ctypes.sizeof(SolveInfo), dtype=torch.uint8, device=dev)
        minfo = torch.zeros(ctypes.sizeof(MixedInfo), dtype=torch.uint8, device=dev)
        hp = torch.zeros(1, dtype=torch.float64, device=dev)
        flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    x, y = loop.initial_rounds(x0, y0, init_rounds)
    rows = []
    fx, fy = loop.fx, loop.fy
    # untimed: every solver's buffers allocated once, and the learned
    # network's per-netlist trunk embedding computed (it depends on the
    # topology only, so it belongs with the netlist upload)
    for vctx in {id(c): c for c in vctxs.values()}.values():
        vctx.build_b2b(x, y, 0.0, None, None, fx, fy)
        if learned is not None:
            learned.prepare_coarse(vctx)
        for pre, coarse in ((0, 0), (2, 2)):
            vctx.set_option("precond", pre)
            vctx.set_option("coarse", coarse)
            vctx.solve_mixed(x, y, TOL, MIXED_INNER_TOL)
        vctx.set_option("precond", 0)
        vctx.set_option("coarse", 0)
        vctx.solve(x, y, TOL, MAX_ITER)
    for st in loop.iterations(x, y, iters):
        row = {"it": st.it, "alpha": st.alpha}
        ref = None
        for name, pre, coarse, reuse in variants:
            if coarse == 3 and learned is None:
                continue
            vctx = vctxs[name]
            vctx.build_b2b(st.x, st.y, st.alpha, st.ux, st.uy, fx, fy)  # fresh systems
            with torch.cuda.stream(stream):
                dx.copy_(torch.from_numpy(st.x))
                dy.copy_(torch.from_numpy(st.y))
                flush.zero_()
            torch.cuda.synchronize(dev)
            if pre is not None:
                vctx.set_option("precond", pre)
                vctx.set_option("coarse", coarse)
                # the run's first global iteration builds its aggregates fresh
                vctx.set_option("agg_reuse", reuse if st.it > 0 else 0)
            with torch.cuda.stream(stream):
                e0.record(stream)
                if coarse == 3:
                    learned.prepare_coarse_dev(vctx)
                if pre is None:
                    vctx.solve_dev(dx, dy, TOL, MAX_ITER, info)
                else:
                    vctx.solve_mixed_dev(dx, dy, TOL, MIXED_INNER_TOL, MAX_ITER, 50, minfo)
                e1.record(stream)
                vctx.hpwl_dev(dx, dy, hp)
            e1.synchronize()
            ms = e0.elapsed_time(e1)
            vctx.set_option("precond", 0)
            vctx.set_option("coarse", 0)
            sol = np.concatenate([dx.cpu().numpy(), dy.cpu().numpy()])
            h = float(hp.item())
            if pre is None:
                inf = SolveInfo.from_buffer_copy(bytes(info.cpu().numpy()))
                ref = (sol, h)
                row[name] = {"ms": ms, "iters": [int(inf.iters_x), int(inf.iters_y)],
                             "resid": [inf.resid_x, inf.resid_y], "hpwl": h}
            else:
                mi = MixedInfo.from_buffer_copy(bytes(minfo.cpu().numpy()))
                row[name] = {"ms": ms, "iters": [int(mi.inner_x), int(mi.inner_y)],
                             "outer": [int(mi.outer_x), int(mi.outer_y)],
                             "true_resid": [mi.resid_x, mi.resid_y],
                             "fp64_fallback_iters": [int(mi.fp64_iters_x), int(mi.fp64_iters_y)],
                             "sol_rel_vs_fp64": float(np.linalg.norm(sol - ref[0]) /
                                                      np.linalg.norm(ref[0])),
                             "hpwl_rel_vs_fp64": (h - ref[1]) / ref[1]}
        rows.append(row)
    for c in {id(c): c for c in vctxs.values()}.values():
        c.close()
    names = [v[0] for v in variants if v[0] in rows[0]]
    summary = {}
    base = sum(r["fp64_jacobi"]["ms"] for r in rows)
    for nm in names:
        tot = sum(r[nm]["ms"] for r in rows)
        d = {"ms_per_iter": tot / len(rows), "speedup_vs_fp64": base / tot,
             "iters_mean": float(np.mean([sum(r[nm]["iters"]) / 2 for r in rows]))}
        if nm != "fp64_jacobi":
            d["max_true_resid"] = max(max(r[nm]["true_resid"]) for r in rows)
            d["max_abs_hpwl_rel_vs_fp64"] = max(abs(r[nm]["hpwl_rel_vs_fp64"]) for r in rows)
            d["max_sol_rel_vs_fp64"] = max(r[nm]["sol_rel_vs_fp64"] for r in rows)
        summary[nm] = d
    return {"workload": f"{iters} SimPL global iterations on synth211k after {init_rounds} B2B "
                        "initial rounds: anchors at ktg_lal positions, alpha 0.01 -> 1.0 "
                        "linear, x+y solved to rtol 1e-6 from the previous FP64 solution",
            "summary": summary, "iterations": rows}


def kraftwerk2_leg(torch, dev, stream, raw, reps: int, cpu: bool) -> dict:
    """Kraftwerk2's initial-placement step on the same 211k-cell netlist
    (Kraftwerk2Placer::Impl::placeInitially, kraftwerk2_placer.cc:422-453):
    buildSystem with rhs for x and y, diag floor 1e-12, CG to its default
    tolerance 1e-5 with at most 150 iterations, from the bench positions. GPU:
    ktg_build_b2b_kraftwerk2 + ktg_kraftwerk2_adjust + ktg_solve (CUDA events).
    Beside it, the reference's own buildSystem and solve (oracle/_ref) on the
    host cores, when the reference library is present."""
    from ktplace_b200 import netlist
    from ktplace_b200.gpu import Context
    from ktplace_b200._lib import SolveInfo
    nl = netlist.flatten(raw, kraftwerk2=True)
    n = nl.num_movable
    fx, fy = nl.floors()
    rng = np.random.default_rng(5)
    lx, ly, ux, uy = nl.die
    x0 = rng.uniform(lx, ux - nl.width)
    y0 = rng.uniform(ly, uy - nl.height)
    ctx = Context(dev.index or 0)
    ctx.upload_netlist(nl)
    ctx.set_stream(stream.cuda_stream)
    with torch.cuda.stream(stream):
        dx = torch.tensor(x0, device=dev)
        dy = torch.tensor(y0, device=dev)
        wx = torch.empty_like(dx)
        wy = torch.empty_like(dy)
        info = torch.zeros(ctypes.sizeof(SolveInfo), dtype=torch.uint8, device=dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    ms = []
    for k in range(reps + 1):
        with torch.cuda.stream(stream):
            wx.copy_(dx)
            wy.copy_(dy)
            e0.record(stream)
            ctx.build_kraftwerk2_dev(wx, wy, True, fx, fy)
            ctx.kraftwerk2_adjust_dev(None, None, None, 1e-12)
            ctx.solve_dev(wx, wy, 1e-5, 150, info)
            e1.record(stream)
        e1.synchronize()
        if k > 0:
            ms.append(e0.elapsed_time(e1))
    inf = SolveInfo.from_buffer_copy(bytes(info.cpu().numpy()))
    out = {"workload": "Kraftwerk2 initial-placement step on synth211k: buildSystem x+y with rhs, "
                       "diag floor 1e-12, Jacobi-PCG to 1e-5 (max 150)",
           "gpu_ms": statistics.median(ms), "iters": [int(inf.iters_x), int(inf.iters_y)]}
    ctx.close()
    if cpu:
        import oracle
        if oracle.ref_available():
            threads = os.cpu_count() or 1
            oracle.set_ref_threads(threads)
            ref = oracle.Kraftwerk2Ref(nl)
            t = []
            for k in range(2):
                t0 = time.perf_counter()
                for axis, p in ((0, x0), (1, y0)):
                    r = ref.build(x0, y0, axis == 0, True, fx, fy)
                    ref.set_diag_rhs(np.maximum(r["diag"], 1e-12), r["rhs"])
                    ref.solve(p, 1e-5, 150)
                t.append(1000.0 * (time.perf_counter() - t0))
            out["reference_cpu_ms"] = min(t)
            out["reference_cpu_cores"] = threads
            out["speedup_vs_reference"] = out["reference_cpu_ms"] / out["gpu_ms"]
    return out


def lal_leg(torch, dev, stream, nl, x0, y0, reps: int, cpu: bool) -> dict:
    """SimPL's look-ahead legalization (LookAheadLegalizer::legalize,
    simpl_lal.cc:43-123) of the bench step's solved positions on the 211k-cell
    netlist, SimPL's default grid (getDefaultBinsPerAxis) at density 1.0 and
    the default options (20 levels, 4 cells, stripe fraction 0.1). GPU:
    ktg_lal on device positions (host wall clock around the call, which ends
    synchronised) and through the host-pointer C ABI (copies included).
    Beside it, the reference's own legalizer (oracle/_ref) on all host cores,
    with a bit-identity check of the two results."""
    from ktplace_b200 import grid
    from ktplace_b200.gpu import Context
    bins = grid.default_bins_per_axis(nl.num_movable)
    g = grid.build_grid(nl, bins, 1.0)
    fs = grid.build_free_space(nl)
    ctx = Context(dev.index or 0)
    ctx.upload_netlist(nl)
    ctx.set_stream(stream.cuda_stream)
    ctx.set_grid(g)
    ctx.set_free_space(fs)
    with torch.cuda.stream(stream):
        bx = torch.tensor(x0, device=dev)
        by = torch.tensor(y0, device=dev)
        wx = torch.empty_like(bx)
        wy = torch.empty_like(by)
    ms, e2e = [], []
    for k in range(reps + 1):
        with torch.cuda.stream(stream):
            wx.copy_(bx)
            wy.copy_(by)
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        ctx.lal_dev(wx, wy)
        torch.cuda.synchronize(dev)
        t1 = time.perf_counter()
        if k > 0:
            ms.append(1000.0 * (t1 - t0))
    stats = ctx.lal_stats()
    for k in range(reps):
        t0 = time.perf_counter()
        gx, gy = ctx.lal(x0, y0)
        e2e.append(1000.0 * (time.perf_counter() - t0))
    out = {"workload": f"look-ahead legalization of the bench step's solved positions on "
                       f"synth211k, {bins}x{bins} bins, density 1.0, options 20/4/0.1",
           "gpu_ms": statistics.median(ms), "e2e_ms": statistics.median(e2e),
           "h2d_bytes": 16 * nl.num_movable, "d2h_bytes": 16 * nl.num_movable,
           "moved_fraction": float(np.mean((gx != x0) | (gy != y0))),
           "batches": int(stats["batches"]), "regions": int(stats["regions"]),
           "host_syncs": int(stats["syncs"])}
    ctx.close()
    if cpu:
        import oracle
        if oracle.ref_available():
            import resource
            try:  # the reference's recursion wants more than the default 8 MiB stack
                resource.setrlimit(resource.RLIMIT_STACK,
                                   (resource.RLIM_INFINITY, resource.RLIM_INFINITY))
            except (ValueError, OSError):
                pass
            threads = os.cpu_count() or 1
            oracle.set_ref_threads(threads)
            ref = oracle.RefDesign.from_netlist(nl)
            ref.grid(bins, 1.0)
            t = []
            for k in range(3):
                t0 = time.perf_counter()
                rx, ry = ref.lal(x0, y0)
                t.append(1000.0 * (time.perf_counter() - t0))
            out["reference_cpu_ms"] = min(t)
            out["reference_cpu_cores"] = threads
            out["bit_identical"] = bool(np.array_equal(rx, gx) and np.array_equal(ry, gy))
            out["speedup_vs_reference"] = out["reference_cpu_ms"] / out["gpu_ms"]
            out["e2e_speedup_vs_reference"] = out["reference_cpu_ms"] / out["e2e_ms"]
    return out


def bookshelf_leg(raw, cpu: bool) -> dict:
    """Load time of the 211k-cell workload written as a Bookshelf directory:
    ktg_bookshelf_read (read + flatten, all host threads) beside the
    reference's BookshelfInputAdapter + buildSimplDM (oracle/_ref, same
    threads; it needs more than the default 8 MiB of main-thread stack at this
    size, so the soft stack limit is raised first)."""
    import resource
    import tempfile
    from ktplace_b200 import bookshelf, synth
    threads = os.cpu_count() or 1
    out = {"workload": "Bookshelf read + SimPL flattening of synth211k (nodes/nets/wts/pl/scl)",
           "threads": threads}
    with tempfile.TemporaryDirectory() as tmp:
        d = os.path.join(tmp, raw.name)
        synth.write_bookshelf(raw, d)
        t = []
        for _ in range(3):
            t0 = time.perf_counter()
            nl = bookshelf.read(d, threads)
            t.append(1000.0 * (time.perf_counter() - t0))
        out["ms"] = statistics.median(t)
        out["phases_ms"] = nl.read_ms
        if cpu:
            import oracle
            if oracle.ref_available():
                try:
                    resource.setrlimit(resource.RLIMIT_STACK,
                                       (resource.RLIM_INFINITY, resource.RLIM_INFINITY))
                except (ValueError, OSError):
                    pass
                oracle.set_ref_threads(threads)
                t0 = time.perf_counter()
                ref = oracle.RefDesign.from_bookshelf(d)
                out["reference_ms"] = 1000.0 * (time.perf_counter() - t0)
                out["speedup_vs_reference"] = out["reference_ms"] / out["ms"]
                del ref
    return out


def batch_unit(k: int):
    """Netlist k of the batched-solve workload (log-uniform 5k-200k cells,
    mean degree 3.5, 65% density) with its own seeded positions and anchors:
    (netlist, x, y, anchor_x, anchor_y, alpha)."""
    from ktplace_b200 import synth, netlist
    raw = synth.generate(synth.spec_batch_member(k))
    nl = netlist.flatten(raw)
    x, y = synth.seed_positions(raw, nl.num_movable, 300 + k)
    ax, ay = synth.seed_positions(raw, nl.num_movable, 400 + k)
    return nl, x, y, ax, ay, ALPHA


def batch_workload(count: int = 64):
    """The batched-solve workload loaded into one Batch (x and y of every
    netlist); returns it with the number of rows per system."""
    from ktplace_b200.gpu import Context, Batch
    ctx = Context(0)
    batch = Batch(0)
    rows = []
    for k in range(count):
        nl, x, y, ax, ay, alpha = batch_unit(k)
        fx, fy = nl.floors()
        ctx.upload_netlist(nl)
        ctx.build_b2b(x, y, alpha, ax, ay, fx, fy)
        batch.add_from_context(ctx, x, y)
        rows += [nl.num_movable, nl.num_movable]
    ctx.close()
    return batch, rows


def run_batch_leg(torch, dev, stream, steps: int, rank: int = 0, world: int = 1, dist=None,
                  count: int = 64):
    """The batched solve of `count` netlists (2 systems each). Every rank
    builds and solves its LPT share (shard.ShardPlan over the netlists' row
    counts) as one autotuned Batch on its GPU; the step time is the max over
    ranks, and the host slices of the solutions are written by
    shard.run_share after the timed steps."""
    from ktplace_b200 import shard, synth
    cells = [synth.spec_batch_member(k).num_movable for k in range(count)]
    plan = shard.ShardPlan([2 * c for c in cells], [2 * c for c in cells], world)
    mine = plan.share(rank)
    solver = shard.BatchShardSolver(batch_unit, device=dev.index or 0, tol=TOL, max_iter=MAX_ITER,
                                    precision=1, inner_tol=MIXED_INNER_TOL,
                                    stream=stream.cuda_stream)
    if mine:
        solver.load(mine)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    times, lat, iters = [], [], []
    for k in range(steps + 3):
        if mine:
            solver.batch.reset_x()
        with torch.cuda.stream(stream):
            flush.zero_()
        torch.cuda.synchronize(dev)
        if dist:
            dist.barrier()
        e0.record(stream)
        if mine:
            solver.solve(reset=False)
        e1.record(stream)
        e1.synchronize()
        if k >= 3:
            times.append(e0.elapsed_time(e1))
            if mine:
                res = solver.batch.results()
                lat += [r["latency_ns"] / 1e6 for r in res]
                iters += [r["iters"] for r in res]
                bad = [r for r in res if r["status"] != 0 or r["resid"] > TOL]
                if bad:
                    raise RuntimeError(f"batched solve left {len(bad)} systems unconverged")
    ms = statistics.median(times)
    out = np.zeros(plan.total)
    shard.run_share(plan, rank, solver, out)  # host slices (untimed)
    t = torch.tensor([ms], dtype=torch.float64, device=dev)
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    shape, split, offload = solver.shape, solver.split, solver.offload
    solver.close()
    systems = 2 * count
    return {"workload": f"{count} synthetic netlists (log-uniform 5k-200k cells), x+y = "
                        f"{systems} systems, FP32 PCG in FP64 refinement to true rtol 1e-6; "
                        "the largest x/y pairs on the whole GPU (aggregation-preconditioned), "
                        "the rest in persistent cluster launches (size classes) replayed as "
                        "one graph",
            "systems": systems, "rows_total": int(plan.total), "ms_per_batch": ms_max,
            "systems_per_s": systems / (ms_max * 1e-3),
            "sharding": {"ranks": world, "units_per_rank": len(mine),
                         "rows_this_rank": int(sum(plan.sizes[u] for u in mine)),
                         "lpt_makespan_rows": plan.makespan(), "scaling": "strong"},
            "latency_ms_p50": float(np.percentile(lat, 50)) if lat else None,
            "latency_ms_p99": float(np.percentile(lat, 99)) if lat else None,
            "inner_iters_p50": float(np.percentile(iters, 50)) if iters else None,
            "autotuned_shape": {"cluster": shape[0], "threads": shape[1]} if shape else None,
            "size_split": split,
            "whole_gpu_pairs": offload}


def profile_once():
    """The capture workload of the 211k kernel profiles: one build, one FP64
    and one mixed solve, HPWL and the 512x512 density map."""
    from ktplace_b200.gpu import Context
    from ktplace_b200 import grid as kgrid
    raw, nl, x, y, ax, ay = make_workload(1)
    fx, fy = nl.floors()
    ctx = Context(0)
    ctx.upload_netlist(nl)
    ctx.set_grid(kgrid.build_grid(nl, GRID, 1.0))
    ctx.build_b2b(x, y, ALPHA, ax, ay, fx, fy)
    r = ctx.solve(x, y, TOL, MAX_ITER)
    m = ctx.solve_mixed(x, y, TOL, MIXED_INNER_TOL)
    h = ctx.hpwl(r["x"], r["y"])
    _, ov = ctx.occupancy(r["x"], r["y"])
    print(f"profile-once: {r['iters']} FP64 iterations, mixed inner {m['inner']}, "
          f"HPWL {h:.6e}, overflow {ov:.4f}")
    ctx.close()
    return 0


def profile_agg():
    """The capture workload of the aggregation profiles: three B2B builds of
    the 211k-cell workload, each followed by a mixed solve with the
    aggregation preconditioner and the coupling-share coarse vector; the
    first two rebuild the aggregates, the third (agg_reuse) keeps the
    second's structure and recomputes only the values."""
    from ktplace_b200.gpu import Context
    raw, nl, x, y, ax, ay = make_workload(1)
    fx, fy = nl.floors()
    ctx = Context(0)
    ctx.upload_netlist(nl)
    ctx.set_option("precond", 2)
    ctx.set_option("coarse", 2)
    for k in range(3):
        ctx.set_option("agg_reuse", 4 if k == 2 else 0)
        ctx.build_b2b(x, y, ALPHA, ax, ay, fx, fy)
        m = ctx.solve_mixed(x, y, TOL, MIXED_INNER_TOL)
        print(f"profile-agg: build {k}: inner {m['inner']}, outer {m['outer']}, "
              f"resid {m['resid']}")
    ctx.close()
    return 0


def profile_dense(reps: int = 5) -> int:
    """The learned network's forward pass on the 211k-cell workload's x and
    y systems with each dense-layer engine: tensor_cores 2 (tcgen05.mma, FP32
    accumulator in tensor memory), 1 (mma.sync) and 0 (FP32 CUDA cores).
    Times are host wall clock around ktg_learned_prepare (features, trunk and
    head for both axes; it synchronises its streams before returning), median
    of `reps` after one warm-up; the dense layers' FLOPs are 2 x rows x K x
    OUT summed over the trunk's layers and both axes."""
    import torch
    from ktplace_b200.gpu import Context
    from ktplace_b200.learned import Learned
    raw, nl, x, y, ax, ay = make_workload(1)
    fx, fy = nl.floors()
    ctx = Context(0)
    ctx.upload_netlist(nl)
    ctx.build_b2b(x, y, ALPHA, ax, ay, fx, fy)
    n, N = nl.num_movable, len(nl.net_start) - 1
    hid, proj = 64, 16
    flops = 2 * 2.0 * (n * 16 * hid + 3 * (N * hid * hid + n * 2 * hid * hid) + n * hid * proj)
    learned = Learned(0, seed=1)
    out = {"workload": "learned network forward (features, 3-layer trunk, head) on synth211k",
           "cells": n, "nets": N, "dense_gflop": flops / 1e9}
    for mode, name in ((2, "tcgen05"), (1, "mma_sync"), (0, "fp32_cores")):
        learned.set_option("tensor_cores", mode)
        learned.prepare(ctx)
        ts = []
        for _ in range(reps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            learned.prepare(ctx)
            ts.append((time.perf_counter() - t0) * 1e3)
        out[name + "_ms"] = float(np.median(ts))
    learned.close()
    ctx.close()
    print(json.dumps(out))
    return 0


def profile_lal():
    """The capture workload of the legalizer profiles: one B2B build and
    FP64 PCG solve of the 211k-cell workload from its seed positions, then
    the look-ahead legalization of the solved positions, twice."""
    from ktplace_b200 import grid
    from ktplace_b200.gpu import Context
    raw, nl, x, y, ax, ay = make_workload(1)
    fx, fy = nl.floors()
    ctx = Context(0)
    ctx.upload_netlist(nl)
    ctx.build_b2b(x, y, ALPHA, ax, ay, fx, fy)
    px, py = np.array(x, dtype=np.float64), np.array(y, dtype=np.float64)
    ctx.solve(px, py, TOL, MAX_ITER, inplace=True)
    bins = grid.default_bins_per_axis(nl.num_movable)
    ctx.set_grid(grid.build_grid(nl, bins, 1.0))
    ctx.set_free_space(grid.build_free_space(nl))
    for _ in range(2):
        lx, ly = ctx.lal(px, py)
    st = ctx.lal_stats()
    print(f"profile-lal: {int(st['batches'])} batches, {int(st['regions'])} regions, "
          f"{st['ms_total']:.1f} ms, moved {float(np.mean((lx != px) | (ly != py))):.3f}")
    ctx.close()
    return 0


def profile_pcg(cells: int) -> int:
    """A design of `cells` movable cells with the 211k design's proportions
    (nets 1.05x, rows and pads by the square root, macros by the cell count),
    seed 7: one B2B build (alpha 0.2, anchors) and three FP64 solves to rtol
    1e-6 from the same start, timed with CUDA events; prints the median time,
    iterations and the algorithmic bytes per second of the solve (pcg_bytes)."""
    import math
    import torch
    from ktplace_b200 import netlist, synth
    from ktplace_b200.gpu import Context
    from ktplace_b200._lib import SolveInfo
    k = cells / 211_000
    spec = synth.SynthSpec(num_movable=cells, num_nets=int(round(1.0474 * cells)),
                           num_pads=int(round(1000 * math.sqrt(k))),
                           num_rows=int(round(890 * math.sqrt(k))), utilization=0.6,
                           num_macros=int(round(550 * k)), seed=7, name=f"synth{cells}")
    raw = synth.generate(spec)
    nl = netlist.flatten(raw)
    x, y = synth.seed_positions(raw, nl.num_movable, 107)
    ax, ay = synth.seed_positions(raw, nl.num_movable, 207)
    fx, fy = nl.floors()
    dev = torch.device("cuda", 0)
    stream = torch.cuda.Stream(dev)
    ctx = Context(0)
    ctx.upload_netlist(nl)
    ctx.set_stream(stream.cuda_stream)
    with torch.cuda.stream(stream):
        dx, dy = torch.tensor(x, device=dev), torch.tensor(y, device=dev)
        dax, day = torch.tensor(ax, device=dev), torch.tensor(ay, device=dev)
        wx, wy = torch.empty_like(dx), torch.empty_like(dy)
        info = torch.zeros(ctypes.sizeof(SolveInfo), dtype=torch.uint8, device=dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    ms = []
    for _ in range(3):
        with torch.cuda.stream(stream):
            ctx.build_b2b_dev(dx, dy, ALPHA, dax, day, fx, fy)
            wx.copy_(dx)
            wy.copy_(dy)
            e0.record(stream)
            ctx.solve_dev(wx, wy, TOL, MAX_ITER, info)
            e1.record(stream)
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
    inf = SolveInfo.from_buffer_copy(bytes(info.cpu().numpy()))
    _, mx = ctx.system_info(0)
    _, my = ctx.system_info(1)
    n = nl.num_movable
    byts = pcg_bytes(n, mx, inf.iters_x) + pcg_bytes(n, my, inf.iters_y)
    t = statistics.median(ms)
    peak, kind = measured_peak()
    print(json.dumps({"cells": n, "nnz": [mx, my], "iters": [int(inf.iters_x), int(inf.iters_y)],
                      "solve_ms": t, "algorithmic_bytes": byts,
                      "achieved_gbs": byts / (t * 1e-3) / 1e9, "peak_gbs": peak,
                      "peak_kind": kind, "frac": byts / (t * 1e-3) / 1e9 / peak}))
    ctx.close()
    return 0


def profile_spmv(cells: int) -> int:
    """Standalone SpMV (ktg_spmv, SparseSystem::multiply's row sums) on the
    scaled design of --profile-pcg: one B2B build, then 20 timed rounds of
    A v on both axes with CUDA events; prints ms per SpMV and the
    algorithmic bytes per second (spmv_bytes) against the measured HBM peak.
    Inputs larger than L2 (from about 1M cells) need no flush."""
    import math
    import torch
    from ktplace_b200 import netlist, synth
    from ktplace_b200.gpu import Context
    k = cells / 211_000
    spec = synth.SynthSpec(num_movable=cells, num_nets=int(round(1.0474 * cells)),
                           num_pads=int(round(1000 * math.sqrt(k))),
                           num_rows=int(round(890 * math.sqrt(k))), utilization=0.6,
                           num_macros=int(round(550 * k)), seed=7, name=f"synth{cells}")
    raw = synth.generate(spec)
    nl = netlist.flatten(raw)
    x, y = synth.seed_positions(raw, nl.num_movable, 107)
    ax, ay = synth.seed_positions(raw, nl.num_movable, 207)
    fx, fy = nl.floors()
    dev = torch.device("cuda", 0)
    stream = torch.cuda.Stream(dev)
    ctx = Context(0)
    ctx.upload_netlist(nl)
    ctx.set_stream(stream.cuda_stream)
    with torch.cuda.stream(stream):
        dx, dy = torch.tensor(x, device=dev), torch.tensor(y, device=dev)
        dax, day = torch.tensor(ax, device=dev), torch.tensor(ay, device=dev)
        ox, oy = torch.empty_like(dx), torch.empty_like(dy)
        ctx.build_b2b_dev(dx, dy, ALPHA, dax, day, fx, fy)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    rounds = 20
    with torch.cuda.stream(stream):
        for _ in range(3):  # warm-up
            ctx.spmv_dev(0, dx, ox)
            ctx.spmv_dev(1, dy, oy)
        e0.record(stream)
        for _ in range(rounds):
            ctx.spmv_dev(0, dx, ox)
            ctx.spmv_dev(1, dy, oy)
        e1.record(stream)
    e1.synchronize()
    t = e0.elapsed_time(e1) / (2 * rounds)
    n = nl.num_movable
    _, mx = ctx.system_info(0)
    _, my = ctx.system_info(1)
    byts = (spmv_bytes(n, mx) + spmv_bytes(n, my)) / 2
    peak, kind = measured_peak()
    gbs = byts / (t * 1e-3) / 1e9
    print(json.dumps({"cells": n, "nnz": [mx, my], "ms_per_spmv": t, "algorithmic_bytes": byts,
                      "achieved_gbs": gbs, "peak_gbs": peak, "peak_kind": kind,
                      "frac": gbs / peak}))
    ctx.close()
    return 0


def run_config4(args) -> int:
    """The solve comparison of `solve_variants` on the 2.2M-cell design (2.25M
    nets, 8,000 macros; seed positions and anchors), the configuration the
    learned preconditioner is specified at. One GPU; not part of the default
    run (the design alone takes tens of seconds to generate)."""
    import torch
    from ktplace_b200 import netlist, synth
    from ktplace_b200.gpu import Context
    from ktplace_b200._lib import SolveInfo
    raw = synth.generate(synth.spec_2m(4))
    nl = netlist.flatten(raw)
    x, y = synth.seed_positions(raw, nl.num_movable, 104)
    ax, ay = synth.seed_positions(raw, nl.num_movable, 204)
    fx, fy = nl.floors()
    dev = torch.device("cuda", 0)
    stream = torch.cuda.Stream(dev)
    ctx = Context(0)
    ctx.upload_netlist(nl)
    ctx.set_stream(stream.cuda_stream)
    with torch.cuda.stream(stream):
        dx, dy = torch.tensor(x, device=dev), torch.tensor(y, device=dev)
        dax, day = torch.tensor(ax, device=dev), torch.tensor(ay, device=dev)
        wx, wy = torch.empty_like(dx), torch.empty_like(dy)
        info = torch.zeros(ctypes.sizeof(SolveInfo), dtype=torch.uint8, device=dev)
        scal = torch.zeros(8, dtype=torch.float64, device=dev)
        flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    torch.cuda.synchronize(dev)
    variants = solve_variants(torch, dev, stream, ctx, dx, dy, dax, day, fx, fy, wx, wy, info,
                              scal, flush, max(3, args.steps // 20))
    print(json.dumps({"config": "2.2M cells, 2.25M nets, 8,000 macros (seed 4), positions seed "
                                "104, anchors seed 204, alpha 0.2, rtol 1e-6",
                      "cells": nl.num_movable, "nets": nl.num_nets, "pins": nl.num_pins,
                      "solve_variants": variants}))
    ctx.close()
    return 0


def run_simpl_report(iters: int, weights: str = None) -> int:
    import torch
    dev = torch.device("cuda:0")
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream(device=dev)
    raw, nl, x, y, ax, ay = make_workload(1)
    learned = load_coarse_network(dev, weights)
    rep = simpl_report(torch, dev, stream, nl, x, y, iters, learned=learned)
    if learned is not None:
        learned.close()
    print(json.dumps(rep))
    return 0


COARSE_WEIGHTS = os.path.join(ROOT, "ktplace_b200", "weights", "learned_coarse.npy")


def load_coarse_network(dev, path: str = None):
    """The trained coarse-vector network, or None when no weights exist."""
    path = path or COARSE_WEIGHTS
    if not os.path.exists(path):
        return None
    from ktplace_b200.learned import Learned
    learned = Learned(dev.index or 0)
    learned.load(path)
    return learned


def main():
    args = parse()
    if args.profile_pcg:
        return profile_pcg(args.profile_pcg)
    if args.profile_spmv:
        return profile_spmv(args.profile_spmv)
    if args.config4:
        return run_config4(args)
    if args.simpl_report:
        return run_simpl_report(args.simpl_report, args.coarse_weights)
    if args.profile_once:
        return profile_once()
    if args.profile_dense:
        return profile_dense()
    if args.profile_lal:
        return profile_lal()
    if args.profile_agg:
        return profile_agg()
    if args.profile_batch_full:
        batch, rows = batch_workload(64)
        batch.set_shape(4, 1024)
        batch.set_offload(44725, precond=2, coarse=0)
        batch.solve(TOL, MAX_ITER, precision=1, inner_tol=MIXED_INNER_TOL)
        res = batch.results()
        bad = [r for r in res if r["status"] != 0 or r["resid"] > TOL]
        print(f"profile-batch-full: {len(rows)} systems, {batch.offload()['pairs']} pairs on the "
              f"whole GPU, {len(bad)} unconverged")
        return 1 if bad else 0
    if args.profile_batch:
        batch, rows = batch_workload(16)
        batch.solve(TOL, MAX_ITER, precision=1, inner_tol=MIXED_INNER_TOL)
        res = batch.results()
        print(f"profile-batch: {len(rows)} systems, inner iterations p50 "
              f"{float(np.median([r['iters'] for r in res]))}")
        return 0
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
