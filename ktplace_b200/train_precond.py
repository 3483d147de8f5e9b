"""Trains the learned networks of the mixed solve and writes their weights.

    python -m ktplace_b200.train_precond --coarse [--designs 64] [--iters 30]
        [--min-cells 5000] [--max-cells 500000] [--epochs-from-dataset E]
        [--out ktplace_b200/weights/learned_coarse.npy]
        [--dataset ktplace_b200/weights/coarse_dataset.bin]
    python -m ktplace_b200.train_precond --coarse --from-dataset FILE
        [--epochs-from-dataset E]

trains the learned coarse vector of the two-level aggregation preconditioner
on the systems of the GPU SimPL loop (B2B initial rounds, then global
iterations anchored at the look-ahead-legalized positions, anchor weight
0.01 -> 1.0) of seeded synthetic netlists with log-uniform cell counts,
designs x iters x 2 systems (3,840 with the defaults). The first epoch
streams the systems as the loop produces them and writes the training set's
record file (learned.CoarseDataset); further epochs, or a run from an
existing file, consume that file: each recorded system is regenerated from
its design and iteration and checked against its recorded digests before it
is used.

    python -m ktplace_b200.train_precond [--designs 40] [--iters 25] [--epochs 3]
                                          [--out ktplace_b200/weights/learned_precond.npy]

trains the learned sparse approximate inverse (precond 1):

Training systems: the B2B x and y systems of every iteration of a SimPL-style
run (ktplace_b200.learned.simpl_like_systems) on seeded synthetic netlists in
the shapes of the single-netlist and batch configurations (5k-100k cells,
mean degree 3.5-3.9), designs x iters x 2 systems in all (2,000 with the
defaults). Everything runs on the GPU through the C ABI.
"""
from __future__ import annotations

import argparse
import math
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_OUT = os.path.join(HERE, "weights", "learned_precond.npy")
COARSE_OUT = os.path.join(HERE, "weights", "learned_coarse.npy")
COARSE_DATASET = os.path.join(HERE, "weights", "coarse_dataset.bin")


def coarse_design(k: int, cells: int, s: int):
    """Training design k: `cells` movable cells, generator seed s; returns
    (netlist, x0, y0, s). Odd designs have mean degree 3.5 and 60% density,
    even ones a heavier-tailed degree law and 70%; every third carries
    macros."""
    from . import synth, netlist
    spec = synth.SynthSpec(num_movable=cells, num_nets=int(cells * 1.05),
                           num_pads=max(50, int(200 * math.sqrt(cells / 12_000))),
                           num_rows=max(20, int(120 * math.sqrt(cells / 12_000))),
                           utilization=0.6 if k % 2 else 0.7,
                           num_macros=int(cells / 400) if k % 3 == 0 else 0,
                           degree_exponent=synth.exponent_for_mean(3.5) if k % 2 else 2.5,
                           seed=s, name=f"coarse{k}")
    raw = synth.generate(spec)
    nl = netlist.flatten(raw)
    x0, y0 = synth.seed_positions(raw, nl.num_movable, s + 500)
    return nl, x0, y0, s


def coarse_designs(count: int, seed: int = 9000, min_cells: int = 5_000,
                   max_cells: int = 500_000):
    """Seeded synthetic netlists in the shape of the single-netlist and batch
    configurations, cell counts log-uniform in [min_cells, max_cells];
    yields (netlist, x0, y0, seed)."""
    rng = np.random.default_rng(seed)
    for k in range(count):
        cells = int(round(math.exp(rng.uniform(math.log(min_cells), math.log(max_cells)))))
        yield coarse_design(k, cells, seed + k)


def dataset_designs(records):
    """The designs a recorded training set was drawn from, regenerated from
    the records (design index, cells, seed), with the global iterations
    recorded for each: yields (design index, (netlist, x0, y0, seed),
    iterations)."""
    seen = {}
    for r in records:
        key = (int(r["design"]), int(r["cells"]), int(r["seed"]))
        seen.setdefault(key, set()).add(int(r["iteration"]))
    for (k, cells, s), its in seen.items():
        yield k, coarse_design(k, cells, s), sorted(its)


def training_designs(count: int, seed: int = 7000, max_cells: int = 100_000):
    from . import synth, netlist
    rng = np.random.default_rng(seed)
    for k in range(count):
        cells = int(round(math.exp(rng.uniform(math.log(5_000), math.log(max_cells)))))
        if k % 2 == 0:
            spec = synth.SynthSpec(num_movable=cells, num_nets=int(cells * 13 / 12),
                                   num_pads=max(50, int(200 * math.sqrt(cells / 12_000))),
                                   num_rows=max(20, int(120 * math.sqrt(cells / 12_000))),
                                   utilization=0.7, seed=seed + k, name=f"train{k}")
        else:
            spec = synth.SynthSpec(num_movable=cells, num_nets=int(cells * 13 / 12),
                                   num_pads=max(50, int(200 * math.sqrt(cells / 12_000))),
                                   num_rows=max(20, int(120 * math.sqrt(cells / 12_000))),
                                   utilization=0.65, degree_exponent=synth.exponent_for_mean(3.5),
                                   seed=seed + k, name=f"train{k}")
        raw = synth.generate(spec)
        nl = netlist.flatten(raw)
        x0, y0 = synth.seed_positions(raw, nl.num_movable, seed + 500 + k)
        yield nl, x0, y0


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--designs", type=int, default=40)
    ap.add_argument("--iters", type=int, default=25)
    ap.add_argument("--epochs", type=int, default=3)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--out", default=None)
    ap.add_argument("--coarse", action="store_true",
                    help="train the learned coarse vector instead of the approximate inverse")
    ap.add_argument("--min-cells", type=int, default=5_000)
    ap.add_argument("--max-cells", type=int, default=500_000)
    ap.add_argument("--dataset", default=COARSE_DATASET)
    ap.add_argument("--epochs-from-dataset", type=int, default=0,
                    help="further epochs over the recorded training set (regenerated and "
                         "checked against its digests)")
    ap.add_argument("--from-dataset", default=None,
                    help="train only from this recorded training set")
    args = ap.parse_args(argv)
    if args.coarse:
        return main_coarse(args)
    args.out = args.out or DEFAULT_OUT
    from .gpu import Context
    from .learned import Learned, train
    t0 = time.time()
    designs = list(training_designs(args.designs))
    print(f"{len(designs)} designs, {sum(d[0].num_movable for d in designs)} cells "
          f"({time.time() - t0:.1f}s)", flush=True)
    learned = Learned(0, seed=args.seed)
    learned.set_option("lr", args.lr)
    ctx = Context(0)
    t0 = time.time()
    losses = train(learned, designs, iters=args.iters, epochs=args.epochs, ctx=ctx,
                   log=lambda m: print(m, flush=True))
    n = len(losses) // args.epochs
    print(f"{len(losses)} steps in {time.time() - t0:.1f}s; mean loss first epoch "
          f"{np.mean(losses[:n]):.4e}, last epoch {np.mean(losses[-n:]):.4e}", flush=True)
    os.makedirs(os.path.dirname(args.out), exist_ok=True)
    learned.save(args.out)
    print("wrote", args.out)
    ctx.close()
    learned.close()
    return 0


def main_coarse(args) -> int:
    from .gpu import Context
    from .learned import Learned, CoarseDataset, train_coarse, train_coarse_recorded
    out = args.out or COARSE_OUT
    learned = Learned(0, seed=args.seed)
    learned.set_option("lr", args.lr)
    ctx = Context(0)
    t0 = time.time()
    log = lambda m: print(m, f"({time.time() - t0:.0f}s)", flush=True)  # noqa: E731
    losses = []
    if args.from_dataset:
        records = CoarseDataset.load(args.from_dataset)
        epochs = max(1, args.epochs_from_dataset)
    else:
        ds = CoarseDataset()
        designs = coarse_designs(args.designs, min_cells=args.min_cells, max_cells=args.max_cells)
        losses = train_coarse(learned, designs, iters=args.iters, epochs=1, ctx=ctx, dataset=ds,
                              log=log)
        ds.save(args.dataset)
        print("wrote", args.dataset, f"({len(ds.records)} systems)", flush=True)
        records = CoarseDataset.load(args.dataset)
        epochs = args.epochs_from_dataset
    for ep in range(epochs):
        losses += train_coarse_recorded(learned, records, ctx=ctx, log=log, epoch=ep)
    k = max(1, len(losses) // 10)
    print(f"{len(losses)} steps in {time.time() - t0:.1f}s; mean loss first tenth "
          f"{np.mean(losses[:k]):.4e}, last tenth {np.mean(losses[-k:]):.4e}", flush=True)
    os.makedirs(os.path.dirname(out), exist_ok=True)
    learned.save(out)
    print("wrote", out)
    ctx.close()
    learned.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
