"""Trains the learned preconditioner and writes its weights.

    python -m ktplace_b200.train_precond [--designs 40] [--iters 25] [--epochs 3]
                                          [--out ktplace_b200/weights/learned_precond.npy]

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
    ap.add_argument("--out", default=DEFAULT_OUT)
    args = ap.parse_args(argv)
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


if __name__ == "__main__":
    sys.exit(main())
