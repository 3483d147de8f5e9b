"""Learned networks of the mixed-precision solve: training data, training
loops, the training-set file and evaluation.

The networks, their training and their use all run in the CUDA library
(csrc/ktg_learned.cu, include/ktplace_b200.h); this module orchestrates them.

Two uses of the same message-passing network over the cell-net graph:
  * the learned coarse vector of the two-level aggregation preconditioner
    ("coarse" = 3): trained on systems of the GPU SimPL loop
    (simpl.GlobalLoop: B2B initial rounds, then global iterations anchored
    at the look-ahead-legalized positions, ktg_lal), with test vectors taken
    from the solves themselves (train_coarse, CoarseDataset);
  * the learned sparse approximate inverse on A's pattern (precond 1), kept
    for comparison; its training systems come from simpl_like_systems, whose
    anchors are a 1-D area-proportional spread.
"""
from __future__ import annotations

import ctypes
from typing import Iterable, Iterator, Optional

import numpy as np

from . import _lib
from ._lib import KtgError
from .gpu import Context


def alpha_schedule(it: int, iters: int = 30) -> float:
    """Anchor weight rising linearly from 0.01 to 1.0 over `iters` iterations."""
    return 0.01 + (1.0 - 0.01) * min(it, iters - 1) / max(iters - 1, 1)


def spread(nl, x, y):
    """Area-proportional 1-D redistribution of the movable cells per axis."""
    lx, ly, ux, uy = nl.die
    area = nl.width * nl.height
    total = area.sum()
    out = []
    for pos, size, lo, hi in ((x, nl.width, lx, ux), (y, nl.height, ly, uy)):
        order = np.argsort(pos + 0.5 * size, kind="stable")
        cum = np.cumsum(area[order]) - 0.5 * area[order]
        centre = lo + (hi - lo) * cum / total
        p = np.empty_like(pos)
        p[order] = np.clip(centre - 0.5 * size[order], lo, hi - size[order])
        out.append(p)
    return out[0], out[1]


def simpl_like_systems(ctx: Context, nl, x0, y0, iters: int, tol: float = 1e-6,
                       max_iter: int = 100000) -> Iterator[tuple]:
    """Runs `iters` SimPL-style iterations on `ctx` (netlist already
    uploaded); right after each B2B build, while ctx holds that iteration's
    systems, yields (iteration, x, y) with the positions they were built at
    (the warm start of that iteration's solve)."""
    fx, fy = nl.floors()
    x, y = np.array(x0, dtype=np.float64), np.array(y0, dtype=np.float64)
    for it in range(iters):
        ax, ay = spread(nl, x, y)
        ctx.build_b2b(x, y, alpha_schedule(it), ax, ay, fx, fy)
        yield it, x.copy(), y.copy()
        r = ctx.solve(x, y, tol, max_iter)
        x, y = r["x"], r["y"]


class Learned:
    """Owns a ``ktg_learned`` handle (network weights + Adam state)."""

    def __init__(self, device: int = 0, seed: int = 0):
        self.lib = _lib.load()
        h = ctypes.c_void_p()
        rc = self.lib.ktg_learned_create(device, seed, ctypes.byref(h))
        if rc != 0:
            raise KtgError(rc, "ktg_learned_create failed")
        self.h = h
        self.num_params = int(self.lib.ktg_learned_num_params())

    def close(self):
        if getattr(self, "h", None):
            self.lib.ktg_learned_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def launches(self) -> int:
        """Kernels this handle has launched."""
        return int(self.lib.ktg_learned_launch_count(self.h))

    def _check(self, rc: int):
        if rc != 0:
            raise KtgError(rc, self.lib.ktg_learned_last_error(self.h).decode())

    def set_option(self, key: str, value: float):
        self._check(self.lib.ktg_learned_set_option(self.h, key.encode(), float(value)))

    def get_params(self) -> np.ndarray:
        w = np.zeros(self.num_params, np.float32)
        self._check(self.lib.ktg_learned_get_params(self.h, ctypes.c_void_p(w.ctypes.data)))
        return w

    def set_params(self, w):
        w = np.ascontiguousarray(w, dtype=np.float32)
        assert w.shape[0] == self.num_params
        self._check(self.lib.ktg_learned_set_params(self.h, ctypes.c_void_p(w.ctypes.data)))

    def loss_grad(self, ctx: Context, axis: int, seed: int = 0):
        loss = ctypes.c_double()
        g = np.zeros(self.num_params, np.float32)
        self._check(self.lib.ktg_learned_loss_grad(self.h, ctx.h, axis, seed, ctypes.byref(loss),
                                                   ctypes.c_void_p(g.ctypes.data)))
        return float(loss.value), g

    def train_step(self, ctx: Context, axis: int, seed: int) -> float:
        loss = ctypes.c_double()
        self._check(self.lib.ktg_learned_train_step(self.h, ctx.h, axis, seed,
                                                    ctypes.byref(loss)))
        return float(loss.value)

    def prepare(self, ctx: Context):
        self._check(self.lib.ktg_learned_prepare(self.h, ctx.h))

    # -- learned coarse vector ---------------------------------------------------
    def coarse_loss_grad(self, ctx: Context, axis: int, vectors):
        """Projection loss of the test vectors ([T, n], T <= 4) on the
        predicted coarse vector of one axis, and the parameter gradient."""
        e = np.ascontiguousarray(np.atleast_2d(vectors), dtype=np.float64)
        loss = ctypes.c_double()
        g = np.zeros(self.num_params, np.float32)
        self._check(self.lib.ktg_learned_coarse_loss_grad(
            self.h, ctx.h, axis, ctypes.c_void_p(e.ctypes.data), e.shape[0], ctypes.byref(loss),
            ctypes.c_void_p(g.ctypes.data)))
        return float(loss.value), g

    def coarse_train_step(self, ctx: Context, axis: int, vectors) -> float:
        e = np.ascontiguousarray(np.atleast_2d(vectors), dtype=np.float64)
        loss = ctypes.c_double()
        self._check(self.lib.ktg_learned_coarse_train_step(
            self.h, ctx.h, axis, ctypes.c_void_p(e.ctypes.data), e.shape[0], ctypes.byref(loss)))
        return float(loss.value)

    def prepare_coarse(self, ctx: Context):
        """Coarse vectors of ctx's current systems for "coarse" = 3 (enqueued
        on ctx's stream)."""
        self._check(self.lib.ktg_learned_prepare_coarse(self.h, ctx.h))

    prepare_coarse_dev = prepare_coarse

    def save(self, path: str):
        np.save(path, self.get_params())

    def load(self, path: str):
        w = np.load(path).astype(np.float32)
        if w.shape[0] < self.num_params:
            # weights saved before the coarse-vector head existed: keep the
            # freshly initialised head (the constant coarse vector)
            cur = self.get_params()
            cur[:w.shape[0]] = w
            w = cur
        self.set_params(w)


def train(learned: Learned, designs: Iterable, iters: int = 8, epochs: int = 2,
          ctx: Optional[Context] = None, seed: int = 0, log=None) -> list:
    """Trains on the systems of a SimPL-style run of every design.

    `designs` yields (netlist, x0, y0). Each epoch replays the runs (the
    systems are rebuilt on the GPU, not stored) and takes one Adam step per
    axis system. Returns the per-step losses."""
    own = ctx is None
    ctx = ctx or Context(0)
    designs = list(designs)
    losses = []
    step = 0
    for ep in range(epochs):
        for d, (nl, x0, y0) in enumerate(designs):
            ctx.upload_netlist(nl)
            for _ in simpl_like_systems(ctx, nl, x0, y0, iters):
                for axis in (0, 1):
                    loss = learned.train_step(ctx, axis, seed + step)
                    losses.append(loss)
                    step += 1
            if log:
                log(f"epoch {ep} design {d}: loss {np.mean(losses[-2 * iters:]):.4e}")
    if own:
        ctx.close()
    return losses


def compare_solvers(learned: Learned, ctx: Context, nl, x0, y0, iters: int, tol: float = 1e-6,
                    inner_tol: float = 1e-3) -> list:
    """For each iteration of a SimPL-style run, solves that iteration's
    systems twice with the FP32-in-FP64 PCG, Jacobi and learned
    preconditioner, from the same warm start."""
    out = []
    for it, x, y in simpl_like_systems(ctx, nl, x0, y0, iters):
        row = {"iteration": it}
        for name, pre in (("jacobi", 0), ("learned", 1)):
            ctx.set_option("precond", pre)
            if pre:
                learned.prepare(ctx)
            row[name] = ctx.solve_mixed(x, y, tol, inner_tol)
        ctx.set_option("precond", 0)
        out.append(row)
    return out


# ---- learned coarse vector ----------------------------------------------------

DATASET_MAGIC = b"KTGCOARS"
DATASET_VERSION = 2
_REC = np.dtype([("design", "<i4"), ("seed", "<i8"), ("cells", "<i8"), ("nets", "<i8"),
                 ("iteration", "<i4"), ("alpha", "<f8"), ("n", "<i8"), ("nnz_x", "<i8"),
                 ("nnz_y", "<i8"), ("fp64_iters_x", "<i4"), ("fp64_iters_y", "<i4"),
                 ("agg_iters_x", "<i4"), ("agg_iters_y", "<i4"), ("loss_x", "<f8"),
                 ("loss_y", "<f8"), ("system_sha", "u1", (32,)),
                 ("solution_sha", "u1", (32,))])


class CoarseDataset:
    """The training set of the learned coarse vector as a versioned binary
    file: the 8-byte magic KTGCOARS, a little-endian u32 version and u32
    record count, then one fixed-size record per (A, b, x*) system. A record
    names the system by how it is produced (training design index and
    generator seed, SimPL global iteration, anchor weight: the GPU SimPL loop
    is deterministic, so these regenerate the system exactly) and pins it by
    SHA-256 digests of A, b (CSR, diag, rhs of both axes) and of the FP64
    solution x*, beside its sizes, the FP64 and aggregation iteration counts
    and the training loss of each axis. The arrays themselves are not stored
    (a 2,000-system set of 5k-500k-cell netlists would take tens of GB)."""

    def __init__(self):
        self.records = []

    def add(self, **fields):
        self.records.append(fields)

    def save(self, path: str):
        arr = np.zeros(len(self.records), dtype=_REC)
        for i, r in enumerate(self.records):
            for k in _REC.names:
                v = r[k]
                arr[i][k] = np.frombuffer(v, dtype=np.uint8) if isinstance(v, bytes) else v
        with open(path, "wb") as f:
            f.write(DATASET_MAGIC)
            f.write(np.array([DATASET_VERSION, len(arr)], dtype="<u4").tobytes())
            f.write(arr.tobytes())

    @staticmethod
    def load(path: str) -> np.ndarray:
        with open(path, "rb") as f:
            if f.read(8) != DATASET_MAGIC:
                raise ValueError(f"{path}: not a coarse-vector training set")
            version, count = np.frombuffer(f.read(8), dtype="<u4")
            if version != DATASET_VERSION:
                raise ValueError(f"{path}: version {version}, expected {DATASET_VERSION}")
            return np.frombuffer(f.read(), dtype=_REC, count=int(count))


def _sha(*arrays) -> bytes:
    import hashlib
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.digest()


def coarse_test_vectors(ctx: Context, x, y, xs, ys, ks=(4, 8), tol: float = 1e-6):
    """Errors the aggregation-preconditioned FP32 PCG leaves after k inner
    iterations from the warm start (x, y), against the FP64 solution (xs, ys):
    the slow error components a coarse vector has to capture. Returns
    ([T, n] for x, [T, n] for y) and the inner iterations of a full solve."""
    ctx.set_option("precond", 2)
    ctx.set_option("coarse", 0)
    ex, ey = [], []
    for k in ks:
        r = ctx.solve_mixed(x, y, tol, 1e-3, max_inner=k)
        ex.append(r["x"] - xs)
        ey.append(r["y"] - ys)
    full = ctx.solve_mixed(x, y, tol, 1e-3)
    ctx.set_option("precond", 0)
    return np.stack(ex), np.stack(ey), full["inner"]


def coarse_training_systems(ctx: Context, nl, x0, y0, iters: int, init_rounds: int = 3,
                            tol: float = 1e-6):
    """Runs the GPU SimPL loop (simpl.GlobalLoop) on netlist nl and, after
    every global iteration's build, yields (state, FP64 result, test vectors
    per axis, aggregation inner iterations) while ctx holds that system."""
    from . import grid as kgrid
    from . import simpl
    g = kgrid.build_grid(nl, kgrid.default_bins_per_axis(nl.num_movable), 1.0)
    loop = simpl.GlobalLoop(ctx, nl, g, kgrid.build_free_space(nl), tol=tol)
    x, y = loop.initial_rounds(x0, y0, init_rounds)
    last = {}

    def solve(px, py):
        return last["x"], last["y"]

    for st in loop.iterations(x, y, iters, solve=solve):
        f = ctx.solve(st.x, st.y, tol, 100000)
        last["x"], last["y"] = f["x"], f["y"]
        ex, ey, agg_inner = coarse_test_vectors(ctx, st.x, st.y, f["x"], f["y"], tol=tol)
        yield st, f, (ex, ey), agg_inner


def train_coarse(learned: Learned, designs: Iterable, iters: int = 30, epochs: int = 1,
                 ctx: Optional[Context] = None, dataset: Optional[CoarseDataset] = None,
                 log=None) -> list:
    """Trains the coarse-vector head and trunk: one Adam step per axis system
    of every global iteration of the GPU SimPL loop on every design
    ((netlist, x0, y0, seed) tuples). Returns the per-step losses; records
    every system in `dataset` (first epoch) when given."""
    own = ctx is None
    ctx = ctx or Context(0)
    if epochs > 1:
        designs = list(designs)  # replayed; one epoch streams them
    losses = []
    for ep in range(epochs):
        for d, (nl, x0, y0, seed) in enumerate(designs):
            ctx.upload_netlist(nl)
            for st, f, (ex, ey), agg_inner in coarse_training_systems(ctx, nl, x0, y0, iters):
                lx = learned.coarse_train_step(ctx, 0, ex)
                ly = learned.coarse_train_step(ctx, 1, ey)
                losses += [lx, ly]
                if dataset is not None and ep == 0:
                    sx, sy = ctx.system(0), ctx.system(1)
                    dataset.add(design=d, seed=seed, cells=nl.num_movable, nets=nl.num_nets,
                                iteration=st.it, alpha=st.alpha, n=nl.num_movable,
                                nnz_x=len(sx["val"]), nnz_y=len(sy["val"]),
                                fp64_iters_x=f["iters_x"], fp64_iters_y=f["iters_y"],
                                agg_iters_x=agg_inner[0], agg_iters_y=agg_inner[1],
                                loss_x=lx, loss_y=ly,
                                system_sha=_sha(*[sx[k] for k in ("row_ptr", "col", "val",
                                                                  "diag", "rhs")],
                                                *[sy[k] for k in ("row_ptr", "col", "val",
                                                                  "diag", "rhs")]),
                                solution_sha=_sha(f["x"], f["y"]))
            if log:
                log(f"epoch {ep} design {d} ({nl.num_movable} cells): "
                    f"loss {np.mean(losses[-2 * iters:]):.4e}")
    if own:
        ctx.close()
    return losses


def train_coarse_recorded(learned: Learned, records, ctx: Optional[Context] = None, log=None,
                          epoch: int = 0) -> list:
    """One epoch over a recorded training set (CoarseDataset.load): every
    design is regenerated from its record, its GPU SimPL loop rerun, and each
    recorded system checked against its digests (A, b and the FP64 solution
    x*) before its Adam steps. Returns the per-step losses."""
    from .train_precond import dataset_designs
    own = ctx is None
    ctx = ctx or Context(0)
    want = {(int(r["design"]), int(r["iteration"])): r for r in records}
    losses = []
    try:
        for k, (nl, x0, y0, _), its in dataset_designs(records):
            ctx.upload_netlist(nl)
            for st, f, (ex, ey), _ in coarse_training_systems(ctx, nl, x0, y0, its[-1] + 1):
                rec = want.get((k, st.it))
                if rec is None:
                    continue
                sx, sy = ctx.system(0), ctx.system(1)
                sha = _sha(*[sx[q] for q in ("row_ptr", "col", "val", "diag", "rhs")],
                           *[sy[q] for q in ("row_ptr", "col", "val", "diag", "rhs")])
                if (sha != rec["system_sha"].tobytes() or
                        _sha(f["x"], f["y"]) != rec["solution_sha"].tobytes()):
                    raise RuntimeError(f"design {k} iteration {st.it}: regenerated system "
                                       "differs from the recorded one")
                losses += [learned.coarse_train_step(ctx, 0, ex),
                           learned.coarse_train_step(ctx, 1, ey)]
            if log:
                log(f"epoch {epoch} (recorded) design {k} ({nl.num_movable} cells): "
                    f"loss {np.mean(losses[-2 * len(its):]):.4e}")
    finally:
        if own:
            ctx.close()
    return losses


def compare_coarse(learned: Optional[Learned], ctx: Context, nl, x0, y0, iters: int,
                   tol: float = 1e-6, init_rounds: int = 3) -> list:
    """For each global iteration of the GPU SimPL loop, the aggregation mixed
    solve of that iteration's systems with no coarse vector, the constant one
    (the network switched off), the coupling share and the learned one, from
    the same warm start: inner iterations, rounds and the true residuals."""
    from . import grid as kgrid
    from . import simpl
    g = kgrid.build_grid(nl, kgrid.default_bins_per_axis(nl.num_movable), 1.0)
    loop = simpl.GlobalLoop(ctx, nl, g, kgrid.build_free_space(nl), tol=tol)
    x, y = loop.initial_rounds(x0, y0, init_rounds)
    out = []
    for st in loop.iterations(x, y, iters):
        row = {"iteration": st.it}
        ctx.set_option("precond", 2)
        for name, mode in (("none", 0), ("constant", 1), ("coupling", 2), ("learned", 3)):
            if mode == 3:
                if learned is None:
                    continue
                learned.prepare_coarse(ctx)
            ctx.set_option("coarse", mode)
            row[name] = ctx.solve_mixed(st.x, st.y, tol, 1e-3)
        ctx.set_option("coarse", 0)
        ctx.set_option("precond", 0)
        out.append(row)
    return out
