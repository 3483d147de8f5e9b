"""Learned preconditioner: training data, training loop and evaluation.

The network, its training and its use all run in the CUDA library
(csrc/ktg_learned.cu, include/ktplace_b200.h); this module orchestrates them.

Training systems come from a SimPL-style loop run on the GPU path itself:
each iteration builds the B2B systems at the current lower-bound positions
with anchors at a spread (upper-bound) placement and an anchor weight that
grows linearly from 0.01 to 1.0 over 30 iterations, then solves them warm
started. The spread placement is a 1-D area-proportional redistribution per
axis (cells keep their order, their centres move to equal-area slots of the
die), a stand-in for look-ahead legalization, which is not part of this path.
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
