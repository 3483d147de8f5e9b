"""Python handle on one ktplace_b200 context (one device, one stream).

Thin wrapper over the C ABI (include/ktplace_b200.h). Host-mode calls take
numpy arrays; device-mode calls (``*_dev``) take torch CUDA tensors and only
enqueue work on the context's stream.
"""
from __future__ import annotations

import ctypes
from typing import Optional

import numpy as np

from . import _lib
from ._lib import KtgError, NetlistView, GridView, SolveInfo, MixedInfo


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


def _c(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


def _tptr(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


class Context:
    """Owns a ``ktg_ctx``: the device-resident netlist, systems and grid."""

    def __init__(self, device: int = 0):
        self.lib = _lib.load()
        h = ctypes.c_void_p()
        rc = self.lib.ktg_create(device, ctypes.byref(h))
        if rc != 0:
            raise KtgError(rc, f"ktg_create(device={device}) failed")
        self.h = h
        self.device = device
        self._mode = _lib.KTG_PTR_HOST
        self._keep = None
        self.nl = None

    def close(self):
        if getattr(self, "h", None):
            self.lib.ktg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- plumbing --------------------------------------------------------------
    def _check(self, rc: int):
        if rc != 0:
            raise KtgError(rc, self.lib.ktg_last_error(self.h).decode())

    def set_stream(self, stream_handle: int):
        self._check(self.lib.ktg_set_stream(self.h, ctypes.c_void_p(stream_handle)))

    def _set_mode(self, mode: int):
        if mode != self._mode:
            self._check(self.lib.ktg_set_pointer_mode(self.h, mode))
            self._mode = mode

    def set_option(self, key: str, value: int):
        self._check(self.lib.ktg_set_option(self.h, key.encode(), int(value)))

    @property
    def launches(self) -> int:
        return int(self.lib.ktg_launch_count(self.h))

    # -- netlist -----------------------------------------------------------------
    def upload_netlist(self, nl):
        k = dict(
            mov_vertex=_c(nl.mov_vertex, np.int32), var_of_vertex=_c(nl.var_of_vertex, np.int32),
            fixed_x=_c(nl.fixed_x, np.float64), fixed_y=_c(nl.fixed_y, np.float64),
            net_start=_c(nl.net_start, np.int64), pin_cell=_c(nl.pin_cell, np.int32),
            off_x=_c(nl.off_x, np.float64), off_y=_c(nl.off_y, np.float64),
            net_weight=_c(nl.net_weight, np.float64), pin_start=_c(nl.pin_start, np.int64),
            pin_net=_c(nl.pin_net, np.int32), pin_q=_c(nl.pin_q, np.int32),
            width=_c(nl.width, np.float64), height=_c(nl.height, np.float64))

        def p(name, t):
            return k[name].ctypes.data_as(ctypes.POINTER(t))
        i32, i64, f64 = ctypes.c_int32, ctypes.c_int64, ctypes.c_double
        v = NetlistView(nl.num_vertices, nl.num_movable, nl.num_nets, p("mov_vertex", i32),
                        p("var_of_vertex", i32), p("fixed_x", f64), p("fixed_y", f64),
                        p("net_start", i64), p("pin_cell", i32), p("off_x", f64),
                        p("off_y", f64), p("net_weight", f64), p("pin_start", i64),
                        p("pin_net", i32), p("pin_q", i32), p("width", f64), p("height", f64))
        self._check(self.lib.ktg_upload_netlist(self.h, ctypes.byref(v)))
        self.nl = nl

    # -- B2B ---------------------------------------------------------------------
    def build_b2b(self, x, y, alpha, ax=None, ay=None, floor_x=1.0, floor_y=1.0):
        self._set_mode(_lib.KTG_PTR_HOST)
        x, y = _c(x, np.float64), _c(y, np.float64)
        ax = None if ax is None else _c(ax, np.float64)
        ay = None if ay is None else _c(ay, np.float64)
        self._check(self.lib.ktg_build_b2b(self.h, _ptr(x), _ptr(y), alpha, _ptr(ax), _ptr(ay),
                                           floor_x, floor_y))

    def build_kraftwerk2(self, x, y, with_rhs: bool, floor_x: float, floor_y: float):
        """Kraftwerk2's buildSystem for both axes (host mode)."""
        self._set_mode(_lib.KTG_PTR_HOST)
        x, y = _c(x, np.float64), _c(y, np.float64)
        self._check(self.lib.ktg_build_b2b_kraftwerk2(self.h, _ptr(x), _ptr(y), int(with_rhs),
                                                      floor_x, floor_y))

    def build_kraftwerk2_dev(self, x, y, with_rhs: bool, floor_x: float, floor_y: float):
        self._set_mode(_lib.KTG_PTR_DEVICE)
        self._check(self.lib.ktg_build_b2b_kraftwerk2(self.h, _tptr(x), _tptr(y), int(with_rhs),
                                                      floor_x, floor_y))

    def kraftwerk2_adjust_dev(self, move_weight=None, toward_x=None, toward_y=None,
                              diag_floor: float = 0.0):
        self._set_mode(_lib.KTG_PTR_DEVICE)
        self._check(self.lib.ktg_kraftwerk2_adjust(self.h, _tptr(move_weight), _tptr(toward_x),
                                                   _tptr(toward_y), diag_floor))

    def kraftwerk2_adjust(self, move_weight=None, toward_x=None, toward_y=None,
                          diag_floor: float = 0.0):
        self._set_mode(_lib.KTG_PTR_HOST)
        mw = None if move_weight is None else _c(move_weight, np.float64)
        tx = None if toward_x is None else _c(toward_x, np.float64)
        ty = None if toward_y is None else _c(toward_y, np.float64)
        self._check(self.lib.ktg_kraftwerk2_adjust(self.h, _ptr(mw), _ptr(tx), _ptr(ty),
                                                   diag_floor))

    def build_b2b_dev(self, x, y, alpha, ax=None, ay=None, floor_x=1.0, floor_y=1.0):
        self._set_mode(_lib.KTG_PTR_DEVICE)
        self._check(self.lib.ktg_build_b2b(self.h, _tptr(x), _tptr(y), alpha, _tptr(ax),
                                           _tptr(ay), floor_x, floor_y))

    def build_star(self) -> int:
        """LinearSystems::buildStar on the GPU; returns the system size."""
        size = ctypes.c_int64()
        self._check(self.lib.ktg_build_star(self.h, ctypes.byref(size)))
        return int(size.value)

    def build_hpwl(self) -> float:
        self._set_mode(_lib.KTG_PTR_HOST)
        out = ctypes.c_double()
        self._check(self.lib.ktg_build_hpwl(self.h, ctypes.byref(out)))
        return float(out.value)

    def build_hpwl_dev(self, out):
        self._set_mode(_lib.KTG_PTR_DEVICE)
        self._check(self.lib.ktg_build_hpwl(self.h, _tptr(out)))

    def system_info(self, axis: int):
        n, m = ctypes.c_int64(), ctypes.c_int64()
        self._check(self.lib.ktg_system_info(self.h, axis, ctypes.byref(n), ctypes.byref(m)))
        return int(n.value), int(m.value)

    def aggregates(self) -> dict:
        """Aggregation preconditioner of the current systems (built if needed):
        order [2n], meta [2n] and the block-inverse rows minv [2n, 8]."""
        n, _ = self.system_info(0)
        out = dict(order=np.zeros(max(2 * n, 1), np.int32), meta=np.zeros(max(2 * n, 1), np.int32),
                   minv=np.zeros((max(2 * n, 1), 8), np.float32))
        P = ctypes.POINTER
        self._check(self.lib.ktg_download_aggregates(
            self.h, out["order"].ctypes.data_as(P(ctypes.c_int32)),
            out["meta"].ctypes.data_as(P(ctypes.c_int32)),
            out["minv"].ctypes.data_as(P(ctypes.c_float))))
        return {k: v[:2 * n] for k, v in out.items()}

    def coarse(self) -> dict:
        """Coarse correction of the aggregation preconditioner (option
        "coarse" > 0): z and A z per permuted row [2n], 1 / (z^T A z) per axis."""
        n, _ = self.system_info(0)
        z = np.zeros(max(2 * n, 1), np.float32)
        az = np.zeros(max(2 * n, 1), np.float32)
        einv = np.zeros(2)
        P = ctypes.POINTER
        self._check(self.lib.ktg_download_coarse(self.h, z.ctypes.data_as(P(ctypes.c_float)),
                                                 az.ctypes.data_as(P(ctypes.c_float)),
                                                 einv.ctypes.data_as(P(ctypes.c_double))))
        return dict(z=z[:2 * n], az=az[:2 * n], einv=einv)

    def mixed_trace(self, cap: int) -> np.ndarray:
        """Phase stamps of the last mixed solve (option "mixed_trace"): rows
        of (tag, ns)."""
        w = np.zeros(cap, np.uint64)
        self._check(self.lib.ktg_download_mixed_trace(self.h, ctypes.c_void_p(w.ctypes.data), cap))
        w = w[w != 0]
        return np.stack([w >> np.uint64(56), w & np.uint64((1 << 56) - 1)], 1).astype(np.int64)

    def system(self, axis: int) -> dict:
        n, m = self.system_info(axis)
        s = dict(row_ptr=np.zeros(n + 1, np.int64), col=np.zeros(max(m, 1), np.int32),
                 val=np.zeros(max(m, 1)), diag=np.zeros(max(n, 1)), rhs=np.zeros(max(n, 1)))
        P = ctypes.POINTER
        self._check(self.lib.ktg_download_system(
            self.h, axis, s["row_ptr"].ctypes.data_as(P(ctypes.c_int64)),
            s["col"].ctypes.data_as(P(ctypes.c_int32)), s["val"].ctypes.data_as(P(ctypes.c_double)),
            s["diag"].ctypes.data_as(P(ctypes.c_double)),
            s["rhs"].ctypes.data_as(P(ctypes.c_double))))
        s["col"], s["val"] = s["col"][:m], s["val"][:m]
        s["diag"], s["rhs"] = s["diag"][:n], s["rhs"][:n]
        return s

    def bound_pins(self, axis: int):
        N = self.nl.num_nets
        lo = np.zeros(max(N, 1), np.uint32)
        hi = np.zeros(max(N, 1), np.uint32)
        P = ctypes.POINTER(ctypes.c_uint32)
        self._check(self.lib.ktg_download_bound_pins(self.h, axis, lo.ctypes.data_as(P),
                                                     hi.ctypes.data_as(P)))
        return lo[:N], hi[:N]

    def upload_system(self, axis: int, s: dict):
        rp = _c(s["row_ptr"], np.int64)
        col = _c(s["col"], np.int32)
        val, diag, rhs = (_c(s[k], np.float64) for k in ("val", "diag", "rhs"))
        P = ctypes.POINTER
        self._check(self.lib.ktg_upload_system(
            self.h, axis, diag.shape[0], rp.ctypes.data_as(P(ctypes.c_int64)),
            col.ctypes.data_as(P(ctypes.c_int32)), val.ctypes.data_as(P(ctypes.c_double)),
            diag.ctypes.data_as(P(ctypes.c_double)), rhs.ctypes.data_as(P(ctypes.c_double))))

    # -- PCG ---------------------------------------------------------------------
    def solve(self, x, y, tol: float, max_iter: int, hist_cap: int = 0,
              inplace: bool = False) -> dict:
        """Host-mode solve; returns new x, y, residuals and iteration counts.
        With ``inplace`` the given float64 arrays are updated directly (e.g.
        pinned buffers); otherwise copies are solved and returned."""
        self._set_mode(_lib.KTG_PTR_HOST)
        if inplace:
            for a in (x, y):
                if a.dtype != np.float64 or not a.flags["C_CONTIGUOUS"]:
                    raise ValueError("inplace solve needs contiguous float64 arrays")
        else:
            x, y = _c(x, np.float64).copy(), _c(y, np.float64).copy()
        info = SolveInfo()
        hx = np.zeros(hist_cap) if hist_cap else None
        hy = np.zeros(hist_cap) if hist_cap else None
        self._check(self.lib.ktg_solve(self.h, _ptr(x), _ptr(y), tol, max_iter,
                                       ctypes.byref(info), _ptr(hx), _ptr(hy), hist_cap))
        k = int(info.iters)
        return dict(x=x, y=y, resid=(info.resid_x, info.resid_y), iters=k,
                    iters_x=int(info.iters_x), iters_y=int(info.iters_y), live=int(info.live),
                    hist_x=None if hx is None else hx[:min(k, hist_cap)],
                    hist_y=None if hy is None else hy[:min(k, hist_cap)])

    def solve_dev(self, x, y, tol: float, max_iter: int, info=None, hist_x=None, hist_y=None,
                  hist_cap: int = 0):
        """Device-mode solve: x, y (and info: a uint8 tensor of
        ctypes.sizeof(SolveInfo) bytes) are CUDA tensors updated in place."""
        self._set_mode(_lib.KTG_PTR_DEVICE)
        self._check(self.lib.ktg_solve(self.h, _tptr(x), _tptr(y), tol, max_iter, _tptr(info),
                                       _tptr(hist_x), _tptr(hist_y), hist_cap))

    def solve_mixed(self, x, y, tol: float, inner_tol: float = 1e-3, max_inner: int = 100000,
                    max_outer: int = 50, hist_cap: int = 0, inplace: bool = False) -> dict:
        """FP32 Jacobi-PCG inside FP64 iterative refinement (host mode)."""
        self._set_mode(_lib.KTG_PTR_HOST)
        if not inplace:
            x, y = _c(x, np.float64).copy(), _c(y, np.float64).copy()
        info = MixedInfo()
        hx = np.zeros(hist_cap) if hist_cap else None
        hy = np.zeros(hist_cap) if hist_cap else None
        self._check(self.lib.ktg_solve_mixed(self.h, _ptr(x), _ptr(y), tol, inner_tol, max_inner,
                                             max_outer, ctypes.byref(info), _ptr(hx), _ptr(hy),
                                             hist_cap))
        k = max(info.outer_x, info.outer_y)
        return dict(x=x, y=y, resid=(info.resid_x, info.resid_y),
                    inner=(int(info.inner_x), int(info.inner_y)),
                    outer=(int(info.outer_x), int(info.outer_y)), stalled=int(info.stalled),
                    fp64_iters=(int(info.fp64_iters_x), int(info.fp64_iters_y)),
                    hist_x=None if hx is None else hx[:min(k, hist_cap)],
                    hist_y=None if hy is None else hy[:min(k, hist_cap)])

    def solve_mixed_dev(self, x, y, tol: float, inner_tol: float = 1e-3,
                        max_inner: int = 100000, max_outer: int = 50, info=None):
        self._set_mode(_lib.KTG_PTR_DEVICE)
        self._check(self.lib.ktg_solve_mixed(self.h, _tptr(x), _tptr(y), tol, inner_tol,
                                             max_inner, max_outer, _tptr(info), None, None, 0))

    # -- HPWL / density ------------------------------------------------------------
    def hpwl(self, x, y) -> float:
        self._set_mode(_lib.KTG_PTR_HOST)
        x, y = _c(x, np.float64), _c(y, np.float64)
        out = ctypes.c_double()
        self._check(self.lib.ktg_hpwl(self.h, _ptr(x), _ptr(y), ctypes.byref(out)))
        return float(out.value)

    def spmv(self, axis: int, v) -> np.ndarray:
        """A v for the system of `axis` from the last build (host mode):
        SparseSystem::multiply's row sums, bit for bit."""
        self._set_mode(_lib.KTG_PTR_HOST)
        v = _c(v, np.float64)
        out = np.empty_like(v)
        self._check(self.lib.ktg_spmv(self.h, axis, _ptr(v), _ptr(out)))
        return out

    def spmv_dev(self, axis: int, v, out):
        self._set_mode(_lib.KTG_PTR_DEVICE)
        self._check(self.lib.ktg_spmv(self.h, axis, _tptr(v), _tptr(out)))

    def hpwl_dev(self, x, y, out):
        self._set_mode(_lib.KTG_PTR_DEVICE)
        self._check(self.lib.ktg_hpwl(self.h, _tptr(x), _tptr(y), _tptr(out)))

    def set_grid(self, g):
        self._grid_avail = _c(g.avail, np.float64)
        v = GridView(g.origin_x, g.origin_y, g.dx, g.dy, g.nx, g.ny,
                     self._grid_avail.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                     g.total_avail, g.density_limit)
        self._check(self.lib.ktg_set_grid(self.h, ctypes.byref(v)))
        self.grid = g

    def occupancy(self, x, y, want_map: bool = True):
        self._set_mode(_lib.KTG_PTR_HOST)
        x, y = _c(x, np.float64), _c(y, np.float64)
        occ = np.zeros(self.grid.size) if want_map else None
        ov = ctypes.c_double()
        self._check(self.lib.ktg_occupancy(self.h, _ptr(x), _ptr(y), _ptr(occ), ctypes.byref(ov)))
        return occ, float(ov.value)

    def occupancy_dev(self, x, y, occ, overflow):
        self._set_mode(_lib.KTG_PTR_DEVICE)
        self._check(self.lib.ktg_occupancy(self.h, _tptr(x), _tptr(y), _tptr(occ),
                                           _tptr(overflow)))

    def set_free_space(self, fs):
        """Installs a ``grid.FreeSpace`` (rows, spans, obstacles, die) for
        ``lal``."""
        self._fs = (_c(fs.row_y, np.float64), _c(fs.row_span, np.int64),
                    _c(fs.spans, np.float64), _c(fs.obstacles, np.float64),
                    _c(np.asarray(fs.die, np.float64), np.float64))
        ry, rs, sp, ob, die = self._fs
        self._check(self.lib.ktg_set_free_space(self.h, ry.shape[0], _ptr(ry), _ptr(rs), _ptr(sp),
                                                ob.shape[0], _ptr(ob), _ptr(die)))

    def lal(self, x, y, max_level: int = 20, min_cells_to_split: int = 4,
            stripe_area_fraction: float = 0.1):
        """LookAheadLegalizer::legalize on host positions; returns new (x, y)."""
        self._set_mode(_lib.KTG_PTR_HOST)
        x = _c(x, np.float64).copy()
        y = _c(y, np.float64).copy()
        self._check(self.lib.ktg_lal(self.h, _ptr(x), _ptr(y), max_level, min_cells_to_split,
                                     stripe_area_fraction))
        return x, y

    def lal_stats(self) -> dict:
        out = np.zeros(16)
        self._check(self.lib.ktg_lal_stats(self.h, _ptr(out), 16))
        keys = ("batches", "regions", "levels", "syncs", "blocks", "ms_bisect", "ms_refresh",
                "ms_total", "ms_subtree", "big_levels", "subtree_blocks", "subtree_handed_back",
                "back_size_or_obstacles", "back_sub_blocks", "back_sort_buffer", "back_stripes")
        return dict(zip(keys, out.tolist()))

    def lal_dev(self, x, y, max_level: int = 20, min_cells_to_split: int = 4,
                stripe_area_fraction: float = 0.1):
        """In place on device tensors x, y."""
        self._set_mode(_lib.KTG_PTR_DEVICE)
        self._check(self.lib.ktg_lal(self.h, _tptr(x), _tptr(y), max_level, min_cells_to_split,
                                     stripe_area_fraction))


class Batch:
    """Owns a ``ktg_batch``: many independent systems solved in one
    persistent cluster launch (see include/ktplace_b200.h)."""

    def __init__(self, device: int = 0):
        self.lib = _lib.load()
        h = ctypes.c_void_p()
        rc = self.lib.ktg_batch_create(device, ctypes.byref(h))
        if rc != 0:
            raise KtgError(rc, f"ktg_batch_create(device={device}) failed")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.lib.ktg_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, rc: int):
        if rc != 0:
            raise KtgError(rc, self.lib.ktg_batch_last_error(self.h).decode())

    def __len__(self):
        return int(self.lib.ktg_batch_size(self.h))

    def set_stream(self, stream_handle: int):
        self._check(self.lib.ktg_batch_set_stream(self.h, ctypes.c_void_p(stream_handle)))

    def add_system(self, s: dict, x0) -> int:
        rp = _c(s["row_ptr"], np.int64)
        col = _c(s["col"], np.int32)
        val, diag, rhs = (_c(s[k], np.float64) for k in ("val", "diag", "rhs"))
        x0 = _c(x0, np.float64)
        P = ctypes.POINTER
        sid = ctypes.c_int64()
        self._check(self.lib.ktg_batch_add_system(
            self.h, diag.shape[0], rp.ctypes.data_as(P(ctypes.c_int64)),
            col.ctypes.data_as(P(ctypes.c_int32)), val.ctypes.data_as(P(ctypes.c_double)),
            diag.ctypes.data_as(P(ctypes.c_double)), rhs.ctypes.data_as(P(ctypes.c_double)),
            x0.ctypes.data_as(P(ctypes.c_double)), ctypes.byref(sid)))
        return int(sid.value)

    def add_from_context(self, ctx: Context, x0, y0) -> int:
        x0, y0 = _c(x0, np.float64), _c(y0, np.float64)
        P = ctypes.POINTER(ctypes.c_double)
        sid = ctypes.c_int64()
        self._check(self.lib.ktg_batch_add_from_context(self.h, ctx.h, x0.ctypes.data_as(P),
                                                        y0.ctypes.data_as(P), ctypes.byref(sid)))
        return int(sid.value)

    def set_shape(self, cluster: int, threads: int):
        self._check(self.lib.ktg_batch_set_shape(self.h, cluster, threads))

    def shape(self):
        c, t = ctypes.c_int(), ctypes.c_int()
        self._check(self.lib.ktg_batch_get_shape(self.h, ctypes.byref(c), ctypes.byref(t)))
        return int(c.value), int(t.value)

    def autotune(self, tol: float, precision: int = 1, inner_tol: float = 1e-3,
                 probe_iter: int = 40):
        c, t, ms = ctypes.c_int(), ctypes.c_int(), ctypes.c_float()
        self._check(self.lib.ktg_batch_autotune(self.h, tol, precision, inner_tol, probe_iter,
                                                ctypes.byref(c), ctypes.byref(t),
                                                ctypes.byref(ms)))
        return int(c.value), int(t.value), float(ms.value)

    def set_split(self, rows: int, cluster: int = 16, threads: int = 1024, clusters: int = 1):
        """Systems of >= rows rows go to a concurrent launch of `clusters`
        clusters of cluster x threads (rows 0: no split)."""
        self._check(self.lib.ktg_batch_set_split(self.h, rows, cluster, threads, clusters))

    def split(self) -> dict:
        r, c, t, n, nl = (ctypes.c_int64(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int(),
                          ctypes.c_int())
        self._check(self.lib.ktg_batch_get_split(self.h, ctypes.byref(r), ctypes.byref(c),
                                                 ctypes.byref(t), ctypes.byref(n),
                                                 ctypes.byref(nl)))
        return dict(rows=int(r.value), cluster=int(c.value), threads=int(t.value),
                    clusters=int(n.value), num_large=int(nl.value))

    def autotune_split(self, tol: float, precision: int = 1, inner_tol: float = 1e-3,
                       max_iter: int = 100000):
        """Picks the size split by timing full solves; returns
        (split dict, unsplit ms, kept ms)."""
        base, best = ctypes.c_float(), ctypes.c_float()
        self._check(self.lib.ktg_batch_autotune_split(self.h, tol, precision, inner_tol, max_iter,
                                                      ctypes.byref(base), ctypes.byref(best)))
        return self.split(), float(base.value), float(best.value)

    def set_offload(self, rows: int, precond: int = 2, coarse: int = 0):
        """Pairs of consecutive equal-size systems of >= rows rows are solved
        on the whole GPU before the cluster launches (rows 0: off)."""
        self._check(self.lib.ktg_batch_set_offload(self.h, rows, precond, coarse))

    def offload(self) -> dict:
        r, k = ctypes.c_int64(), ctypes.c_int()
        self._check(self.lib.ktg_batch_get_offload(self.h, ctypes.byref(r), ctypes.byref(k)))
        return dict(rows=int(r.value), pairs=int(k.value))

    def autotune_offload(self, tol: float, precision: int = 1, inner_tol: float = 1e-3,
                         max_iter: int = 100000):
        """Picks the whole-GPU threshold by timing full solves; returns
        (offload dict, ms without, kept ms)."""
        base, best = ctypes.c_float(), ctypes.c_float()
        self._check(self.lib.ktg_batch_autotune_offload(self.h, tol, precision, inner_tol,
                                                        max_iter, ctypes.byref(base),
                                                        ctypes.byref(best)))
        return self.offload(), float(base.value), float(best.value)

    def reset_x(self):
        self._check(self.lib.ktg_batch_reset_x(self.h))

    def solve(self, tol: float, max_iter: int = 100000, precision: int = 0,
              inner_tol: float = 1e-3):
        """Enqueues the batch solve (asynchronous)."""
        self._check(self.lib.ktg_batch_solve(self.h, tol, max_iter, precision, inner_tol))

    def results(self):
        n = len(self)
        arr = (_lib.BatchResult * max(n, 1))()
        self._check(self.lib.ktg_batch_results(self.h, ctypes.cast(arr, ctypes.c_void_p)))
        return [dict(iters=int(r.iters), outer=int(r.outer), status=int(r.status),
                     resid=float(r.resid), latency_ns=int(r.latency_ns)) for r in arr[:n]]

    def get_x(self, sid: int, n: int) -> np.ndarray:
        x = np.zeros(max(n, 1))
        self._check(self.lib.ktg_batch_get_x(self.h, sid,
                                             x.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return x[:n]

    @property
    def launches(self) -> int:
        return int(self.lib.ktg_batch_launch_count(self.h))
