"""Oracle for the SimPL quadratic-solve path (test infrastructure only).

Two checkers live here, both CPU-only:

* ``RefDesign`` drives ``_ref/libktref.so``: the reference's own SimPL sources
  compiled unmodified (see Makefile, ref_harness.cc). Built only where the
  reference tree is present; the built library travels with the repository
  snapshot.
* ``port`` drives ``_build/libktp_oracle.so``: ktp_oracle.c, a plain-C
  restatement of the same functions, pinned against ``RefDesign`` and against
  the committed golden vectors in tests/golden/.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg may
import this package. The CUDA product never does and has no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(HERE, "_ref", "libktref.so")
# The reference's SimPL linked with the ktplace_b200 drop-in (GPU path).
REF_GPU_LIB = os.path.join(HERE, "_ref", "libktref_gpu.so")
PORT_LIB = os.path.join(HERE, "_build", "libktp_oracle.so")

_u64p = ctypes.POINTER(ctypes.c_uint64)
_u32p = ctypes.POINTER(ctypes.c_uint32)
_i32p = ctypes.POINTER(ctypes.c_int32)
_i64p = ctypes.POINTER(ctypes.c_int64)
_f64p = ctypes.POINTER(ctypes.c_double)
_vp = ctypes.c_void_p


def _p(a, t):
    if a is None:
        return None
    return a.ctypes.data_as(t)


def _c(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


_refs = {}


def ref_available(variant: str = "cpu") -> bool:
    return os.path.exists(REF_LIB if variant == "cpu" else REF_GPU_LIB)


def load_ref(variant: str = "cpu"):
    if variant not in _refs:
        lib = ctypes.CDLL(REF_LIB if variant == "cpu" else REF_GPU_LIB)
        lib.ref_set_threads.argtypes = [ctypes.c_int]
        lib.ref_set_threads.restype = ctypes.c_int
        lib.ref_last_error.argtypes = [_vp]
        lib.ref_last_error.restype = ctypes.c_char_p
        lib.ref_design_load_bookshelf.argtypes = [ctypes.c_char_p]
        lib.ref_design_load_bookshelf.restype = _vp
        lib.ref_design_from_arrays.argtypes = [
            ctypes.c_uint64, ctypes.c_uint64, _u32p, _f64p, _f64p, ctypes.c_uint64, _u64p, _u32p,
            _f64p, _f64p, _f64p, _f64p, _f64p, ctypes.c_uint64, _f64p, ctypes.c_uint64, _f64p,
            _f64p]
        lib.ref_design_from_arrays.restype = _vp
        lib.ref_design_free.argtypes = [_vp]
        lib.ref_netlist_sizes.argtypes = [_vp, _u64p]
        lib.ref_netlist_export.argtypes = [_vp, _u32p, _u32p, _f64p, _f64p, _u64p, _u32p, _f64p,
                                           _f64p, _f64p, _u64p, _u32p, _u32p, _f64p, _f64p,
                                           _f64p, _f64p, _f64p]
        lib.ref_floors.argtypes = [_vp, _f64p, _f64p]
        lib.ref_build_b2b.argtypes = [_vp, _f64p, _f64p, ctypes.c_double, _f64p, _f64p,
                                      ctypes.c_double, ctypes.c_double]
        lib.ref_build_star.argtypes = [_vp, _u64p]
        lib.ref_system_sizes.argtypes = [_vp, ctypes.c_int, _u64p, _u64p]
        lib.ref_system_export.argtypes = [_vp, ctypes.c_int, _u64p, _u32p, _f64p, _f64p, _f64p]
        lib.ref_system_import.argtypes = [_vp, ctypes.c_int, ctypes.c_uint64, _u64p, _u32p,
                                          _f64p, _f64p, _f64p]
        lib.ref_solve.argtypes = [_vp, _f64p, _f64p, ctypes.c_double, ctypes.c_uint64, _f64p,
                                  _f64p, _f64p, ctypes.c_uint64, _u64p]
        lib.ref_hpwl.argtypes = [_vp, _f64p, _f64p]
        lib.ref_hpwl.restype = ctypes.c_double
        lib.ref_grid.argtypes = [_vp, ctypes.c_uint64, ctypes.c_double, _f64p, _f64p]
        lib.ref_occupancy.argtypes = [_vp, _f64p, _f64p, _f64p, _f64p]
        lib.ref_run_simpl.argtypes = [_vp, _f64p, ctypes.c_char_p, _f64p, _f64p]
        for f in ("ref_netlist_sizes", "ref_netlist_export", "ref_floors", "ref_build_b2b",
                  "ref_build_star", "ref_system_sizes", "ref_system_export",
                  "ref_system_import", "ref_solve", "ref_grid", "ref_occupancy", "ref_run_simpl"):
            getattr(lib, f).restype = ctypes.c_int
        _refs[variant] = lib
    return _refs[variant]


class RefDesign:
    """One design inside the reference's SimPL data structures."""

    def __init__(self, handle, variant: str = "cpu"):
        if not handle:
            raise RuntimeError("reference design could not be created")
        self.h = handle
        self.lib = load_ref(variant)
        s = (ctypes.c_uint64 * 8)()
        self.lib.ref_netlist_sizes(self.h, s)
        (self.V, self.n, self.N, self.P, self.Pm, self.num_fixed, self.num_obstacles,
         self.num_rows) = [int(v) for v in s]

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.ref_design_free(self.h)
            self.h = None

    @classmethod
    def from_bookshelf(cls, directory: str, variant: str = "cpu") -> "RefDesign":
        lib = load_ref(variant)
        return cls(lib.ref_design_load_bookshelf(directory.encode()), variant)

    @classmethod
    def from_netlist(cls, nl, variant: str = "cpu") -> "RefDesign":
        lib = load_ref(variant)
        mv = _c(nl.mov_vertex, np.uint32)
        fx, fy = _c(nl.fixed_x, np.float64), _c(nl.fixed_y, np.float64)
        ns = _c(nl.net_start, np.uint64)
        pc = _c(nl.pin_cell, np.uint32)
        ox, oy = _c(nl.off_x, np.float64), _c(nl.off_y, np.float64)
        w = _c(nl.net_weight, np.float64)
        cw, ch = _c(nl.width, np.float64), _c(nl.height, np.float64)
        ob = _c(nl.obstacles.reshape(-1), np.float64)
        rw = _c(nl.rows.reshape(-1), np.float64)
        die = _c(np.array(nl.die, dtype=np.float64), np.float64)
        h = lib.ref_design_from_arrays(
            nl.num_vertices, nl.num_movable, _p(mv, _u32p), _p(fx, _f64p), _p(fy, _f64p),
            nl.num_nets, _p(ns, _u64p), _p(pc, _u32p), _p(ox, _f64p), _p(oy, _f64p),
            _p(w, _f64p), _p(cw, _f64p), _p(ch, _f64p), nl.obstacles.shape[0], _p(ob, _f64p),
            nl.rows.shape[0], _p(rw, _f64p), _p(die, _f64p))
        return cls(h, variant)

    def export(self) -> dict:
        o = dict(
            mov_vertex=np.zeros(self.n, np.uint32), var_of_vertex=np.zeros(self.V, np.uint32),
            fixed_x=np.zeros(self.V), fixed_y=np.zeros(self.V),
            net_start=np.zeros(self.N + 1, np.uint64), pin_cell=np.zeros(self.P, np.uint32),
            off_x=np.zeros(self.P), off_y=np.zeros(self.P), net_weight=np.zeros(self.N),
            pin_start=np.zeros(self.n + 1, np.uint64), pin_net=np.zeros(self.Pm, np.uint32),
            pin_q=np.zeros(self.Pm, np.uint32), width=np.zeros(self.n), height=np.zeros(self.n),
            die=np.zeros(4), obstacles=np.zeros((self.num_obstacles, 4)),
            rows=np.zeros((self.num_rows, 5)))
        self.lib.ref_netlist_export(
            self.h, _p(o["mov_vertex"], _u32p), _p(o["var_of_vertex"], _u32p),
            _p(o["fixed_x"], _f64p), _p(o["fixed_y"], _f64p), _p(o["net_start"], _u64p),
            _p(o["pin_cell"], _u32p), _p(o["off_x"], _f64p), _p(o["off_y"], _f64p),
            _p(o["net_weight"], _f64p), _p(o["pin_start"], _u64p), _p(o["pin_net"], _u32p),
            _p(o["pin_q"], _u32p), _p(o["width"], _f64p), _p(o["height"], _f64p),
            _p(o["die"], _f64p), _p(o["obstacles"], _f64p), _p(o["rows"], _f64p))
        return o

    def floors(self):
        fx, fy = ctypes.c_double(), ctypes.c_double()
        self.lib.ref_floors(self.h, ctypes.byref(fx), ctypes.byref(fy))
        return fx.value, fy.value

    def _check(self, rc):
        if rc != 0:
            raise RuntimeError(self.lib.ref_last_error(self.h).decode())

    def build_b2b(self, x, y, alpha, ax=None, ay=None, floor_x=0.0, floor_y=0.0):
        x, y = _c(x, np.float64), _c(y, np.float64)
        ax = None if ax is None else _c(ax, np.float64)
        ay = None if ay is None else _c(ay, np.float64)
        self._check(self.lib.ref_build_b2b(self.h, _p(x, _f64p), _p(y, _f64p), alpha,
                                           _p(ax, _f64p), _p(ay, _f64p), floor_x, floor_y))

    def build_star(self) -> int:
        s = ctypes.c_uint64()
        self._check(self.lib.ref_build_star(self.h, ctypes.byref(s)))
        return int(s.value)

    def system(self, axis: int) -> dict:
        n, m = ctypes.c_uint64(), ctypes.c_uint64()
        self.lib.ref_system_sizes(self.h, axis, ctypes.byref(n), ctypes.byref(m))
        n, m = int(n.value), int(m.value)
        s = dict(row_ptr=np.zeros(n + 1, np.uint64), col=np.zeros(m, np.uint32),
                 val=np.zeros(m), diag=np.zeros(n), rhs=np.zeros(n))
        self.lib.ref_system_export(self.h, axis, _p(s["row_ptr"], _u64p), _p(s["col"], _u32p),
                                   _p(s["val"], _f64p), _p(s["diag"], _f64p),
                                   _p(s["rhs"], _f64p))
        return s

    def set_system(self, axis: int, s: dict):
        rp = _c(s["row_ptr"], np.uint64)
        col = _c(s["col"], np.uint32)
        val, diag, rhs = (_c(s[k], np.float64) for k in ("val", "diag", "rhs"))
        self.lib.ref_system_import(self.h, axis, diag.shape[0], _p(rp, _u64p), _p(col, _u32p),
                                   _p(val, _f64p), _p(diag, _f64p), _p(rhs, _f64p))

    def solve(self, x, y, tol, max_iter, hist_cap=0):
        x, y = _c(x, np.float64).copy(), _c(y, np.float64).copy()
        r = np.zeros(2)
        hx = np.zeros(hist_cap) if hist_cap else None
        hy = np.zeros(hist_cap) if hist_cap else None
        it = ctypes.c_uint64()
        self._check(self.lib.ref_solve(self.h, _p(x, _f64p), _p(y, _f64p), tol, max_iter,
                                       _p(r, _f64p), _p(hx, _f64p), _p(hy, _f64p), hist_cap,
                                       ctypes.byref(it)))
        k = int(it.value)
        return dict(x=x, y=y, resid=(float(r[0]), float(r[1])), iters=k,
                    hist_x=None if hx is None else hx[:min(k, hist_cap)],
                    hist_y=None if hy is None else hy[:min(k, hist_cap)])

    def hpwl(self, x, y) -> float:
        x, y = _c(x, np.float64), _c(y, np.float64)
        return float(self.lib.ref_hpwl(self.h, _p(x, _f64p), _p(y, _f64p)))

    def grid(self, per_axis: int, density_limit: float = 1.0):
        info = np.zeros(7)
        self._check(self.lib.ref_grid(self.h, per_axis, density_limit, _p(info, _f64p), None))
        nx, ny = int(info[4]), int(info[5])
        avail = np.zeros(nx * ny)
        self._check(self.lib.ref_grid(self.h, per_axis, density_limit, _p(info, _f64p),
                                      _p(avail, _f64p)))
        return dict(origin=(info[0], info[1]), dx=info[2], dy=info[3], nx=nx, ny=ny,
                    total_avail=info[6], avail=avail)

    def lal(self, x, y):
        """The reference's look-ahead legalization on the grid of the last
        grid() call; returns the new (x, y)."""
        lib = self.lib
        if not hasattr(lib, "_lal_ready"):
            lib.ref_lal.argtypes = [_vp, _f64p, _f64p]
            lib.ref_lal.restype = ctypes.c_int
            lib.ref_free_space.argtypes = [_vp, _u64p, _f64p, _u64p, _f64p]
            lib.ref_free_space.restype = ctypes.c_int
            lib._lal_ready = True
        x, y = _c(x, np.float64).copy(), _c(y, np.float64).copy()
        self._check(lib.ref_lal(self.h, _p(x, _f64p), _p(y, _f64p)))
        return x, y

    def free_space(self):
        """FreeSpace rows of the last grid() call: rows [R, 2] (y0, y1),
        row_span [R + 1], spans [S, 2] (x0, x1)."""
        self.lal.__func__  # argtypes are set up by lal()
        lib = self.lib
        if not hasattr(lib, "_lal_ready"):
            self.lal(np.zeros(self.n), np.zeros(self.n))
        counts = np.zeros(2, np.uint64)
        self._check(lib.ref_free_space(self.h, _p(counts, _u64p), None, None, None))
        R, S = int(counts[0]), int(counts[1])
        rows = np.zeros((max(R, 1), 2))
        rs = np.zeros(R + 1, np.uint64)
        spans = np.zeros((max(S, 1), 2))
        self._check(lib.ref_free_space(self.h, _p(counts, _u64p), _p(rows, _f64p), _p(rs, _u64p),
                                       _p(spans, _f64p)))
        return rows[:R], rs.astype(np.int64), spans[:S]

    def occupancy_map(self, x, y, nbins: int):
        x, y = _c(x, np.float64), _c(y, np.float64)
        occ = np.zeros(nbins)
        ov = ctypes.c_double()
        self._check(self.lib.ref_occupancy(self.h, _p(x, _f64p), _p(y, _f64p), _p(occ, _f64p),
                                           ctypes.byref(ov)))
        return occ, float(ov.value)


    def run_simpl(self, cg_tol=1e-4, cg_max_iter=60, max_iters=100, init_iters=15,
                  seed=20240607, alpha_base=0.02, bins=0, density=1.0, refine_iters=10,
                  init_net="star"):
        """Full SimPL (simplDM::run) on a copy of this design; returns the
        final look-ahead-legalized positions."""
        o = np.array([cg_tol, cg_max_iter, max_iters, init_iters, seed, alpha_base, bins,
                      density, refine_iters], dtype=np.float64)
        x = np.zeros(self.n)
        y = np.zeros(self.n)
        self._check(self.lib.ref_run_simpl(self.h, _p(o, _f64p), init_net.encode(),
                                           _p(x, _f64p), _p(y, _f64p)))
        return x, y


def set_ref_threads(n: int, variant: str = "cpu") -> int:
    return int(load_ref(variant).ref_set_threads(n))


# ---- the C restatement ---------------------------------------------------------

class _KtoNetlist(ctypes.Structure):
    _fields_ = [("num_vertices", ctypes.c_int64), ("num_movable", ctypes.c_int64),
                ("num_nets", ctypes.c_int64), ("mov_vertex", _i32p), ("var_of_vertex", _i32p),
                ("fixed_x", _f64p), ("fixed_y", _f64p), ("net_start", _i64p),
                ("pin_cell", _i32p), ("off_x", _f64p), ("off_y", _f64p),
                ("net_weight", _f64p), ("pin_start", _i64p), ("pin_net", _i32p),
                ("pin_q", _i32p)]


_port = None


def load_port():
    global _port
    if _port is None:
        lib = ctypes.CDLL(PORT_LIB)
        np_ = ctypes.POINTER(_KtoNetlist)
        lib.kto_b2b_axis.argtypes = [np_, ctypes.c_int, _f64p, ctypes.c_double, ctypes.c_double,
                                     _f64p, _u32p, _u32p, _i64p, _i32p, _f64p, ctypes.c_int64,
                                     _f64p, _f64p]
        lib.kto_b2b_axis.restype = ctypes.c_int
        lib.kto_pcg_axis.argtypes = [ctypes.c_int64, _i64p, _i32p, _f64p, _f64p, _f64p, _f64p,
                                     ctypes.c_double, ctypes.c_int64, _f64p, _i64p, _f64p,
                                     ctypes.c_int64]
        lib.kto_pcg_axis.restype = ctypes.c_int
        lib.kto_hpwl.argtypes = [np_, _f64p, _f64p]
        lib.kto_hpwl.restype = ctypes.c_double
        lib.kto_hpwl_terms.argtypes = [np_, _f64p, _f64p, _f64p]
        lib.kto_occupancy.argtypes = [ctypes.c_int64, _f64p, _f64p, _f64p, _f64p, _f64p,
                                      ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                      ctypes.c_double, ctypes.c_int64, ctypes.c_int64, _f64p]
        lib.kto_overflow.argtypes = [ctypes.c_int64, _f64p, _f64p, ctypes.c_double,
                                     ctypes.c_double]
        lib.kto_overflow.restype = ctypes.c_double
        lib.kto_dot.argtypes = [ctypes.c_int64, _f64p, _f64p]
        lib.kto_dot.restype = ctypes.c_double
        _port = lib
    return _port


class PortNetlist:
    """Holds contiguous copies of a Netlist's arrays for the C restatement."""

    def __init__(self, nl):
        self.nl = nl
        self._keep = dict(
            mov_vertex=_c(nl.mov_vertex, np.int32), var_of_vertex=_c(nl.var_of_vertex, np.int32),
            fixed_x=_c(nl.fixed_x, np.float64), fixed_y=_c(nl.fixed_y, np.float64),
            net_start=_c(nl.net_start, np.int64), pin_cell=_c(nl.pin_cell, np.int32),
            off_x=_c(nl.off_x, np.float64), off_y=_c(nl.off_y, np.float64),
            net_weight=_c(nl.net_weight, np.float64), pin_start=_c(nl.pin_start, np.int64),
            pin_net=_c(nl.pin_net, np.int32), pin_q=_c(nl.pin_q, np.int32))
        k = self._keep
        self.s = _KtoNetlist(
            nl.num_vertices, nl.num_movable, nl.num_nets, _p(k["mov_vertex"], _i32p),
            _p(k["var_of_vertex"], _i32p), _p(k["fixed_x"], _f64p), _p(k["fixed_y"], _f64p),
            _p(k["net_start"], _i64p), _p(k["pin_cell"], _i32p), _p(k["off_x"], _f64p),
            _p(k["off_y"], _f64p), _p(k["net_weight"], _f64p), _p(k["pin_start"], _i64p),
            _p(k["pin_net"], _i32p), _p(k["pin_q"], _i32p))
        self.lib = load_port()

    def b2b_axis(self, vertical: bool, pos, floor_len: float, alpha: float, anchor=None) -> dict:
        nl = self.nl
        pos = _c(pos, np.float64)
        anc = None if anchor is None else _c(anchor, np.float64)
        lo = np.zeros(nl.num_nets, np.uint32)
        hi = np.zeros(nl.num_nets, np.uint32)
        rp = np.zeros(nl.num_movable + 1, np.int64)
        rc = self.lib.kto_b2b_axis(ctypes.byref(self.s), int(vertical), _p(pos, _f64p), floor_len,
                                   alpha, _p(anc, _f64p), _p(lo, _u32p), _p(hi, _u32p),
                                   _p(rp, _i64p), None, None, 0, None, None)
        m = int(rp[-1])
        col = np.zeros(max(m, 1), np.int32)
        val = np.zeros(max(m, 1))
        diag = np.zeros(nl.num_movable)
        rhs = np.zeros(nl.num_movable)
        rc = self.lib.kto_b2b_axis(ctypes.byref(self.s), int(vertical), _p(pos, _f64p), floor_len,
                                   alpha, _p(anc, _f64p), _p(lo, _u32p), _p(hi, _u32p),
                                   _p(rp, _i64p), _p(col, _i32p), _p(val, _f64p), m,
                                   _p(diag, _f64p), _p(rhs, _f64p))
        if rc != 0:
            raise RuntimeError("kto_b2b_axis failed")
        return dict(lo=lo, hi=hi, row_ptr=rp, col=col[:m], val=val[:m], diag=diag, rhs=rhs)

    def hpwl(self, x, y) -> float:
        x, y = _c(x, np.float64), _c(y, np.float64)
        return float(self.lib.kto_hpwl(ctypes.byref(self.s), _p(x, _f64p), _p(y, _f64p)))

    def hpwl_terms(self, x, y):
        x, y = _c(x, np.float64), _c(y, np.float64)
        out = np.zeros(self.nl.num_nets)
        self.lib.kto_hpwl_terms(ctypes.byref(self.s), _p(x, _f64p), _p(y, _f64p),
                                _p(out, _f64p))
        return out


def port_pcg_axis(sys: dict, x, tol: float, max_iter: int, hist_cap: int = 0):
    lib = load_port()
    rp = _c(sys["row_ptr"], np.int64)
    col = _c(sys["col"], np.int32)
    val, diag, rhs = (_c(sys[k], np.float64) for k in ("val", "diag", "rhs"))
    x = _c(x, np.float64).copy()
    resid = ctypes.c_double()
    it = ctypes.c_int64()
    hist = np.zeros(hist_cap) if hist_cap else None
    rc = lib.kto_pcg_axis(diag.shape[0], _p(rp, _i64p), _p(col, _i32p), _p(val, _f64p),
                          _p(diag, _f64p), _p(rhs, _f64p), _p(x, _f64p), tol, max_iter,
                          ctypes.byref(resid), ctypes.byref(it), _p(hist, _f64p), hist_cap)
    if rc != 0:
        raise RuntimeError("kto_pcg_axis failed")
    k = int(it.value)
    return dict(x=x, resid=float(resid.value), iters=k,
                hist=None if hist is None else hist[:min(k, hist_cap)])


def port_solve_both(sys_x: dict, x, sys_y: dict, y, tol: float, max_iter: int,
                    hist_cap: int = 0) -> dict:
    """solveBothAxes semantics: both axes step in lock-step while live; the
    observer history holds (resid_x, resid_y) after every loop iteration."""
    rx = port_pcg_axis(sys_x, x, tol, max_iter, hist_cap)
    ry = port_pcg_axis(sys_y, y, tol, max_iter, hist_cap)
    k = max(rx["iters"], ry["iters"])
    out = dict(x=rx["x"], y=ry["x"], resid=(rx["resid"], ry["resid"]), iters=k)
    if hist_cap:
        def fill(h, it, final):
            a = np.empty(min(k, hist_cap))
            a[:min(it, hist_cap)] = h[:min(it, hist_cap)]
            a[min(it, hist_cap):] = final
            return a
        out["hist_x"] = fill(rx["hist"], rx["iters"], rx["resid"])
        out["hist_y"] = fill(ry["hist"], ry["iters"], ry["resid"])
    return out


def port_occupancy(nl, x, y, grid: dict):
    lib = load_port()
    x, y = _c(x, np.float64), _c(y, np.float64)
    w, h = _c(nl.width, np.float64), _c(nl.height, np.float64)
    area = _c(nl.width * nl.height, np.float64)
    occ = np.zeros(grid["nx"] * grid["ny"])
    lib.kto_occupancy(nl.num_movable, _p(x, _f64p), _p(y, _f64p), _p(w, _f64p), _p(h, _f64p),
                      _p(area, _f64p), grid["origin"][0], grid["origin"][1], grid["dx"],
                      grid["dy"], grid["nx"], grid["ny"], _p(occ, _f64p))
    return occ


def port_overflow(occ, avail, density_limit: float, total_avail: float) -> float:
    lib = load_port()
    occ, avail = _c(occ, np.float64), _c(avail, np.float64)
    return float(lib.kto_overflow(occ.shape[0], _p(occ, _f64p), _p(avail, _f64p),
                                  density_limit, total_avail))


def port_dot(a, b) -> float:
    a, b = _c(a, np.float64), _c(b, np.float64)
    return float(load_port().kto_dot(a.shape[0], _p(a, _f64p), _p(b, _f64p)))


class Kraftwerk2Ref:
    """The reference's Kraftwerk2 buildSystem / solve on a Design filled from a
    Netlist (oracle/ref_kraftwerk2.cc): movable cells as slots, each net's
    pins as (slot or none, offset, fixedPosition = fixed position + offset)."""

    def __init__(self, nl):
        lib = load_ref("cpu")
        if not hasattr(lib, "_kw2_ready"):
            lib.kw2_create.argtypes = [ctypes.c_int64, _f64p, _f64p, ctypes.c_int64, _i64p, _i64p,
                                       _f64p, _f64p, _f64p, _f64p, _f64p, ctypes.c_double,
                                       ctypes.c_double, ctypes.c_double, ctypes.c_double]
            lib.kw2_create.restype = _vp
            lib.kw2_destroy.argtypes = [_vp]
            lib.kw2_build.argtypes = [_vp, _f64p, _f64p, ctypes.c_int, ctypes.c_int,
                                      ctypes.c_double, ctypes.c_double]
            lib.kw2_build.restype = ctypes.c_int64
            lib.kw2_get_system.argtypes = [_vp, _i64p, _i32p, _f64p, _f64p, _f64p]
            lib.kw2_set_diag_rhs.argtypes = [_vp, _f64p, _f64p]
            lib.kw2_solve.argtypes = [_vp, _f64p, ctypes.c_double, ctypes.c_int64]
            lib._kw2_ready = True
        self.lib = lib
        self.n = nl.num_movable
        slot = nl.var_of_vertex[nl.pin_cell].astype(np.int64)
        fixed = slot < 0
        fx = np.where(fixed, nl.fixed_x[nl.pin_cell] + nl.off_x, 0.0)
        fy = np.where(fixed, nl.fixed_y[nl.pin_cell] + nl.off_y, 0.0)
        k = dict(w=_c(nl.width, np.float64), h=_c(nl.height, np.float64),
                 ns=_c(nl.net_start, np.int64), slot=_c(slot, np.int64),
                 ox=_c(nl.off_x, np.float64), oy=_c(nl.off_y, np.float64),
                 fx=_c(fx, np.float64), fy=_c(fy, np.float64),
                 wt=_c(nl.net_weight, np.float64))
        self._keep = k
        lx, ly, ux, uy = nl.die
        self.h = lib.kw2_create(self.n, _p(k["w"], _f64p), _p(k["h"], _f64p), nl.num_nets,
                                _p(k["ns"], _i64p), _p(k["slot"], _i64p), _p(k["ox"], _f64p),
                                _p(k["oy"], _f64p), _p(k["fx"], _f64p), _p(k["fy"], _f64p),
                                _p(k["wt"], _f64p), lx, ly, ux, uy)
        if not self.h:
            raise RuntimeError("kw2_create failed")

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.kw2_destroy(self.h)
            self.h = None

    def build(self, x, y, horizontal: bool, with_rhs: bool, floor_x: float, floor_y: float) -> dict:
        x, y = _c(x, np.float64), _c(y, np.float64)
        m = int(self.lib.kw2_build(self.h, _p(x, _f64p), _p(y, _f64p), int(horizontal),
                                   int(with_rhs), floor_x, floor_y))
        s = dict(row_ptr=np.zeros(self.n + 1, np.int64), col=np.zeros(max(m, 1), np.int32),
                 val=np.zeros(max(m, 1)), diag=np.zeros(max(self.n, 1)),
                 rhs=np.zeros(max(self.n, 1)))
        self.lib.kw2_get_system(self.h, _p(s["row_ptr"], _i64p), _p(s["col"], _i32p),
                                _p(s["val"], _f64p), _p(s["diag"], _f64p), _p(s["rhs"], _f64p))
        s["col"], s["val"] = s["col"][:m], s["val"][:m]
        s["diag"], s["rhs"] = s["diag"][:self.n], s["rhs"][:self.n]
        return s

    def set_diag_rhs(self, diag, rhs):
        d, r = _c(diag, np.float64), _c(rhs, np.float64)
        self.lib.kw2_set_diag_rhs(self.h, _p(d, _f64p), _p(r, _f64p))

    def solve(self, x, tol: float, max_iter: int):
        x = _c(x, np.float64).copy()
        self.lib.kw2_solve(self.h, _p(x, _f64p), tol, max_iter)
        return x
