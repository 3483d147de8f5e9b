"""Bookshelf designs through the library's own reader (ktg_bookshelf_read).

``read(directory)`` returns the same ``Netlist`` that ``netlist.flatten``
builds, read and flattened by the C ABI's multithreaded host reader, whose
rules are the reference's BookshelfInputAdapter (adaptor/
bookshelfToKTAdaptor.cc) and buildSimplDM (globalPlacer/simpl/simpl_dm.cc).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import KtgError
from .netlist import Netlist


def read(directory: str, threads: int = 0) -> Netlist:
    lib = _lib.load()
    h = ctypes.c_void_p()
    rc = lib.ktg_bookshelf_read(directory.encode(), int(threads), ctypes.byref(h))
    if rc != 0:
        raise KtgError(rc, lib.ktg_bookshelf_last_error().decode())
    try:
        sz = np.zeros(9, np.int64)
        lib.ktg_bookshelf_sizes(h, sz.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)))
        V, n, N, P, Pm, _, K, R, S = (int(v) for v in sz)
        view = _lib.NetlistView()
        lib.ktg_bookshelf_view(h, ctypes.byref(view))

        def arr(ptr, count, dtype):
            if count == 0:
                return np.zeros(0, dtype)
            return np.ctypeslib.as_array(ptr, shape=(count,)).astype(dtype, copy=True)

        die = np.zeros(4)
        obst = np.zeros(max(K, 1) * 4)
        rows = np.zeros(max(R, 1) * 5)
        sub = np.zeros(max(S, 1) * 3)
        f64 = ctypes.POINTER(ctypes.c_double)
        lib.ktg_bookshelf_geometry(h, die.ctypes.data_as(f64), obst.ctypes.data_as(f64),
                                   rows.ctypes.data_as(f64), sub.ctypes.data_as(f64))
        nl = Netlist(
            num_vertices=V, num_movable=n,
            mov_vertex=arr(view.mov_vertex, n, np.int32),
            var_of_vertex=arr(view.var_of_vertex, V, np.int32),
            fixed_x=arr(view.fixed_x, V, np.float64), fixed_y=arr(view.fixed_y, V, np.float64),
            net_start=arr(view.net_start, N + 1, np.int64),
            pin_cell=arr(view.pin_cell, P, np.int32),
            off_x=arr(view.off_x, P, np.float64), off_y=arr(view.off_y, P, np.float64),
            net_weight=arr(view.net_weight, N, np.float64),
            pin_start=arr(view.pin_start, n + 1, np.int64),
            pin_net=arr(view.pin_net, Pm, np.int32), pin_q=arr(view.pin_q, Pm, np.int32),
            width=arr(view.width, n, np.float64), height=arr(view.height, n, np.float64),
            obstacles=obst[:4 * K].reshape(K, 4), rows=rows[:5 * R].reshape(R, 5),
            die=tuple(float(v) for v in die))
        nl.subrows = sub[:3 * S].reshape(S, 3)
        ms = np.zeros(6)
        lib.ktg_bookshelf_times(h, ms.ctypes.data_as(f64))
        nl.read_ms = dict(zip(("nodes", "wts", "nets", "pl", "scl", "flatten"), ms.tolist()))
        return nl
    finally:
        lib.ktg_bookshelf_free(h)
