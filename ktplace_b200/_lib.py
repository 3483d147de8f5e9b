"""ctypes binding of the C ABI in include/ktplace_b200.h.

Loads ``_build/libktplace_b200.so`` (built in-tree by ``ktplace_b200.build``).
There is no fallback: if the library is missing or cannot be loaded, every
entry point raises.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libktplace_b200.so")

KTG_OK = 0
KTG_ERR_ARG = -1
KTG_ERR_CUDA = -2
KTG_ERR_NOMEM = -3
KTG_ERR_STATE = -4
KTG_ERR_TIMEOUT = -5
KTG_ERR_RANGE = -6
KTG_PTR_HOST = 0
KTG_PTR_DEVICE = 1

_i32p = ctypes.POINTER(ctypes.c_int32)
_i64p = ctypes.POINTER(ctypes.c_int64)
_u32p = ctypes.POINTER(ctypes.c_uint32)
_f64p = ctypes.POINTER(ctypes.c_double)
_f32p = ctypes.POINTER(ctypes.c_float)
_vp = ctypes.c_void_p


class NetlistView(ctypes.Structure):
    _fields_ = [("num_vertices", ctypes.c_int64), ("num_movable", ctypes.c_int64),
                ("num_nets", ctypes.c_int64), ("mov_vertex", _i32p), ("var_of_vertex", _i32p),
                ("fixed_x", _f64p), ("fixed_y", _f64p), ("net_start", _i64p),
                ("pin_cell", _i32p), ("off_x", _f64p), ("off_y", _f64p),
                ("net_weight", _f64p), ("pin_start", _i64p), ("pin_net", _i32p),
                ("pin_q", _i32p), ("width", _f64p), ("height", _f64p)]


class GridView(ctypes.Structure):
    _fields_ = [("origin_x", ctypes.c_double), ("origin_y", ctypes.c_double),
                ("dx", ctypes.c_double), ("dy", ctypes.c_double), ("nx", ctypes.c_int64),
                ("ny", ctypes.c_int64), ("avail", _f64p), ("total_avail", ctypes.c_double),
                ("density_limit", ctypes.c_double)]


class SolveInfo(ctypes.Structure):
    _fields_ = [("resid_x", ctypes.c_double), ("resid_y", ctypes.c_double),
                ("iters", ctypes.c_int64), ("iters_x", ctypes.c_int64),
                ("iters_y", ctypes.c_int64), ("status", ctypes.c_int32),
                ("live", ctypes.c_int32)]


class MixedInfo(ctypes.Structure):
    _fields_ = [("resid_x", ctypes.c_double), ("resid_y", ctypes.c_double),
                ("inner_x", ctypes.c_int64), ("inner_y", ctypes.c_int64),
                ("outer_x", ctypes.c_int32), ("outer_y", ctypes.c_int32),
                ("status", ctypes.c_int32), ("stalled", ctypes.c_int32),
                ("fp64_iters_x", ctypes.c_int64), ("fp64_iters_y", ctypes.c_int64)]


class BatchResult(ctypes.Structure):
    _fields_ = [("iters", ctypes.c_int64), ("outer", ctypes.c_int32), ("status", ctypes.c_int32),
                ("resid", ctypes.c_double), ("latency_ns", ctypes.c_int64)]


# (name, restype, argtypes) of every entry point in include/ktplace_b200.h
SIGNATURES = [
    ("ktg_create", ctypes.c_int, [ctypes.c_int, ctypes.POINTER(_vp)]),
    ("ktg_destroy", None, [_vp]),
    ("ktg_last_error", ctypes.c_char_p, [_vp]),
    ("ktg_version", ctypes.c_char_p, []),
    ("ktg_set_stream", ctypes.c_int, [_vp, _vp]),
    ("ktg_set_pointer_mode", ctypes.c_int, [_vp, ctypes.c_int]),
    ("ktg_upload_netlist", ctypes.c_int, [_vp, ctypes.POINTER(NetlistView)]),
    ("ktg_build_b2b", ctypes.c_int, [_vp, _vp, _vp, ctypes.c_double, _vp, _vp, ctypes.c_double,
                                     ctypes.c_double]),
    ("ktg_build_hpwl", ctypes.c_int, [_vp, _vp]),
    ("ktg_build_star", ctypes.c_int, [_vp, _i64p]),
    ("ktg_system_info", ctypes.c_int, [_vp, ctypes.c_int, _i64p, _i64p]),
    ("ktg_download_system", ctypes.c_int, [_vp, ctypes.c_int, _i64p, _i32p, _f64p, _f64p,
                                           _f64p]),
    ("ktg_download_bound_pins", ctypes.c_int, [_vp, ctypes.c_int, _u32p, _u32p]),
    ("ktg_upload_system", ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int64, _i64p, _i32p,
                                         _f64p, _f64p, _f64p]),
    ("ktg_spmv", ctypes.c_int, [_vp, ctypes.c_int32, _vp, _vp]),
    ("ktg_solve", ctypes.c_int, [_vp, _vp, _vp, ctypes.c_double, ctypes.c_int64, _vp, _vp, _vp,
                                 ctypes.c_int64]),
    ("ktg_solve_mixed", ctypes.c_int, [_vp, _vp, _vp, ctypes.c_double, ctypes.c_double,
                                       ctypes.c_int64, ctypes.c_int32, _vp, _vp, _vp,
                                       ctypes.c_int64]),
    ("ktg_hpwl", ctypes.c_int, [_vp, _vp, _vp, _vp]),
    ("ktg_set_grid", ctypes.c_int, [_vp, ctypes.POINTER(GridView)]),
    ("ktg_occupancy", ctypes.c_int, [_vp, _vp, _vp, _vp, _vp]),
    ("ktg_set_free_space", ctypes.c_int, [_vp, ctypes.c_int64, _vp, _vp, _vp, ctypes.c_int64,
                                          _vp, _vp]),
    ("ktg_lal", ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int32, ctypes.c_int32, ctypes.c_double]),
    ("ktg_lal_stats", ctypes.c_int, [_vp, _vp, ctypes.c_int32]),
    ("ktg_launch_count", ctypes.c_int64, [_vp]),
    ("ktg_selftest_wait_timeout", ctypes.c_int, [_vp, ctypes.c_int64,
                                                 ctypes.POINTER(ctypes.c_int)]),
    ("ktg_set_option", ctypes.c_int, [_vp, ctypes.c_char_p, ctypes.c_int64]),
    ("ktg_download_aggregates", ctypes.c_int, [_vp, _i32p, _i32p, _f32p]),
    ("ktg_download_coarse", ctypes.c_int, [_vp, _f32p, _f32p, _f64p]),
    ("ktg_download_mixed_trace", ctypes.c_int, [_vp, _vp, ctypes.c_int64]),
    ("ktg_bookshelf_read", ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(_vp)]),
    ("ktg_bookshelf_free", None, [_vp]),
    ("ktg_bookshelf_last_error", ctypes.c_char_p, []),
    ("ktg_bookshelf_sizes", ctypes.c_int, [_vp, _i64p]),
    ("ktg_bookshelf_view", ctypes.c_int, [_vp, ctypes.POINTER(NetlistView)]),
    ("ktg_bookshelf_times", ctypes.c_int, [_vp, _f64p]),
    ("ktg_bookshelf_geometry", ctypes.c_int, [_vp, _f64p, _f64p, _f64p, _f64p]),
    ("ktg_build_b2b_kraftwerk2", ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int, ctypes.c_double,
                                                ctypes.c_double]),
    ("ktg_kraftwerk2_adjust", ctypes.c_int, [_vp, _vp, _vp, _vp, ctypes.c_double]),
    ("ktg_batch_create", ctypes.c_int, [ctypes.c_int, ctypes.POINTER(_vp)]),
    ("ktg_batch_destroy", None, [_vp]),
    ("ktg_batch_last_error", ctypes.c_char_p, [_vp]),
    ("ktg_batch_set_stream", ctypes.c_int, [_vp, _vp]),
    ("ktg_batch_size", ctypes.c_int64, [_vp]),
    ("ktg_batch_add_system", ctypes.c_int, [_vp, ctypes.c_int64, _i64p, _i32p, _f64p, _f64p,
                                            _f64p, _f64p, _i64p]),
    ("ktg_batch_add_from_context", ctypes.c_int, [_vp, _vp, _f64p, _f64p, _i64p]),
    ("ktg_batch_set_shape", ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int]),
    ("ktg_batch_get_shape", ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_int),
                                           ctypes.POINTER(ctypes.c_int)]),
    ("ktg_batch_autotune", ctypes.c_int, [_vp, ctypes.c_double, ctypes.c_int, ctypes.c_double,
                                          ctypes.c_int64, ctypes.POINTER(ctypes.c_int),
                                          ctypes.POINTER(ctypes.c_int),
                                          ctypes.POINTER(ctypes.c_float)]),
    ("ktg_batch_set_split", ctypes.c_int, [_vp, ctypes.c_int64, ctypes.c_int, ctypes.c_int,
                                           ctypes.c_int]),
    ("ktg_batch_get_split", ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_int64),
                                           ctypes.POINTER(ctypes.c_int),
                                           ctypes.POINTER(ctypes.c_int),
                                           ctypes.POINTER(ctypes.c_int),
                                           ctypes.POINTER(ctypes.c_int)]),
    ("ktg_batch_autotune_split", ctypes.c_int, [_vp, ctypes.c_double, ctypes.c_int,
                                                ctypes.c_double, ctypes.c_int64,
                                                ctypes.POINTER(ctypes.c_float),
                                                ctypes.POINTER(ctypes.c_float)]),
    ("ktg_batch_set_offload", ctypes.c_int, [_vp, ctypes.c_int64, ctypes.c_int, ctypes.c_int]),
    ("ktg_batch_get_offload", ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_int64),
                                             ctypes.POINTER(ctypes.c_int)]),
    ("ktg_batch_autotune_offload", ctypes.c_int, [_vp, ctypes.c_double, ctypes.c_int,
                                                  ctypes.c_double, ctypes.c_int64,
                                                  ctypes.POINTER(ctypes.c_float),
                                                  ctypes.POINTER(ctypes.c_float)]),
    ("ktg_batch_reset_x", ctypes.c_int, [_vp]),
    ("ktg_batch_solve", ctypes.c_int, [_vp, ctypes.c_double, ctypes.c_int64, ctypes.c_int,
                                       ctypes.c_double]),
    ("ktg_batch_results", ctypes.c_int, [_vp, _vp]),
    ("ktg_batch_get_x", ctypes.c_int, [_vp, ctypes.c_int64, _f64p]),
    ("ktg_batch_launch_count", ctypes.c_int64, [_vp]),
    ("ktg_learned_num_params", ctypes.c_int64, []),
    ("ktg_learned_create", ctypes.c_int, [ctypes.c_int, ctypes.c_uint64, ctypes.POINTER(_vp)]),
    ("ktg_learned_destroy", None, [_vp]),
    ("ktg_learned_last_error", ctypes.c_char_p, [_vp]),
    ("ktg_learned_set_option", ctypes.c_int, [_vp, ctypes.c_char_p, ctypes.c_double]),
    ("ktg_learned_get_params", ctypes.c_int, [_vp, _vp]),
    ("ktg_learned_set_params", ctypes.c_int, [_vp, _vp]),
    ("ktg_learned_loss_grad", ctypes.c_int, [_vp, _vp, ctypes.c_int, ctypes.c_uint64,
                                             ctypes.POINTER(ctypes.c_double), _vp]),
    ("ktg_learned_train_step", ctypes.c_int, [_vp, _vp, ctypes.c_int, ctypes.c_uint64,
                                              ctypes.POINTER(ctypes.c_double)]),
    ("ktg_learned_prepare", ctypes.c_int, [_vp, _vp]),
    ("ktg_learned_launch_count", ctypes.c_int64, [_vp]),
    ("ktg_learned_coarse_loss_grad", ctypes.c_int,
     [_vp, _vp, ctypes.c_int, _vp, ctypes.c_int32, ctypes.POINTER(ctypes.c_double), _vp]),
    ("ktg_learned_coarse_train_step", ctypes.c_int,
     [_vp, _vp, ctypes.c_int, _vp, ctypes.c_int32, ctypes.POINTER(ctypes.c_double)]),
    ("ktg_learned_prepare_coarse", ctypes.c_int, [_vp, _vp]),
    ("ktg_hpwl_noalloc", ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                                        ctypes.c_int64, _vp, _vp]),
]

_lib = None


def load():
    """Loads the CUDA library; raises if it is missing (no CPU fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"ktplace_b200 CUDA library not built: {LIB_PATH} is missing "
                "(run `python -m ktplace_b200.build`)")
        lib = ctypes.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


class KtgError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"ktplace_b200 error {code}: {msg}")
        self.code = code
