"""Failure detection without a GPU fault: a bounded wait is made to run out
(one block of a cooperative launch never arrives), the kernel reports
KTG_ERR_TIMEOUT through the status word, and the same context then solves
normally. Host-side failures (bad arguments, calls out of order) return
error codes."""
import ctypes
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

from cases import build_case, TOL, MAX_ITER  # noqa: E402

pytestmark = pytest.mark.gpu


def test_wait_timeout_is_reported_and_context_survives(gpu_ctx):
    from ktplace_b200 import _lib
    st = ctypes.c_int(0)
    rc = gpu_ctx.lib.ktg_selftest_wait_timeout(gpu_ctx.h, 50_000_000, ctypes.byref(st))
    assert rc == 0
    assert st.value == _lib.KTG_ERR_TIMEOUT
    raw, nl, x, y, ax, ay, alpha, _ = build_case("tiny_macros")
    gpu_ctx.upload_netlist(nl)
    fx, fy = nl.floors()
    gpu_ctx.build_b2b(x, y, alpha, ax, ay, fx, fy)
    r = gpu_ctx.solve(x, y, TOL, MAX_ITER)
    assert r["iters"] > 0 and max(r["resid"]) <= TOL


def test_host_side_errors(gpu_ctx):
    from ktplace_b200 import _lib
    from ktplace_b200._lib import KtgError
    with pytest.raises(KtgError) as e:
        gpu_ctx.set_option("pcg_lanes", 3)
    assert e.value.code == _lib.KTG_ERR_ARG
    st = ctypes.c_int(0)
    assert gpu_ctx.lib.ktg_selftest_wait_timeout(gpu_ctx.h, 0, ctypes.byref(st)) == _lib.KTG_ERR_ARG
    x = np.zeros(4)
    with pytest.raises(KtgError):
        gpu_ctx.solve_mixed(x, x, TOL, inner_tol=1.5)
