"""ktg_hpwl_noalloc: the HPWL entry point for callers that cannot allocate GPU
memory (host callbacks, foreign allocators, fixed memory budgets).

It is called through the C ABI with caller-owned device arrays, twice in a
row on the same scratch, and must agree with the regular entry point
(ktg_hpwl) within the HPWL tolerance of the parity tests. The file is named
so that pytest collects it last.
"""
import ctypes
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

from cases import build_case  # noqa: E402

pytestmark = pytest.mark.gpu
HPWL_RTOL = 1e-12


def _dev(torch, a, dtype):
    return torch.tensor(np.ascontiguousarray(a), dtype=dtype, device="cuda:0")


@pytest.mark.parametrize("name", ["tiny_macros", "small12k"])
def test_noalloc_matches_ktg_hpwl(name):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from ktplace_b200 import _lib, synth
    from ktplace_b200.gpu import Context
    lib = _lib.load()
    raw, nl, x, y, ax, ay, *_ = build_case(name)
    x2, y2 = synth.seed_positions(raw, nl.num_movable, 999)
    torch.cuda.set_device(0)
    ns = _dev(torch, nl.net_start.astype(np.int32), torch.int32)
    pc = _dev(torch, nl.pin_cell, torch.int32)
    vv = _dev(torch, nl.var_of_vertex, torch.int32)
    ox, oy = _dev(torch, nl.off_x, torch.float64), _dev(torch, nl.off_y, torch.float64)
    fx, fy = _dev(torch, nl.fixed_x, torch.float64), _dev(torch, nl.fixed_y, torch.float64)
    out = torch.zeros(2, dtype=torch.float64, device="cuda:0")
    stream = torch.cuda.Stream()
    P = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    got = []
    with Context(0) as ctx:
        ctx.upload_netlist(nl)
        for k, (px, py) in enumerate(((x, y), (x2, y2))):
            dx, dy = _dev(torch, px, torch.float64), _dev(torch, py, torch.float64)
            torch.cuda.synchronize()
            rc = lib.ktg_hpwl_noalloc(P(ns), P(pc), P(vv), P(ox), P(oy), P(fx), P(fy), P(dx),
                                      P(dy), nl.num_nets, ctypes.c_void_p(out.data_ptr() + 8 * k),
                                      ctypes.c_void_p(stream.cuda_stream))
            assert rc == 0
            stream.synchronize()
            want = ctx.hpwl(px, py)
            got.append(float(out[k].item()))
            assert abs(got[-1] - want) <= HPWL_RTOL * abs(want), (k, got[-1], want)
    assert got[0] != got[1]


def test_noalloc_rejects_oversize():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from ktplace_b200 import _lib
    lib = _lib.load()
    one = torch.zeros(1, dtype=torch.int32, device="cuda:0")
    out = torch.zeros(1, dtype=torch.float64, device="cuda:0")
    P = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    rc = lib.ktg_hpwl_noalloc(P(one), P(one), P(one), P(out), P(out), P(out), P(out), P(out),
                              P(out), (1 << 22) + 1, P(out), None)
    assert rc == _lib.KTG_ERR_RANGE
