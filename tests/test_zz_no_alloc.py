"""ktg_hpwl_noalloc: the HPWL entry point for callers that cannot allocate GPU
memory (host callbacks, foreign allocators, fixed memory budgets).

It is called through the C ABI with caller-owned device arrays, twice in a
row on the same scratch, and must give the regular entry point's (ktg_hpwl)
result bit for bit (the same per-net terms summed by the same fixed-shape
tree); the first call's positions are also checked against the golden HPWL
the reference computed for them. A second test calls it from a context the
caller created itself on the same device, where the scratch array sits at
another address. The file is named so that pytest collects it last.
"""
import ctypes
import json
import os
import subprocess
import sys
import textwrap

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

from cases import build_case  # noqa: E402

pytestmark = pytest.mark.gpu
HPWL_RTOL = 1e-12
GOLDEN = json.load(open(os.path.join(HERE, "golden", "golden.json")))


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
            assert got[-1] == want, (k, got[-1], want)
            if k == 0 and name in GOLDEN:
                ref = GOLDEN[name]["hpwl_in"]
                assert abs(got[-1] - ref) <= HPWL_RTOL * abs(ref), (got[-1], ref)
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


_CONTEXTS_SCRIPT = textwrap.dedent("""
    import ctypes, json, sys
    import numpy as np
    from cuda.bindings import driver as cu

    def ok(r):
        err = r[0] if isinstance(r, tuple) else r
        if err != cu.CUresult.CUDA_SUCCESS:
            raise RuntimeError(str(err))
        return r[1] if isinstance(r, tuple) and len(r) == 2 else None

    lib = ctypes.CDLL(sys.argv[1])
    f = lib.ktg_hpwl_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_void_p] * 9 + [ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p]
    arrays = np.load(sys.argv[2])
    names = ["net_start", "pin_cell", "var_of_vertex", "off_x", "off_y", "fixed_x", "fixed_y",
             "x", "y"]
    num_nets = int(arrays["net_start"].shape[0] - 1)

    def hpwl_here():
        ptrs = []
        for nm in names:
            a = np.ascontiguousarray(arrays[nm])
            d = ok(cu.cuMemAlloc(max(a.nbytes, 8)))
            ok(cu.cuMemcpyHtoD(d, a.ctypes.data, a.nbytes))
            ptrs.append(d)
        out = ok(cu.cuMemAlloc(8))
        rc = f(*[int(p) for p in ptrs], num_nets, int(out), None)
        if rc != 0:
            raise RuntimeError(f"ktg_hpwl_noalloc returned {rc}")
        ok(cu.cuCtxSynchronize())
        v = np.zeros(1)
        ok(cu.cuMemcpyDtoH(v.ctypes.data, out, 8))
        for p in ptrs + [out]:
            ok(cu.cuMemFree(p))
        return float(v[0])

    ok(cu.cuInit(0))
    dev = ok(cu.cuDeviceGet(0))
    primary = ok(cu.cuDevicePrimaryCtxRetain(dev))
    ok(cu.cuCtxSetCurrent(primary))
    res = {"primary": [hpwl_here(), hpwl_here()]}
    other = ok(cu.cuCtxCreate(0, dev))  # becomes current
    res["created"] = [hpwl_here(), hpwl_here()]
    ok(cu.cuCtxSetCurrent(primary))
    res["primary_again"] = [hpwl_here()]
    ok(cu.cuCtxDestroy(other))
    print(json.dumps(res))
""")


def test_noalloc_in_caller_created_context(tmp_path):
    """A caller may keep its own CUDA context on the device. The library's
    module, and with it the scratch array, is then loaded into that context at
    another address; the entry point must find that context's copy (its
    cached address is keyed by the context, not by the device ordinal). Run
    in a fresh process that drives the contexts through the driver API."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    pytest.importorskip("cuda.bindings.driver")
    from ktplace_b200 import _lib
    raw, nl, x, y, *_ = build_case("small12k")
    arrays = dict(net_start=nl.net_start.astype(np.int32), pin_cell=nl.pin_cell.astype(np.int32),
                  var_of_vertex=nl.var_of_vertex.astype(np.int32), off_x=nl.off_x,
                  off_y=nl.off_y, fixed_x=nl.fixed_x, fixed_y=nl.fixed_y,
                  x=np.asarray(x, np.float64), y=np.asarray(y, np.float64))
    npz = tmp_path / "in.npz"
    np.savez(npz, **arrays)
    script = tmp_path / "contexts.py"
    script.write_text(_CONTEXTS_SCRIPT)
    r = subprocess.run([sys.executable, str(script), _lib.LIB_PATH, str(npz)],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    res = json.loads(r.stdout.strip().splitlines()[-1])
    want = GOLDEN["small12k"]["hpwl_in"]
    vals = res["primary"] + res["created"] + res["primary_again"]
    assert all(v == vals[0] for v in vals), res
    assert abs(vals[0] - want) <= HPWL_RTOL * abs(want)
