"""One SimPL step end to end from Bookshelf files: the library's reader feeds
the GPU path (B2B, the solve in the reference's summation order, HPWL,
occupancy, look-ahead legalization), the reference's reader feeds the
reference's own code (oracle/_ref), and the two must agree bit for bit.

The design is the seeded 12k generator's, written as Bookshelf with every
fourth row split into two subrows around a gap that no obstacle covers, so
the grid's free area and the legalizer's free space come from the subrows
(buildGrid, simpl_placer.cc:199-212)."""
import os
import re

import numpy as np
import pytest

import oracle
from ktplace_b200 import bookshelf, grid, synth

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not oracle.ref_available(), reason="reference library not built")]


def gap_rows(scl_path, sites, site_width):
    """Rewrite the single subrow of every fourth row as two subrows with a gap
    of 15% of the row between them."""
    a = int(sites * 0.40)
    b = int(sites * 0.55)
    text = open(scl_path).read()
    rows = text.split("CoreRow Horizontal\n")
    out = [rows[0]]
    for r, body in enumerate(rows[1:]):
        if r % 4 == 1:
            body = re.sub(r"  SubrowOrigin : 0 NumSites : \d+\n",
                          f"  SubrowOrigin : 0 NumSites : {a}\n"
                          f"  SubrowOrigin : {repr(b * site_width)} NumSites : {sites - b}\n",
                          body)
        out.append(body)
    with open(scl_path, "w") as f:
        f.write("CoreRow Horizontal\n".join(out))


@pytest.fixture(scope="module")
def design(tmp_path_factory):
    raw = synth.generate(synth.spec_small(seed=5))
    d = os.path.join(str(tmp_path_factory.mktemp("bs")), raw.name)
    synth.write_bookshelf(raw, d)
    gap_rows(os.path.join(d, raw.name + ".scl"), raw.sites_per_row, raw.site_width)
    nl = bookshelf.read(d)
    assert len(nl.subrows) == raw.num_rows + (raw.num_rows + 2) // 4
    ref = oracle.RefDesign.from_bookshelf(d)
    x, y = synth.seed_positions(raw, nl.num_movable, 31)
    ax, ay = synth.seed_positions(raw, nl.num_movable, 32)
    return nl, ref, x, y, ax, ay


def test_step_from_bookshelf_bit_identical(design, gpu_ctx):
    nl, ref, x, y, ax, ay = design
    ctx = gpu_ctx
    ctx.upload_netlist(nl)
    fx, fy = nl.floors()
    ctx.build_b2b(x, y, 0.2, ax, ay, fx, fy)
    ref.build_b2b(x, y, 0.2, ax, ay)
    for axis in (0, 1):
        g, r = ctx.system(axis), ref.system(axis)
        m = int(r["row_ptr"][-1])
        assert np.array_equal(g["row_ptr"].astype(np.int64), r["row_ptr"].astype(np.int64)), axis
        assert np.array_equal(g["col"][:m].astype(np.int64), r["col"].astype(np.int64)), axis
        assert np.array_equal(g["val"][:m], r["val"]), axis
        assert np.array_equal(g["diag"], r["diag"]) and np.array_equal(g["rhs"], r["rhs"]), axis

    rr = ref.solve(x, y, 1e-6, 1000)
    try:
        ctx.set_option("pcg_form", 2)
        e = ctx.solve(x, y, 1e-6, 1000)
    finally:
        ctx.set_option("pcg_form", -1)
    assert e["iters"] == rr["iters"]
    assert np.array_equal(e["x"], rr["x"]) and np.array_equal(e["y"], rr["y"])
    px, py = rr["x"], rr["y"]
    h, hr = ctx.hpwl(px, py), ref.hpwl(px, py)
    assert abs(h - hr) <= 1e-12 * abs(hr)

    bins = grid.default_bins_per_axis(nl.num_movable)
    g = grid.build_grid(nl, bins, 1.0)
    rg = ref.grid(bins, 1.0)
    assert np.array_equal(g.avail, rg["avail"]) and g.total_avail == rg["total_avail"]
    ctx.set_grid(g)
    occ, _ = ctx.occupancy(px, py)
    rocc, _ = ref.occupancy_map(px, py, bins * bins)
    assert np.array_equal(occ, rocc)

    ctx.set_free_space(grid.build_free_space(nl))
    gx, gy = ctx.lal(px, py)
    lx, ly = ref.lal(px, py)
    assert np.array_equal(gx, lx) and np.array_equal(gy, ly)
    assert np.mean(gx != px) > 0.1
    # the split rows' gaps are in the legalizer's free space
    fs = grid.build_free_space(nl)
    assert len(fs.spans) > len(fs.row_y)
