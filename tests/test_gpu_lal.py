"""Look-ahead legalization on the GPU (ktg_lal) against the reference's own
LookAheadLegalizer (oracle/_ref, RefDesign.lal) and the Python restatement
(oracle/lal_ref.py).

Bar: bit-identical positions. Designs: seeded tiny designs with macros (the
restatement and the reference both check), and a 12k-cell design whose cells
start in a tight cluster, so that one region holds every cell and the long
segment sort (chunks + merge passes) runs; uniform starts give many small
clusters and batches. Each case runs with blocks of up to 2048 cells
finished in one CTA (the default), with every level run level by level
(lal_subtree_cells = 0), and with the hand-off at 64 cells; and with the
area sums read off exact integer prefixes (the default for these integer
areas) as well as summed sequentially (lal_exact_sums = 0)."""
import resource

import numpy as np
import pytest

import oracle
from oracle import lal_ref
from ktplace_b200 import grid, netlist, synth

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True, scope="module")
def big_stack():
    # the reference's recursion wants more than the default main-thread stack
    try:
        resource.setrlimit(resource.RLIMIT_STACK, (resource.RLIM_INFINITY, resource.RLIM_INFINITY))
    except (ValueError, OSError):
        pass


def clustered(raw, n, seed, spread):
    """Lower-left positions around the die centre (normal, `spread` of the
    die's extent), so the centre bins are far over their room."""
    rng = np.random.default_rng(seed)
    lx, ly, ux, uy = raw.die
    x = 0.5 * (lx + ux) + spread * (ux - lx) * rng.standard_normal(n)
    y = 0.5 * (ly + uy) + spread * (uy - ly) * rng.standard_normal(n)
    return x, y


def run_gpu(ctx, nl, bins, density, x, y, subtree=2048, exact=1, **opts):
    ctx.set_option("lal_subtree_cells", subtree)
    ctx.set_option("lal_exact_sums", exact)
    ctx.upload_netlist(nl)
    ctx.set_grid(grid.build_grid(nl, bins, density))
    ctx.set_free_space(grid.build_free_space(nl))
    return ctx.lal(x, y, **opts)


def run_oracle(nl, bins, density, x, y, **opts):
    g = grid.build_grid(nl, bins, density)
    fs = grid.build_free_space(nl)
    rows = lal_ref.free_rows(fs.row_y, fs.row_span, fs.spans)
    gd = dict(origin=(g.origin_x, g.origin_y), dx=g.dx, dy=g.dy, nx=g.nx, ny=g.ny, avail=g.avail)
    L = lal_ref.LAL(nl.width, nl.height, gd, rows, nl.obstacles, nl.die, g.density_limit, **opts)
    px, py = L.legalize(x, y)
    return np.array(px), np.array(py)


@pytest.mark.parametrize("exact", [1, 0])
@pytest.mark.parametrize("subtree", [2048, 0, 64])
@pytest.mark.parametrize("seed,cells,macros,bins,density,start", [
    (2, 400, 3, 16, 1.0, "uniform"),
    (5, 900, 4, 24, 1.0, "cluster"),
    (7, 600, 0, 8, 0.8, "uniform"),
    (9, 700, 2, 12, 0.9, "cluster"),
])
def test_lal_tiny_bit_exact(seed, cells, macros, bins, density, start, subtree, exact, gpu_ctx):
    raw = synth.generate(synth.spec_tiny(seed=seed, macros=macros, cells=cells, nets=cells + 30))
    nl = netlist.flatten(raw)
    if start == "uniform":
        x, y = synth.seed_positions(raw, nl.num_movable, seed + 10)
    else:
        x, y = clustered(raw, nl.num_movable, seed + 10, 0.08)
    gx, gy = run_gpu(gpu_ctx, nl, bins, density, x, y, subtree, exact)
    ox, oy = run_oracle(nl, bins, density, x, y)
    assert np.array_equal(gx, ox) and np.array_equal(gy, oy)
    assert np.mean(gx != x) > 0.1  # legalization did move cells
    if oracle.ref_available():
        ref = oracle.RefDesign.from_netlist(nl)
        ref.grid(bins, density)
        rx, ry = ref.lal(x, y)
        assert np.array_equal(gx, rx) and np.array_equal(gy, ry)


@pytest.mark.parametrize("subtree", [2048, 0])
@pytest.mark.parametrize("opts", [dict(max_level=6, min_cells_to_split=2, stripe_area_fraction=0.05),
                                  dict(max_level=30, min_cells_to_split=0, stripe_area_fraction=0.3),
                                  # many stripes: the one-CTA path runs out of stripe slots
                                  # below the top level and hands the blocks back
                                  dict(max_level=20, min_cells_to_split=4,
                                       stripe_area_fraction=0.002)])
def test_lal_options(opts, subtree, gpu_ctx):
    raw = synth.generate(synth.spec_tiny(seed=3, macros=2, cells=500, nets=530))
    nl = netlist.flatten(raw)
    x, y = clustered(raw, nl.num_movable, 21, 0.1)
    gx, gy = run_gpu(gpu_ctx, nl, 16, 1.0, x, y, subtree, **opts)
    ox, oy = run_oracle(nl, 16, 1.0, x, y, max_level=opts["max_level"],
                        min_cells=opts["min_cells_to_split"],
                        stripe_fraction=opts["stripe_area_fraction"])
    assert np.array_equal(gx, ox) and np.array_equal(gy, oy)


@pytest.mark.parametrize("subtree,exact", [(2048, 1), (0, 1), (2048, 0)])
@pytest.mark.parametrize("start", ["uniform", "cluster"])
def test_lal_12k_matches_reference(start, subtree, exact, gpu_ctx):
    if not oracle.ref_available():
        pytest.skip("reference library not built")
    raw = synth.generate(synth.spec_small(seed=3))
    nl = netlist.flatten(raw)
    if start == "uniform":
        x, y = synth.seed_positions(raw, nl.num_movable, 5)
    else:
        x, y = clustered(raw, nl.num_movable, 5, 0.03)
    bins = grid.default_bins_per_axis(nl.num_movable)
    gx, gy = run_gpu(gpu_ctx, nl, bins, 1.0, x, y, subtree, exact)
    ref = oracle.RefDesign.from_netlist(nl)
    ref.grid(bins, 1.0)
    rx, ry = ref.lal(x, y)
    assert np.array_equal(gx, rx) and np.array_equal(gy, ry)


def test_lal_no_overflow_only_clamps(gpu_ctx):
    """Nothing overfilled: positions only clamped to the die."""
    raw = synth.generate(synth.spec_tiny(seed=4, cells=200, nets=220))
    nl = netlist.flatten(raw)
    x, y = synth.seed_positions(raw, nl.num_movable, 1)
    x = x.copy()
    x[:5] = raw.die[2] + 50.0  # outside the die, but their bin is not overfilled
    gx, gy = run_gpu(gpu_ctx, nl, 4, 1.0, x, y)
    ox, oy = run_oracle(nl, 4, 1.0, x, y)
    assert np.array_equal(gx, ox) and np.array_equal(gy, oy)


def test_lal_stats_count_the_work(gpu_ctx):
    raw = synth.generate(synth.spec_tiny(seed=5, macros=4, cells=900, nets=930))
    nl = netlist.flatten(raw)
    x, y = clustered(raw, nl.num_movable, 15, 0.08)
    run_gpu(gpu_ctx, nl, 24, 1.0, x, y)
    st = gpu_ctx.lal_stats()
    assert st["batches"] >= 1 and st["regions"] >= st["batches"]
    assert st["levels"] >= 1 and st["syncs"] >= 2 and st["ms_total"] > 0.0


def test_lal_requires_free_space(gpu_ctx):
    from ktplace_b200.gpu import KtgError
    raw = synth.generate(synth.spec_tiny(seed=4, cells=100, nets=110))
    nl = netlist.flatten(raw)
    gpu_ctx.upload_netlist(nl)
    gpu_ctx.set_grid(grid.build_grid(nl, 8, 1.0))
    x, y = synth.seed_positions(raw, nl.num_movable, 1)
    if getattr(gpu_ctx, "_fs", None) is None:
        with pytest.raises(KtgError):
            gpu_ctx.lal(x, y)
    with pytest.raises(KtgError):
        gpu_ctx.lal(x, y, stripe_area_fraction=0.0)


def test_simpl_mirror_legalizes_in_place(gpu_ctx):
    """simpl.LookAheadLegalizer reads like the reference's (simpl_placer.cc:
    299-310): built from the grid, the free space and the options, legalize()
    updates x and y in place."""
    from ktplace_b200 import simpl
    raw = synth.generate(synth.spec_tiny(seed=5, macros=4, cells=900, nets=930))
    nl = netlist.flatten(raw)
    x, y = clustered(raw, nl.num_movable, 15, 0.08)
    gpu_ctx.set_option("lal_subtree_cells", 2048)
    gpu_ctx.set_option("lal_exact_sums", 1)
    gpu_ctx.upload_netlist(nl)
    legalizer = simpl.LookAheadLegalizer(gpu_ctx, grid.build_grid(nl, 24, 1.0),
                                         grid.build_free_space(nl), simpl.SimplOptions())
    px, py = x.copy(), y.copy()
    legalizer.legalize(px, py)
    ox, oy = run_oracle(nl, 24, 1.0, x, y)
    assert np.array_equal(px, ox) and np.array_equal(py, oy)
