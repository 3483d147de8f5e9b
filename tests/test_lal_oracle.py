"""The look-ahead-legalization restatement (oracle/lal_ref.py) pinned against
the reference's own LookAheadLegalizer (oracle/_ref): bit-identical positions
on seeded designs with macros. CPU only."""
import resource

import numpy as np
import pytest

import oracle
from oracle import lal_ref
from ktplace_b200 import grid, netlist, synth

pytestmark = pytest.mark.skipif(not oracle.ref_available(), reason="reference library not built")


@pytest.fixture(autouse=True, scope="module")
def big_stack():
    # the reference's recursion wants more than the default main-thread stack
    try:
        resource.setrlimit(resource.RLIMIT_STACK, (resource.RLIM_INFINITY, resource.RLIM_INFINITY))
    except (ValueError, OSError):
        pass


@pytest.mark.parametrize("seed,cells,macros,bins", [(2, 400, 3, 16), (5, 900, 4, 24), (7, 600, 0, 8)])
def test_restatement_matches_reference(seed, cells, macros, bins):
    raw = synth.generate(synth.spec_tiny(seed=seed, macros=macros, cells=cells, nets=cells + 30))
    nl = netlist.flatten(raw)
    for pos_seed in (11, 12):
        x, y = synth.seed_positions(raw, nl.num_movable, pos_seed)
        ref = oracle.RefDesign.from_netlist(nl)
        g = ref.grid(bins, 1.0)
        rx, ry = ref.lal(x, y)
        rows, rs, spans = ref.free_space()
        L = lal_ref.LAL(nl.width, nl.height, g, lal_ref.free_rows(rows, rs, spans),
                        nl.obstacles, nl.die, 1.0)
        px, py = L.legalize(x, y)
        assert np.array_equal(np.array(px), rx)
        assert np.array_equal(np.array(py), ry)
        assert np.mean(rx != x) > 0.1  # legalization did move cells


def _clustered(raw, n, seed, spread):
    rng = np.random.default_rng(seed)
    lx, ly, ux, uy = raw.die
    return (0.5 * (lx + ux) + spread * (ux - lx) * rng.standard_normal(n),
            0.5 * (ly + uy) + spread * (uy - ly) * rng.standard_normal(n))


@pytest.mark.parametrize("seed,cells,macros,bins,density", [(5, 900, 4, 24, 1.0), (9, 700, 2, 12, 0.9),
                                                            (7, 600, 0, 8, 0.8)])
def test_restatement_clustered_and_density(seed, cells, macros, bins, density):
    """Cells started in a tight cluster (one region, deep bisection) and
    density limits below 1, on the host free space the GPU path installs."""
    raw = synth.generate(synth.spec_tiny(seed=seed, macros=macros, cells=cells, nets=cells + 30))
    nl = netlist.flatten(raw)
    x, y = _clustered(raw, nl.num_movable, seed + 10, 0.08)
    ref = oracle.RefDesign.from_netlist(nl)
    g = ref.grid(bins, density)
    rx, ry = ref.lal(x, y)
    fs = grid.build_free_space(nl)
    L = lal_ref.LAL(nl.width, nl.height, g, lal_ref.free_rows(fs.row_y, fs.row_span, fs.spans),
                    fs.obstacles, fs.die, density)
    px, py = L.legalize(x, y)
    assert np.array_equal(np.array(px), rx) and np.array_equal(np.array(py), ry)


@pytest.mark.parametrize("seed,cells,macros", [(2, 400, 3), (5, 900, 4), (7, 600, 0)])
def test_host_free_space_matches_reference(seed, cells, macros):
    """grid.build_free_space (what ktg_set_free_space receives) equals the
    reference's FreeSpace rows and spans."""
    raw = synth.generate(synth.spec_tiny(seed=seed, macros=macros, cells=cells, nets=cells + 30))
    nl = netlist.flatten(raw)
    ref = oracle.RefDesign.from_netlist(nl)
    ref.grid(16, 1.0)
    rows, rs, spans = ref.free_space()
    fs = grid.build_free_space(nl)
    assert np.array_equal(rows, fs.row_y)
    assert np.array_equal(rs, fs.row_span)
    assert np.array_equal(spans, fs.spans)
