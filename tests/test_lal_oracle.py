"""The look-ahead-legalization restatement (oracle/lal_ref.py) pinned against
the reference's own LookAheadLegalizer (oracle/_ref): bit-identical positions
on seeded designs with macros. CPU only."""
import resource

import numpy as np
import pytest

import oracle
from oracle import lal_ref
from ktplace_b200 import synth, netlist

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
