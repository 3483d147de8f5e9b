"""The library's Bookshelf reader (ktg_bookshelf_read) against the
reference's own reader + buildSimplDM (oracle/_ref), CPU only.

Bar: every flattened array, the obstacles, the rows and the die are
bit-identical, on synthetic designs and on hand-written files that hit the
reader's corner cases (comments, CRLF, terminal_NI, repeated names, name-less
and repeated nets, short degrees, pins without offsets or with unknown cells,
/FIXED_NI, lowercase .scl keys, two subrows in a row, gzip)."""
import gzip
import os
import shutil

import numpy as np
import pytest

import oracle
from ktplace_b200 import bookshelf, synth

pytestmark = pytest.mark.skipif(not oracle.ref_available(), reason="reference library not built")

KEYS = ("mov_vertex", "fixed_x", "fixed_y", "net_start", "pin_cell", "off_x", "off_y",
        "net_weight", "pin_start", "pin_net", "pin_q", "width", "height")


def check_same(d):
    nl = bookshelf.read(d)
    e = oracle.RefDesign.from_bookshelf(d).export()
    for k in KEYS:
        assert np.array_equal(np.asarray(getattr(nl, k)).astype(e[k].dtype), e[k]), k
    var = e["var_of_vertex"].astype(np.int64)
    var[var == 2 ** 32 - 1] = -1
    assert np.array_equal(nl.var_of_vertex, var)
    assert tuple(nl.die) == tuple(e["die"])
    assert np.array_equal(nl.obstacles, e["obstacles"])
    assert np.array_equal(nl.rows, e["rows"])
    return nl


@pytest.mark.parametrize("spec", [synth.spec_tiny(seed=3, macros=3, cells=500, nets=520),
                                  synth.spec_small(seed=0)])
def test_synthetic_designs(spec, tmp_path):
    raw = synth.generate(spec)
    d = os.path.join(str(tmp_path), raw.name)
    synth.write_bookshelf(raw, d)
    check_same(d)


NODES = """UCLA nodes 1.0
# a comment line
NumNodes : 9\r
NumTerminals : 3

a  4 12
b  2 12   # trailing comment
c  3 12
b  9 12
d  x 12
e  1 12
m  20 24 terminal
p1 0 0 terminal
p2 0 0 terminal_NI
"""

WTS = """UCLA wts 1.0
n_ab 2.5
n_ab 3.0
nnn 7
"""

NETS = """UCLA nets 1.0
NumNets : 6
NumPins : 15

NetDegree : 3 n_ab
  a I : 0.5 -1.0
  b O : -0.25 2
  m B
NetDegree 2 n_cd
  c I : 1 1
  zz I : 0 0
  d I : 0 0
NetDegree : 2
  a I : 0 0
  p1 O : 0 0
NetDegree : 2 n_ab
  e I : 0.125 0
  c O
NetDegree : 1 lonely
  x
  e O : 0 0
NetDegree : 4 wide
  a I : 0 0
  b I : 0 0
  e I : 0 0
  p2 I : 0 0
"""

PL = """UCLA pl 1.0

a 10 12 : N
b 20.5 24 : N
c 30 36 : FS
e 3 0 : N /FIXED
m 40 0 : N /FIXED
p1 0 0 : N /FIXED
p2 100 60 : N /FIXED_NI
ghost 5 5 : N
"""

SCL = """UCLA scl 1.0
NumRows : 4

CoreRow Horizontal
  coordinate : 0
  height : 12
  sitewidth : 1
  sitespacing : 1
  SubrowOrigin : 0 numsites : 50
  SubrowOrigin : 60 NumSites : 40
End
CoreRow Horizontal
  Coordinate : 12
  Height : 12
  Sitewidth : 2
  Sitespacing : 0
  SubrowOrigin : 0 NumSites : 60
End
CoreRow Horizontal
  Coordinate : 24
  Height : 12
End
CoreRow Horizontal
  Coordinate : 36
  Height : 12
  Sitewidth : 1
  Sitespacing : 1
  SubrowOrigin : 5 NumSites : 80
End
"""


def write_edge(d, gz=False):
    os.makedirs(d, exist_ok=True)
    name = os.path.basename(d)
    for ext, text in ((".nodes", NODES), (".wts", WTS), (".nets", NETS), (".pl", PL),
                      (".scl", SCL)):
        path = os.path.join(d, name + ext)
        if gz:
            with gzip.open(path + ".gz", "wt") as f:
                f.write(text)
        else:
            with open(path, "w", newline="") as f:
                f.write(text)


def test_hand_written_corner_cases(tmp_path):
    d = os.path.join(str(tmp_path), "edgecase")
    write_edge(d)
    nl = check_same(d)
    # the checks above compare with the reference; a few facts for the reader
    assert nl.num_vertices == 7           # repeated "b" and malformed "d" dropped
    assert nl.num_movable == 4            # e is /FIXED, m and p1 terminals; p2 terminal_NI
    assert nl.net_weight[0] == 3.0        # last .wts line wins, first net keeps it


def test_gzip_inputs(tmp_path):
    d = os.path.join(str(tmp_path), "edgegz")
    write_edge(d, gz=True)
    check_same(d)


def test_missing_nodes_is_an_error(tmp_path):
    d = os.path.join(str(tmp_path), "nothing")
    os.makedirs(d)
    from ktplace_b200._lib import KtgError
    with pytest.raises(KtgError):
        bookshelf.read(d)


def test_grid_and_free_space_follow_subrows(tmp_path):
    """A row split into subrows with a gap that no obstacle covers: the bin
    grid's free area and the legalizer's free space come from the subrows,
    as the reference's buildGrid takes them, and match the reference."""
    if not oracle.ref_available():
        pytest.skip("reference library not built")
    from ktplace_b200 import grid
    scl = SCL.replace("""  Sitespacing : 0
  SubrowOrigin : 0 NumSites : 60
End""", """  Sitespacing : 0
  SubrowOrigin : 0 NumSites : 15
  SubrowOrigin : 70 NumSites : 25
End""")
    d = os.path.join(str(tmp_path), "gapped")
    os.makedirs(d)
    for ext, text in ((".nodes", NODES), (".wts", WTS), (".nets", NETS), (".pl", PL), (".scl", scl)):
        with open(os.path.join(d, "gapped" + ext), "w", newline="") as f:
            f.write(text)
    nl = bookshelf.read(d)
    ref = oracle.RefDesign.from_bookshelf(d)
    for bins in (4, 8):
        g = ref.grid(bins, 1.0)
        mine = grid.build_grid(nl, bins, 1.0)
        assert np.array_equal(mine.avail, g["avail"]) and mine.total_avail == g["total_avail"]
    rows, rs, spans = ref.free_space()
    fs = grid.build_free_space(nl)
    assert np.array_equal(rows, fs.row_y) and np.array_equal(rs, fs.row_span)
    assert np.array_equal(spans, fs.spans)
    assert [30.0, 70.0] in [[a, b] for a, b in zip(spans[:-1, 1], spans[1:, 0])]  # the gap
