"""CPU checks of the staged kernels' shared-memory index arithmetic, with the
box constants read from the CUDA headers themselves
(nmhd_b200/csrc/cell_flux_staged.cuh, cell_epilogue.cuh), so that a change of
tile or box shape that would read outside a staged box fails here, before any
GPU run.

Staged flux kernel: every read face_flux() makes for the three lower faces of
each cell of a 32 x 4 x 2 tile (the 4-cell stencil along the face axis, the
+1 transverse neighbours of the face-centred B, the shear half-kick's two
cells and the normal B) lies inside its field's box, and that box position
holds the cell the reference's periodic neighbour offsets name.

Fused epilogue: the staged boxes cover every cell, edge and face its phases
read (corner EMFs of the tile and its upper halo edges, new face B, the
cell update's lower and upper faces)."""
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "..", "nmhd_b200", "csrc")


def header(name):
    with open(os.path.join(CSRC, name)) as f:
        return f.read()


def sfx_constants():
    t = header("cell_flux_staged.cuh")
    m = re.search(r"constexpr int P = (\d+), NJ = (\d+), NK = (\d+), XO = (\d+);", t)
    assert m, "staged box constants not found"
    P, NJ, NK, XO = map(int, m.groups())
    # the box origin relative to the tile: x0 - XO, y0 - 2, z0 - 2 (tensor copy
    # coordinates and the wrapped offset tables)
    assert '"r"(x0 - XO), "r"(y0 - 2), "r"(z0 - 2)' in t
    assert "wrap_any(x0 - XO + tid, g.sx)" in t and "wrap_any(y0 - 2 + (tid - P), g.sy)" in t
    assert re.search(r"return \(\(c \+ 2\) \* NJ \+ \(b \+ 2\)\) \* P \+ XO \+ a;", t), "at() changed"
    return P, NJ, NK, XO


def test_staged_flux_reads_stay_in_their_boxes():
    P, NJ, NK, XO = sfx_constants()
    DY, DZ, FS = P, P * NJ, P * NJ * NK

    def at(a, b, c):
        return ((c + 2) * NJ + (b + 2)) * P + XO + a

    def cell_of(idx):
        """Tile-local cell held at shared index idx (within one field)."""
        assert 0 <= idx < FS, idx
        k, r = divmod(idx, P * NJ)
        j, i = divmod(r, P)
        return i - XO, j - 2, k - 2

    for c in range(2):
        for b in range(4):
            for a in range(32):
                ci = at(a, b, c)
                for ax in range(3):
                    sa = (1, DY, DZ)[ax]
                    t1 = (DY, DZ, 1)[ax]
                    t2 = (DZ, 1, DY)[ax]
                    unit = [(1, 0, 0), (0, 1, 0), (0, 0, 1)]
                    e1, e2 = (ax + 1) % 3, (ax + 2) % 3
                    for s, d in ((-2 * sa, -2), (-sa, -1), (0, 0), (sa, 1)):
                        want = tuple(p + d * u for p, u in zip((a, b, c), unit[ax]))
                        assert cell_of(ci + s) == want
                        # face-centred transverse B: the cell and its +1 along e1 / e2
                        assert cell_of(ci + s + t1) == tuple(w + u for w, u in zip(want, unit[e1]))
                        assert cell_of(ci + s + t2) == tuple(w + u for w, u in zip(want, unit[e2]))


def epi_boxes():
    t = header("cell_epilogue.cuh")
    boxes = {}
    for name, ni, nj, nk, oi, oj, ok in re.findall(
            r"using (\w+) = Staged<(\d+), (\d+), (\d+), (-?\d+), (-?\d+), (-?\d+)>;", t):
        boxes[name] = tuple(map(int, (ni, nj, nk, oi, oj, ok)))
    for name, ni, nj, nk, oi, oj, ok in re.findall(
            r"using (\w+) = Box<(\d+), (\d+), (\d+), (-?\d+), (-?\d+), (-?\d+)>;", t):
        boxes[name] = tuple(map(int, (ni, nj, nk, oi, oj, ok)))
    return boxes


def covers(box, a, b, c):
    ni, nj, nk, oi, oj, ok = box
    return oi <= a < oi + ni and oj <= b < oj + nj and ok <= c < ok + nk


def test_epilogue_boxes_cover_every_read():
    B = epi_boxes()
    for n in ("VelBox", "XYF", "YXF", "XZF", "ZXF", "YZF", "ZYF", "BXs", "BYs", "BZs", "ZEdge", "YEdge", "XEdge"):
        assert n in B, n
    # corner EMFs at the edges of tile-local cell (a, b, c) for the tile's
    # cells and the upper halo edges (z-edges at b = 4 and a = 32, y-edges at
    # c = 2 and a = 32, x-edges at b = 4 and c = 2)
    z_edges = {(a, b, c) for a in range(33) for b in range(5) for c in range(2)}
    y_edges = {(a, b, c) for a in range(33) for b in range(4) for c in range(3)}
    x_edges = {(a, b, c) for a in range(32) for b in range(5) for c in range(3)}
    for (a, b, c) in z_edges:
        assert covers(B["ZEdge"], a, b, c)
        for da, db in ((0, 0), (-1, 0), (0, -1), (-1, -1)):  # the 4 cells' v around the edge
            assert covers(B["VelBox"], a + da, b + db, c)
        assert covers(B["XYF"], a, b, c) and covers(B["XYF"], a, b - 1, c)
        assert covers(B["YXF"], a, b, c) and covers(B["YXF"], a - 1, b, c)
    for (a, b, c) in y_edges:
        assert covers(B["YEdge"], a, b, c)
        for da, dc in ((0, 0), (-1, 0), (0, -1), (-1, -1)):
            assert covers(B["VelBox"], a + da, b, c + dc)
        assert covers(B["XZF"], a, b, c) and covers(B["XZF"], a, b, c - 1)
        assert covers(B["ZXF"], a, b, c) and covers(B["ZXF"], a - 1, b, c)
    for (a, b, c) in x_edges:
        assert covers(B["XEdge"], a, b, c)
        for db, dc in ((0, 0), (-1, 0), (0, -1), (-1, -1)):
            assert covers(B["VelBox"], a, b + db, c + dc)
        assert covers(B["YZF"], a, b, c) and covers(B["YZF"], a, b, c - 1)
        assert covers(B["ZYF"], a, b, c) and covers(B["ZYF"], a, b - 1, c)
    # new face B of the tile's faces and the upper halo faces read the edges
    # at the face and one step up the two transverse axes
    for a in range(33):
        for b in range(4):
            for c in range(2):
                assert covers(B["BXs"], a, b, c)
                for e, pts in (("ZEdge", ((a, b, c), (a, b + 1, c))), ("YEdge", ((a, b, c), (a, b, c + 1)))):
                    assert all(covers(B[e], *p) for p in pts)
    for a in range(32):
        for b in range(5):
            for c in range(2):
                assert covers(B["BYs"], a, b, c)
                assert covers(B["ZEdge"], a, b, c) and covers(B["ZEdge"], a + 1, b, c)
                assert covers(B["XEdge"], a, b, c) and covers(B["XEdge"], a, b, c + 1)
        for b in range(4):
            for c in range(3):
                assert covers(B["BZs"], a, b, c)
                assert covers(B["YEdge"], a, b, c) and covers(B["YEdge"], a + 1, b, c)
                assert covers(B["XEdge"], a, b, c) and covers(B["XEdge"], a, b + 1, c)
