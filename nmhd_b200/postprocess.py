"""Snapshot post-processing: a snapshot folder of per-rank dumps stitched onto
the global grid, with the shearing-box displacement un-applied.

Restates the reference's post-processors src/tools/parallel/to_gnuplot.cpp
(whole grid as gnuplot text on stdout, at most 720 cells per axis) and
to_gnuplot_3d.cpp (three mid-plane cross sections, at most 120 cells per axis,
cells that wrapped across the radial boundary dropped).  A folder holds, for
each rank r of the run, ``%04d.bin`` and ``%04d_setup.txt`` as save_state
writes them (MHDSolver.save_state and nmhd::MHDSolver::save_state write rank
0000 of a one-rank run; reference runs write one pair per MPI rank).

Every rank's cells (margins included) are placed by their centres: the
azimuthal coordinate shifted by the displacement accumulated over the radial
ranks below, v_x raised by the accumulated shear velocity, then binned onto the
output grid and averaged.  The float operations follow the tools' Real =
float arithmetic and the accumulation their order, so the text is theirs.

    python -m nmhd_b200.postprocess FOLDER               # to_gnuplot
    python -m nmhd_b200.postprocess FOLDER OUT_PREFIX    # to_gnuplot_3d
"""
from __future__ import annotations

import os
import sys

import numpy as np

from .binio import read_bin
from .checkpoint import parse_setup

F = np.float32
ITEMS = 8


def _pods(path):
    with open(path) as fp:
        return parse_setup(fp.read())


def _get(glob, loc, key, typ):
    # read_hash: the rank's LocalSetup first, then GlobalSetup
    v = loc[key] if key in loc else glob[key]
    return int(v) if typ is int else F(float(v))


def stitch(folder, max_resolution=720, drop_wrapped=False):
    """Average of every field on the output grid.  Returns (sizes (nx, ny,
    nz), corner (3 floats), extent (3 floats), numerators, denominators):
    numerators[item] float64 and denominators int64, shape (nz, ny, nx)."""
    prefix = os.path.join(folder, "")
    glob, loc = _pods(prefix + "0000_setup.txt")
    if _get(glob, loc, "real_size", int) != 4:
        raise ValueError("only Real = float snapshots are supported")
    size = [min(max_resolution, _get(glob, loc, "global_size_" + a, int)) for a in "xyz"]
    corner = [_get(glob, loc, "global_corner_" + a, float) for a in "xyz"]
    extent = [_get(glob, loc, "global_extent_" + a, float) for a in "xyz"]
    n_out = size[0] * size[1] * size[2]
    num = np.zeros((ITEMS, n_out), np.float64)
    den = np.zeros((ITEMS, n_out), np.int64)
    py = _get(glob, loc, "parallel_size_y", int)
    ranks = _get(glob, loc, "parallel_size", int)
    disp = np.zeros(py, np.float64)  # integrated_displacement
    vel = np.zeros(py, np.float64)   # integrated_velocity
    for rank in range(ranks):
        g1, loc = _pods(prefix + "%04d_setup.txt" % rank)
        if g1 != glob:
            raise ValueError("global setup differs: %04d_setup.txt" % rank)
        isz = [_get(glob, loc, "computational_size_" + a, int) for a in "xyz"]
        icorner = [_get(glob, loc, "computational_corner_" + a, float) for a in "xyz"]
        iextent = [_get(glob, loc, "computational_extent_" + a, float) for a in "xyz"]
        ry_rank = rank % py
        if ry_rank < py - 1:
            disp[ry_rank + 1] = disp[ry_rank] + float(_get(glob, loc, "relative_displacement", float))
            vel[ry_rank + 1] = vel[ry_rank] + float(_get(glob, loc, "relative_velocity", float))
        state = read_bin(prefix + "%04d.bin" % rank)
        if tuple(state.shape[1:]) != (isz[2], isz[1], isz[0]):
            raise ValueError("size mismatch in %04d.bin" % rank)
        # cell centres (decode_real), x shifted by the accumulated displacement
        z, y, x = np.meshgrid(np.arange(isz[2]), np.arange(isz[1]), np.arange(isz[0]), indexing="ij")
        pos = []
        for c, sz, co, ex in ((x, isz[0], icorner[0], iextent[0]), (y, isz[1], icorner[1], iextent[1]),
                              (z, isz[2], icorner[2], iextent[2])):
            pos.append(co + (c.astype(F) + F(0.5)) / F(sz) * ex)
        pos[0] = (pos[0].astype(np.float64) + disp[ry_rank]).astype(F)
        # output cell (encode_real), periodic, and the radial wrap count
        idx = []
        carry = None
        for k in range(3):
            i0 = np.floor((pos[k] - corner[k]) / extent[k] * F(size[k])).astype(np.int64)
            iw = ((i0 % size[k]) + size[k]) % size[k]
            if k == 1:
                carry = (iw - i0) // size[k]
            idx.append(iw)
        addr = ((idx[2] * size[1] + idx[1]) * size[0] + idx[0]).ravel()
        keep = np.ones(addr.shape, bool) if not drop_wrapped else (carry.ravel() == 0)
        for item in range(ITEMS):
            val = state[item].ravel()
            if item == 1:
                if drop_wrapped:
                    boost = (vel[ry_rank] + (F(py) * _get(glob, loc, "relative_velocity", float)
                                             * carry.ravel().astype(F)).astype(np.float64)).astype(F)
                else:
                    boost = F(vel[ry_rank])
                val = (val + boost).astype(F)
            np.add.at(num[item], addr[keep], val[keep].astype(np.float64))
            np.add.at(den[item], addr[keep], 1)
    shape = (ITEMS, size[2], size[1], size[0])
    return size, corner, extent, num.reshape(shape), den.reshape(shape)


def _centre(k, i, size, corner, extent):
    return corner[k] + (F(i) + F(0.5)) / F(size[k]) * extent[k]


def _lines(size, corner, extent, num, den, xr, yr, zr):
    with np.errstate(invalid="ignore", divide="ignore"):
        avg = num / den
    out = []
    for z in range(*zr):
        for y in range(*yr):
            for x in range(*xr):
                vals = " ".join("%.6g" % avg[i, z, y, x] for i in range(ITEMS))
                out.append("%.6g %.6g %.6g %s" % (_centre(0, x, size, corner, extent),
                                                   _centre(1, y, size, corner, extent),
                                                   _centre(2, z, size, corner, extent), vals))
                if xr[1] - xr[0] > 1:
                    out.append("\n")
            if yr[1] - yr[0] > 1:
                out.append("\n")
        if zr[1] - zr[0] > 1:
            out.append("\n")
    # as in the tools, a data line ends with a newline only when the x range
    # has more than one cell
    return "".join(out)


def gnuplot_text(folder, max_resolution=720):
    """The text to_gnuplot prints for a snapshot folder."""
    size, corner, extent, num, den = stitch(folder, max_resolution)
    return _lines(size, corner, extent, num, den, (0, size[0]), (0, size[1]), (0, size[2]))


def sections(folder, max_resolution=120):
    """{"yz": text, "xz": text, "xy": text}: the three mid-plane sections
    to_gnuplot_3d writes to OUT_PREFIX_<plane>.txt."""
    size, corner, extent, num, den = stitch(folder, max_resolution, drop_wrapped=True)
    out = {}
    for axis, name in ((0, "yz"), (1, "xz"), (2, "xy")):
        r = [(0, size[0]), (0, size[1]), (0, size[2])]
        r[axis] = (size[axis] // 2, size[axis] // 2 + 1)
        out[name] = _lines(size, corner, extent, num, den, *r)
    return out


def main(argv):
    if len(argv) < 2:
        print(__doc__.strip().splitlines()[-2].strip(), file=sys.stderr)
        return 2
    if len(argv) == 2:
        sys.stdout.write(gnuplot_text(argv[1]))
        return 0
    for name, text in sections(argv[1]).items():
        with open("%s_%s.txt" % (argv[2], name), "w") as fp:
            fp.write(text)
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv))
