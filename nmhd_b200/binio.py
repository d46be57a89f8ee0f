"""Reader/writer for the reference's state dump format (``.bin``).

Layout (``MHDSolver::read``/``write``, src/library/mhd_solver.inlrb:995-1014,
helpers ``fread_singlet``/``fread_device`` src/library/mhd_solver.hrb:216-235):

* three native int32: the computational sizes Sx, Sy, Sz (margins included);
* eight arrays of Sx*Sy*Sz ``Real`` (float32 here; float64 for double
  builds): density, velocity x, y, z, pressure, magnet x, y, z;
* every array is x-fastest, i.e. element (x, y, z) sits at
  ``(z*Sy + y)*Sx + x`` (src/library/crystal.hrb:45).  As numpy arrays they
  have shape (Sz, Sy, Sx).

Magnet component d at index (x, y, z) is the field on the lower d-face of cell
(x, y, z) (src/library/crystal.hrb:106-131).
"""
from __future__ import annotations

import numpy as np

FIELDS = ("density", "velocity_x", "velocity_y", "velocity_z", "pressure",
          "magnet_x", "magnet_y", "magnet_z")


def write_bin(path, state, dtype=np.float32):
    """Write ``state`` (array (8, Sz, Sy, Sx)) in the reference's format."""
    state = np.asarray(state)
    if state.ndim != 4 or state.shape[0] != 8:
        raise ValueError("state must have shape (8, Sz, Sy, Sx)")
    sz, sy, sx = state.shape[1:]
    with open(path, "wb") as fp:
        np.array([sx, sy, sz], dtype=np.int32).tofile(fp)
        np.ascontiguousarray(state, dtype=dtype).tofile(fp)


def read_bin(path, dtype=np.float32, expect_shape=None):
    """Read a reference ``.bin`` dump; returns an array (8, Sz, Sy, Sx).

    Raises ``ValueError`` on a size mismatch with ``expect_shape`` (Sx, Sy, Sz)
    or a truncated file, where the reference's ``read`` returns false.
    """
    with open(path, "rb") as fp:
        head = np.fromfile(fp, dtype=np.int32, count=3)
        if head.size != 3:
            raise ValueError(f"{path}: truncated header")
        sx, sy, sz = (int(v) for v in head)
        if expect_shape is not None and tuple(expect_shape) != (sx, sy, sz):
            raise ValueError(f"{path}: sizes {(sx, sy, sz)} != expected {tuple(expect_shape)}")
        n = sx * sy * sz
        data = np.fromfile(fp, dtype=dtype, count=8 * n)
    if data.size != 8 * n:
        raise ValueError(f"{path}: truncated data ({data.size} of {8 * n} values)")
    return data.reshape(8, sz, sy, sx)
