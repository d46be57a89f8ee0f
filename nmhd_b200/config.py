"""Runtime solver configuration (the reference's compile-time constants).

The reference fixes sizes, extents and physics at compile time in a generated
``simulation_config.h`` (defaults src/library/simulation_config_default.h,
overrides src/application/*/simulation_config.hrb).  Here they form one
runtime struct, ``nmhd_config`` in include/nmhd.h, mirrored by
:class:`SolverConfig`.  :meth:`SolverConfig.derived` restates the float32
chains the reference uses to derive spacings and extents
(simulation_config_default.h:56-103), so a solver built from this struct uses
bit-identical constants.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, asdict

import numpy as np

PROBLEMS = {"none": 0, "shearing_box": 1}
# nmhd_config.flags bits (nmhd_flag in include/nmhd.h)
FLAG_HALO_PER_STAGE = 1  # refill the RK2 predictor's margins before the second stage
FLAG_FAST_ARITHMETIC = 2  # contracted, approximate face-flux arithmetic (not bitwise)


class NmhdConfig(ctypes.Structure):
    """ctypes mirror of ``nmhd_config`` (include/nmhd.h)."""

    _fields_ = [
        ("size_x", ctypes.c_int32), ("size_y", ctypes.c_int32), ("size_z", ctypes.c_int32),
        ("margin_y", ctypes.c_int32), ("margin_z", ctypes.c_int32),
        ("extent_x", ctypes.c_float), ("extent_y", ctypes.c_float), ("extent_z", ctypes.c_float),
        ("gamma", ctypes.c_float), ("cfl", ctypes.c_float),
        ("problem", ctypes.c_int32), ("q", ctypes.c_float), ("omega", ctypes.c_float),
        ("space_order", ctypes.c_int32), ("time_order", ctypes.c_int32),
        ("flags", ctypes.c_int32), ("parallel_size_y", ctypes.c_int32),
    ]


@dataclass
class SolverConfig:
    """Sizes include margins (the reference's kSize{X,Y,Z}); extents are of the
    interior (kGlobalExtent{X,Y,Z}).  Margins exist only in Y (shearing
    direction) and Z, as in the reference's slab decomposition."""

    size_x: int
    size_y: int
    size_z: int
    margin_y: int = 0
    margin_z: int = 0
    extent_x: float = 1.0
    extent_y: float = 1.0
    extent_z: float = 1.0
    gamma: float = 5.0 / 3.0
    cfl: float = 0.4
    problem: str = "none"
    q: float = 1.5
    omega: float = 1.0
    space_order: int = 2
    time_order: int = 2
    flags: int = 0
    # kParallelSizeY: > 1 makes this one radial slab of a box split over that
    # many ranks (size_y: the slab's rows and margins; extent_y: the box's)
    parallel_size_y: int = 1

    @property
    def shape(self):
        """numpy shape of one field: (Sz, Sy, Sx)."""
        return (self.size_z, self.size_y, self.size_x)

    @property
    def cells(self):
        return self.size_x * self.size_y * self.size_z

    @property
    def interior_cells(self):
        return self.size_x * (self.size_y - 2 * self.margin_y) * (self.size_z - 2 * self.margin_z)

    def to_ctypes(self):
        d = asdict(self)
        d["problem"] = PROBLEMS[self.problem]
        return NmhdConfig(**d)

    def derived(self):
        """Spacings and extents exactly as the reference's float32 chains give them."""
        f = np.float32
        loc = (self.size_x, self.size_y - 2 * self.margin_y, self.size_z - 2 * self.margin_z)
        g = (loc[0], max(1, self.parallel_size_y) * loc[1], loc[2])
        s = (self.size_x, self.size_y, self.size_z)
        ext = (self.extent_x, self.extent_y, self.extent_z)
        out = {}
        for name, gi, si, li, ni in zip("xyz", g, s, ext, loc):
            comp_ext = f(f(f(li) / f(gi)) * f(si))          # kExtent
            local_ext = f(f(f(li) / f(gi)) * f(ni))         # kLocalExtent
            out["extent_" + name] = comp_ext
            out["local_extent_" + name] = local_ext
            out["d" + name] = f(comp_ext / f(si))           # kD
            out["corner_" + name] = f(-comp_ext / f(2))     # -gExtent/2
        out["relative_velocity"] = float(f(f(f(-self.q) * f(self.omega)) * out["local_extent_y"]))
        return out
