"""nmhd_diagnostics (the FP64 reduction kernel k_diag) against an independent
FP64 numpy computation from the state read back through the C ABI.

The quantities follow the reference's two diagnostics:
  * the conservation dump of src/application/convergence_demo/
    mhd_solver.curb:61-100: momentum, kinetic, internal, magnetic and total
    energy summed over the cells times dV (there over all kSize cells with
    e_mag = (Bx^2 + By^2 + Bz^2)/2 of each cell's lower faces; its sums square
    float values in float, sq() of src/library/math.h:25, so the comparison
    here is with the exact FP64 sums, which the kernel computes);
  * the Kepler monitor of src/application/kepler_disk_demo/
    mhd_solver.curb:107-130: <Bx^2> and <By^2> over every entry of the face
    arrays, margins included;
and the two added ones: -<Bx By> with B averaged to cell centres, and
max |div B| over the interior cells.

Tolerance: 1e-12 relative to each quantity's scale (FP64 sums in a different
order).
"""

import numpy as np
import pytest

from nmhd_b200.problems import orszag_tang_3d, shearing_box
from nmhd_b200.solver import MHDSolver

pytestmark = pytest.mark.gpu

TOL = 1e-12


def fp64_diagnostics(cfg, state):
    """The diagnostics of `state` (8, Sz, Sy, Sx) in FP64: sums over the
    interior cells (Y and Z margins excluded), upper faces by periodic wrap."""
    d = cfg.derived()
    dx, dy, dz = float(d["dx"]), float(d["dy"]), float(d["dz"])
    w = state.astype(np.float64)
    rho, vx, vy, vz, p, bx, by, bz = w
    bxh = np.roll(bx, -1, axis=2)
    byh = np.roll(by, -1, axis=1)
    bzh = np.roll(bz, -1, axis=0)
    my, mz = cfg.margin_y, cfg.margin_z
    inner = (slice(mz, cfg.size_z - mz), slice(my, cfg.size_y - my), slice(None))
    dv = dx * dy * dz
    I = lambda a: a[inner]
    mass = I(rho).sum() * dv
    mom = [(I(rho) * I(v)).sum() * dv for v in (vx, vy, vz)]
    kin = (0.5 * I(rho) * (I(vx) ** 2 + I(vy) ** 2 + I(vz) ** 2)).sum() * dv
    eint = (I(p) / (float(np.float32(cfg.gamma)) - 1.0)).sum() * dv
    mag = (0.25 * (I(bx) ** 2 + I(bxh) ** 2 + I(by) ** 2 + I(byh) ** 2 + I(bz) ** 2 + I(bzh) ** 2)).sum() * dv
    vol = I(rho).size * dv
    stress = (-(0.25 * (I(bx) + I(bxh)) * (I(by) + I(byh)))).sum() * dv / vol
    divb = np.abs((I(bxh) - I(bx)) / dx + (I(byh) - I(by)) / dy + (I(bzh) - I(bz)) / dz).max()
    return {"mass": mass, "momentum": mom, "kinetic_energy": kin, "internal_energy": eint,
            "magnetic_energy": mag, "total_energy": kin + eint + mag, "volume": vol,
            "maxwell_stress": stress, "max_div_b": divb,
            # Kepler monitor: every entry of the face arrays
            "bx2_mean": (bx ** 2).mean(), "by2_mean": (by ** 2).mean(),
            # scales for quantities that can be near zero
            "_mom_scale": (np.abs(I(rho) * np.sqrt(I(vx) ** 2 + I(vy) ** 2 + I(vz) ** 2))).sum() * dv,
            "_stress_scale": (0.25 * np.abs((I(bx) + I(bxh)) * (I(by) + I(byh)))).sum() * dv / vol,
            "_b2_scale": max((bx ** 2).mean(), (by ** 2).mean(), (bz ** 2).mean())}


def reference_dump_form(cfg, state):
    """The convergence demo's dump (convergence_demo/mhd_solver.curb:74-95)
    over all kSize cells with each cell's lower-face B, in exact FP64."""
    d = cfg.derived()
    dv = float(d["dx"]) * float(d["dy"]) * float(d["dz"])
    rho, vx, vy, vz, p, bx, by, bz = state.astype(np.float64)
    kin = (0.5 * rho * (vx ** 2 + vy ** 2 + vz ** 2)).sum() * dv
    eint = (p / (float(np.float32(cfg.gamma)) - 1.0)).sum() * dv
    mag = (0.5 * (bx ** 2 + by ** 2 + bz ** 2)).sum() * dv
    return {"momentum": [(rho * v).sum() * dv for v in (vx, vy, vz)], "kinetic_energy": kin,
            "internal_energy": eint, "magnetic_energy": mag, "total_energy": kin + eint + mag}


def close(a, b, scale):
    return abs(a - b) <= TOL * max(abs(b), scale)


@pytest.mark.parametrize("case", ["orszag_tang_32", "mri_box_with_margins"])
def test_diagnostics_match_fp64_numpy(gpu, case):
    if case == "orszag_tang_32":
        cfg, s = orszag_tang_3d(32)
        steps = 12
    else:
        cfg, s = shearing_box(n_radial=32, n_azimuthal=64, n_vertical=16, l_azimuthal=2.0, seed=41)
        cfg.margin_z, cfg.size_z = 2, 20
        s = np.ascontiguousarray(np.concatenate([s[:, -2:], s, s[:, :2]], axis=1))
        steps = 15
    with MHDSolver(cfg) as sol:
        sol.set_state(s)
        sol.step(steps)
        st = sol.get_state()
        got = sol.diagnostics()
    ref = fp64_diagnostics(cfg, st)
    for k in ("mass", "kinetic_energy", "internal_energy", "magnetic_energy", "total_energy", "volume"):
        assert close(got[k], ref[k], 0.0), (k, got[k], ref[k])
    for a, b in zip(got["momentum"], ref["momentum"]):
        assert close(a, b, ref["_mom_scale"]), ("momentum", a, b)
    assert close(got["maxwell_stress"], ref["maxwell_stress"], ref["_stress_scale"])
    assert close(got["bx2_mean"], ref["bx2_mean"], ref["_b2_scale"])
    assert close(got["by2_mean"], ref["by2_mean"], ref["_b2_scale"])
    assert close(got["max_div_b"], ref["max_div_b"], 0.0)
    assert got["max_div_b"] > 0.0 and got["magnetic_energy"] > 0.0
    if case == "orszag_tang_32":
        # a periodic box without margins: every face is one cell's lower face
        # and another's upper face, so the face-averaged magnetic energy is the
        # reference dump's lower-face sum; the other totals are its sums
        dump = reference_dump_form(cfg, st)
        for k in ("kinetic_energy", "internal_energy", "magnetic_energy", "total_energy"):
            assert close(got[k], dump[k], 0.0), (k, got[k], dump[k])
        for a, b in zip(got["momentum"], dump["momentum"]):
            assert close(a, b, ref["_mom_scale"])
