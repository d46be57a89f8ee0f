"""The per-stage margin fill (nmhd_config flag HALO_PER_STAGE), on the oracle.

The reference fills the margins once per step and advances them like the
interior: the second RK2 stage then reads margin cells that the first stage
computed in the margin's own frame (and, within two cells of the box edge,
from wrapped neighbours), so its interior depends on the margin width.  With
the flag, the predictor's margins are refilled from the interior predictor
(shear-shifted at t + dt/2) before the second stage: the interior results no
longer depend on the margin width, bitwise, from 2 cells up, and equal the
reference's scheme to truncation error.  The CUDA path is pinned bitwise to
this oracle mode in tests/test_parity_gpu.py.
"""
import numpy as np
import pytest

from nmhd_b200.config import FLAG_HALO_PER_STAGE
from nmhd_b200.problems import orszag_tang_3d, shearing_box
from oracle import oracle

STEPS = 12


def _ot(margin, flags):
    """16^3 Orszag-Tang box with periodic Y margins (no shear boost)."""
    cfg, s = orszag_tang_3d(16)
    cfg.margin_y, cfg.size_y, cfg.flags = margin, 16 + 2 * margin, flags
    return cfg, np.concatenate([s[:, :, -margin:], s, s[:, :, :margin]], axis=2)


def _shear(margin, flags, mz=0):
    cfg, s = shearing_box(n_radial=16, n_azimuthal=32, n_vertical=8, l_azimuthal=4.0, seed=21, margin=margin)
    cfg.flags = flags
    if mz:
        cfg.margin_z, cfg.size_z = mz, cfg.size_z + 2 * mz
        s = np.concatenate([s[:, -mz:], s, s[:, :mz]], axis=1)
    return cfg, s


def _interior(cfg, steps):
    def run(s):
        o = oracle.proceed(cfg, s, steps)
        st = o["state"]
        z0, y0 = cfg.margin_z, cfg.margin_y
        return st[:, z0:cfg.size_z - z0, y0:cfg.size_y - y0], o["time"], o["dts"]
    return run


def _case(kind, margin, flags):
    if kind == "ot":
        return _ot(margin, flags)
    if kind == "shear":
        return _shear(margin, flags)
    return _shear(margin, flags, mz=margin)


@pytest.mark.parametrize("kind", ["ot", "shear", "shear_mz"])
def test_per_stage_fill_is_independent_of_margin_width(kind):
    runs = {}
    for margin in (2, 3, 4):
        cfg, s = _case(kind, margin, FLAG_HALO_PER_STAGE)
        runs[margin] = _interior(cfg, STEPS)(s)
    for margin in (2, 3):
        st, t, dts = runs[margin]
        assert np.array_equal(st, runs[4][0]), margin
        assert t == runs[4][1] and np.array_equal(dts, runs[4][2])


def test_reference_scheme_depends_on_thin_margins():
    cfg2, s2 = _ot(2, 0)
    cfg4, s4 = _ot(4, 0)
    a = _interior(cfg2, STEPS)(s2)[0]
    b = _interior(cfg4, STEPS)(s4)[0]
    assert np.abs(a - b).max() > 1e-3


def test_per_stage_fill_agrees_with_the_reference_scheme_to_truncation():
    """Same box, margins 4: the two schemes differ only by how the margins of
    the predictor are obtained, a truncation-size difference."""
    cfg0, s0 = _ot(4, 0)
    cfg1, s1 = _ot(4, FLAG_HALO_PER_STAGE)
    a, ta, _ = _interior(cfg0, STEPS)(s0)
    b, tb, _ = _interior(cfg1, STEPS)(s1)
    # per quantity: density, velocity (all components), pressure, B (all components)
    groups = [[0], [1, 2, 3], [4], [5, 6, 7]]
    for grp in groups:
        scale = np.abs(a[grp]).max()
        assert (np.abs(a[grp] - b[grp]) / scale).max() < 0.1, grp
    assert np.abs(a - b).max() > 0
    assert abs(ta - tb) < 1e-4 * ta
