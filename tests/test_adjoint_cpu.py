"""CPU checks of the differentiated step (host build of nmhd_b200/csrc/ad_*.cuh,
the same functors the CUDA adjoint kernels run).

- The generic forward (float / double) is bitwise the oracle, so the adjoint's
  recomputation takes the production branches and the FP64 runs are the
  reference's Real = double build.
- The tangent-linear HLLD flux matches central differences.
- The hand-written adjoint is the transpose of the tangent-linear map, for the
  HLLD flux alone and for whole steps (dot-product test: <grad, d> = dJ[d]).
- Along initial-velocity directions the tangent matches central differences
  of the FP64 loss on shearing boxes, and the FP32 adjoint is close to FP64.
"""
import numpy as np
import pytest

import adcheck
from nmhd_b200.problems import orszag_tang_3d, shearing_box
from oracle import oracle

GAMMA = 5.0 / 3.0


def _random_states(rng, n):
    """Riemann inputs covering all six fan regions (subsonic, supersonic both
    ways, Bx = 0)."""
    out = []
    for k in range(n):
        lr = np.empty(14)
        lr[0:2] = rng.uniform(0.3, 2.0, 2)
        lr[2:8] = rng.normal(0.0, 1.0, 6)
        if k % 7 == 0:
            lr[2:4] += rng.choice([-4.0, 4.0])  # supersonic: regions 0 and 5
        lr[8:10] = rng.uniform(0.2, 2.0, 2)
        lr[10:14] = rng.normal(0.0, 1.0, 4)
        bx = 0.0 if k % 5 == 0 else rng.normal(0.0, 1.0)
        out.append((bx, lr))
    return out


def test_generic_hlld_is_bitwise_the_oracle_in_all_regions():
    rng = np.random.default_rng(0)
    regions = np.zeros(6, int)
    for bx, lr in _random_states(rng, 4000):
        a = adcheck.hlld(GAMMA, np.float32(bx), lr.astype(np.float32), np.float32)
        b = oracle.hlld(np.float32(GAMMA), np.float32(bx), lr.astype(np.float32), np.float32)
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
        a = adcheck.hlld(GAMMA, bx, lr, np.float64)
        b = oracle.hlld(GAMMA, bx, lr, np.float64)
        assert np.array_equal(a, b)
        regions[adcheck.hlld_region(GAMMA, bx, lr)] += 1
    assert (regions > 0).all(), regions


def test_hlld_tangent_matches_central_differences():
    rng = np.random.default_rng(1)
    errs = []
    for bx, lr in _random_states(rng, 600):
        d = rng.normal(0.0, 1.0, 14)
        dbx = 0.0 if bx == 0.0 else rng.normal()
        eps = 1e-6
        if adcheck.hlld_region(GAMMA, bx + eps * dbx, lr + eps * d) != adcheck.hlld_region(
                GAMMA, bx - eps * dbx, lr - eps * d):
            continue  # the perturbation crosses a fan boundary
        _, df = adcheck.hlld_tangent(GAMMA, bx, lr, dbx, d)
        fd = (adcheck.hlld(GAMMA, bx + eps * dbx, lr + eps * d) -
              adcheck.hlld(GAMMA, bx - eps * dbx, lr - eps * d)) / (2 * eps)
        errs.append(np.max(np.abs(fd - df)) / (np.max(np.abs(df)) + 1e-300))
    assert len(errs) > 500
    assert np.max(errs) < 1e-6


@pytest.mark.parametrize("dtype,tol", [(np.float64, 1e-11), (np.float32, 2e-3)])
def test_hlld_adjoint_is_the_transpose_of_the_tangent(dtype, tol):
    rng = np.random.default_rng(2)
    errs = []
    for bx, lr in _random_states(rng, 1500):
        d = rng.normal(0.0, 1.0, 14)
        dbx = rng.normal()
        lf = rng.normal(0.0, 1.0, 7)
        _, df = adcheck.hlld_tangent(GAMMA, float(dtype(bx)), lr.astype(dtype).astype(np.float64), dbx, d)
        lin, lbx = adcheck.hlld_adjoint(GAMMA, bx, lr, lf, dtype)
        lhs = float(np.dot(lin.astype(np.float64), d) + lbx * dbx)
        rhs = float(np.dot(lf, df))
        scale = np.sum(np.abs(lin.astype(np.float64) * d)) + abs(lbx * dbx) + 1e-300
        errs.append(abs(lhs - rhs) / scale)
    assert np.max(errs) < tol


def _case(name):
    if name == "ot":
        cfg, s = orszag_tang_3d(12, ny=10, nz=8)
    elif name == "shear":
        cfg, s = shearing_box(n_radial=12, n_azimuthal=16, n_vertical=6, l_azimuthal=4.0, seed=5)
    elif name == "shear_mz":
        cfg, s = shearing_box(n_radial=12, n_azimuthal=16, n_vertical=6, l_azimuthal=4.0, seed=3)
        cfg.margin_z, cfg.size_z = 2, 10
        s = np.concatenate([s[:, -2:], s, s[:, :2]], axis=1)
    elif name == "euler":
        cfg, s = shearing_box(n_radial=12, n_azimuthal=16, n_vertical=6, l_azimuthal=4.0, seed=4)
        cfg.time_order = 1
    elif name == "shear_thin":  # interior rows = margin_y: both shear images share their sources
        cfg, s = shearing_box(n_radial=4, n_azimuthal=16, n_vertical=6, l_radial=0.25, l_azimuthal=4.0, seed=6)
    else:  # first-order reconstruction
        cfg, s = orszag_tang_3d(12, ny=10, nz=8)
        cfg.space_order = 1
    return cfg, s


CASES = ["ot", "shear", "shear_mz", "euler", "order1", "shear_thin"]


@pytest.mark.parametrize("case", CASES)
def test_generic_forward_is_bitwise_the_oracle(case):
    cfg, s = _case(case)
    o32 = oracle.proceed(cfg, s, 6)
    a32 = adcheck.forward(cfg, s, o32["dts"], dtype=np.float32)
    assert np.array_equal(a32.view(np.uint32), o32["state"].view(np.uint32))
    o64 = oracle.proceed(cfg, s.astype(np.float64), 6, dtype=np.float64)
    a64 = adcheck.forward(cfg, s.astype(np.float64), o64["dts"], dtype=np.float64)
    assert np.array_equal(a64, o64["state"])


def _velocity_direction(s, seed):
    rng = np.random.default_rng(seed)
    d = np.zeros(s.shape)
    d[1:4] = rng.normal(0.0, 1.0, s[1:4].shape) * 0.01
    return d


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("window", [(2, 6), (0, 6), (6, 6)])
def test_adjoint_is_the_transpose_of_the_tangent_linear_step(case, window):
    cfg, s = _case(case)
    dts = oracle.proceed(cfg, s, 6)["dts"].astype(np.float64)
    s64 = s.astype(np.float64)
    rng = np.random.default_rng(11)
    # a direction in every field (B too): the transpose must hold everywhere
    scale = np.abs(s64).reshape(8, -1).mean(axis=1).reshape(8, 1, 1, 1) + 1e-3
    d = rng.normal(0.0, 1.0, s64.shape) * scale
    J, dJ = adcheck.tlm(cfg, s64, d, dts, *window)
    Ja, g = adcheck.adjoint(cfg, s64, dts, *window, dtype=np.float64)
    assert Ja == pytest.approx(J, rel=1e-13, abs=1e-300)
    assert float(np.sum(g * d)) == pytest.approx(dJ, rel=1e-11, abs=1e-14 * abs(J) + 1e-300)


@pytest.mark.parametrize("case", ["shear", "shear_mz", "euler"])
def test_tangent_matches_central_differences_along_velocity(case):
    cfg, s = _case(case)
    dts = oracle.proceed(cfg, s, 6)["dts"].astype(np.float64)
    s64 = s.astype(np.float64)
    d = _velocity_direction(s64, 3)
    _, dJ = adcheck.tlm(cfg, s64, d, dts, 2, 6)
    eps = 1e-6
    Jp, _ = adcheck.tlm(cfg, s64 + eps * d, None, dts, 2, 6)
    Jm, _ = adcheck.tlm(cfg, s64 - eps * d, None, dts, 2, 6)
    assert (Jp - Jm) / (2 * eps) == pytest.approx(dJ, rel=2e-3)


@pytest.mark.parametrize("case", ["shear", "shear_mz", "euler"])
def test_fp32_adjoint_is_close_to_fp64(case):
    cfg, s = _case(case)
    o = oracle.proceed(cfg, s, 6)
    s64 = s.astype(np.float64)
    d = _velocity_direction(s64, 4)
    _, dJ = adcheck.tlm(cfg, s64, d, o["dts"].astype(np.float64), 2, 6)
    _, g32 = adcheck.adjoint(cfg, s, o["dts"], 2, 6, dtype=np.float32)
    assert float(np.sum(g32.astype(np.float64) * d)) == pytest.approx(dJ, rel=1e-2)


def test_margin_entries_overwritten_by_the_fill_have_zero_gradient():
    cfg, s = _case("shear")
    dts = oracle.proceed(cfg, s, 4)["dts"]
    _, g = adcheck.adjoint(cfg, s.astype(np.float64), dts.astype(np.float64), 1, 4)
    m = cfg.margin_y
    lo = g[:, :, :m, :]
    hi = g[:, :, -m:, :]
    assert not lo.any()
    # By of the first top margin row is the upper face of the last interior row
    # and is kept by the fill
    keep = np.zeros_like(hi, dtype=bool)
    keep[6, :, 0, :] = True
    assert not hi[~keep].any()
    assert hi[keep].any()
