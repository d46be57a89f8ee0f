"""Pins the oracle (oracle/mhd_oracle.c) to the reference.

* Against the committed golden fixtures (tests/golden/*.npz, produced by the
  host-compiled reference solver with tests/golden/make_golden.py): bitwise
  equal states and identical step times.
* Against the reference binaries themselves (oracle/_ref), when they are built
  in this checkout: more sizes, Z margins, the FP64 build.
"""
import hashlib
import os

import numpy as np
import pytest

from nmhd_b200.problems import orszag_tang_3d, shearing_box
from oracle import oracle

def scheme(built, space=2, time=2):
    """A problem with generate_config.rb's scheme options (-s space, -t time)."""
    cfg, state = built
    cfg.space_order, cfg.time_order = space, time
    return cfg, state


GOLDEN = {
    "ot16": lambda: orszag_tang_3d(16),
    "ot16_goal": lambda: orszag_tang_3d(16),
    "ot24x20x12": lambda: orszag_tang_3d(24, ny=20, nz=12),
    "shear32x16x8": lambda: shearing_box(n_radial=16, n_azimuthal=32, n_vertical=8, l_azimuthal=4.0),
    "shear48x20x12": lambda: shearing_box(n_radial=20, n_azimuthal=48, n_vertical=12, l_azimuthal=2.0),
    # the reference's piecewiseconst1 / euler1 expansions (oracle/expand_variant.py)
    "ot24x20x12_s1": lambda: scheme(orszag_tang_3d(24, ny=20, nz=12), space=1),
    "shear32x16x8_t1": lambda: scheme(shearing_box(n_radial=16, n_azimuthal=32, n_vertical=8,
                                                   l_azimuthal=4.0, seed=4), time=1),
    "shear48x20x12_s1t1": lambda: scheme(shearing_box(n_radial=20, n_azimuthal=48, n_vertical=12,
                                                      l_azimuthal=2.0, seed=5), space=1, time=1),
}


def load_golden(golden_dir, name):
    """(config, input state, fixture dict) for a golden case."""
    fx = dict(np.load(os.path.join(golden_dir, name + ".npz")))
    cfg, state = GOLDEN[name]()
    if "input" in fx:
        state = fx["input"]
    digest = hashlib.sha256(np.ascontiguousarray(state).tobytes()).hexdigest()
    assert digest == fx["input_sha256"].item().decode(), "regenerated input differs from the fixture's"
    return cfg, state, fx


@pytest.mark.parametrize("name", sorted(GOLDEN))
def test_oracle_matches_golden(golden_dir, name):
    cfg, state, fx = load_golden(golden_dir, name)
    steps = int(fx["steps"])
    r = oracle.proceed(cfg, state, steps, goal_time=float(fx["goal_time"]))
    assert r["steps"] == steps
    assert np.array_equal(r["state"], fx["output"]), "oracle state differs from the reference's"
    assert np.array_equal(r["times"][:len(fx["times"])], fx["times"])
    assert r["goal_reached"] == bool(fx["goal_reached"])


def test_goal_clamp_lands_on_goal(golden_dir):
    cfg, state, fx = load_golden(golden_dir, "ot16_goal")
    r = oracle.proceed(cfg, state, 100, goal_time=0.05)
    assert r["goal_reached"]
    assert r["time"] == float(np.float64(np.float32(0.05)))


needs_ref = pytest.mark.skipif(oracle.ref_binary("ot16") is None,
                               reason="reference binaries not built (make -C oracle ref)")


@needs_ref
def test_oracle_matches_reference_long_run():
    cfg, state = orszag_tang_3d(16)
    ref, times, _ = oracle.run_ref("ot16", state, 150)
    r = oracle.proceed(cfg, state, 150)
    assert np.array_equal(ref, r["state"])
    assert np.array_equal(times, r["times"])


@needs_ref
def test_oracle_matches_reference_z_margins():
    cfg, s = shearing_box(n_radial=32, n_azimuthal=64, n_vertical=16, l_azimuthal=4.0)
    cfg.margin_z, cfg.size_z = 4, 24
    s2 = np.concatenate([s[:, -4:], s, s[:, :4]], axis=1)
    ref, times, _ = oracle.run_ref("shear64x32x16_mz", s2, 12)
    r = oracle.proceed(cfg, s2, 12)
    assert np.array_equal(ref, r["state"])
    assert np.array_equal(times, r["times"])


@needs_ref
def test_oracle_matches_reference_fp64():
    cfg, s = shearing_box(n_radial=16, n_azimuthal=32, n_vertical=8, l_azimuthal=4.0)
    s = s.astype(np.float64)
    ref, times, _ = oracle.run_ref("shear32x16x8_f64", s, 25, dtype=np.float64)
    r = oracle.proceed(cfg, s, 25, dtype=np.float64)
    assert np.array_equal(ref, r["state"])
    assert np.array_equal(times, r["times"])


def test_hlld_consistency_and_mirror():
    """F(U, U) is the physical flux; mirroring x -> -x flips the odd fluxes."""
    rng = np.random.default_rng(5)
    g = np.float32(5.0 / 3.0)
    for _ in range(50):
        d, u, v, w, p, by, bz, bx = rng.uniform(-1, 1, 8).astype(np.float32)
        d, p = np.float32(abs(d) + 0.5), np.float32(abs(p) + 0.5)
        lr = np.array([d, d, u, u, v, v, w, w, p, p, by, by, bz, bz], np.float32)
        f = oracle.hlld(g, bx, lr).astype(np.float64)
        D, U, V, W, P, BY, BZ, BX = (float(t) for t in (d, u, v, w, p, by, bz, bx))
        b2 = BX * BX + BY * BY + BZ * BZ
        pt = P + 0.5 * b2
        e = P / (5.0 / 3.0 - 1) + 0.5 * D * (U * U + V * V + W * W) + 0.5 * b2
        vb = U * BX + V * BY + W * BZ
        phys = [D * U, D * U * U + pt - BX * BX, D * V * U - BX * BY, D * W * U - BX * BZ,
                (e + pt) * U - BX * vb, BY * U - BX * V, BZ * U - BX * W]
        assert np.allclose(f, phys, rtol=2e-5, atol=2e-5)
        # mirror: reflect the normal axis
        l2 = np.array([d, d * 1.3, u, -u * 0.5, v, v, w, w, p, p * 0.8, by, by, bz, bz], np.float32)
        m2 = np.array([l2[1], l2[0], -l2[3], -l2[2], l2[5], l2[4], l2[7], l2[6], l2[9], l2[8],
                       l2[11], l2[10], l2[13], l2[12]], np.float32)
        fa = oracle.hlld(g, bx, l2).astype(np.float64)
        fb = oracle.hlld(g, -bx, m2).astype(np.float64)
        sign = np.array([-1, 1, -1, -1, -1, -1, -1])
        assert np.allclose(fa, sign * fb, rtol=1e-4, atol=1e-5)


@pytest.mark.parametrize("name,nr,k,nz,q,beta", [("shear64x32x32_q12", 32, 2, 32, 1.2, 1e2),
                                                 ("shear144x48x32_q18", 48, 3, 32, 1.8, 1e4)])
def test_oracle_matches_reference_at_ensemble_q_extremes(name, nr, k, nz, q, beta):
    """The reference built with kDifferentialRotationIndex 1.2 and 1.8 (the
    ends of the batched ensemble's q range) equals the restatement with that
    q, at the ends of the ensemble's beta range."""
    if oracle.ref_binary(name) is None:
        pytest.skip(f"reference binary ref_{name} not built")
    cfg, s = shearing_box(n_radial=nr, n_azimuthal=k * nr, n_vertical=nz, l_radial=1.0,
                          l_azimuthal=float(k), l_vertical=1.0, q=q, beta=beta, seed=77)
    ref, times, _ = oracle.run_ref(name, s, 15)
    r = oracle.proceed(cfg, s, 15)
    assert np.array_equal(ref, r["state"])
    assert np.array_equal(times, r["times"])
