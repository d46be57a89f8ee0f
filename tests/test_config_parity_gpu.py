"""Parity at the benchmark configurations themselves, against the reference's
own solver (host-compiled from its sources into oracle/_ref), through the C ABI.

Tolerance: bitwise equality of every state value and identical FP64 clocks
after the stated number of steps (the CUDA path keeps the reference's
operation order and float/double promotions).

  * the 64^3 Orszag-Tang vortex, 100 steps (the plain method's small case);
  * the 128 (radial) x 256 (azimuthal) x 64 MRI shearing box, 100 steps;
  * the batched ensemble at the ends of its physics range: boxes with
    q = 1.2 and 1.8 (reference binaries built with those
    kDifferentialRotationIndex values) and beta = 1e2 and 1e4, advanced in
    one batch with other ensemble boxes, each compared with the reference
    run of that box alone.
"""
import numpy as np
import pytest

from nmhd_b200.batch import BatchSolver
from nmhd_b200.problems import mri_ensemble, orszag_tang_3d, shearing_box
from nmhd_b200.solver import MHDSolver
from oracle import oracle

pytestmark = pytest.mark.gpu


def needs_ref(name):
    if oracle.ref_binary(name) is None:
        pytest.skip(f"reference binary ref_{name} not built")


def assert_same(a, b):
    diff = np.argwhere(a != b)
    assert diff.size == 0, f"{len(diff)} values differ, first at {diff[:3].tolist()}"


def gpu_run(cfg, state, steps):
    with MHDSolver(cfg) as s:
        s.set_state(state)
        s.step(steps)
        return s.get_state(), s.current_time(), s.generation()


def test_orszag_tang_64_cubed_100_steps_matches_reference(gpu):
    """The plain method's small configuration as stated: 64^3 periodic
    Orszag-Tang vortex, gamma 5/3, CFL 0.4, 100 steps."""
    needs_ref("ot64")
    cfg, s = orszag_tang_3d(64)
    ref, times, info = oracle.run_ref("ot64", s, 100)
    assert info["steps"] == 100
    got, t, gen = gpu_run(cfg, s, 100)
    assert gen == 100 and t == times[-1]
    assert_same(got, ref)


def test_mri_box_128x256x64_100_steps_matches_reference(gpu):
    """The MRI benchmark box as stated (128 radial x 256 azimuthal x 64,
    beta 400, q 1.5, seeded noise), 100 steps: the reference binary takes
    tens of seconds on the host cores."""
    needs_ref("shear256x128x64")
    cfg, s = shearing_box()
    ref, times, info = oracle.run_ref("shear256x128x64", s, 100)
    assert info["steps"] == 100
    got, t, gen = gpu_run(cfg, s, 100)
    assert gen == 100 and t == times[-1]
    assert_same(got, ref)


# (reference binary, radial, azimuthal ratio, vertical, q) of the two built
# ends of the ensemble's q range; each is run at both ends of its beta range
EXTREMES = [("shear64x32x32_q12", 32, 2, 32, 1.2), ("shear144x48x32_q18", 48, 3, 32, 1.8)]


def test_batched_ensemble_extremes_match_reference(gpu):
    """Four boxes at the corners of the ensemble's (q, beta) range, batched
    together with eight boxes of the 64-box ensemble, 100 steps: each corner
    box equals the reference's own run of that box bitwise (state and clock);
    the ensemble boxes equal their single-box runs."""
    for name, *_ in EXTREMES:
        needs_ref(name)
    corners = []
    for name, nr, k, nz, q in EXTREMES:
        for beta in (1e2, 1e4):
            cfg, s = shearing_box(n_radial=nr, n_azimuthal=k * nr, n_vertical=nz, l_radial=1.0,
                                  l_azimuthal=float(k), l_vertical=1.0, q=q, beta=beta,
                                  seed=4000 + len(corners))
            corners.append((name, cfg, s))
    others, _ = mri_ensemble(n_boxes=8, seed=0)
    steps = 100
    with BatchSolver([c for _, c, _ in corners] + [c for c, _ in others]) as b:
        for i, (_, _, s) in enumerate(corners):
            b.set_state(i, s)
        for j, (_, s) in enumerate(others):
            b.set_state(len(corners) + j, s)
        b.step(steps)
        for i, (name, cfg, s) in enumerate(corners):
            ref, times, info = oracle.run_ref(name, s, steps)
            t, gen = b.clock(i)
            assert gen == steps and t == times[-1], (name, i)
            assert_same(b.get_state(i), ref)
        for j, (cfg, s) in enumerate(others[:3]):
            got, t, gen = gpu_run(cfg, s, steps)
            assert b.clock(len(corners) + j) == (t, gen)
            assert_same(b.get_state(len(corners) + j), got)


# The reference's other scheme choices (generate_config.rb -s 1 / -t 1),
# host-compiled from its shipped expansion through oracle/expand_variant.py:
# (binary, problem, space order, time order)
SCHEMES = [
    ("ot24x20x12_s1", lambda: orszag_tang_3d(24, ny=20, nz=12), 1, 2),
    ("shear32x16x8_t1", lambda: shearing_box(n_radial=16, n_azimuthal=32, n_vertical=8, l_azimuthal=4.0,
                                             seed=11), 2, 1),
    ("shear48x20x12_s1t1", lambda: shearing_box(n_radial=20, n_azimuthal=48, n_vertical=12, l_azimuthal=2.0,
                                                seed=12), 1, 1),
]


@pytest.mark.parametrize("variant", [4, 2, 5])
@pytest.mark.parametrize("case", range(len(SCHEMES)))
def test_scheme_variants_match_the_reference_expansions(gpu, case, variant):
    """Piecewise-constant reconstruction and Euler stepping, 60 steps, against
    the reference's own piecewiseconst1 / euler1 code (its template's rules
    applied to the shipped expansion), for the default, the three-kernel and
    the staged-flux variant."""
    name, make, so, to = SCHEMES[case]
    needs_ref(name)
    cfg, s = make()
    cfg.space_order, cfg.time_order = so, to
    ref, times, info = oracle.run_ref(name, s, 60)
    with MHDSolver(cfg) as sol:
        sol.set_kernel(variant, 8, 0)
        sol.set_state(s)
        sol.step(60)
        assert sol.current_time() == times[-1]
        assert_same(sol.get_state(), ref)
