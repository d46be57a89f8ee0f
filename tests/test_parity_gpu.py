"""Parity of the CUDA time step (libnmhd.so, called through the C ABI) with the
reference.  Tolerance: bitwise equality of every state value after every
tested number of steps, and identical step times; the CUDA path mirrors the
reference's operation order and promotions, so anything else is a bug."""
import math
import os

import numpy as np
import pytest

from nmhd_b200.binio import read_bin, write_bin
from nmhd_b200.config import SolverConfig
from nmhd_b200.problems import orszag_tang_3d, shearing_box
from nmhd_b200.solver import MHDSolver
from nmhd_b200 import _lib
from oracle import oracle

from test_oracle_pin import GOLDEN, load_golden

pytestmark = pytest.mark.gpu


def run_gpu(cfg, state, steps, goal=math.inf):
    with MHDSolver(cfg) as s:
        s.set_state(state)
        reached = s.proceed(goal, -1.0, steps)
        return {"state": s.get_state(), "time": s.current_time(), "generation": s.generation(),
                "dts": s.dt_history(steps), "reached": reached}


def assert_same(a, b):
    diff = np.argwhere(a != b)
    assert diff.size == 0, f"{len(diff)} values differ, first at {diff[:3].tolist()}"


@pytest.mark.parametrize("name", sorted(GOLDEN))
def test_gpu_matches_reference_golden(gpu, golden_dir, name):
    cfg, state, fx = load_golden(golden_dir, name)
    steps = int(fx["steps"])
    goal = float(fx["goal_time"])
    r = run_gpu(cfg, state, 1000 if goal < 1e29 else steps, goal if goal < 1e29 else math.inf)
    assert r["generation"] == steps
    assert_same(r["state"], fx["output"])
    times = fx["times"]
    assert r["time"] == (times[-1] if goal > 1e29 else float(np.float32(goal)))


@pytest.mark.parametrize("case", ["ot32", "ot_2d", "shear64x40x16", "shear_mz", "euler", "order1"])
def test_gpu_matches_oracle(gpu, case):
    if case == "ot32":
        cfg, s = orszag_tang_3d(32)
        steps = 25
    elif case == "ot_2d":
        cfg, s = orszag_tang_3d(40, ny=24, nz=1)
        steps = 30
    elif case == "shear64x40x16":
        cfg, s = shearing_box(n_radial=32, n_azimuthal=64, n_vertical=16, l_azimuthal=4.0, seed=7)
        steps = 30
    elif case == "shear_mz":
        cfg, s = shearing_box(n_radial=16, n_azimuthal=32, n_vertical=8, l_azimuthal=4.0, seed=3)
        cfg.margin_z, cfg.size_z = 4, 16
        s = np.concatenate([s[:, -4:], s, s[:, :4]], axis=1)
        steps = 15
    elif case == "euler":
        cfg, s = shearing_box(n_radial=16, n_azimuthal=32, n_vertical=8, l_azimuthal=4.0, seed=4)
        cfg.time_order = 1
        steps = 20
    else:
        cfg, s = orszag_tang_3d(24, ny=20, nz=12)
        cfg.space_order = 1
        steps = 20
    o = oracle.proceed(cfg, s, steps)
    r = run_gpu(cfg, s, steps)
    assert r["generation"] == steps
    assert r["time"] == o["time"]
    assert np.array_equal(r["dts"], o["dts"])
    assert_same(r["state"], o["state"])


def test_gpu_full_size_mri_box_matches_oracle_and_keeps_div_b(gpu):
    """128(radial) x 256(azimuthal) x 64 box of the MRI benchmark, a few steps."""
    cfg, s = shearing_box()
    o = oracle.proceed(cfg, s, 3)
    with MHDSolver(cfg) as sol:
        sol.set_state(s)
        d0 = sol.diagnostics()
        sol.step(3)
        assert_same(sol.get_state(), o["state"])
        d1 = sol.diagnostics()
    assert d1["max_div_b"] < 1e-4 * math.sqrt(2 / 400) * 128
    assert abs(d1["mass"] - d0["mass"]) < 1e-6 * d0["mass"]


def test_gpu_large_box_matches_oracle_and_keeps_div_b(gpu):
    """The 512(radial) x 1024(azimuthal) x 256 box of the large-box benchmark
    (136 M cells with margins): one step bitwise against the oracle, then div B
    at roundoff and mass conserved after ten more steps.  The oracle's step takes
    ~22 GB of host memory and a minute or two on the host cores."""
    import psutil
    if psutil.virtual_memory().available < 32 * 2 ** 30:
        pytest.skip("not enough host memory for the oracle at this size")
    cfg, s = shearing_box(n_radial=512, n_azimuthal=1024, n_vertical=256, seed=3)
    o = oracle.proceed(cfg, s, 1)
    with MHDSolver(cfg) as sol:
        sol.set_state(s)
        del s
        d0 = sol.diagnostics()
        sol.step(1)
        assert sol.current_time() == o["time"]
        assert_same(sol.get_state(), o["state"])
        del o
        sol.step(10)
        d1 = sol.diagnostics()
    assert d1["max_div_b"] < 1e-4 * math.sqrt(2 / 400) * 512
    assert abs(d1["mass"] - d0["mass"]) < 1e-6 * d0["mass"]


@pytest.mark.parametrize("case", ["ot_m2", "shear_m2", "shear_m4_mz2"])
@pytest.mark.parametrize("variant", [2, 0, 4, 5])
def test_per_stage_margin_fill_matches_oracle(gpu, case, variant):
    """NMHD_FLAG_HALO_PER_STAGE: the predictor's margins refilled before the
    second stage; bitwise the oracle's mode, for the default and the tiled
    kernels."""
    from nmhd_b200.config import FLAG_HALO_PER_STAGE
    if case == "ot_m2":
        cfg, s = orszag_tang_3d(16)
        cfg.margin_y, cfg.size_y = 2, 20
        s = np.concatenate([s[:, :, -2:], s, s[:, :, :2]], axis=2)
    else:
        m = 2 if case == "shear_m2" else 4
        cfg, s = shearing_box(n_radial=16, n_azimuthal=32, n_vertical=8, l_azimuthal=4.0, seed=23, margin=m)
        if case == "shear_m4_mz2":
            cfg.margin_z, cfg.size_z = 2, 12
            s = np.concatenate([s[:, -2:], s, s[:, :2]], axis=1)
    cfg.flags = FLAG_HALO_PER_STAGE
    o = oracle.proceed(cfg, s, 10)
    with MHDSolver(cfg) as sol:
        sol.set_kernel(variant, 8, 0)
        sol.set_state(s)
        sol.step(10)
        assert sol.current_time() == o["time"]
        assert_same(sol.get_state(), o["state"])


def _rel_by_quantity(a, b):
    """Largest |a - b| over each quantity (density, velocity, pressure, B),
    relative to that quantity's largest |b|."""
    out = []
    for grp in ([0], [1, 2, 3], [4], [5, 6, 7]):
        d = np.abs(a[grp].astype(np.float64) - b[grp].astype(np.float64)).max()
        out.append(d / max(np.abs(b[grp]).max(), 1e-30))
    return max(out)


@pytest.mark.parametrize("case", ["mri_128x256x64", "mri_96x192x48"])
def test_fast_arithmetic_within_tolerance(gpu, case):
    """NMHD_FLAG_FAST_ARITHMETIC on the noisy MRI boxes: one step from the
    reference's own state (the oracle's) is within 1e-5 of the reference's,
    relative to each quantity's scale (the per-step FP32 tolerance this mode
    is held to); after 20 steps mass is conserved and div B stays at roundoff.
    (Not on flows with exact symmetries: there the reference's corner wind
    sums are exactly zero, CT takes the mean, and rounding-size differences
    in the predictor pick one side instead.)"""
    from nmhd_b200.config import FLAG_FAST_ARITHMETIC
    if case == "mri_128x256x64":
        cfg, s = shearing_box()
    else:
        cfg, s = shearing_box(n_radial=96, n_azimuthal=192, n_vertical=48, l_azimuthal=2.0, seed=17)
    o1 = oracle.proceed(cfg, s, 1)
    cfg.flags = FLAG_FAST_ARITHMETIC
    with MHDSolver(cfg) as sol:
        sol.set_state(s)
        d0 = sol.diagnostics()
        sol.step(1)
        one = sol.get_state()
        assert not np.array_equal(one, o1["state"])  # fast: not bitwise
        # the interior (margin cells are overwritten by the next step's fill;
        # their outer rows are advanced from wrapped neighbours)
        ys = slice(cfg.margin_y, cfg.size_y - cfg.margin_y)
        dev = _rel_by_quantity(one[:, :, ys], o1["state"][:, :, ys])
        assert dev < 1e-5, dev
        sol.step(19)
        d1 = sol.diagnostics()
    assert abs(d1["mass"] - d0["mass"]) < 1e-6 * d0["mass"]
    bscale = max(abs(d0["bx2_mean"]), abs(d0["by2_mean"]), 1e-30) ** 0.5 + math.sqrt(2 / 400)
    assert d1["max_div_b"] < 1e-4 * bscale * cfg.size_x


def test_chunked_proceed_equals_single_call(gpu):
    cfg, s = shearing_box(n_radial=16, n_azimuthal=32, n_vertical=8, l_azimuthal=4.0, seed=9)
    with MHDSolver(cfg) as a, MHDSolver(cfg) as b:
        a.set_state(s)
        b.set_state(s)
        a.step(37)
        for k in (1, 16, 3, 17):
            b.step(k)
        assert a.generation() == b.generation() == 37
        assert a.current_time() == b.current_time()
        assert_same(a.get_state(), b.get_state())


def test_read_write_bin_roundtrip(gpu, tmp_path):
    cfg, s = orszag_tang_3d(16)
    p_in, p_out = tmp_path / "in.bin", tmp_path / "out.bin"
    write_bin(p_in, s)
    with MHDSolver(cfg) as sol:
        assert sol.read(p_in)
        assert sol.write(p_out)
        assert open(p_in, "rb").read() == open(p_out, "rb").read()
        bad = tmp_path / "bad.bin"
        write_bin(bad, np.zeros((8, 4, 4, 4), np.float32))
        assert not sol.read(bad)
        assert sol.last_status == -4
        assert not sol.read(tmp_path / "missing.bin")


def test_save_load_state_resumes_bitwise(gpu, tmp_path):
    cfg, s = shearing_box(n_radial=16, n_azimuthal=32, n_vertical=8, l_azimuthal=4.0, seed=11)
    with MHDSolver(cfg) as a:
        a.set_state(s)
        a.step(10)
        assert a.save_state(tmp_path / "c")
        a.step(10)
        ref = a.get_state()
        t_ref = a.current_time()
    with MHDSolver(cfg) as b:
        assert b.load_state(tmp_path / "c")
        assert b.generation() == 10
        b.step(10)
        assert b.current_time() == t_ref
        assert_same(b.get_state(), ref)


def test_numerical_failure_is_reported_not_faulted(gpu):
    """A state with negative pressure: the kernels produce NaN, the host sees
    NMHD_ERR_NUMERICAL; the GPU context stays usable."""
    cfg, s = orszag_tang_3d(16)
    s = s.copy()
    s[4, 3, 3, 3] = -1.0
    with MHDSolver(cfg) as sol:
        sol.set_state(s)
        with pytest.raises(_lib.NmhdError) as e:
            sol.step(5)
        assert e.value.code == -5
        cfg2, good = orszag_tang_3d(16)
        sol.set_state(good)  # a new state keeps the clock, like initialize_state()
        g0 = sol.generation()
        sol.step(2)
        assert sol.generation() == g0 + 2


def test_goal_time_semantics(gpu):
    cfg, s = orszag_tang_3d(16)
    with MHDSolver(cfg) as sol:
        sol.set_state(s)
        assert sol.proceed(0.02)
        assert sol.current_time() == float(np.float32(0.02))
        g = sol.generation()
        assert not sol.proceed(1.0, -1.0, 3)
        assert sol.generation() == g + 3


@pytest.mark.parametrize("variant,rows,zc", [(2, 8, 0), (1, 8, 0), (0, 4, 0), (0, 8, 16), (0, 16, 5),
                                             (0, 8, 3), (3, 8, 1), (3, 8, 2), (3, 8, 3), (3, 8, 4),
                                             (3, 8, 64), (4, 8, 0), (5, 8, 0)])
@pytest.mark.parametrize("case", ["ot_ragged", "shear_ragged", "shear_mz"])
def test_kernel_variants_and_tile_shapes_bitwise(gpu, variant, rows, zc, case):
    """Every kernel variant and tile shape, on boxes whose sizes are not
    multiples of the tile (partial tiles in x, y and z)."""
    _variant_case(variant, rows, zc, case)


@pytest.mark.parametrize("variant", [2, 4, 5])
@pytest.mark.parametrize("case", ["tiny", "ot_2d", "euler_order1", "shear_tma"])
def test_cell_kernels_on_tiny_flat_and_first_order_boxes(gpu, variant, case):
    """The per-cell kernels, the fused epilogue and the staged flux kernel
    (whose shared-memory tiles with their halos are larger than these boxes:
    every halo entry wraps periodically) on a 5 x 9 x 1 box, a single-plane
    box, Euler stepping with piecewise-constant reconstruction, and a box
    with interior tiles (staged by tensor copies) beside edge tiles."""
    _variant_case(variant, 8, 0, case)


def _variant_case(variant, rows, zc, case):
    if case == "ot_ragged":
        cfg, s = orszag_tang_3d(40, ny=20, nz=13)
        steps = 12
    elif case == "shear_ragged":
        cfg, s = shearing_box(n_radial=12, n_azimuthal=48, n_vertical=7, l_azimuthal=2.0, seed=5)
        steps = 12
    elif case == "shear_mz":
        cfg, s = shearing_box(n_radial=16, n_azimuthal=32, n_vertical=8, l_azimuthal=4.0, seed=6)
        cfg.margin_z, cfg.size_z = 4, 16
        s = np.concatenate([s[:, -4:], s, s[:, :4]], axis=1)
        steps = 10
    elif case == "tiny":  # boxes smaller than a tile and its halo in every axis
        cfg, s = shearing_box(n_radial=3, n_azimuthal=5, n_vertical=1, l_azimuthal=2.0, seed=8, margin=3)
        steps = 8
    elif case == "ot_2d":
        cfg, s = orszag_tang_3d(40, ny=24, nz=1)
        steps = 10
    elif case == "shear_tma":  # 96 x 24 x 8: tiles at x0 = 32, 2 <= y0 <= 19, z0 = 2 lie inside
        cfg, s = shearing_box(n_radial=16, n_azimuthal=96, n_vertical=8, l_azimuthal=6.0, seed=9)
        steps = 8
    else:  # Euler stepping with piecewise-constant reconstruction
        cfg, s = shearing_box(n_radial=12, n_azimuthal=40, n_vertical=5, l_azimuthal=2.0, seed=10)
        cfg.time_order, cfg.space_order = 1, 1
        steps = 10
    o = oracle.proceed(cfg, s, steps)
    with MHDSolver(cfg) as sol:
        sol.set_kernel(variant, rows, zc)
        sol.set_state(s)
        sol.step(steps)
        assert sol.current_time() == o["time"]
        assert_same(sol.get_state(), o["state"])


def test_autotune_restores_state_and_keeps_results_bitwise(gpu):
    cfg, s = shearing_box(n_radial=16, n_azimuthal=64, n_vertical=16, l_azimuthal=4.0, seed=13)
    o = oracle.proceed(cfg, s, 6)
    with MHDSolver(cfg) as sol:
        sol.set_state(s)
        sol.step(2)
        mid = sol.get_state()
        t_mid = sol.current_time()
        trials = sol.autotune(steps=2)
        assert len(trials) >= 5
        best = min(trials, key=lambda r: r[3])
        assert sol.kernel() == best[:3]
        assert sol.generation() == 2 and sol.current_time() == t_mid
        assert_same(sol.get_state(), mid)
        sol.step(4)
        assert sol.current_time() == o["time"]
        assert_same(sol.get_state(), o["state"])
    # a later solver for a box of the same shape and scheme starts with the
    # tuned selection; another shape keeps the default
    with MHDSolver(cfg) as again:
        assert again.kernel() == best[:3]
    other, _ = shearing_box(n_radial=16, n_azimuthal=64, n_vertical=12, l_azimuthal=4.0, seed=13)
    with MHDSolver(other) as fresh:
        assert fresh.kernel()[0] == 5


@pytest.mark.parametrize("zc", [1, 2, 5])
@pytest.mark.parametrize("case", ["ot_2d", "euler", "order1"])
def test_chunked_pipeline_variant_bitwise(gpu, zc, case):
    """Variant 3 (z-chunked pipeline): single-plane boxes, Euler stepping and
    first-order reconstruction, chunks of 1, 2 and 5 planes."""
    if case == "ot_2d":
        cfg, s = orszag_tang_3d(40, ny=24, nz=1)
    elif case == "euler":
        cfg, s = shearing_box(n_radial=16, n_azimuthal=32, n_vertical=9, l_azimuthal=4.0, seed=4)
        cfg.time_order = 1
    else:
        cfg, s = orszag_tang_3d(24, ny=20, nz=11)
        cfg.space_order = 1
    o = oracle.proceed(cfg, s, 10)
    with MHDSolver(cfg) as sol:
        sol.set_kernel(3, 8, zc)
        sol.set_state(s)
        sol.step(10)
        assert sol.current_time() == o["time"]
        assert_same(sol.get_state(), o["state"])


def test_monitor_hook_runs_before_every_step(gpu):
    """A monitor() override is called before every step, as in the
    reference's loop; a non-zero return stops the run before that step; the
    steps taken are bitwise the batched ones."""
    cfg, s = shearing_box(n_radial=16, n_azimuthal=32, n_vertical=8, l_azimuthal=4.0, seed=31)

    class Counting(MHDSolver):
        def __init__(self, cfg, stop_at):
            super().__init__(cfg)
            self.calls, self.gens, self.stop_at = 0, [], stop_at

        def monitor(self):
            self.calls += 1
            self.gens.append(self.generation())
            return self.generation() >= self.stop_at

    with Counting(cfg, 7) as sol:
        sol.set_state(s)
        assert sol.proceed(1e30) is False
        assert sol.gens == list(range(8)) and sol.generation() == 7
        got = sol.get_state()
    with MHDSolver(cfg) as ref:
        ref.set_state(s)
        ref.step(7)
        assert np.array_equal(got, ref.get_state())
    # reaching the goal ends the loop without another monitor call
    with Counting(cfg, 10 ** 6) as sol:
        sol.set_state(s)
        assert sol.proceed(0.05) is True
        assert sol.calls == sol.generation()


@pytest.mark.parametrize("variant,zc,mz,expect", [(2, 0, 0, 8), (2, 0, 2, 9), (0, 0, 0, 6), (3, 4, 0, 2 + 2 * 3 * 2),
                                                 (4, 0, 0, 6), (4, 0, 2, 7), (5, 0, 0, 6)])
def test_profile_counts_kernel_launches(gpu, variant, zc, mz, expect):
    """nmhd_profile reports each class's kernel launches per step (the bench's
    gpu_launches): fill (Y, Z), margin CFL, flux and update of each stage;
    the profiled steps advance the state as the graph path would."""
    cfg, s = shearing_box(n_radial=16, n_azimuthal=32, n_vertical=8, l_azimuthal=4.0, seed=61)
    if mz:
        cfg.margin_z, cfg.size_z = mz, 8 + 2 * mz
        s = np.concatenate([s[:, -mz:], s, s[:, :mz]], axis=1)
    o = oracle.proceed(cfg, s, 3)
    with MHDSolver(cfg) as sol:
        sol.set_kernel(variant, 8, zc)
        sol.set_state(s)
        prof = sol.profile(3)
        assert sum(n for _, n in prof.values()) == expect
        assert all(ms >= 0 for ms, _ in prof.values())
        assert sol.generation() == 3
        assert_same(sol.get_state(), o["state"])


def test_full_size_runs_keep_the_conservation_properties(gpu):
    """Size-independent properties at the benchmarks' full sizes, where the
    oracle would take too long: the 256^3 Orszag-Tang box (fully periodic, no
    source) conserves mass, momentum and total energy to roundoff over 100
    steps (the scheme updates them in flux form) with div B at roundoff; the
    128 x 256 x 64 MRI box runs the benchmark's 1000 steps with div B at
    roundoff and a valid state."""
    cfg, s = orszag_tang_3d(256)
    with MHDSolver(cfg) as sol:
        sol.set_state(s)
        del s
        d0 = sol.diagnostics()
        sol.step(100)
        assert sol.generation() == 100
        d1 = sol.diagnostics()
    b0 = 1.0 / math.sqrt(4.0 * math.pi)
    assert abs(d1["mass"] - d0["mass"]) < 1e-5 * d0["mass"]
    assert abs(d1["total_energy"] - d0["total_energy"]) < 1e-5 * d0["total_energy"]
    for a, b in zip(d0["momentum"], d1["momentum"]):
        assert abs(b - a) < 1e-5 * d0["mass"]
    assert d1["max_div_b"] < 1e-4 * b0 * 256

    cfg, s = shearing_box()
    with MHDSolver(cfg) as sol:
        sol.set_state(s)
        d0 = sol.diagnostics()
        sol.step(1000)
        assert sol.generation() == 1000
        st = sol.get_state()
        d1 = sol.diagnostics()
    assert np.isfinite(st).all() and (st[0] > 0).all() and (st[4] > 0).all()
    assert d1["max_div_b"] < 1e-4 * math.sqrt(2 / 400) * 128
    assert abs(d1["mass"] - d0["mass"]) < 1e-6 * d0["mass"]
