"""Batched ensemble (nmhd_batch_*): every box of a batch is bitwise the box
advanced alone by the single-box solver (which is pinned to the oracle), with
its own CFL time step and clock."""
import ctypes
import math

import numpy as np
import pytest

from nmhd_b200 import _lib
from nmhd_b200.config import SolverConfig
from nmhd_b200.problems import mri_ensemble, orszag_tang_3d, shearing_box


def small_ensemble(n=7, seed=3):
    return mri_ensemble(n_boxes=n, seed=seed, sides=(8, 12, 16), ratios=(2, 3, 4))


def test_ensemble_draws_follow_the_spec():
    boxes, params = mri_ensemble(n_boxes=64, seed=0)
    assert len(boxes) == 64
    for (cfg, state), p in zip(boxes, params):
        assert p["n_radial"] in (32, 48, 64, 96) and p["n_vertical"] in (32, 48, 64, 96)
        assert p["n_azimuthal"] // p["n_radial"] in (2, 3, 4)
        assert 1e2 <= p["beta"] <= 1e4 and 1.2 <= p["q"] <= 1.8
        assert state.shape == (8,) + cfg.shape
        assert cfg.size_x == p["n_azimuthal"] and cfg.size_y == p["n_radial"] + 8
    total = sum(c.interior_cells for (c, _) in boxes)
    assert 20e6 < total < 120e6


def test_batch_rejects_unsupported_configs_on_cpu():
    L = _lib.lib()
    cfg, _ = shearing_box(n_radial=16, n_azimuthal=32, n_vertical=8)
    bad = SolverConfig(**{**cfg.__dict__, "time_order": 1})
    arr = (type(cfg.to_ctypes()) * 2)(cfg.to_ctypes(), bad.to_ctypes())
    h = ctypes.c_void_p()
    assert L.nmhd_batch_create(arr, 2, ctypes.byref(h)) == -1
    assert b"box 1" in L.nmhd_batch_last_error(None)


@pytest.mark.gpu
@pytest.mark.parametrize("schedule", ["per_tile", "persistent", "mixed", "unsplit", "unsplit_persistent",
                                      "fused", "fused_persistent", "staged", "staged_persistent"])
def test_batch_boxes_equal_single_box_runs(gpu, schedule):
    """Every box of a batch equals its single-box run, in each schedule of the
    stage kernels (persistent tile ranges or one tile per CTA, and the fused
    constrained-transport + update pass of the 32 x 4 x 2 boxes)."""
    from nmhd_b200.batch import BatchSolver
    from nmhd_b200.solver import MHDSolver
    persist = {"per_tile": (0, 0, 0), "persistent": (1, 1, 1), "mixed": (1, 0, 1), "unsplit": (0, 0, 0),
               "unsplit_persistent": (1, 1, 1), "fused": (0, 0, 0), "fused_persistent": (1, 1, 1),
               "staged": (0, 0, 0), "staged_persistent": (1, 1, 1)}[schedule]
    split = not schedule.startswith("unsplit")
    boxes, _ = small_ensemble()
    # add two non-shearing boxes of other shapes (power-of-two and not)
    boxes.append(orszag_tang_3d(16))
    boxes.append(orszag_tang_3d(24, ny=20, nz=12))
    # and a box with interior tiles (cells and their +-1 neighbours away from
    # every edge), which the CT kernel addresses without the periodic wrap
    boxes.append(shearing_box(n_radial=24, n_azimuthal=128, n_vertical=8, l_azimuthal=4.0, seed=5))
    # and a single-plane box (its tile is one plane deep)
    boxes.append(orszag_tang_3d(40, ny=24, nz=1))
    steps = 9
    with BatchSolver([c for c, _ in boxes]) as batch:
        # the boxes' tile shapes (fewest padded cells) include narrow ones
        shapes = {batch.tile_shape(i) for i in range(len(boxes))}
        assert all(x * y * z == 256 and x >= 8 for x, y, z in shapes) and len(shapes) >= 3, shapes
        for k, p in enumerate(persist):
            batch.set_schedule(k, p, split)
        if schedule.startswith("fused"):
            launches = batch.launches_per_step()
            batch.set_schedule(3, schedule == "fused_persistent", True)
            assert batch.launches_per_step() != launches
        if schedule.startswith("staged"):
            batch.set_schedule(4, schedule == "staged_persistent", True)
        for i, (c, s) in enumerate(boxes):
            batch.set_state(i, s)
        batch.step(4)
        batch.step(steps - 4)
        for i, (c, s) in enumerate(boxes):
            with MHDSolver(c) as one:
                one.set_state(s)
                one.step(steps)
                t, g = batch.clock(i)
                assert g == steps and t == one.current_time(), f"box {i} clock"
                assert np.array_equal(batch.get_state(i), one.get_state()), f"box {i} state"


@pytest.mark.gpu
def test_batch_goal_time_per_box(gpu):
    """Per-box goal times, with the batch on a caller's stream."""
    import torch
    from nmhd_b200.batch import BatchSolver
    from nmhd_b200.solver import MHDSolver
    boxes, _ = small_ensemble(n=4, seed=8)
    stream = torch.cuda.Stream(device=gpu)
    with BatchSolver([c for c, _ in boxes]) as batch:
        batch.set_stream(stream.cuda_stream)
        batch.set_states([s for _, s in boxes])  # all boxes in one call
        assert batch.proceed(0.05)
        for i, (c, s) in enumerate(boxes):
            with MHDSolver(c) as one:
                one.set_state(s)
                assert one.proceed(0.05)
                t, g = batch.clock(i)
                assert t == float(np.float32(0.05)) and g == one.generation()
                out = np.empty((8,) + c.shape, dtype=np.float32)
                assert batch.get_state(i, out=out) is out
                assert np.array_equal(out, one.get_state())
                assert np.array_equal(batch.get_states()[i], out)


@pytest.mark.gpu
def test_batch_of_more_boxes_than_one_launch_group(gpu):
    """Batches beyond one launch group (128 boxes) are split into several
    launches per kernel; boxes on both sides of a group boundary still equal
    their single-box runs."""
    from nmhd_b200.batch import BatchSolver
    from nmhd_b200.solver import MHDSolver
    boxes, _ = mri_ensemble(n_boxes=131, seed=11, sides=(8,), ratios=(2, 3))
    steps = 5
    with BatchSolver([c for c, _ in boxes]) as batch:
        for i, (c, s) in enumerate(boxes):
            batch.set_state(i, s)
        batch.step(steps)
        for i in (0, 1, 126, 127, 128, 129, 130):
            c, s = boxes[i]
            with MHDSolver(c) as one:
                one.set_state(s)
                one.step(steps)
                t, g = batch.clock(i)
                assert g == steps and t == one.current_time(), f"box {i} clock"
                assert np.array_equal(batch.get_state(i), one.get_state()), f"box {i} state"


@pytest.mark.gpu
def test_batch_autotune_keeps_states_clocks_and_results(gpu):
    """The schedule autotuner times both schedules of every stage kernel on the
    current states, leaves states and clocks unchanged, and the batch then
    still advances every box bitwise as its single-box run."""
    from nmhd_b200.batch import BatchSolver
    from nmhd_b200.solver import MHDSolver
    boxes, _ = small_ensemble(n=5, seed=4)
    with BatchSolver([c for c, _ in boxes]) as batch:
        for i, (c, s) in enumerate(boxes):
            batch.set_state(i, s)
        batch.step(3)
        before = [(batch.clock(i), batch.get_state(i)) for i in range(len(boxes))]
        trials = batch.autotune(reps=2)
        assert sorted((k, p, s) for k, p, s, _ in trials if k < 3) == [(k, p, s) for k in range(3)
                                                                       for p in (False, True)
                                                                       for s in (False, True)]
        # the fused pass against the update kernels: off, and where boxes have
        # 32 x 4 x 2 tiles, per tile and persistent
        fixed = any(batch.tile_shape(i) == (32, 4, 2) for i in range(len(boxes)))
        for kk in (3, 4):  # fused update, staged fluxes
            assert sorted((p, s) for k, p, s, _ in trials if k == kk) == (
                [(False, False), (False, True), (True, True)] if fixed else [(False, False)])
        assert all(ms > 0 for _, _, _, ms in trials)
        for i, (clk, st) in enumerate(before):
            assert batch.clock(i) == clk and np.array_equal(batch.get_state(i), st)
        batch.step(4)
        for i, (c, s) in enumerate(boxes):
            with MHDSolver(c) as one:
                one.set_state(s)
                one.step(7)
                assert np.array_equal(batch.get_state(i), one.get_state()), f"box {i}"


def test_batch_schedule_arguments_are_checked_on_cpu():
    L = _lib.lib()
    assert L.nmhd_batch_set_schedule(None, 0, 0, 1) == -1
    assert L.nmhd_batch_autotune(None, 3, None, 0) == -1
    assert L.nmhd_batch_set_stream(None, None) == -1
    assert L.nmhd_batch_launches_per_step(None) == -1
    assert L.nmhd_batch_set_states(None, None, 0) == -1 and L.nmhd_batch_get_states(None, None, 0) == -1


def test_batch_tile_rule_launches_the_fewest_padded_cells_on_cpu():
    """nmhd_batch_tile_rule (the tile of a box in the batched kernels): 256
    threads as 2^a x 2^b x 2^c cells with x at least 8 wide, the fewest padded
    cells; among equals the widest x, then the shape nearest 32 x 4 x 2, then
    the taller y.  Checked against a brute force over seeded box sizes."""
    L = _lib.lib()
    rng = np.random.default_rng(7)

    def padded(n, e):
        return -(-n // (1 << e)) << e

    def brute(sx, sy, sz):
        shapes = [(a, b, 8 - a - b) for a in (5, 4, 3) for b in range(0, 9 - a)]
        key = lambda s: (padded(sx, s[0]) * padded(sy, s[1]) * padded(sz, s[2]), -s[0],
                         abs(s[1] - 2) + abs(s[2] - 1), -s[1])
        best = min(shapes, key=key)
        if key(best) == key((5, 2, 1)):
            best = (5, 2, 1)
        return tuple(1 << e for e in best)

    cfg, _ = shearing_box(n_radial=16, n_azimuthal=32, n_vertical=8)
    sizes = [(16, 16, 16), (48, 24, 16), (40, 24, 1), (256, 136, 64), (1, 1, 1), (24, 20, 12)]
    sizes += [tuple(int(v) for v in rng.integers(1, 200, size=3)) for _ in range(300)]
    for sx, sy, sz in sizes:
        c = SolverConfig(**{**cfg.__dict__, "size_x": sx, "size_y": sy, "size_z": sz, "margin_y": 0,
                            "problem": "none"})
        v = [ctypes.c_int() for _ in range(3)]
        assert L.nmhd_batch_tile_rule(ctypes.byref(c.to_ctypes()), *[ctypes.byref(x) for x in v]) == 0
        got = tuple(x.value for x in v)
        assert got == brute(sx, sy, sz), (sx, sy, sz, got)
        assert got[0] * got[1] * got[2] == 256 and got[0] >= 8
    assert L.nmhd_batch_tile_rule(None, None, None, None) == -1
