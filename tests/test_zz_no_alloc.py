"""The allocation-free entry point, nmhd_advance_noalloc, called through the C ABI.

It is for callers that cannot allocate device memory: a host framework whose
caching allocator has reserved the device's memory, or a real-time loop where
a device allocation and the synchronisation it can bring are not allowed.
This file is named so pytest collects it last; it passes alone in a fresh
process and after the other tests.

Tolerance: bitwise equality with the existing entry point (nmhd_create +
nmhd_proceed), the same bar as every other parity test here.
"""
import ctypes
import math

import numpy as np
import pytest

from nmhd_b200 import _lib
from nmhd_b200.problems import orszag_tang_3d, shearing_box
from nmhd_b200.solver import MHDSolver

pytestmark = pytest.mark.gpu


def noalloc(cfg, dev_in, dev_out, time, generation, steps, goal=math.inf):
    L = _lib.lib()
    c = cfg.to_ctypes()
    t = ctypes.c_double(time)
    g = ctypes.c_int64(generation)
    done = ctypes.c_int64(0)
    code = L.nmhd_advance_noalloc(ctypes.byref(c), ctypes.c_void_p(dev_in.data_ptr()),
                                  ctypes.c_void_p(dev_out.data_ptr()), ctypes.byref(t),
                                  ctypes.byref(g), goal, steps, ctypes.byref(done), None)
    return code, t.value, g.value, done.value


@pytest.mark.parametrize("case", ["orszag_tang", "shearing_box", "euler", "z_margins"])
def test_noalloc_matches_existing_entry_point_twice(gpu, case):
    import torch
    if case == "orszag_tang":
        cfg, s = orszag_tang_3d(24, ny=20, nz=12)
    elif case == "shearing_box":
        cfg, s = shearing_box(n_radial=16, n_azimuthal=32, n_vertical=8, l_azimuthal=4.0, seed=21)
    elif case == "euler":  # time_order 1
        cfg, s = shearing_box(n_radial=16, n_azimuthal=32, n_vertical=8, l_azimuthal=4.0, seed=22)
        cfg.time_order = 1
    else:  # Z margins filled by copy, as the reference's kMarginSizeZ
        cfg, s = shearing_box(n_radial=16, n_azimuthal=32, n_vertical=8, l_azimuthal=4.0, seed=23)
        cfg.margin_z, cfg.size_z = 4, 16
        s = np.ascontiguousarray(np.concatenate([s[:, -4:], s, s[:, :4]], axis=1))
    steps = 7
    # existing entry point: the same box after `steps` and after 2*`steps` steps
    with MHDSolver(cfg) as sol:
        sol.set_state(s)
        sol.step(steps)
        ref1, t1 = sol.get_state(), sol.current_time()
        sol.step(steps)
        ref2, t2 = sol.get_state(), sol.current_time()
    a = torch.from_numpy(s).to(gpu)
    b = torch.empty_like(a)
    c = torch.empty_like(a)
    torch.cuda.synchronize()
    code, t, g, done = noalloc(cfg, a, b, 0.0, 0, steps)
    assert code == _lib.STEP_LIMIT, _lib.lib().nmhd_noalloc_last_error()
    assert (g, done, t) == (steps, steps, t1)
    assert np.array_equal(b.cpu().numpy(), ref1)
    free_before = torch.cuda.mem_get_info()[0]
    code, t, g, done = noalloc(cfg, b, c, t, g, steps)  # second call, continuing
    free_after = torch.cuda.mem_get_info()[0]
    assert code == _lib.STEP_LIMIT, _lib.lib().nmhd_noalloc_last_error()
    assert (g, t) == (2 * steps, t2)
    assert np.array_equal(c.cpu().numpy(), ref2)
    assert free_after == free_before, "the call changed the free device memory"


def test_noalloc_goal_time_and_size_limit(gpu):
    import torch
    cfg, s = orszag_tang_3d(16)
    a = torch.from_numpy(s).to(gpu)
    b = torch.empty_like(a)
    code, t, g, _ = noalloc(cfg, a, b, 0.0, 0, 1000, goal=0.02)
    assert code == _lib.GOAL_REACHED
    assert t == float(np.float32(0.02))
    with MHDSolver(cfg) as sol:
        sol.set_state(s)
        assert sol.proceed(0.02)
        assert np.array_equal(b.cpu().numpy(), sol.get_state())
    big, _ = orszag_tang_3d(65)  # 65^3 cells > NMHD_NOALLOC_MAX_CELLS
    code, _, _, _ = noalloc(big, a, b, 0.0, 0, 1)
    assert code == -1
    assert b"at most 262144" in _lib.lib().nmhd_noalloc_last_error()


def test_noalloc_stops_at_the_goal_within_a_large_step_cap(gpu):
    """nsteps is a cap: with a goal a few steps away and a cap of 10^12 the
    call returns once the goal step is done (the control block is read back
    every 16 steps)."""
    import time as _time
    import torch
    cfg, s = orszag_tang_3d(16)
    a = torch.from_numpy(s).to(gpu)
    b = torch.empty_like(a)
    t0 = _time.perf_counter()
    code, t, g, done = noalloc(cfg, a, b, 0.0, 0, 10 ** 12, goal=0.01)
    assert code == _lib.GOAL_REACHED
    assert t == float(np.float32(0.01)) and done == g
    assert _time.perf_counter() - t0 < 60
