"""GPU checks of the differentiation entry points (nmhd_loss_run,
nmhd_adjoint_run, nmhd_adjoint_run_f64, nmhd_tlm_run).

The FP32 runs use the production kernels for the forward pass, so their time
steps and trajectory are the oracle's; the adjoint kernels are checked against
the host build of the same per-cell adjoint (tests/native), against the GPU
tangent-linear run (transpose identity in FP64), and against FP64 central
differences of the loss along initial-velocity directions.  A
torch.autograd.Function wrapper (test harness only) exposes the adjoint as a
backward pass.
"""
import numpy as np
import pytest

import adcheck
from nmhd_b200._lib import NmhdError
from nmhd_b200.problems import orszag_tang_3d, shearing_box
from nmhd_b200.solver import MHDSolver
from oracle import oracle

pytestmark = pytest.mark.gpu


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
    elif name == "ragged":
        cfg, s = shearing_box(n_radial=10, n_azimuthal=36, n_vertical=5, l_azimuthal=4.0, seed=9)
    else:  # first-order reconstruction
        cfg, s = orszag_tang_3d(12, ny=10, nz=8)
        cfg.space_order = 1
    return cfg, s


CASES = ["ot", "shear", "shear_mz", "euler", "ragged", "order1"]


def _velocity_direction(shape, seed, amp=0.01):
    rng = np.random.default_rng(seed)
    d = np.zeros(shape)
    d[1:4] = rng.normal(0.0, 1.0, (3,) + shape[1:]) * amp
    return d


@pytest.mark.parametrize("case", CASES)
def test_loss_run_takes_the_oracle_steps_and_leaves_the_solver_alone(gpu, case):
    cfg, s = _case(case)
    o = oracle.proceed(cfg, s, 6)
    with MHDSolver(cfg) as sol:
        sol.set_state(s)
        J, dts = sol.loss_run(6, window=(2, 6))
        assert np.array_equal(dts, o["dts"])
        assert np.array_equal(sol.get_state().view(np.uint32), s.view(np.uint32))
        assert sol.generation() == 0 and sol.current_time() == 0.0
        Jf, _ = sol.loss_run(6, window=(2, 6), dt=dts)
        assert Jf == J
    Jh, _ = adcheck.adjoint(cfg, s, o["dts"], 2, 6, dtype=np.float32)
    assert J == pytest.approx(Jh, rel=1e-12, abs=1e-300)


@pytest.mark.parametrize("case", CASES)
def test_fp32_adjoint_matches_the_host_build(gpu, case):
    cfg, s = _case(case)
    with MHDSolver(cfg) as sol:
        sol.set_state(s)
        J, g, dts = sol.adjoint(6, window=(2, 6), ckpt_every=4)
    Jh, gh = adcheck.adjoint(cfg, s, dts, 2, 6, dtype=np.float32)
    assert J == pytest.approx(Jh, rel=1e-12, abs=1e-300)
    scale = np.max(np.abs(gh))
    assert scale > 0
    assert np.max(np.abs(g - gh)) <= 1e-5 * scale


@pytest.mark.parametrize("ckpt", [1, 2, 5, 6, 20])
@pytest.mark.parametrize("budget", ["last", "two", "auto"])
def test_checkpoint_interval_and_tape_budget_do_not_change_the_gradient(gpu, ckpt, budget):
    """Checkpoint interval and the number of segments kept on the tape (the
    last only: every earlier segment recomputed; two; all that fit) leave the
    gradient bitwise unchanged."""
    cfg, s = _case("shear")
    nseg = -(-6 // ckpt)
    seg_bytes = min(ckpt, 6) * 24 * cfg.cells * 4  # 24 tape fields per step
    with MHDSolver(cfg) as sol:
        sol.set_state(s)
        sol.set_adjoint_tape_budget(0)
        J0, g0, _ = sol.adjoint(6, window=(1, 6), ckpt_every=3)
        assert sol.adjoint_kept_segments() == 1
        sol.set_adjoint_tape_budget({"last": 0, "two": seg_bytes, "auto": -1}[budget])
        J, g, _ = sol.adjoint(6, window=(1, 6), ckpt_every=ckpt)
        assert sol.adjoint_kept_segments() == {"last": 1, "two": min(2, nseg), "auto": nseg}[budget]
        if budget == "auto":
            assert sol.adjoint_timing()["recompute"] < 0.05  # nothing to recompute
    assert J == J0
    assert np.array_equal(g.view(np.uint32), g0.view(np.uint32))


@pytest.mark.parametrize("case", CASES)
def test_fp64_adjoint_is_the_transpose_of_the_gpu_tangent_linear_run(gpu, case):
    cfg, s = _case(case)
    o = oracle.proceed(cfg, s, 6)
    rng = np.random.default_rng(5)
    scale = np.abs(s.astype(np.float64)).reshape(8, -1).mean(axis=1).reshape(8, 1, 1, 1) + 1e-3
    d = rng.normal(0.0, 1.0, s.shape) * scale
    with MHDSolver(cfg) as sol:
        sol.set_state(s)
        J, dJ = sol.tlm(6, o["dts"], d, window=(2, 6))
        Ja, g = sol.adjoint_f64(6, o["dts"], window=(2, 6), ckpt_every=4)
    assert Ja == pytest.approx(J, rel=1e-12, abs=1e-300)
    assert float(np.sum(g * d)) == pytest.approx(dJ, rel=1e-10, abs=1e-13 * abs(J) + 1e-300)
    # and the same numbers as the host build of the tangent-linear step
    Jh, dJh = adcheck.tlm(cfg, s.astype(np.float64), d, o["dts"].astype(np.float64), 2, 6)
    assert J == pytest.approx(Jh, rel=1e-12, abs=1e-300)
    assert dJ == pytest.approx(dJh, rel=1e-10, abs=1e-13 * abs(J) + 1e-300)


def test_gradient_agrees_with_fp64_central_differences_on_a_shearing_box(gpu):
    """Central differences in FP64 around the same float state (shift), with
    eps far below the perturbation at which limiter, upwind-corner or sign(Bx)
    choices start to flip: the discrete step is only piecewise smooth, so a
    larger eps measures those jumps, not the derivative."""
    cfg, s = shearing_box(n_radial=24, n_azimuthal=32, n_vertical=16, l_radial=1.0, l_azimuthal=1.0, seed=2)
    steps, window = 30, (21, 30)
    with MHDSolver(cfg) as sol:
        sol.set_state(s)
        J, g, dts = sol.adjoint(steps, window=window, ckpt_every=10)
        _, g64 = sol.adjoint_f64(steps, dts, window=window, ckpt_every=10)
        for k in range(3):
            d = _velocity_direction(s.shape, 100 + k)
            eps = 1e-8
            Jp, _ = sol.tlm(steps, dts, d, window=window, shift=eps)
            Jm, _ = sol.tlm(steps, dts, d, window=window, shift=-eps)
            fd = (Jp - Jm) / (2 * eps)
            _, dJ = sol.tlm(steps, dts, d, window=window)
            assert dJ == pytest.approx(fd, rel=1e-4)
            assert float(np.sum(g64 * d)) == pytest.approx(fd, rel=1e-4)
            assert float(np.sum(g.astype(np.float64) * d)) == pytest.approx(fd, rel=1e-2)


def test_window_edges_and_initial_state_term(gpu):
    cfg, s = _case("shear")
    o = oracle.proceed(cfg, s, 4)
    d = _velocity_direction(s.shape, 7, amp=1.0)
    d[5:7] = np.random.default_rng(8).normal(0.0, 1e-3, d[5:7].shape)
    with MHDSolver(cfg) as sol:
        sol.set_state(s)
        for window in [(0, 0), (0, 4), (4, 4)]:
            _, dJ = sol.tlm(4, o["dts"], d, window=window)
            _, g = sol.adjoint_f64(4, o["dts"], window=window, ckpt_every=2)
            assert float(np.sum(g * d)) == pytest.approx(dJ, rel=1e-10, abs=1e-300)


def test_invalid_arguments_are_rejected(gpu):
    cfg, s = _case("shear")
    with MHDSolver(cfg) as sol:
        sol.set_state(s)
        with pytest.raises(NmhdError):
            sol.loss_run(0)
        with pytest.raises(NmhdError):
            sol.loss_run(5000)
        with pytest.raises(NmhdError):
            sol.loss_run(4, window=(3, 5))
        with pytest.raises(NmhdError):
            sol.adjoint(4, ckpt_every=0)
        # the solver still steps like the oracle afterwards
        sol.step(3)
        assert np.array_equal(sol.get_state(), oracle.proceed(cfg, s, 3)["state"])


def test_autograd_function_wraps_the_adjoint(gpu):
    torch = pytest.importorskip("torch")
    cfg, s = _case("shear")
    steps, window = 6, (2, 6)

    class MaxwellStressLoss(torch.autograd.Function):
        """J(initial velocity) through the C ABI; backward = nmhd_adjoint_run."""

        @staticmethod
        def forward(ctx, velocity):
            st = s.copy()
            st[1:4] = velocity.detach().cpu().numpy()
            with MHDSolver(cfg) as sol:
                sol.set_state(st)
                J, g, _ = sol.adjoint(steps, window=window, ckpt_every=3)
            ctx.save_for_backward(torch.from_numpy(g[1:4].copy()))
            return torch.tensor(J, dtype=torch.float64)

        @staticmethod
        def backward(ctx, grad_out):
            (g,) = ctx.saved_tensors
            return grad_out * g.to(torch.float64)

    v = torch.tensor(s[1:4].astype(np.float64), requires_grad=True)
    J = MaxwellStressLoss.apply(v)
    J.backward()
    with MHDSolver(cfg) as sol:
        sol.set_state(s)
        _, g, _ = sol.adjoint(steps, window=window, ckpt_every=3)
    assert np.array_equal(v.grad.numpy(), g[1:4].astype(np.float64))
    # a small step against the gradient lowers J by about |grad|^2 * step
    step = 1e-3 / float(np.linalg.norm(g[1:4]))
    with torch.no_grad():
        J2 = MaxwellStressLoss.apply(v - step * v.grad)
    predicted_drop = step * float((v.grad ** 2).sum())
    assert float(J) - float(J2) == pytest.approx(predicted_drop, rel=0.05)
