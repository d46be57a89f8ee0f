"""Host-side mirror of the reference's solver interface.

:class:`MHDSolver` keeps the member names, argument meaning and error
behaviour of the reference's ``class MHDSolver``
(src/library/mhd_solver.hrb:150-276): ``read``/``write`` return ``False`` on
failure, ``proceed`` returns ``True`` when the goal time was reached and
``False`` on a wallclock timeout, ``current_time``/``generation`` report the
clock.  Problem hooks cannot cross the C ABI, so ``initialize_state`` takes the
initial primitive state as an array (see :mod:`nmhd_b200.problems`).

Every call goes through libnmhd.so (include/nmhd.h); the compute runs only on
the GPU.
"""
from __future__ import annotations

import ctypes
import math
import os

import numpy as np

from . import _lib, checkpoint
from .config import SolverConfig


class NmhdDiag(ctypes.Structure):
    _fields_ = [
        ("mass", ctypes.c_double), ("momentum", ctypes.c_double * 3),
        ("kinetic_energy", ctypes.c_double), ("internal_energy", ctypes.c_double),
        ("magnetic_energy", ctypes.c_double), ("total_energy", ctypes.c_double),
        ("bx2_mean", ctypes.c_double), ("by2_mean", ctypes.c_double),
        ("maxwell_stress", ctypes.c_double), ("max_div_b", ctypes.c_double),
        ("volume", ctypes.c_double),
    ]


def _check(L, handle, code):
    if code < 0:
        raise _lib.NmhdError(code, L.nmhd_last_error(handle).decode())
    return code


class MHDSolver:
    """One box advanced by the B200 time step (MHDSolver::MHDSolver(LocalSetup&))."""

    def __init__(self, config: SolverConfig):
        self.config = config
        self._L = _lib.lib()
        self._c = config.to_ctypes()
        h = ctypes.c_void_p()
        code = self._L.nmhd_create(ctypes.byref(self._c), ctypes.byref(h))
        if code != 0:
            raise _lib.NmhdError(code, self._L.nmhd_last_error(None).decode())
        self._h = h
        self.last_status = _lib.OK

    # -- lifetime --------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            self._L.nmhd_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- state -----------------------------------------------------------
    def _ptrs(self, arr):
        n = self.config.cells
        base = arr.ctypes.data
        return (ctypes.c_void_p * 8)(*[base + 4 * n * v for v in range(8)])

    def initialize_state(self, state):
        """Set the primitive state (8, Sz, Sy, Sx) float32 (replaces the
        reference's set_initial_condition hook)."""
        self.set_state(state)

    def set_state(self, state):
        st = np.ascontiguousarray(state, dtype=np.float32)
        if st.shape != (8,) + self.config.shape:
            raise ValueError(f"state shape {st.shape} != {(8,) + self.config.shape}")
        _check(self._L, self._h, self._L.nmhd_set_state(self._h, self._ptrs(st), 0))

    def set_state_device(self, tensor):
        """Set the state from a CUDA tensor (8, Sz, Sy, Sx) float32 on this device."""
        n = self.config.cells
        t = tensor.contiguous()
        base = t.data_ptr()
        ptrs = (ctypes.c_void_p * 8)(*[base + 4 * n * v for v in range(8)])
        _check(self._L, self._h, self._L.nmhd_set_state(self._h, ptrs, 1))

    def get_state(self, out=None):
        if out is None:
            out = np.empty((8,) + self.config.shape, dtype=np.float32)
        _check(self._L, self._h, self._L.nmhd_get_state(self._h, self._ptrs(out), 0))
        return out

    def get_state_device(self, tensor):
        n = self.config.cells
        base = tensor.data_ptr()
        ptrs = (ctypes.c_void_p * 8)(*[base + 4 * n * v for v in range(8)])
        _check(self._L, self._h, self._L.nmhd_get_state(self._h, ptrs, 1))
        return tensor

    def read(self, path) -> bool:
        """MHDSolver::read: False when the file cannot be read or sizes differ."""
        code = self._L.nmhd_read(self._h, os.fsencode(path))
        self.last_status = code
        return code == 0

    def write(self, path) -> bool:
        code = self._L.nmhd_write(self._h, os.fsencode(path))
        self.last_status = code
        return code == 0

    # -- time stepping ---------------------------------------------------
    def monitor(self) -> int:
        """MHDSolver::monitor(): the application's per-step hook.  A subclass
        that overrides it makes proceed() call it before every step, as the
        reference's loop does (mhd_solver.inlrb:857-860); a non-zero return
        stops the run before that step."""
        return 0

    def dump(self, tag) -> bool:
        """MHDSolver::dump(tag): the state dump ``tag.bin`` (the reference's
        applications define their own)."""
        return self.write(str(tag) + ".bin")

    def initial_event(self) -> int:
        """Application hook called by the host program before the run."""
        return 0

    def final_event(self) -> int:
        """Application hook called by the host program after the run."""
        return 0

    def _proceed_monitored(self, goal_time, wallclock_time_limit, max_steps):
        import time as _t
        t0 = _t.monotonic()
        steps = 0
        while True:
            if max_steps > 0 and steps >= max_steps:
                self.last_steps = steps
                return False
            if self.monitor():
                self.last_steps = steps
                return False
            left = -1.0
            if wallclock_time_limit > 0:
                left = wallclock_time_limit - (_t.monotonic() - t0)
                if left <= 0:
                    self.last_steps = steps
                    return False
            done = ctypes.c_int64(0)
            code = self._L.nmhd_proceed(self._h, float(goal_time), float(left), 1, ctypes.byref(done))
            self.last_status = code
            steps += done.value
            _check(self._L, self._h, code)
            if code == _lib.GOAL_REACHED:
                self.last_steps = steps
                return True
            if code == _lib.TIMEOUT:
                self.last_steps = steps
                return False

    def proceed(self, goal_time, wallclock_time_limit=-1.0, max_steps=0) -> bool:
        """MHDSolver::proceed: integrate until ``goal_time`` (True) or until the
        wallclock limit in seconds passes (False); ``max_steps`` > 0 also stops
        after that many steps (False).  Raises on numerical or CUDA errors.
        Steps run in device-resident batches unless a subclass overrides
        monitor()."""
        if type(self).monitor is not MHDSolver.monitor:
            return self._proceed_monitored(goal_time, wallclock_time_limit, max_steps)
        done = ctypes.c_int64(0)
        code = self._L.nmhd_proceed(self._h, float(goal_time), float(wallclock_time_limit),
                                    int(max_steps), ctypes.byref(done))
        self.last_status = code
        self.last_steps = done.value
        _check(self._L, self._h, code)
        return code == _lib.GOAL_REACHED

    def prepare(self, max_steps=0):
        """Build the CUDA graphs a later proceed(..., max_steps) launches,
        without running them (nmhd_prepare)."""
        _check(self._L, self._h, self._L.nmhd_prepare(self._h, int(max_steps)))

    def step(self, nsteps):
        """Advance exactly ``nsteps`` steps (no goal time); returns steps done."""
        self.proceed(math.inf, -1.0, nsteps)
        return self.last_steps

    def current_time(self) -> float:
        return self._L.nmhd_current_time(self._h)

    def generation(self) -> int:
        return self._L.nmhd_generation(self._h)

    def set_time(self, current_time, generation):
        _check(self._L, self._h, self._L.nmhd_set_time(self._h, float(current_time), int(generation)))

    def dt_history(self, n):
        out = np.zeros(n, np.float32)
        k = self._L.nmhd_dt_history(self._h, out.ctypes.data, n)
        return out[:k]

    def diagnostics(self):
        d = NmhdDiag()
        _check(self._L, self._h, self._L.nmhd_diagnostics(self._h, ctypes.byref(d)))
        return {
            "mass": d.mass, "momentum": list(d.momentum), "kinetic_energy": d.kinetic_energy,
            "internal_energy": d.internal_energy, "magnetic_energy": d.magnetic_energy,
            "total_energy": d.total_energy, "bx2_mean": d.bx2_mean, "by2_mean": d.by2_mean,
            "maxwell_stress": d.maxwell_stress, "max_div_b": d.max_div_b, "volume": d.volume,
        }

    # -- checkpoint ------------------------------------------------------
    def save_state(self, prefix, rank=0) -> bool:
        """MHDSolver::save_state (src/library/mhd_solver.inlrb:1023-1036):
        ``prefix.bin`` plus ``prefix_setup.txt`` in the reference's pod text
        (see :mod:`nmhd_b200.checkpoint`); the reference's load_state reads
        both.  ``rank``: this solver's rank when it is a radial slab."""
        prefix = str(prefix)
        if not self.write(prefix + ".bin"):
            return False
        text = checkpoint.setup_text(self.config, self.generation(), self.current_time(),
                                     output_directory=os.path.dirname(os.path.abspath(prefix)), rank=rank)
        try:
            with open(prefix + "_setup.txt", "w") as fp:
                fp.write(text)
        except OSError:
            return False
        return True

    def load_state(self, prefix) -> bool:
        """MHDSolver::load_state (mhd_solver.inlrb:1038-1050): the clock from
        ``prefix_setup.txt`` (written here or by the reference) and the state
        from ``prefix.bin``; False, with state and clock unchanged, when a file
        cannot be read."""
        prefix = str(prefix)
        try:
            with open(prefix + "_setup.txt") as fp:
                gen, t = checkpoint.clock_from_setup(fp.read())
        except (OSError, ValueError, KeyError, IndexError):
            return False
        if not self.read(prefix + ".bin"):
            return False
        self.set_time(t, gen)
        return True

    def set_kernel(self, variant=0, tile_rows=8, z_chunk=16):
        """Select the kernel variant and tile shape (results are identical)."""
        _check(self._L, self._h, self._L.nmhd_set_kernel(self._h, int(variant), int(tile_rows),
                                                         int(z_chunk)))

    def kernel(self):
        """The current kernel selection: (variant, tile_rows, z_chunk)."""
        v, r, z = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _check(self._L, self._h, self._L.nmhd_get_kernel(self._h, ctypes.byref(v), ctypes.byref(r),
                                                         ctypes.byref(z)))
        return v.value, r.value, z.value

    def autotune(self, steps=5):
        """Time every kernel variant / tile shape on this box and keep the
        fastest (solvers created later for boxes of the same shape and scheme
        start with it); returns [(variant, tile_rows, z_chunk, ms_per_step), ...]."""
        out = np.zeros((64, 4), np.float64)
        k = _check(self._L, self._h, self._L.nmhd_autotune(self._h, int(steps), out.ctypes.data, 64))
        return [(int(a), int(b), int(c), float(d)) for a, b, c, d in out[:k]]

    def profile(self, steps):
        """Per kernel class: (mean device ms per step, kernel launches per
        step), from CUDA events around separately launched kernels."""
        ms = np.zeros(16, np.float64)
        launches = np.zeros(16, np.float64)
        k = _check(self._L, self._h, self._L.nmhd_profile(self._h, int(steps), ms.ctypes.data,
                                                          launches.ctypes.data, 16))
        return {self._L.nmhd_kernel_name(i).decode(): (float(ms[i]), float(launches[i]))
                for i in range(k)}

    @property
    def device(self):
        return self._L.nmhd_device(self._h)

    def set_stream(self, stream_ptr):
        _check(self._L, self._h, self._L.nmhd_set_stream(self._h, ctypes.c_void_p(stream_ptr)))

    # -- differentiation (no counterpart in the reference) ------------------
    def _loss(self, nsteps, window):
        first, last = (0, nsteps) if window is None else window
        return _lib.LossSpec(_lib.LOSS_MAXWELL_STRESS, int(first), int(last), 0)

    @staticmethod
    def _dts(dt, nsteps):
        if dt is None:
            return None
        d = np.ascontiguousarray(dt, np.float32)
        if d.shape != (nsteps,):
            raise ValueError(f"dt must have {nsteps} entries")
        return d

    def loss_run(self, nsteps, window=None, dt=None):
        """FP32 forward run of ``nsteps`` steps from the current state (which
        stays unchanged).  Returns (J, dts): J the mean over the states
        window=(first, last) of the Maxwell stress -<Bx By> (default: all
        states 0..nsteps), dts the time steps taken (``dt`` freezes them)."""
        spec = self._loss(nsteps, window)
        d = self._dts(dt, nsteps)
        loss = ctypes.c_double()
        dts = np.zeros(nsteps, np.float32)
        _check(self._L, self._h, self._L.nmhd_loss_run(
            self._h, int(nsteps), ctypes.byref(spec), None if d is None else d.ctypes.data,
            ctypes.byref(loss), dts.ctypes.data))
        return loss.value, dts

    def adjoint(self, nsteps, window=None, dt=None, ckpt_every=20, out=None):
        """FP32 adjoint: (J, dJ/d(initial state) as (8, Sz, Sy, Sx) float32, dts)."""
        spec = self._loss(nsteps, window)
        d = self._dts(dt, nsteps)
        if out is None:
            out = np.zeros((8,) + self.config.shape, np.float32)
        loss = ctypes.c_double()
        dts = np.zeros(nsteps, np.float32)
        _check(self._L, self._h, self._L.nmhd_adjoint_run(
            self._h, int(nsteps), int(ckpt_every), ctypes.byref(spec), None if d is None else d.ctypes.data,
            ctypes.byref(loss), dts.ctypes.data, self._ptrs(out), 0))
        return loss.value, out, dts

    def adjoint_f64(self, nsteps, dt, window=None, ckpt_every=20):
        """FP64 adjoint with the time steps frozen to ``dt``: (J, gradient float64)."""
        spec = self._loss(nsteps, window)
        d = self._dts(dt, nsteps)
        out = np.zeros((8,) + self.config.shape, np.float64)
        n = self.config.cells
        ptrs = (ctypes.c_void_p * 8)(*[out.ctypes.data + 8 * n * v for v in range(8)])
        loss = ctypes.c_double()
        _check(self._L, self._h, self._L.nmhd_adjoint_run_f64(
            self._h, int(nsteps), int(ckpt_every), ctypes.byref(spec), d.ctypes.data, ctypes.byref(loss), ptrs))
        return loss.value, out

    def tlm(self, nsteps, dt, direction=None, window=None, shift=0.0):
        """FP64 tangent-linear run with frozen ``dt`` from the current state
        plus ``shift * direction`` (in double): (J, dJ[direction])."""
        spec = self._loss(nsteps, window)
        d = self._dts(dt, nsteps)
        ptrs = None
        if direction is not None:
            dr = np.ascontiguousarray(direction, np.float64)
            if dr.shape != (8,) + self.config.shape:
                raise ValueError("direction must have the state's shape")
            n = self.config.cells
            ptrs = (ctypes.c_void_p * 8)(*[dr.ctypes.data + 8 * n * v for v in range(8)])
        loss = ctypes.c_double()
        dloss = ctypes.c_double()
        _check(self._L, self._h, self._L.nmhd_tlm_run(
            self._h, int(nsteps), ctypes.byref(spec), d.ctypes.data, ptrs, float(shift), ctypes.byref(loss),
            ctypes.byref(dloss)))
        return loss.value, dloss.value

    def set_adjoint_tape_budget(self, nbytes=-1):
        """Device memory for forward tapes beyond the last segment's (-1:
        as many segments as fit in half the free memory; 0: last segment
        only).  The gradient does not depend on it."""
        _check(self._L, self._h, self._L.nmhd_adjoint_set_tape_budget(self._h, int(nbytes)))

    def adjoint_kept_segments(self):
        """Segments whose forward tape the last adjoint run kept (not recomputed)."""
        return int(self._L.nmhd_adjoint_kept_segments(self._h))

    def adjoint_timing(self):
        """Device ms of the last adjoint run: forward (with checkpoints),
        recompute (segment recomputation on its own stream, overlapping the
        reverse sweep), adjoint (the reverse sweep), total (forward + reverse
        sweep)."""
        ms = np.zeros(4, np.float64)
        _check(self._L, self._h, self._L.nmhd_adjoint_timing(self._h, ms.ctypes.data))
        return {"forward": ms[0], "recompute": ms[1], "adjoint": ms[2], "total": ms[3]}
