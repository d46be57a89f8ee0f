"""Batched ensemble of independent boxes (nmhd_batch_* in include/nmhd.h).

Every box keeps its own configuration, state, clock and CFL time step; all
boxes advance together, one persistent launch per kernel per stage.  A box
advanced in a batch is bitwise the box advanced alone by
:class:`~nmhd_b200.solver.MHDSolver`.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np

from . import _lib


class BatchSolver:
    def __init__(self, configs):
        self.configs = list(configs)
        self._L = _lib.lib()
        arr = (type(self.configs[0].to_ctypes()) * len(self.configs))(
            *[c.to_ctypes() for c in self.configs])
        self._arr = arr
        h = ctypes.c_void_p()
        code = self._L.nmhd_batch_create(arr, len(self.configs), ctypes.byref(h))
        if code != 0:
            raise _lib.NmhdError(code, self._L.nmhd_batch_last_error(None).decode())
        self._h = h

    def _check(self, code):
        if code < 0:
            raise _lib.NmhdError(code, self._L.nmhd_batch_last_error(self._h).decode())
        return code

    def close(self):
        if getattr(self, "_h", None):
            self._L.nmhd_batch_destroy(self._h)
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

    def __len__(self):
        return len(self.configs)

    def _ptrs(self, i, arr):
        n = self.configs[i].cells
        base = arr.ctypes.data
        return (ctypes.c_void_p * 8)(*[base + 4 * n * v for v in range(8)])

    def set_state(self, i, state):
        st = np.ascontiguousarray(state, dtype=np.float32)
        if st.shape != (8,) + self.configs[i].shape:
            raise ValueError(f"box {i}: state shape {st.shape} != {(8,) + self.configs[i].shape}")
        self._check(self._L.nmhd_batch_set_state(self._h, i, self._ptrs(i, st), 0))

    def get_state(self, i, out=None):
        """State of box i (8 fields, .bin order); into ``out`` (a C-contiguous
        float32 host array of that shape, e.g. pinned) when given."""
        shape = (8,) + self.configs[i].shape
        if out is None:
            out = np.empty(shape, dtype=np.float32)
        elif out.shape != shape or out.dtype != np.float32 or not out.flags.c_contiguous:
            raise ValueError(f"box {i}: out must be a C-contiguous float32 array of shape {shape}")
        self._check(self._L.nmhd_batch_get_state(self._h, i, self._ptrs(i, out), 0))
        return out

    def set_states(self, states):
        """Every box's state at once (a sequence of arrays, box order)."""
        if len(states) != len(self.configs):
            raise ValueError(f"{len(states)} states for {len(self.configs)} boxes")
        arrs = [np.ascontiguousarray(s, dtype=np.float32) for s in states]
        for i, a in enumerate(arrs):
            if a.shape != (8,) + self.configs[i].shape:
                raise ValueError(f"box {i}: state shape {a.shape} != {(8,) + self.configs[i].shape}")
        ptrs = (ctypes.c_void_p * (8 * len(arrs)))(*[p for i, a in enumerate(arrs) for p in self._ptrs(i, a)])
        self._check(self._L.nmhd_batch_set_states(self._h, ptrs, 0))

    def get_states(self, out=None):
        """Every box's state at once, into ``out`` (C-contiguous float32 host
        arrays, box order) when given."""
        if out is None:
            out = [np.empty((8,) + c.shape, dtype=np.float32) for c in self.configs]
        for i, a in enumerate(out):
            if a.shape != (8,) + self.configs[i].shape or a.dtype != np.float32 or not a.flags.c_contiguous:
                raise ValueError(f"box {i}: out must be a C-contiguous float32 array of shape "
                                 f"{(8,) + self.configs[i].shape}")
        ptrs = (ctypes.c_void_p * (8 * len(out)))(*[p for i, a in enumerate(out) for p in self._ptrs(i, a)])
        self._check(self._L.nmhd_batch_get_states(self._h, ptrs, 0))
        return out

    def clock(self, i):
        t = ctypes.c_double()
        g = ctypes.c_int64()
        self._check(self._L.nmhd_batch_clock(self._h, i, ctypes.byref(t), ctypes.byref(g)))
        return t.value, g.value

    def proceed(self, goal_time=math.inf, max_steps=0):
        done = ctypes.c_int64()
        code = self._check(self._L.nmhd_batch_proceed(self._h, float(goal_time), int(max_steps),
                                                      ctypes.byref(done)))
        self.last_steps = done.value
        return code == _lib.GOAL_REACHED

    def step(self, nsteps):
        self.proceed(math.inf, nsteps)
        return self.last_steps

    def prepare(self, max_steps=0):
        """Build the CUDA graphs a later proceed(..., max_steps) launches,
        without running them (nmhd_batch_prepare)."""
        self._check(self._L.nmhd_batch_prepare(self._h, int(max_steps)))

    def set_stream(self, cuda_stream):
        """Run the batch's work on ``cuda_stream`` (a cudaStream_t as int, e.g.
        torch.cuda.Stream().cuda_stream); None: a stream of its own."""
        self._check(self._L.nmhd_batch_set_stream(self._h, ctypes.c_void_p(cuda_stream or None)))

    def launches_per_step(self):
        """Kernel launches of one batched step with the current schedules."""
        return self._check(self._L.nmhd_batch_launches_per_step(self._h))

    def tile_shape(self, i):
        """Tile of box i in the batched kernels: (x, y, z) cells."""
        v = [ctypes.c_int() for _ in range(3)]
        self._check(self._L.nmhd_batch_tile_shape(self._h, int(i), *[ctypes.byref(c) for c in v]))
        return tuple(c.value for c in v)

    def set_schedule(self, kernel, persistent, split=True):
        """Schedule of stage kernel ``kernel`` (0 fluxes, 1 constrained
        transport, 2 conserved update): persistent or one tile per CTA; with
        ``split`` the boxes with 32 x 4 x 2 tiles run in a launch of their own.
        ``kernel`` 3 is the fused pass (constrained transport and conserved
        update of the 32 x 4 x 2 boxes in one kernel): ``split`` turns it on
        (it then needs kernels 1 and 2 split), ``persistent`` its schedule.
        ``kernel`` 4 is the staged flux pass of the 32 x 4 x 2 boxes (their
        fluxes from a shared copy of each tile's stencil; needs kernel 0
        split), turned on and scheduled the same way."""
        self._check(self._L.nmhd_batch_set_schedule(self._h, int(kernel), int(bool(persistent)),
                                                    int(bool(split))))

    def autotune(self, reps=5):
        """Pick each stage kernel's schedule (persistent or one tile per CTA,
        split or not) by timing all of them on the current states, then the
        face fluxes with and without the staged flux pass and the stage
        update with and without the fused pass; states and clocks are left
        unchanged.  Returns rows (kernel, persistent, split, ms per launch);
        kernel 4 rows are (4, persistent, staged, ms per flux launch), kernel
        3 rows (3, persistent, fused, ms per stage update)."""
        out = np.zeros((20, 4), dtype=np.float64)
        k = self._check(self._L.nmhd_batch_autotune(self._h, int(reps), out.ctypes.data, 20))
        return [(int(a), bool(b), bool(c), float(d)) for a, b, c, d in out[:k]]

    @property
    def cells(self):
        return sum(c.cells for c in self.configs)

    @property
    def interior_cells(self):
        return sum(c.interior_cells for c in self.configs)
