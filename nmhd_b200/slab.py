"""Radial slab decomposition of one box over P ranks (kParallelSizeY = P).

The reference splits a box along Y (radial) over MPI ranks, each rank
advancing its slab in its own shearing frame (positions relative to the slab's
centre).  Every step, MHDSolver::proceed (src/library/mhd_solver.inlrb:850-993)
calls communicate() (:283-493): each rank sends its top margin_y interior rows,
shifted in X by the shear displacement with v_X - relative_velocity, to the
rank above, and its bottom rows, shifted the other way with v_X +
relative_velocity, to the rank below (the last and first ranks are neighbours:
the radial boundary is shear-periodic); then dt is the MPI_Allreduce MIN of the
ranks' CFL times.  The reference stages every message through host memory.

Here each slab is an :class:`~nmhd_b200.solver.MHDSolver` created with
``parallel_size_y = P``, stepped through the split-phase C ABI
(``nmhd_halo_pack`` / transport / ``nmhd_halo_unpack`` / reduce /
``nmhd_step_stages``, include/nmhd.h), with the messages in device memory:

* :class:`SlabGroup` - every slab in this process, on one GPU and one stream:
  a slab unpacks straight from its neighbours' send buffers and the CFL
  minimum is one kernel (``nmhd_cfl_min``); no copies.
* :class:`DistributedSlab` - one slab per process (one process per GPU):
  ``torch.distributed`` point-to-point ``batch_isend_irecv`` of the two
  messages and ``all_reduce(MIN)`` of the CFL time, in the stream order of
  the solver's kernels (NCCL between GPUs).  The transport is written against
  a small backend interface so that the same code runs over ``gloo`` on the
  CPU in tests.

Results are bitwise those of the reference's P-rank run.  A rank's state is in
its own frame; :mod:`nmhd_b200.postprocess` stitches per-rank snapshots
(save_state with the rank) onto the global grid as the reference's tools do.
"""
from __future__ import annotations

import ctypes
import math
import time as _time
from dataclasses import replace

import numpy as np

from . import _lib
from .config import SolverConfig
from .solver import MHDSolver, _check

BATCH = 16  # steps between host polls of the clock and status


def slab_config(whole: SolverConfig, n_slabs: int) -> SolverConfig:
    """Configuration of one of ``n_slabs`` radial slabs of the box ``whole``
    (kLocalSizeY = interior rows / n_slabs, same margins and extents)."""
    rows = whole.size_y - 2 * whole.margin_y
    if n_slabs < 1 or rows % n_slabs:
        raise ValueError(f"{rows} interior rows do not split into {n_slabs} slabs")
    if n_slabs > 1 and (whole.margin_y < 1 or rows // n_slabs < whole.margin_y):
        raise ValueError("each slab needs margin_y >= 1 and at least margin_y interior rows")
    return replace(whole, size_y=rows // n_slabs + 2 * whole.margin_y, parallel_size_y=n_slabs)


def neighbours(rank: int, world: int):
    """(rank below, rank above) along Y, periodic (communicate(),
    mhd_solver.inlrb:337-342)."""
    return (rank - 1) % world, (rank + 1) % world


class SlabGroup:
    """All P slabs of one box in this process, on the current CUDA device.

    ``config`` is one slab's configuration (``parallel_size_y`` = P) and
    ``states[r]`` rank r's primitive state (8, Sz, Sy, Sx) in its own frame.
    Mirrors MHDSolver's clock and ``proceed``; ``get_states`` returns every
    rank's state."""

    def __init__(self, config: SolverConfig, states):
        import torch
        self.P = len(states)
        if max(1, config.parallel_size_y) != self.P:
            raise ValueError("parallel_size_y must equal the number of slab states")
        if self.P > _MAX_SLOTS:
            raise ValueError(f"at most {_MAX_SLOTS} slabs in one process")
        self.config = config
        self._L = _lib.lib()
        self.slabs = [MHDSolver(config) for _ in range(self.P)]
        self._stream = torch.cuda.Stream()
        for s in self.slabs:
            s.set_stream(self._stream.cuda_stream)
        for s, st in zip(self.slabs, states):
            s.set_state(st)
        n = max(1, int(self._L.nmhd_halo_count(self.slabs[0]._h)))
        self._send = torch.zeros((self.P, 2, n), dtype=torch.float32, device="cuda")
        self._handles = (ctypes.c_void_p * self.P)(*[s._h.value for s in self.slabs])
        self.last_steps = 0

    def close(self):
        for s in self.slabs:
            s.close()
        self.slabs = []

    def _ptr(self, r, k):
        return ctypes.c_void_p(self._send[r, k].data_ptr())

    def _step(self):
        L = self._L
        for r, s in enumerate(self.slabs):
            _check(L, s._h, L.nmhd_halo_pack(s._h, self._ptr(r, 0), self._ptr(r, 1)))
        for r, s in enumerate(self.slabs):
            lo, hi = neighbours(r, self.P)
            # the bottom margin takes the rank below's upward message, the top
            # margin the rank above's downward one
            _check(L, s._h, L.nmhd_halo_unpack(s._h, self._ptr(lo, 0), self._ptr(hi, 1)))
        _check(L, self.slabs[0]._h, L.nmhd_cfl_min(self._handles, self.P))
        for s in self.slabs:
            _check(L, s._h, L.nmhd_step_stages(s._h))

    def _poll(self):
        done = False
        gen = ctypes.c_int64()
        tm = ctypes.c_double()
        for s in self.slabs:
            code = self._L.nmhd_slab_poll(s._h, ctypes.byref(gen), ctypes.byref(tm))
            _check(self._L, s._h, code)
            done = done or code == _lib.GOAL_REACHED
        return done, gen.value

    def proceed(self, goal_time, wallclock_time_limit=-1.0, max_steps=0) -> bool:
        """MHDSolver::proceed over all slabs: True when the goal time was
        reached, False on the wallclock limit or after ``max_steps`` steps."""
        t0 = _time.monotonic()
        for s in self.slabs:
            _check(self._L, s._h, self._L.nmhd_slab_begin(s._h, float(goal_time)))
        gen0 = self.slabs[0].generation()
        left = max_steps if max_steps > 0 else -1
        reached = False
        while True:
            k = BATCH if left < 0 else min(BATCH, left)
            if k == 0:
                break
            for _ in range(k):
                self._step()
            if left > 0:
                left -= k
            done, gen = self._poll()
            if done:
                reached = True
                break
            if wallclock_time_limit > 0 and _time.monotonic() - t0 > wallclock_time_limit:
                break
        self.last_steps = self.slabs[0].generation() - gen0
        return reached

    def step(self, nsteps):
        self.proceed(math.inf, -1.0, nsteps)
        return self.last_steps

    def current_time(self):
        return self.slabs[0].current_time()

    def generation(self):
        return self.slabs[0].generation()

    def get_states(self):
        return [s.get_state() for s in self.slabs]

    def save_state(self, folder, tag) -> bool:
        """save_state(tag) of every rank: ``folder/tag/%04d.bin`` and
        ``%04d_setup.txt`` (the reference's layout of one snapshot folder)."""
        import os
        d = os.path.join(str(folder), str(tag))
        os.makedirs(d, exist_ok=True)
        return all(s.save_state(os.path.join(d, "%04d" % r), rank=r) for r, s in enumerate(self.slabs))


_MAX_SLOTS = 64  # kMaxSlots of the library's CFL-minimum kernel


# ---------------------------------------------------------------------------
# One slab per process


class SolverBackend:
    """The split-phase step of one slab on the GPU (libnmhd.so)."""

    def __init__(self, solver: MHDSolver, device):
        import torch
        self.solver = solver
        self._L = _lib.lib()
        self.device = device
        # NCCL work is ordered with torch's current stream: run the solver on it
        solver.set_stream(torch.cuda.current_stream(device).cuda_stream)
        ptr = self._L.nmhd_cfl_slot(solver._h)
        self._slot = torch.as_tensor(_DevicePointer(ptr, 1), device=device)

    def halo_count(self):
        return int(self._L.nmhd_halo_count(self.solver._h))

    def begin(self, goal_time):
        _check(self._L, self.solver._h, self._L.nmhd_slab_begin(self.solver._h, float(goal_time)))

    def pack(self, send_inc, send_dec):
        _check(self._L, self.solver._h, self._L.nmhd_halo_pack(
            self.solver._h, ctypes.c_void_p(send_inc.data_ptr()), ctypes.c_void_p(send_dec.data_ptr())))

    def unpack(self, recv_inc, recv_dec):
        _check(self._L, self.solver._h, self._L.nmhd_halo_unpack(
            self.solver._h, ctypes.c_void_p(recv_inc.data_ptr()), ctypes.c_void_p(recv_dec.data_ptr())))

    def cfl_slot(self):
        return self._slot

    def stages(self):
        _check(self._L, self.solver._h, self._L.nmhd_step_stages(self.solver._h))

    def poll(self):
        """(done, error message or None, generation, time) after the stream drains."""
        gen = ctypes.c_int64()
        tm = ctypes.c_double()
        code = self._L.nmhd_slab_poll(self.solver._h, ctypes.byref(gen), ctypes.byref(tm))
        err = None
        if code < 0:
            err = _lib.NmhdError(code, self._L.nmhd_last_error(self.solver._h).decode())
        return code == _lib.GOAL_REACHED, err, gen.value, tm.value


class _DevicePointer:
    """A float32 vector at a device address, for torch.as_tensor."""

    def __init__(self, ptr, n):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f4", "data": (ptr, False), "version": 2}


class DistributedSlab:
    """This process's slab of a box split over the ranks of ``group``
    (torch.distributed; rank r of P holds radial slab r).  ``backend`` is a
    :class:`SolverBackend` (GPU) or any object with the same methods."""

    def __init__(self, backend, group=None):
        import torch
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.b = backend
        n = max(1, backend.halo_count())
        dev = getattr(backend, "device", "cpu")
        self._send = torch.zeros((2, n), dtype=torch.float32, device=dev)
        self._recv = torch.zeros((2, n), dtype=torch.float32, device=dev)
        self._flags_device = dev
        self.last_steps = 0

    def _exchange(self):
        dist = self.dist
        lo, hi = neighbours(self.rank, self.world)
        if self.world == 1:
            return self._send[0], self._send[1]
        to = lambda r: dist.get_global_rank(self.group, r) if self.group is not None else r
        ops = [dist.P2POp(dist.isend, self._send[0], to(hi), self.group),
               dist.P2POp(dist.irecv, self._recv[0], to(lo), self.group),
               dist.P2POp(dist.isend, self._send[1], to(lo), self.group),
               dist.P2POp(dist.irecv, self._recv[1], to(hi), self.group)]
        for req in dist.batch_isend_irecv(ops):
            req.wait()
        return self._recv[0], self._recv[1]

    def step_once(self):
        """One step: pack, exchange, unpack, CFL minimum over the ranks, stages."""
        self.b.pack(self._send[0], self._send[1])
        recv_inc, recv_dec = self._exchange()
        self.b.unpack(recv_inc, recv_dec)
        self.dist.all_reduce(self.b.cfl_slot(), op=self.dist.ReduceOp.MIN, group=self.group)
        self.b.stages()

    def proceed(self, goal_time, wallclock_time_limit=-1.0, max_steps=0) -> bool:
        """MHDSolver::proceed on every rank together: True when the goal time
        was reached, False on the wallclock limit (any rank's) or after
        ``max_steps``; an error on any rank raises on every rank."""
        import torch
        dist = self.dist
        t0 = _time.monotonic()
        self.b.begin(goal_time)
        _, _, gen0, _ = self.b.poll()
        left = max_steps if max_steps > 0 else -1
        reached = False
        while True:
            k = BATCH if left < 0 else min(BATCH, left)
            if k == 0:
                break
            for _ in range(k):
                self.step_once()
            if left > 0:
                left -= k
            done, err, gen, _ = self.b.poll()
            timeout = wallclock_time_limit > 0 and _time.monotonic() - t0 > wallclock_time_limit
            flags = torch.tensor([int(done), int(err is not None), int(timeout)], dtype=torch.int32,
                                 device=self._flags_device)
            dist.all_reduce(flags, op=dist.ReduceOp.MAX, group=self.group)
            f = flags.tolist()
            self.last_steps = gen - gen0
            if f[1]:
                raise err if err is not None else RuntimeError("a slab on another rank failed")
            if f[0]:
                reached = True
                break
            if f[2]:
                break
        return reached
