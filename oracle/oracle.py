"""ctypes front end of the oracle (TEST INFRASTRUCTURE ONLY).

Loads ``oracle/liboracle.so`` (this repository's C restatement of the
reference time step, mhd_oracle.c) and runs the host-compiled reference
binaries in ``oracle/_ref`` (built by ``make -C oracle ref`` where the
reference sources are present).  Only tests/, ``__graft_entry__.smoke()`` and
bench.py's CPU-baseline leg use this module, as the correctness reference or
the timed CPU baseline.
"""
from __future__ import annotations

import ctypes
import json
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")

_lib = None


def build():
    """Compile liboracle.so (gcc only; works on any box with this image)."""
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
        f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
        for suf, rp in (("f32", f32p), ("f64", f64p)):
            fn = getattr(L, "oracle_proceed_" + suf)
            fn.restype = ctypes.c_int
            fn.argtypes = [ctypes.c_void_p, rp, ctypes.POINTER(ctypes.c_double),
                           ctypes.POINTER(ctypes.c_int64), ctypes.c_double, ctypes.c_int,
                           ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)]
            fn = getattr(L, "oracle_shear_fill_" + suf)
            fn.restype = None
            fn.argtypes = [ctypes.c_void_p, rp, ctypes.c_double]
            fn = getattr(L, "oracle_halo_pack_" + suf)
            fn.restype = None
            fn.argtypes = [ctypes.c_void_p, rp, ctypes.c_double, rp, rp]
            fn = getattr(L, "oracle_halo_unpack_" + suf)
            fn.restype = None
            fn.argtypes = [ctypes.c_void_p, rp, rp, rp]
            fn = getattr(L, "oracle_stages_" + suf)
            fn.restype = None
            fn.argtypes = [ctypes.c_void_p, rp, ctypes.c_float if suf == "f32" else ctypes.c_double]
        L.oracle_hlld_f32.restype = None
        L.oracle_hlld_f32.argtypes = [ctypes.c_float, ctypes.c_float, f32p, f32p]
        L.oracle_hlld_f64.restype = None
        L.oracle_hlld_f64.argtypes = [ctypes.c_double, ctypes.c_double, f64p, f64p]
        L.oracle_cfl_f32.restype = ctypes.c_float
        L.oracle_cfl_f32.argtypes = [ctypes.c_void_p, f32p, ctypes.c_float]
        L.oracle_cfl_f64.restype = ctypes.c_double
        L.oracle_cfl_f64.argtypes = [ctypes.c_void_p, f64p, ctypes.c_double]
        _lib = L
    return _lib


def proceed(cfg, state, steps, goal_time=1.0e30, time=0.0, generation=0, dtype=np.float32):
    """Advance ``state`` (8, Sz, Sy, Sx) by ``steps`` steps; returns a dict with
    the new state, times (steps+1), dts, time, generation, goal_reached."""
    suf = "f32" if dtype == np.float32 else "f64"
    st = np.ascontiguousarray(state, dtype=dtype).copy()
    c = cfg.to_ctypes()
    t = ctypes.c_double(time)
    g = ctypes.c_int64(generation)
    times = np.zeros(steps + 1, np.float64)
    dts = np.zeros(max(steps, 1), dtype)
    reached = ctypes.c_int(0)
    n = getattr(lib(), "oracle_proceed_" + suf)(
        ctypes.byref(c), st, ctypes.byref(t), ctypes.byref(g), goal_time, steps,
        times.ctypes.data, dts.ctypes.data, ctypes.byref(reached))
    return {"state": st, "steps": n, "times": times[:n + 1], "dts": dts[:n], "time": t.value,
            "generation": g.value, "goal_reached": bool(reached.value)}


def hlld(gamma, bx, lr, dtype=np.float32):
    suf = "f32" if dtype == np.float32 else "f64"
    out = np.zeros(7, dtype)
    getattr(lib(), "oracle_hlld_" + suf)(gamma, bx, np.ascontiguousarray(lr, dtype), out)
    return out


def cfl(cfg, state, goal=1.0e30):
    c = cfg.to_ctypes()
    return float(lib().oracle_cfl_f32(ctypes.byref(c), np.ascontiguousarray(state, np.float32), goal))


def shear_fill(cfg, state, time, dtype=np.float32):
    suf = "f32" if dtype == np.float32 else "f64"
    st = np.ascontiguousarray(state, dtype=dtype).copy()
    c = cfg.to_ctypes()
    getattr(lib(), "oracle_shear_fill_" + suf)(ctypes.byref(c), st, time)
    return st


def halo_count(cfg):
    """Values in one Y-halo message: 8 fields x Sx x margin_y x Sz."""
    return 8 * cfg.size_x * cfg.margin_y * cfg.size_z


def halo_pack(cfg, state, time, dtype=np.float32):
    """The two outgoing Y messages of a radial slab at ``time``: (to the rank
    above, to the rank below)."""
    suf = "f32" if dtype == np.float32 else "f64"
    st = np.ascontiguousarray(state, dtype=dtype)
    inc = np.zeros(max(1, halo_count(cfg)), dtype)
    dec = np.zeros_like(inc)
    c = cfg.to_ctypes()
    getattr(lib(), "oracle_halo_pack_" + suf)(ctypes.byref(c), st, time, inc, dec)
    return inc, dec


def halo_unpack(cfg, state, recv_inc, recv_dec, dtype=np.float32):
    """Scatter the received messages into the Y margins and copy the Z
    margins, in place (``state`` must be C-contiguous of ``dtype``)."""
    suf = "f32" if dtype == np.float32 else "f64"
    c = cfg.to_ctypes()
    getattr(lib(), "oracle_halo_unpack_" + suf)(ctypes.byref(c), state, np.ascontiguousarray(recv_inc, dtype),
                                                np.ascontiguousarray(recv_dec, dtype))


def stages(cfg, state, dt, dtype=np.float32):
    """The RK stages of one step with time step ``dt``, in place."""
    suf = "f32" if dtype == np.float32 else "f64"
    c = cfg.to_ctypes()
    getattr(lib(), "oracle_stages_" + suf)(ctypes.byref(c), state, dt)


def ref_binary(name):
    """Path of a host-compiled reference binary, or None when not built."""
    p = os.path.join(REF_DIR, "ref_" + name)
    return p if os.path.exists(p) else None


def run_ref(name, state, steps, goal_time=1.0e30, threads=None, dtype=np.float32, ckpt_dir=None,
            load_tag=None, save_tag=None):
    """Run the reference binary ``name`` on ``state`` until generation
    ``steps``; returns (state, times, info).  With ``ckpt_dir``, the run starts
    from the reference's own load_state(load_tag) (``state`` is then unused)
    and/or ends with save_state(save_tag), under ckpt_dir/<tag>/0000."""
    from nmhd_b200.binio import read_bin, write_bin
    exe = ref_binary(name)
    if exe is None:
        raise FileNotFoundError(f"reference binary ref_{name} is not built")
    env = dict(os.environ)
    if threads:
        env["OMP_NUM_THREADS"] = str(threads)
    if ckpt_dir:
        env["NMHD_REF_DIR"] = str(ckpt_dir)
        if load_tag:
            env["NMHD_REF_LOAD"] = load_tag
        if save_tag:
            env["NMHD_REF_SAVE"] = save_tag
    with tempfile.TemporaryDirectory() as d:
        fin, fout, ftimes = (os.path.join(d, x) for x in ("in.bin", "out.bin", "t.txt"))
        write_bin(fin, state, dtype=dtype)
        r = subprocess.run([exe, fin, fout, str(steps), repr(float(goal_time)), ftimes],
                           check=True, capture_output=True, text=True, env=env)
        info = json.loads(r.stdout.strip().splitlines()[-1])
        out = read_bin(fout, dtype=dtype)
        times = np.loadtxt(ftimes, ndmin=1)
    return out, times, info


def run_ref_slabs(name, states, steps, goal_time=1.0e30, threads=1, dtype=np.float32, timeout=600,
                  ckpt_dir=None, save_tag=None):
    """Run the reference binary ``name`` (built with NMHD_REF_PY = len(states)
    ranks along Y) as one process per rank, rank r starting from
    ``states[r]`` (its radial slab, margins included), until generation
    ``steps``.  The ranks exchange their halos and reduce dt through the
    file mailbox of refshim/mpi.h.  With ``ckpt_dir`` and ``save_tag`` every
    rank ends with save_state(save_tag) under ckpt_dir/<tag>/.  Returns
    (per-rank states, times of rank 0, per-rank infos)."""
    from nmhd_b200.binio import read_bin, write_bin
    exe = ref_binary(name)
    if exe is None:
        raise FileNotFoundError(f"reference binary ref_{name} is not built")
    n = len(states)
    with tempfile.TemporaryDirectory() as d:
        box = os.path.join(d, "mailbox")
        logs = str(ckpt_dir) if ckpt_dir else os.path.join(d, "logs")
        os.makedirs(box)
        os.makedirs(logs, exist_ok=True)
        for r, s in enumerate(states):
            write_bin(os.path.join(d, "in%04d.bin" % r), s, dtype=dtype)
        procs = []
        for r in range(n):
            env = dict(os.environ, NMHD_REF_RANK=str(r), NMHD_REF_NRANKS=str(n), NMHD_REF_MAILBOX=box,
                       NMHD_REF_DIR=logs, NMHD_REF_MPI_TIMEOUT=str(timeout), OMP_NUM_THREADS=str(threads))
            if save_tag:
                env["NMHD_REF_SAVE"] = save_tag
            procs.append(subprocess.Popen(
                [exe, os.path.join(d, "in%04d.bin"), os.path.join(d, "out%04d.bin"), str(steps),
                 repr(float(goal_time)), os.path.join(d, "t%04d.txt")],
                stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True, env=env))
        outs = []
        for p in procs:
            try:
                o, e = p.communicate(timeout=timeout + 60)
            except subprocess.TimeoutExpired:
                for q in procs:
                    q.kill()
                raise
            outs.append((p.returncode, o, e))
        for r, (rc, o, e) in enumerate(outs):
            if rc != 0:
                raise RuntimeError(f"reference rank {r} exited {rc}: {e.strip()[-400:]}")
        infos = [json.loads(o.strip().splitlines()[-1]) for _, o, _ in outs]
        res = [read_bin(os.path.join(d, "out%04d.bin" % r), dtype=dtype) for r in range(n)]
        times = np.loadtxt(os.path.join(d, "t0000.txt"), ndmin=1)
    return res, times, infos
