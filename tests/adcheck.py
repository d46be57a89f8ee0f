"""ctypes binding of tests/native/libadcheck.so: the host build of the
differentiated step (ad_*.cuh) used by the CPU tests.  Test infrastructure
only; the library itself never loads it."""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

from nmhd_b200._lib import LOSS_MAXWELL_STRESS, LossSpec

HERE = os.path.dirname(os.path.abspath(__file__))
NATIVE = os.path.join(HERE, "native")
LIB = os.path.join(NATIVE, "libadcheck.so")
_lib = None


def build():
    subprocess.run(["make", "-s", "-C", NATIVE], check=True)


def lib():
    global _lib
    if _lib is None:
        # make rebuilds the library when a product header it compiles changed
        build()
        L = ctypes.CDLL(LIB)
        f32, f64, P = ctypes.c_float, ctypes.c_double, ctypes.c_void_p
        L.adh_hlld_f32.argtypes = [f32, f32, P, P]
        L.adh_hlld_f64.argtypes = [f64, f64, P, P]
        L.adh_hlld_tan.argtypes = [f64, f64, P, f64, P, P, P]
        L.adh_hlld_adj_f64.argtypes = [f64, f64, P, P, P, P]
        L.adh_hlld_adj_f32.argtypes = [f32, f32, P, P, P, P]
        L.adh_hlld_region_f32.argtypes = [f32, f32, P]
        L.adh_hlld_region_f32.restype = ctypes.c_int
        L.adh_forward_f32.argtypes = [P, P, f64, P, ctypes.c_int]
        L.adh_forward_f64.argtypes = [P, P, f64, P, ctypes.c_int]
        L.adh_tlm.argtypes = [P, P, P, f64, P, ctypes.c_int, P, P, P]
        L.adh_adjoint_f64.argtypes = [P, P, f64, P, ctypes.c_int, P, P, P]
        L.adh_adjoint_f32.argtypes = [P, P, f64, P, ctypes.c_int, P, P, P]
        _lib = L
    return _lib


def _ptr(a):
    return a.ctypes.data


def hlld(gamma, bx, lr, dtype=np.float64):
    lr = np.ascontiguousarray(lr, dtype)
    out = np.zeros(7, dtype)
    fn = lib().adh_hlld_f32 if dtype == np.float32 else lib().adh_hlld_f64
    fn(gamma, bx, _ptr(lr), _ptr(out))
    return out


def hlld_region(gamma, bx, lr):
    lr = np.ascontiguousarray(lr, np.float32)
    return lib().adh_hlld_region_f32(gamma, bx, _ptr(lr))


def hlld_tangent(gamma, bx, lr, dbx, dlr):
    lr = np.ascontiguousarray(lr, np.float64)
    dlr = np.ascontiguousarray(dlr, np.float64)
    out = np.zeros(7)
    dout = np.zeros(7)
    lib().adh_hlld_tan(gamma, bx, _ptr(lr), dbx, _ptr(dlr), _ptr(out), _ptr(dout))
    return out, dout


def hlld_adjoint(gamma, bx, lr, lf, dtype=np.float64):
    lr = np.ascontiguousarray(lr, dtype)
    lf = np.ascontiguousarray(lf, dtype)
    lin = np.zeros(14, dtype)
    lbx = np.zeros(1, dtype)
    fn = lib().adh_hlld_adj_f32 if dtype == np.float32 else lib().adh_hlld_adj_f64
    fn(gamma, bx, _ptr(lr), _ptr(lf), _ptr(lin), _ptr(lbx))
    return lin, float(lbx[0])


def forward(cfg, state, dts, time=0.0, dtype=np.float32):
    st = np.ascontiguousarray(state, dtype).copy()
    d = np.ascontiguousarray(dts, dtype)
    c = cfg.to_ctypes()
    fn = lib().adh_forward_f32 if dtype == np.float32 else lib().adh_forward_f64
    fn(ctypes.byref(c), _ptr(st), time, _ptr(d), len(d))
    return st


def loss_spec(first, last):
    return LossSpec(LOSS_MAXWELL_STRESS, first, last, 0)


def tlm(cfg, state, direction, dts, first, last, time=0.0):
    st = np.ascontiguousarray(state, np.float64)
    dr = None if direction is None else np.ascontiguousarray(direction, np.float64)
    d = np.ascontiguousarray(dts, np.float64)
    c = cfg.to_ctypes()
    spec = loss_spec(first, last)
    loss = ctypes.c_double()
    dloss = ctypes.c_double()
    lib().adh_tlm(ctypes.byref(c), _ptr(st), None if dr is None else _ptr(dr), time, _ptr(d), len(d),
                  ctypes.byref(spec), ctypes.byref(loss), ctypes.byref(dloss))
    return loss.value, dloss.value


def adjoint(cfg, state, dts, first, last, time=0.0, dtype=np.float64):
    st = np.ascontiguousarray(state, dtype)
    d = np.ascontiguousarray(dts, dtype)
    grad = np.zeros_like(st)
    c = cfg.to_ctypes()
    spec = loss_spec(first, last)
    loss = ctypes.c_double()
    fn = lib().adh_adjoint_f32 if dtype == np.float32 else lib().adh_adjoint_f64
    fn(ctypes.byref(c), _ptr(st), time, _ptr(d), len(d), ctypes.byref(spec), ctypes.byref(loss), _ptr(grad))
    return loss.value, grad
