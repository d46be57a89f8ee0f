"""Loader for libnmhd.so (the C ABI declared in include/nmhd.h).

The compute path exists only as this CUDA library: there is no CPU fallback.
If the library is missing or cannot load, :func:`lib` raises.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libnmhd.so")

# nmhd_status codes
OK = 0
GOAL_REACHED = 1
TIMEOUT = 2
STEP_LIMIT = 3
ERRORS = {
    -1: "invalid argument", -2: "CUDA error", -3: "I/O error", -4: "size mismatch",
    -5: "numerical error", -6: "out of device memory", -7: "not supported",
}



class LossSpec(ctypes.Structure):
    """nmhd_loss_spec: J = mean over states first_step..last_step of the
    volume-averaged Maxwell stress -<Bx By>."""
    _fields_ = [("kind", ctypes.c_int32), ("first_step", ctypes.c_int32),
                ("last_step", ctypes.c_int32), ("reserved", ctypes.c_int32)]


LOSS_MAXWELL_STRESS = 1
ADJOINT_MAX_STEPS = 4096

# Every entry point declared in include/nmhd.h: (name, restype, argtypes)
_P = ctypes.c_void_p
_SIGS = [
    ("nmhd_version", ctypes.c_char_p, []),
    ("nmhd_create", ctypes.c_int, [_P, ctypes.POINTER(_P)]),
    ("nmhd_destroy", None, [_P]),
    ("nmhd_set_state", ctypes.c_int, [_P, ctypes.POINTER(_P), ctypes.c_int]),
    ("nmhd_get_state", ctypes.c_int, [_P, ctypes.POINTER(_P), ctypes.c_int]),
    ("nmhd_read", ctypes.c_int, [_P, ctypes.c_char_p]),
    ("nmhd_write", ctypes.c_int, [_P, ctypes.c_char_p]),
    ("nmhd_proceed", ctypes.c_int, [_P, ctypes.c_double, ctypes.c_double, ctypes.c_int64,
                                    ctypes.POINTER(ctypes.c_int64)]),
    ("nmhd_prepare", ctypes.c_int, [_P, ctypes.c_int64]),
    ("nmhd_current_time", ctypes.c_double, [_P]),
    ("nmhd_generation", ctypes.c_int64, [_P]),
    ("nmhd_set_time", ctypes.c_int, [_P, ctypes.c_double, ctypes.c_int64]),
    ("nmhd_dt_history", ctypes.c_int64, [_P, _P, ctypes.c_int64]),
    ("nmhd_diagnostics", ctypes.c_int, [_P, _P]),
    ("nmhd_device", ctypes.c_int, [_P]),
    ("nmhd_set_stream", ctypes.c_int, [_P, _P]),
    ("nmhd_last_error", ctypes.c_char_p, [_P]),
    ("nmhd_profile", ctypes.c_int, [_P, ctypes.c_int, _P, _P, ctypes.c_int]),
    ("nmhd_kernel_name", ctypes.c_char_p, [ctypes.c_int]),
    ("nmhd_set_kernel", ctypes.c_int, [_P, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    ("nmhd_get_kernel", ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                       ctypes.POINTER(ctypes.c_int)]),
    ("nmhd_autotune", ctypes.c_int, [_P, ctypes.c_int, _P, ctypes.c_int]),
    ("nmhd_advance_noalloc", ctypes.c_int, [_P, _P, _P, ctypes.POINTER(ctypes.c_double),
                                            ctypes.POINTER(ctypes.c_int64), ctypes.c_double,
                                            ctypes.c_int64, ctypes.POINTER(ctypes.c_int64), _P]),
    ("nmhd_noalloc_last_error", ctypes.c_char_p, []),
    ("nmhd_loss_run", ctypes.c_int, [_P, ctypes.c_int32, _P, _P, ctypes.POINTER(ctypes.c_double), _P]),
    ("nmhd_adjoint_run", ctypes.c_int, [_P, ctypes.c_int32, ctypes.c_int32, _P, _P,
                                        ctypes.POINTER(ctypes.c_double), _P, ctypes.POINTER(_P), ctypes.c_int]),
    ("nmhd_adjoint_run_f64", ctypes.c_int, [_P, ctypes.c_int32, ctypes.c_int32, _P, _P,
                                            ctypes.POINTER(ctypes.c_double), ctypes.POINTER(_P)]),
    ("nmhd_tlm_run", ctypes.c_int, [_P, ctypes.c_int32, _P, _P, ctypes.POINTER(_P), ctypes.c_double,
                                    ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]),
    ("nmhd_adjoint_timing", ctypes.c_int, [_P, _P]),
    ("nmhd_adjoint_set_tape_budget", ctypes.c_int, [_P, ctypes.c_int64]),
    ("nmhd_adjoint_kept_segments", ctypes.c_int32, [_P]),
    ("nmhd_batch_create", ctypes.c_int, [_P, ctypes.c_int, ctypes.POINTER(_P)]),
    ("nmhd_batch_destroy", None, [_P]),
    ("nmhd_batch_size", ctypes.c_int, [_P]),
    ("nmhd_batch_set_state", ctypes.c_int, [_P, ctypes.c_int, ctypes.POINTER(_P), ctypes.c_int]),
    ("nmhd_batch_get_state", ctypes.c_int, [_P, ctypes.c_int, ctypes.POINTER(_P), ctypes.c_int]),
    ("nmhd_batch_set_states", ctypes.c_int, [_P, ctypes.POINTER(_P), ctypes.c_int]),
    ("nmhd_batch_get_states", ctypes.c_int, [_P, ctypes.POINTER(_P), ctypes.c_int]),
    ("nmhd_batch_clock", ctypes.c_int, [_P, ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                        ctypes.POINTER(ctypes.c_int64)]),
    ("nmhd_batch_proceed", ctypes.c_int, [_P, ctypes.c_double, ctypes.c_int64,
                                          ctypes.POINTER(ctypes.c_int64)]),
    ("nmhd_batch_prepare", ctypes.c_int, [_P, ctypes.c_int64]),
    ("nmhd_batch_set_schedule", ctypes.c_int, [_P, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    ("nmhd_batch_set_stream", ctypes.c_int, [_P, _P]),
    ("nmhd_batch_launches_per_step", ctypes.c_int, [_P]),
    ("nmhd_batch_tile_rule", ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                            ctypes.POINTER(ctypes.c_int)]),
    ("nmhd_batch_tile_shape", ctypes.c_int, [_P, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                             ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]),
    ("nmhd_batch_autotune", ctypes.c_int, [_P, ctypes.c_int, _P, ctypes.c_int]),
    ("nmhd_batch_last_error", ctypes.c_char_p, [_P]),
    ("nmhd_halo_count", ctypes.c_int64, [_P]),
    ("nmhd_slab_begin", ctypes.c_int, [_P, ctypes.c_double]),
    ("nmhd_halo_pack", ctypes.c_int, [_P, _P, _P]),
    ("nmhd_halo_unpack", ctypes.c_int, [_P, _P, _P]),
    ("nmhd_cfl_slot", _P, [_P]),
    ("nmhd_cfl_min", ctypes.c_int, [ctypes.POINTER(_P), ctypes.c_int]),
    ("nmhd_step_stages", ctypes.c_int, [_P]),
    ("nmhd_slab_poll", ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_double)]),
]
EXPORTS = [s[0] for s in _SIGS]

_lib = None


def build(verbose=False):
    """Compile libnmhd.so for sm_100a (nvcc cross-compiles without a GPU)."""
    subprocess.run(["make", "-s" if not verbose else "-w", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is not built; run nmhd_b200._lib.build()")
        L = ctypes.CDLL(LIB_PATH)
        for name, res, args in _SIGS:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


class NmhdError(RuntimeError):
    def __init__(self, code, message):
        super().__init__(f"{ERRORS.get(code, code)}: {message}")
        self.code = code
