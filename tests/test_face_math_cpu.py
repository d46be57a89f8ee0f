"""CPU checks of the single-box kernels' face arithmetic (nmhd_b200/csrc/
mhd_math.cuh), compiled for the host (tests/native/libcellcheck.so): the HLLD
flux and the minbee reconstruction are bitwise the oracle's, which is pinned
to the reference's own hlld.inl and interpolate() (src/library/hlld.inl:7-284,
src/library/mhd_solver.inlrb:137-155).

The kernels compute the single-star state only for the side(s) the fan
region's formula reads (none in regions 0 and 5, the upwind side in 1 and 4,
both sides' transverse parts in 2 and 3) with the reference's operations;
these tests cover every region, Bx = 0 and both signs of Bx, with the exact
float bit patterns compared.

Tolerance: bitwise (every float of every output)."""
import ctypes
import os
import subprocess

import numpy as np

import adcheck
from oracle import oracle

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "native", "libcellcheck.so")
GAMMA = np.float32(5.0 / 3.0)
_lib = None


def lib():
    global _lib
    if _lib is None:
        # make rebuilds the library when mhd_math.cuh changed
        subprocess.run(["make", "-s", "-C", os.path.join(HERE, "native")], check=True)
        L = ctypes.CDLL(LIB)
        P = ctypes.c_void_p
        L.cellh_hlld_many_f32.argtypes = [ctypes.c_float, P, P, P, ctypes.c_long]
        L.cellh_reconstruct_f32.argtypes = [P, P, ctypes.c_long]
        _lib = L
    return _lib


def riemann_inputs(rng, n):
    """(bx, lr) float32 inputs over all six fan regions: subsonic states,
    supersonic flows both ways, Bx = 0, strong and weak fields, equal states."""
    lr = np.empty((n, 14), np.float32)
    lr[:, 0:2] = rng.uniform(0.3, 2.0, (n, 2))
    lr[:, 2:8] = rng.normal(0.0, 1.0, (n, 6))
    sup = np.arange(n) % 7 == 0
    lr[sup, 2:4] += rng.choice([-4.0, 4.0], (sup.sum(), 1))
    lr[:, 8:10] = rng.uniform(0.2, 2.0, (n, 2))
    lr[:, 10:14] = rng.normal(0.0, 1.0, (n, 4)) * rng.choice([1e-3, 1.0, 3.0], (n, 1))
    eq = np.arange(n) % 11 == 0
    lr[eq, 1::2] = lr[eq, 0::2]
    bx = rng.normal(0.0, 1.0, n).astype(np.float32) * rng.choice([1e-2, 1.0, 4.0], n).astype(np.float32)
    bx[np.arange(n) % 5 == 0] = 0.0
    return bx, np.ascontiguousarray(lr)


def test_device_hlld_is_bitwise_the_oracle_in_all_regions():
    rng = np.random.default_rng(11)
    n = 6000
    bx, lr = riemann_inputs(rng, n)
    out = np.empty((n, 7), np.float32)
    lib().cellh_hlld_many_f32(GAMMA, bx.ctypes.data, lr.ctypes.data, out.ctypes.data, n)
    regions = np.zeros(6, int)
    for i in range(n):
        ref = oracle.hlld(GAMMA, bx[i], lr[i], np.float32)
        assert np.array_equal(out[i].view(np.uint32), ref.view(np.uint32)), (i, bx[i], lr[i], out[i], ref)
        regions[adcheck.hlld_region(float(GAMMA), bx[i], lr[i])] += 1
    assert (regions > 50).all(), regions


def test_device_reconstruction_is_the_minbee_limiter():
    """reconstruct4 against the reference's interpolate() restated in numpy
    (float32 operations): L = x1 + minmod(x1-x0, x2-x1)/2, R = x2 - minmod(x2-x1,
    x3-x2)/2, minmod 0 for products <= 0, else the smaller magnitude (ties: the
    second argument)."""
    rng = np.random.default_rng(3)
    n = 20000
    x = rng.normal(0.0, 1.0, (n, 4)).astype(np.float32)
    x[::9, 2] = x[::9, 1]          # zero slopes
    x[::13, 3] = 2 * x[::13, 2] - x[::13, 1]  # equal slopes (ties)
    lr = np.empty((n, 2), np.float32)
    lib().cellh_reconstruct_f32(np.ascontiguousarray(x).ctypes.data, lr.ctypes.data, n)
    f = np.float32

    def minmod(a, b):
        return np.where(a * b <= f(0), f(0), np.where(np.abs(a) < np.abs(b), a, b)).astype(np.float32)

    d01, d12, d23 = x[:, 1] - x[:, 0], x[:, 2] - x[:, 1], x[:, 3] - x[:, 2]
    left = x[:, 1] + minmod(d01, d12) / f(2)
    right = x[:, 2] - minmod(d12, d23) / f(2)
    assert np.array_equal(lr[:, 0].view(np.uint32), left.view(np.uint32))
    assert np.array_equal(lr[:, 1].view(np.uint32), right.view(np.uint32))
