"""CPU checks of the drop-in boundary: libnmhd.so loads and exports exactly the
entry points include/nmhd.h declares; host-side config and problem setup."""
import ctypes
import os
import re

import numpy as np
import pytest

from nmhd_b200 import _lib
from nmhd_b200.config import NmhdConfig, SolverConfig
from nmhd_b200.problems import orszag_tang_3d, shearing_box

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    text = open(os.path.join(ROOT, "include", "nmhd.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(nmhd_[a-z_0-9]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    if not os.path.exists(_lib.LIB_PATH):
        _lib.build()
    L = ctypes.CDLL(_lib.LIB_PATH)
    syms = header_symbols()
    assert len(syms) >= 15
    for name in syms:
        assert hasattr(L, name), f"libnmhd.so does not export {name}"
    assert sorted(_lib.EXPORTS) == syms, "Python binding and header disagree"


def test_version_string():
    assert b"sm_100a" in _lib.lib().nmhd_version()


def test_create_rejects_bad_config_without_touching_the_gpu():
    L = _lib.lib()
    bad = SolverConfig(size_x=0, size_y=4, size_z=4).to_ctypes()
    h = ctypes.c_void_p()
    assert L.nmhd_create(ctypes.byref(bad), ctypes.byref(h)) == -1
    assert b"sizes" in L.nmhd_last_error(None)
    bad = SolverConfig(size_x=8, size_y=10, size_z=4, margin_y=4).to_ctypes()
    assert L.nmhd_create(ctypes.byref(bad), ctypes.byref(h)) == -1


def test_config_struct_layout_matches_header(tmp_path):
    """Size and every field offset of nmhd_config as the C compiler lays it
    out from include/nmhd.h, against the ctypes mirror."""
    import subprocess
    names = [f[0] for f in NmhdConfig._fields_]
    src = tmp_path / "layout.c"
    src.write_text("#include <stdio.h>\n#include <stddef.h>\n#include \"nmhd.h\"\nint main(void) {\n"
                   '  printf("%zu\\n", sizeof(nmhd_config));\n'
                   + "".join('  printf("%%zu\\n", offsetof(nmhd_config, %s));\n' % n for n in names)
                   + "  return 0;\n}\n")
    exe = tmp_path / "layout"
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    subprocess.run(["gcc", "-I" + os.path.join(root, "include"), str(src), "-o", str(exe)], check=True)
    got = [int(v) for v in subprocess.run([str(exe)], check=True, capture_output=True,
                                          text=True).stdout.split()]
    assert got[0] == ctypes.sizeof(NmhdConfig)
    assert got[1:] == [getattr(NmhdConfig, n).offset for n in names]


def test_derived_constants_follow_reference_float_chains():
    cfg, _ = shearing_box()
    d = cfg.derived()
    assert d["dy"] == np.float32(1.0 / 128)          # 1.0625 / 136
    assert d["dx"] == np.float32(4.0 / 256)
    assert d["extent_y"] == np.float32(1.0625)
    assert d["relative_velocity"] == -1.5
    c48 = SolverConfig(size_x=48, size_y=28, size_z=12, margin_y=4, extent_x=2.0)
    dd = c48.derived()
    f = np.float32
    assert dd["dx"] == f(f(f(f(2.0) / f(48)) * f(48)) / f(48))


def test_shearing_box_background_is_reference_equilibrium():
    cfg, s = shearing_box(n_radial=16, n_azimuthal=32, n_vertical=8, noise=0.0)
    d = cfg.derived()
    y = np.arange(cfg.size_y, dtype=np.float32)
    ly = np.float32(d["corner_y"]) + np.float32(d["dy"]) * (y + np.float32(0.5))
    assert np.array_equal(s[1, 0, :, 0], (np.float32(-1.5) * np.float32(1.0)) * ly)
    assert np.all(s[2:4] == 0) and np.all(s[5:7] == 0)
    assert np.allclose(s[7], np.sqrt(2.0 / 400.0))


def test_orszag_tang_face_field_is_divergence_free():
    cfg, s = orszag_tang_3d(32)
    bx, by = s[5].astype(np.float64), s[6].astype(np.float64)
    div = (np.roll(bx, -1, axis=2) - bx) * 32 + (np.roll(by, -1, axis=1) - by) * 32
    assert np.max(np.abs(div)) < 1e-4


def test_cpp_mirror_compiles_and_links(tmp_path):
    """include/nmhd.hpp (MHDSolver, Batch, checkpoint) compiles as C++17 and
    links against libnmhd.so (nothing runs)."""
    import subprocess
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    src = tmp_path / "m.cpp"
    src.write_text('#include "nmhd.hpp"\n'
                   'int main() { std::vector<nmhd_config> b(1); '
                   'if (b.size() == 7) { nmhd::Batch x(b); nmhd::MHDSolver y(b[0]); x.autotune(); y.proceed(1.f); '
                   'x.initialize_states(x.states()); x.set_schedule(4, false, true); x.prepare(16); '
                   'y.set_kernel(5); y.prepare(16); if (y.autotune(2).size() > 0 && y.kernel_variant() < 0) return 1; } '
                   'return 0; }\n')
    lib = os.path.join(root, "nmhd_b200")
    subprocess.run(["g++", "-std=c++17", "-Wall", "-Werror", "-I" + os.path.join(root, "include"), str(src),
                    "-L" + lib, "-lnmhd", "-Wl,-rpath," + lib, "-o", str(tmp_path / "m")], check=True)


@pytest.mark.parametrize("change,code,text", [
    (dict(size_y=0), -1, b"sizes"),
    (dict(size_x=2048, size_y=1024, size_z=1024), -1, b"too large"),
    (dict(margin_y=-1), -1, b"margins"),
    (dict(size_y=10, margin_y=4), -1, b"interior Y rows"),
    (dict(size_z=5, margin_z=2), -1, b"interior Z planes"),
    (dict(extent_y=0.0), -1, b"extents"),
    (dict(gamma=1.0), -1, b"gamma"),
    (dict(cfl=0.0), -1, b"cfl"),
    (dict(raw_problem=7), -1, b"unknown problem"),
    (dict(space_order=3), -1, b"space_order"),
    (dict(time_order=0), -1, b"time_order"),
    (dict(parallel_size_y=-1), -1, b"parallel_size_y"),
    (dict(flags=4), -1, b"unknown flags"),
    (dict(flags=1, parallel_size_y=2), -7, b"whole boxes"),
    (dict(parallel_size_y=2, margin_y=0, size_y=16), -1, b"margin_y >= 1"),
])
def test_create_validates_every_config_rule_on_cpu(change, code, text):
    """nmhd_create refuses each invalid configuration with its status and a
    message before any device work (the reference's compile-time config has
    no such checks; these are the runtime config's rules)."""
    L = _lib.lib()
    base = dict(size_x=16, size_y=16 + 8, size_z=8, margin_y=4, extent_x=2.0)
    change = dict(change)
    raw = change.pop("raw_problem", None)
    c = SolverConfig(**{**base, **change}).to_ctypes()
    if raw is not None:
        c.problem = raw
    h = ctypes.c_void_p()
    assert L.nmhd_create(ctypes.byref(c), ctypes.byref(h)) == code
    assert text in L.nmhd_last_error(None), L.nmhd_last_error(None)
    assert not h.value


@pytest.mark.parametrize("change,text", [
    (dict(extent_x=0.0), b"extents"),
    (dict(extent_z=-1.0), b"extents"),
    (dict(parallel_size_y=-1), b"parallel_size_y"),
    (dict(parallel_size_y=2), b"whole box"),
    (dict(flags=1), b"whole box"),
    (dict(gamma=0.5), b"gamma"),
    (dict(size_x=65, size_y=72, size_z=64), b"at most 262144"),
])
def test_noalloc_validates_like_create_on_cpu(change, text):
    """nmhd_advance_noalloc checks nmhd_create's configuration rules (the
    same validator) plus its whole-box rules and size limit before any device
    work; the state pointers are never dereferenced on this path."""
    L = _lib.lib()
    base = dict(size_x=16, size_y=16 + 8, size_z=8, margin_y=4, extent_x=2.0)
    c = SolverConfig(**{**base, **change}).to_ctypes()
    t, g, done = ctypes.c_double(0.0), ctypes.c_int64(0), ctypes.c_int64(0)
    code = L.nmhd_advance_noalloc(ctypes.byref(c), ctypes.c_void_p(0x1000), ctypes.c_void_p(0x2000),
                                  ctypes.byref(t), ctypes.byref(g), 1.0, 1, ctypes.byref(done), None)
    assert code in (-1, -7)
    assert text in L.nmhd_noalloc_last_error(), L.nmhd_noalloc_last_error()


def test_batch_create_validates_like_create_on_cpu():
    """nmhd_batch_create applies nmhd_create's rules to every box (extents
    included) before any device work."""
    L = _lib.lib()
    good = SolverConfig(size_x=16, size_y=24, size_z=8, margin_y=4, extent_x=2.0, problem="shearing_box")
    bad = SolverConfig(size_x=16, size_y=24, size_z=8, margin_y=4, extent_x=2.0, extent_y=0.0,
                       problem="shearing_box")
    arr = (NmhdConfig * 2)(good.to_ctypes(), bad.to_ctypes())
    h = ctypes.c_void_p()
    assert L.nmhd_batch_create(arr, 2, ctypes.byref(h)) == -1
    assert b"box 1" in L.nmhd_batch_last_error(None) and b"extents" in L.nmhd_batch_last_error(None)
    assert not h.value
