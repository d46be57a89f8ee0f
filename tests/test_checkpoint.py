"""Checkpoint compatibility with the reference's save_state / load_state
(prefix.bin + prefix_setup.txt, src/library/mhd_solver.inlrb:1023-1050).

- The setup text written here (Python and the C++ header) is the reference's
  own, line for line, plus one extra GlobalSetup member with the exact time.
- The host-compiled reference restarts from a checkpoint written here exactly
  as from its own.
- On the GPU, a reference checkpoint restarts in MHDSolver exactly as in the
  reference, and a checkpoint written here resumes bitwise.
"""
import os
import subprocess

import numpy as np
import pytest

from nmhd_b200 import checkpoint as ck
from nmhd_b200.binio import read_bin, write_bin
from nmhd_b200.problems import orszag_tang_3d, shearing_box
from oracle import oracle

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)

CASES = {  # reference binary -> the box it was built for
    "shear32x16x8": lambda: shearing_box(n_radial=16, n_azimuthal=32, n_vertical=8, l_azimuthal=4.0, seed=3),
    "ot16": lambda: orszag_tang_3d(16),
}


def _need(name):
    if oracle.ref_binary(name) is None:
        pytest.skip(f"reference binary ref_{name} not built")


def _with_exact(ref_text, time):
    """The reference's text with the member written here added."""
    head, tail = ref_text.split("\n\n################", 1)
    lines = head.split("\n")
    lines[0] = str(int(lines[0]) + 1)
    lines.append("current_time_exact %.17g" % time)
    return "\n".join(lines) + "\n\n################" + tail


@pytest.mark.parametrize("name", sorted(CASES))
def test_setup_text_is_the_reference_save_state_text(tmp_path, name):
    _need(name)
    cfg, s = CASES[name]()
    _, _, info = oracle.run_ref(name, s, 5, ckpt_dir=tmp_path, save_tag="c")
    ref = (tmp_path / "c" / "0000_setup.txt").read_text()
    ours = ck.setup_text(cfg, 5, info["time"], output_directory=str(tmp_path))
    assert ours == _with_exact(ref, info["time"])
    assert ck.clock_from_setup(ref) == (5, float("%.6g" % info["time"]))
    assert ck.clock_from_setup(ours) == (5, info["time"])
    assert np.array_equal(read_bin(str(tmp_path / "c" / "0000.bin")), oracle.proceed(cfg, s, 5)["state"])


def test_cpp_header_writes_and_reads_the_same_text(tmp_path):
    src = tmp_path / "ck.cpp"
    src.write_text(r'''
#include "nmhd.hpp"
#include <iostream>
#include <sstream>
int main(int argc, char **argv) {
  nmhd_config c = {};
  c.size_x = 32; c.size_y = 24; c.size_z = 8; c.margin_y = 4;
  c.extent_x = 4; c.extent_y = 1; c.extent_z = 1;
  c.gamma = 5.0f / 3.0f; c.cfl = 0.4f; c.problem = NMHD_PROBLEM_SHEARING_BOX;
  c.q = 1.5f; c.omega = 1.0f; c.space_order = 2; c.time_order = 2;
  const std::string text = nmhd::checkpoint::setup_text(c, 7, 0.1234567890123, "/out dir");
  std::cout << text;
  std::istringstream is(text);
  int g; double t;
  if (!nmhd::checkpoint::clock_from_setup(is, g, t) || g != 7 || t != 0.1234567890123) return 1;
  return 0;
}
''')
    exe = tmp_path / "ck"
    subprocess.run(["g++", "-std=c++17", "-I" + os.path.join(ROOT, "include"), str(src), "-o", str(exe)],
                   check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    cfg, _ = shearing_box(n_radial=16, n_azimuthal=32, n_vertical=8, l_azimuthal=4.0, seed=3)
    assert out == ck.setup_text(cfg, 7, 0.1234567890123, output_directory="/out dir")
    assert "output_directory /out%20dir\n" in out


def test_reference_restarts_from_a_checkpoint_written_here_as_from_its_own(tmp_path):
    name = "shear32x16x8"
    _need(name)
    cfg, s = CASES[name]()
    st5, _, info = oracle.run_ref(name, s, 5, ckpt_dir=tmp_path, save_tag="own")
    os.makedirs(tmp_path / "ours", exist_ok=True)
    write_bin(str(tmp_path / "ours" / "0000.bin"), st5)
    (tmp_path / "ours" / "0000_setup.txt").write_text(
        ck.setup_text(cfg, 5, info["time"], output_directory=str(tmp_path)))
    a, _, ia = oracle.run_ref(name, s, 9, ckpt_dir=tmp_path, load_tag="own")
    b, _, ib = oracle.run_ref(name, s, 9, ckpt_dir=tmp_path, load_tag="ours")
    assert ia["steps"] == ib["steps"] == 9
    assert ia["time"] == ib["time"]
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_load_rejects_unreadable_setup_text():
    with pytest.raises((ValueError, KeyError, IndexError)):
        ck.clock_from_setup("garbage")


@pytest.mark.gpu
def test_reference_checkpoint_restarts_in_the_cuda_solver_as_in_the_reference(gpu, tmp_path):
    name = "shear32x16x8"
    _need(name)
    from nmhd_b200.solver import MHDSolver
    cfg, s = CASES[name]()
    oracle.run_ref(name, s, 5, ckpt_dir=tmp_path, save_tag="c")
    ref9, _, info = oracle.run_ref(name, s, 9, ckpt_dir=tmp_path, load_tag="c", save_tag="r9")
    with MHDSolver(cfg) as sol:
        assert sol.load_state(tmp_path / "c" / "0000")
        assert sol.generation() == 5
        sol.step(4)
        assert sol.current_time() == info["time"]
        assert np.array_equal(sol.get_state().view(np.uint32), ref9.view(np.uint32))
        # the checkpoint MHDSolver writes restarts the reference as its own does
        os.makedirs(tmp_path / "ours", exist_ok=True)
        assert sol.save_state(tmp_path / "ours" / "0000")
    own13, _, i_own = oracle.run_ref(name, s, 13, ckpt_dir=tmp_path, load_tag="r9")
    ours13, _, i_ours = oracle.run_ref(name, s, 13, ckpt_dir=tmp_path, load_tag="ours")
    assert i_own["steps"] == i_ours["steps"] == 13 and i_own["time"] == i_ours["time"]
    assert np.array_equal(own13.view(np.uint32), ours13.view(np.uint32))
