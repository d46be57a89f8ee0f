"""A C++ host program drives the library through include/nmhd.hpp, the way a
reference application drives MHDSolver (read a .bin, proceed with a
monitor, write a .bin): its result equals the Python front end's, bitwise,
and its monitor is called before every step."""
import os
import subprocess

import numpy as np
import pytest

from nmhd_b200.binio import read_bin, write_bin
from nmhd_b200.problems import shearing_box
from nmhd_b200.solver import MHDSolver

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SRC = r'''
#include "nmhd.hpp"
#include <cstdio>
#include <cstdlib>
#include <vector>
int main(int argc, char **argv) {
  nmhd_config c = {};
  c.size_x = 32; c.size_y = 16 + 8; c.size_z = 8; c.margin_y = 4;
  c.extent_x = 4; c.extent_y = 1; c.extent_z = 1;
  c.gamma = 5.0f / 3.0f; c.cfl = 0.4f; c.problem = NMHD_PROBLEM_SHEARING_BOX;
  c.q = 1.5f; c.omega = 1.0f; c.space_order = 2; c.time_order = 2;
  const int stop = std::atoi(argv[3]);
  nmhd::MHDSolver solver(c);
  if (argc > 4) {  // a kernel variant other than the default
    solver.set_kernel(std::atoi(argv[4]));
    if (solver.kernel_variant() != std::atoi(argv[4])) return 6;
  }
  if (!solver.read(argv[1])) return 3;
  std::vector<int> seen;
  solver.set_monitor([&](nmhd::MHDSolver &s) {
    seen.push_back(s.generation());
    return s.generation() >= stop ? 1 : 0;
  });
  const bool reached = solver.proceed(1e30f);
  if (!solver.write(argv[2])) return 4;
  std::printf("%d %d %zu\n", reached ? 1 : 0, solver.generation(), seen.size());
  for (size_t i = 0; i < seen.size(); ++i)
    if (seen[i] != (int)i) return 5;
  return 0;
}
'''


@pytest.mark.parametrize("variant", [None, 4, 2])
def test_cpp_host_program_matches_python_front_end(gpu, tmp_path, variant):
    src = tmp_path / "app.cpp"
    src.write_text(SRC)
    exe = tmp_path / "app"
    lib = os.path.join(ROOT, "nmhd_b200")
    subprocess.run(["g++", "-std=c++17", "-O2", "-I" + os.path.join(ROOT, "include"), str(src), "-L" + lib,
                    "-lnmhd", "-Wl,-rpath," + lib, "-o", str(exe)], check=True)
    cfg, s = shearing_box(n_radial=16, n_azimuthal=32, n_vertical=8, l_azimuthal=4.0, seed=41)
    write_bin(str(tmp_path / "in.bin"), s)
    r = subprocess.run([str(exe), str(tmp_path / "in.bin"), str(tmp_path / "out.bin"), "9"] +
                       ([str(variant)] if variant is not None else []), capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    reached, gen, calls = (int(v) for v in r.stdout.split())
    assert (reached, gen, calls) == (0, 9, 10)
    with MHDSolver(cfg) as sol:
        sol.set_state(s)
        sol.step(9)
        assert np.array_equal(read_bin(str(tmp_path / "out.bin")), sol.get_state())


BATCH_SRC = r'''
#include "nmhd.hpp"
#include <cstdio>
#include <vector>
// Two boxes of different shapes through nmhd::Batch; states in argv[1] and
// argv[2] (8 fields each, .bin order, no header), results written back.
int main(int argc, char **argv) {
  std::vector<nmhd_config> boxes(2);
  for (int i = 0; i < 2; ++i) {
    nmhd_config &c = boxes[i];
    c = nmhd_config{};
    c.size_x = i ? 48 : 32; c.size_y = 16 + 8; c.size_z = i ? 6 : 8; c.margin_y = 4;
    c.extent_x = i ? 3 : 2; c.extent_y = 1; c.extent_z = 1;
    c.gamma = 5.0f / 3.0f; c.cfl = 0.4f; c.problem = NMHD_PROBLEM_SHEARING_BOX;
    c.q = 1.5f; c.omega = 1.0f; c.space_order = 2; c.time_order = 2;
  }
  nmhd::Batch batch(boxes);
  for (int i = 0; i < 2; ++i) {
    std::vector<float> s(8 * batch.cells(i));
    FILE *fp = std::fopen(argv[1 + i], "rb");
    if (!fp || std::fread(s.data(), 4, s.size(), fp) != s.size()) return 3;
    std::fclose(fp);
    batch.initialize_state(i, s);
  }
  batch.autotune(2);
  if (argc > 3) {  // the staged flux and fused update passes pinned, graphs built first
    batch.set_schedule(0, false, true);
    batch.set_schedule(4, false, true);
    batch.set_schedule(3, true, true);
    batch.prepare(7);
  }
  const bool reached = batch.proceed(1e30f, 7);
  const std::vector<std::vector<float>> all = batch.states();
  for (int i = 0; i < 2; ++i) {
    const std::vector<float> s = batch.state(i);
    if (s != all[i]) return 5;
    FILE *fp = std::fopen(argv[1 + i], "wb");
    if (!fp || std::fwrite(s.data(), 4, s.size(), fp) != s.size()) return 4;
    std::fclose(fp);
  }
  std::printf("%d %d %d %lld\n", reached ? 1 : 0, batch.generation(0), batch.generation(1), batch.last_steps());
  return 0;
}
'''


@pytest.mark.parametrize("pinned", [False, True])
def test_cpp_batch_program_matches_single_box_runs(gpu, tmp_path, pinned):
    """nmhd::Batch (include/nmhd.hpp) advances two boxes of different shapes
    bitwise as the single-box solver does (autotuned schedules, or the staged
    and fused passes pinned with the graphs prepared first)."""
    src = tmp_path / "batch.cpp"
    src.write_text(BATCH_SRC)
    exe = tmp_path / "batch"
    lib = os.path.join(ROOT, "nmhd_b200")
    subprocess.run(["g++", "-std=c++17", "-O2", "-I" + os.path.join(ROOT, "include"), str(src), "-L" + lib,
                    "-lnmhd", "-Wl,-rpath," + lib, "-o", str(exe)], check=True)
    cases = [shearing_box(n_radial=16, n_azimuthal=32, n_vertical=8, l_azimuthal=2.0, seed=51),
             shearing_box(n_radial=16, n_azimuthal=48, n_vertical=6, l_azimuthal=3.0, seed=52)]
    paths = [tmp_path / f"box{i}.raw" for i in range(2)]
    for (cfg, s), p in zip(cases, paths):
        np.ascontiguousarray(s, dtype=np.float32).tofile(p)
    r = subprocess.run([str(exe)] + [str(p) for p in paths] + (["pinned"] if pinned else []),
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert r.stdout.split() == ["0", "7", "7", "7"]
    for (cfg, s), p in zip(cases, paths):
        with MHDSolver(cfg) as sol:
            sol.set_state(s)
            sol.step(7)
            got = np.fromfile(p, dtype=np.float32).reshape((8,) + cfg.shape)
            assert np.array_equal(got, sol.get_state())
