"""Snapshot post-processing (nmhd_b200.postprocess) against the reference's own
post-processors, to_gnuplot and to_gnuplot_3d, built from their sources
(oracle/Makefile): the text must be byte-identical on snapshots written by the
reference solver, by this repository's writer, and on a two-rank radial stack
that exercises the shear displacement."""
import os
import subprocess

import pytest

from nmhd_b200 import checkpoint as ck
from nmhd_b200 import postprocess as pp
from nmhd_b200.binio import write_bin
from nmhd_b200.problems import orszag_tang_3d, shearing_box
from oracle import oracle

REF = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref")
CASES = {
    "shear32x16x8": lambda: shearing_box(n_radial=16, n_azimuthal=32, n_vertical=8, l_azimuthal=4.0, seed=3),
    "ot16": lambda: orszag_tang_3d(16),
}


def _tools():
    tg, tg3 = os.path.join(REF, "to_gnuplot"), os.path.join(REF, "to_gnuplot_3d")
    if not (os.path.exists(tg) and os.path.exists(tg3)):
        pytest.skip("reference post-processors not built")
    return tg, tg3


def _compare(folder, tmp_path):
    tg, tg3 = _tools()
    ref = subprocess.run([tg, str(folder)], check=True, capture_output=True, text=True).stdout
    assert pp.gnuplot_text(str(folder)) == ref
    subprocess.run([tg3, str(folder), str(tmp_path / "sec")], check=True)
    ours = pp.sections(str(folder))
    for name in ("yz", "xz", "xy"):
        assert ours[name] == (tmp_path / ("sec_%s.txt" % name)).read_text(), name


@pytest.mark.parametrize("name", sorted(CASES))
def test_reference_snapshot(tmp_path, name):
    _tools()
    if oracle.ref_binary(name) is None:
        pytest.skip(f"reference binary ref_{name} not built")
    cfg, s = CASES[name]()
    oracle.run_ref(name, s, 5, ckpt_dir=tmp_path, save_tag="c")
    _compare(tmp_path / "c", tmp_path)


def test_snapshot_written_here(tmp_path):
    _tools()
    cfg, s = CASES["shear32x16x8"]()
    o = oracle.proceed(cfg, s, 4)
    os.makedirs(tmp_path / "snap")
    write_bin(str(tmp_path / "snap" / "0000.bin"), o["state"])
    (tmp_path / "snap" / "0000_setup.txt").write_text(ck.setup_text(cfg, 4, o["time"]))
    _compare(tmp_path / "snap", tmp_path)


def _two_rank_text(text, rank, disp, corner_y):
    """A one-rank setup text turned into rank `rank` of a 2-rank radial stack."""
    glob, loc = text.split("\n\n################\n")
    glob = (glob.replace("parallel_size 1\n", "parallel_size 2\n")
                .replace("parallel_size_y 1\n", "parallel_size_y 2\n")
                .replace("global_size_y 16\n", "global_size_y 32\n")
                .replace("global_extent_y 1\n", "global_extent_y 2\n"))
    lines = []
    for line in loc.split("\n"):
        key = line.split(" ")[0]
        if key == "mpi_rank":
            line = "mpi_rank %d" % rank
        elif key == "mpi_prefix":
            line = "mpi_prefix %04d" % rank
        elif key == "relative_displacement":
            line = "relative_displacement %g" % disp
        elif key == "computational_corner_y":
            line = "computational_corner_y %g" % corner_y
        lines.append(line)
    return glob + "\n\n################\n" + "\n".join(lines)


def test_two_rank_stack_with_shear_displacement(tmp_path):
    _tools()
    cfg, s = CASES["shear32x16x8"]()
    a = oracle.proceed(cfg, s, 3)
    b = oracle.proceed(cfg, s, 7)
    os.makedirs(tmp_path / "stack")
    text = ck.setup_text(cfg, 3, a["time"])
    for rank, (st, disp, cy) in enumerate([(a["state"], 0.7, -0.25), (b["state"], 1.3, 0.75)]):
        write_bin(str(tmp_path / "stack" / ("%04d.bin" % rank)), st)
        (tmp_path / "stack" / ("%04d_setup.txt" % rank)).write_text(_two_rank_text(text, rank, disp, cy))
    _compare(tmp_path / "stack", tmp_path)


def test_command_line(tmp_path):
    cfg, s = CASES["ot16"]()
    os.makedirs(tmp_path / "snap")
    write_bin(str(tmp_path / "snap" / "0000.bin"), s)
    (tmp_path / "snap" / "0000_setup.txt").write_text(ck.setup_text(cfg, 0, 0.0))
    assert pp.main(["pp", str(tmp_path / "snap"), str(tmp_path / "out")]) == 0
    assert (tmp_path / "out_xy.txt").read_text() == pp.sections(str(tmp_path / "snap"))["xy"]
