"""Radial slab decomposition (nmhd_b200.slab), host side, on the CPU.

- The reference's own P-rank run (one process per rank, oracle.run_ref_slabs)
  is deterministic and matches the committed fixtures; all ranks keep one
  clock.
- The slab problem is the whole box's problem in the ranks' frames.
- The setup text of a rank (Python and the C++ header) is the reference's
  save_state text of that rank, and the reference's snapshot of a P-rank run
  stitches in nmhd_b200.postprocess exactly as in its own to_gnuplot tools.
- DistributedSlab's transport over gloo process groups (2 and 3 ranks), with a
  small host backend, equals the same scheme computed on the global array:
  messages reach the right neighbours and the CFL minimum is global; errors and
  wallclock limits stop every rank together.
"""
import os
import socket
import subprocess

import numpy as np
import pytest

from nmhd_b200 import checkpoint as ck
from nmhd_b200 import postprocess as pp
from nmhd_b200.binio import read_bin
from nmhd_b200.problems import shearing_box, shearing_box_slabs
from nmhd_b200.slab import neighbours, slab_config
from oracle import oracle

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
GOLDEN = os.path.join(HERE, "golden")

SLAB_CASES = {
    "shear32x16x8_p2": (lambda: shearing_box_slabs(2, n_radial=16, n_azimuthal=32, n_vertical=8,
                                                   l_azimuthal=4.0, seed=3), 10),
    "shear32x16x8_p4": (lambda: shearing_box_slabs(4, n_radial=16, n_azimuthal=32, n_vertical=8,
                                                   l_azimuthal=4.0, seed=4), 10),
    "shear48x24x12_p3": (lambda: shearing_box_slabs(3, n_radial=24, n_azimuthal=48, n_vertical=12,
                                                    l_radial=1.5, l_azimuthal=2.0, seed=5), 8),
    "shear64x32x16_mz_p2": (lambda: z_margins(shearing_box_slabs(2, n_radial=32, n_azimuthal=64, n_vertical=16,
                                                                 l_azimuthal=4.0, seed=6)), 6),
}


def z_margins(slabs, m=4):
    """The slabs with m periodic Z-margin planes on each side."""
    cfg, states = slabs
    cfg.margin_z, cfg.size_z = m, cfg.size_z + 2 * m
    return cfg, [np.concatenate([s[:, -m:], s, s[:, :m]], axis=1) for s in states]


def _need(name):
    if oracle.ref_binary(name) is None:
        pytest.skip(f"reference binary ref_{name} not built")


def _digest(a):
    import hashlib
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.mark.parametrize("name", sorted(SLAB_CASES))
def test_reference_ranks_match_fixture(name):
    _need(name)
    make, steps = SLAB_CASES[name]
    cfg, states = make()
    fx = np.load(os.path.join(GOLDEN, name + ".npz"))
    assert [str(h) for h in fx["input_sha256"]] == [_digest(s) for s in states]
    outs, times, infos = oracle.run_ref_slabs(name, states, steps)
    assert len({i["time"] for i in infos}) == 1  # one clock on every rank
    assert all(i["steps"] == steps for i in infos)
    assert [_digest(o) for o in outs] == [str(h) for h in fx["output_sha256"]]
    assert np.array_equal(times, fx["times"])


def test_slab_problem_is_the_whole_box_in_rank_frames():
    whole, s = shearing_box(n_radial=24, n_azimuthal=16, n_vertical=4, l_radial=1.5, seed=9)
    cfg, states = shearing_box_slabs(3, n_radial=24, n_azimuthal=16, n_vertical=4, l_radial=1.5, seed=9)
    assert cfg == slab_config(whole, 3) and cfg.size_y == 8 + 8 and cfg.parallel_size_y == 3
    d, dw = cfg.derived(), whole.derived()
    assert d["dy"] == dw["dy"] and d["extent_y"] == np.float32(1.5) / np.float32(24) * np.float32(16)
    assert d["relative_velocity"] == np.float32(np.float32(-1.5) * d["local_extent_y"])
    m = 4
    for r, st in enumerate(states):
        rows = slice(m, m + 8)
        # noise: the whole box's rows of this slab; background: the slab's own frame
        noise_w = s[2:4, :, m + 8 * r:m + 8 * (r + 1)]
        assert np.array_equal(st[2:4, :, rows], noise_w)
    with pytest.raises(ValueError):
        slab_config(whole, 5)


@pytest.mark.parametrize("world", [1, 2, 3, 4])
def test_neighbours_wrap(world):
    for r in range(world):
        lo, hi = neighbours(r, world)
        assert neighbours(hi, world)[0] == r and neighbours(lo, world)[1] == r


# ---------------------------------------------------------------------------
# checkpoints and snapshots of ranks


def _with_exact(ref_text, time):
    head, tail = ref_text.split("\n\n################", 1)
    lines = head.split("\n")
    lines[0] = str(int(lines[0]) + 1)
    lines.append("current_time_exact %.17g" % time)
    return "\n".join(lines) + "\n\n################" + tail


@pytest.mark.parametrize("name", ["shear32x16x8_p2", "shear48x24x12_p3"])
def test_rank_setup_text_is_the_reference_text(tmp_path, name):
    _need(name)
    make, _ = SLAB_CASES[name]
    cfg, states = make()
    _, _, infos = oracle.run_ref_slabs(name, states, 4, ckpt_dir=tmp_path, save_tag="c")
    for r in range(len(states)):
        ref = (tmp_path / "c" / ("%04d_setup.txt" % r)).read_text()
        ours = ck.setup_text(cfg, 4, infos[r]["time"], output_directory=str(tmp_path), rank=r)
        assert ours == _with_exact(ref, infos[r]["time"])


def test_cpp_header_rank_setup_text(tmp_path):
    _need("shear32x16x8_p2")
    cfg, states = SLAB_CASES["shear32x16x8_p2"][0]()
    _, _, infos = oracle.run_ref_slabs("shear32x16x8_p2", states, 3, ckpt_dir=tmp_path, save_tag="c")
    t = infos[1]["time"]
    src = tmp_path / "ck.cpp"
    src.write_text(r'''
#include "nmhd.hpp"
#include <cstdlib>
#include <iostream>
int main(int argc, char **argv) {
  nmhd_config c = {};
  c.size_x = 32; c.size_y = 16; c.size_z = 8; c.margin_y = 4; c.parallel_size_y = 2;
  c.extent_x = 4; c.extent_y = 1; c.extent_z = 1;
  c.gamma = 5.0f / 3.0f; c.cfl = 0.4f; c.problem = NMHD_PROBLEM_SHEARING_BOX;
  c.q = 1.5f; c.omega = 1.0f; c.space_order = 2; c.time_order = 2;
  std::cout << nmhd::checkpoint::setup_text(c, 3, std::strtod(argv[1], 0), argv[2], 1);
  return 0;
}
''')
    exe = tmp_path / "ck"
    subprocess.run(["g++", "-std=c++17", "-I" + os.path.join(ROOT, "include"), str(src), "-o", str(exe)],
                   check=True)
    out = subprocess.run([str(exe), repr(t), str(tmp_path)], check=True, capture_output=True, text=True).stdout
    assert out == _with_exact((tmp_path / "c" / "0001_setup.txt").read_text(), t)


def test_reference_rank_snapshots_stitch_like_its_tools(tmp_path):
    """A P-rank snapshot of the reference, stitched by nmhd_b200.postprocess,
    is byte-identical to the reference's to_gnuplot / to_gnuplot_3d output."""
    _need("shear48x24x12_p3")
    tg, tg3 = (os.path.join(ROOT, "oracle", "_ref", t) for t in ("to_gnuplot", "to_gnuplot_3d"))
    if not (os.path.exists(tg) and os.path.exists(tg3)):
        pytest.skip("reference post-processors not built")
    cfg, states = SLAB_CASES["shear48x24x12_p3"][0]()
    oracle.run_ref_slabs("shear48x24x12_p3", states, 6, ckpt_dir=tmp_path, save_tag="c")
    folder = tmp_path / "c"
    ref = subprocess.run([tg, str(folder)], check=True, capture_output=True, text=True).stdout
    assert pp.gnuplot_text(str(folder)) == ref
    subprocess.run([tg3, str(folder), str(tmp_path / "sec")], check=True)
    ours = pp.sections(str(folder))
    for plane in ("yz", "xz", "xy"):
        assert ours[plane] == (tmp_path / ("sec_%s.txt" % plane)).read_text(), plane
    assert read_bin(str(folder / "0002.bin")).shape == (8,) + cfg.shape


# ---------------------------------------------------------------------------
# DistributedSlab transport over gloo, with a host backend


class ToyBackend:
    """A 1-D periodic diffusion split into slabs with the slab layout of the
    solver: L interior cells between M margin cells on each side, messages of
    M cells.  CFL time = 0.4 / (1 + max |u|) over every cell, margins
    included (as the solver's).  ``fail_at``: report an error after that
    generation."""

    M = 2

    def __init__(self, u_interior, fail_at=None):
        import torch
        self.L = len(u_interior)
        self.u = np.zeros(self.L + 2 * self.M, np.float32)
        self.u[self.M:self.M + self.L] = u_interior
        self.gen = 0
        self.time = 0.0
        self.goal = np.inf
        self.fail_at = fail_at
        self.done = False
        self._slot = torch.full((1,), np.inf, dtype=torch.float32)
        self.device = "cpu"

    def halo_count(self):
        return self.M

    def begin(self, goal):
        self.goal = goal
        self.done = False

    def pack(self, send_inc, send_dec):
        if self.done:
            return
        M, L = self.M, self.L
        send_inc.copy_(_t(self.u[L:L + M]))      # top interior cells, to the rank above
        send_dec.copy_(_t(self.u[M:2 * M]))      # bottom interior cells, to the rank below

    def unpack(self, recv_inc, recv_dec):
        if self.done:
            return
        M, L = self.M, self.L
        self.u[0:M] = recv_inc.numpy()
        self.u[L + M:] = recv_dec.numpy()
        self._slot[0] = float(np.float32(0.4) / (np.float32(1) + np.abs(self.u).max()))

    def cfl_slot(self):
        return self._slot

    def stages(self):
        if self.done:
            return
        dt = np.float32(self._slot[0].item())
        if self.time + dt > self.goal:
            dt = np.float32(self.goal - self.time)
            self.done = True
        u = self.u
        new = u.copy()
        new[1:-1] = u[1:-1] + dt * (u[:-2] - np.float32(2) * u[1:-1] + u[2:])
        self.u = new
        self.time += float(dt)
        self.gen += 1

    def poll(self):
        err = None
        if self.fail_at is not None and self.gen >= self.fail_at:
            err = RuntimeError("numerical error")
        return self.done, err, self.gen, self.time


def _t(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a))


class OracleSlabBackend:
    """One radial slab of the MHD step on the host, through the oracle's
    split-phase functions (the reference's communicate() halves, its slab CFL
    time and its RK stages): the same interface as SolverBackend, so
    DistributedSlab drives the real step over gloo.  Clock and goal clamp as
    MHDSolver::proceed (mhd_solver.inlrb:870-901): dt = the all-reduced
    minimum of every rank's min(goal, CFL time); past the goal, dt = goal -
    time and the run ends."""

    def __init__(self, cfg, state):
        import torch
        self.cfg = cfg
        self.w = np.ascontiguousarray(state, np.float32).copy()
        self.gen = 0
        self.time = 0.0
        self.goal = np.float32(np.inf)
        self.done = False
        self._slot = torch.full((1,), np.inf, dtype=torch.float32)
        self.device = "cpu"

    def halo_count(self):
        return oracle.halo_count(self.cfg)

    def begin(self, goal):
        self.goal = np.float32(goal)
        self.done = False

    def pack(self, send_inc, send_dec):
        if self.done:
            return
        inc, dec = oracle.halo_pack(self.cfg, self.w, self.time)
        send_inc.copy_(_t(inc))
        send_dec.copy_(_t(dec))

    def unpack(self, recv_inc, recv_dec):
        if self.done:
            return
        oracle.halo_unpack(self.cfg, self.w, recv_inc.numpy(), recv_dec.numpy())
        self._slot[0] = oracle.cfl(self.cfg, self.w, float(self.goal))

    def cfl_slot(self):
        return self._slot

    def stages(self):
        if self.done:
            return
        dt = np.float32(self._slot[0].item())
        if self.time + float(dt) > float(self.goal):
            dt = np.float32(float(self.goal) - self.time)
            self.done = True
        oracle.stages(self.cfg, self.w, dt)
        self.time += float(dt)
        self.gen += 1

    def poll(self):
        return self.done, None, self.gen, self.time


def _global_reference(u0, steps, goal=np.inf):
    """The same scheme on the whole periodic array (the answer the ranks must
    reproduce): margins are periodic copies, dt the global CFL minimum."""
    u = u0.astype(np.float32).copy()
    t = 0.0
    for _ in range(steps):
        dt = np.float32(0.4) / (np.float32(1) + np.abs(u).max())
        if t + dt > goal:
            dt = np.float32(goal - t)
        ext = np.concatenate([u[-1:], u, u[:1]])
        u = ext[1:-1] + dt * (ext[:-2] - np.float32(2) * ext[1:-1] + ext[2:])
        t += float(dt)
        if t >= goal:
            break
    return u, t


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q, mode):
    import torch.distributed as dist
    from nmhd_b200.slab import DistributedSlab
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    os.environ["OMP_NUM_THREADS"] = "1"
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        if mode in SLAB_CASES:  # the MHD step of a reference P-rank case
            make, steps = SLAB_CASES[mode]
            cfg, states = make()
            b = OracleSlabBackend(cfg, states[rank])
            slab = DistributedSlab(b, None)
            reached = slab.proceed(np.inf, max_steps=steps)
            q.put((rank, {"w": b.w, "gen": b.gen, "time": b.time, "reached": reached}))
            return
        u0 = np.sin(np.linspace(0, 2 * np.pi, 12 * world, endpoint=False)).astype(np.float32) + 1.5
        part = u0[12 * rank:12 * (rank + 1)]
        fail_at = 5 if (mode == "error" and rank == world - 1) else None
        b = ToyBackend(part, fail_at=fail_at)
        slab = DistributedSlab(b, None)
        res = {}
        if mode == "steps":
            res["reached"] = slab.proceed(np.inf, max_steps=20)
        elif mode == "goal":
            res["reached"] = slab.proceed(0.5)
        elif mode == "timeout":
            res["reached"] = slab.proceed(np.inf, wallclock_time_limit=1e-9 if rank == 0 else -1.0,
                                          max_steps=64)
        elif mode == "error":
            try:
                slab.proceed(np.inf, max_steps=32)
                res["raised"] = False
            except RuntimeError:
                res["raised"] = True
        res.update(u=b.u[b.M:b.M + b.L].copy(), gen=b.gen, time=b.time)
        q.put((rank, res))
    finally:
        dist.destroy_process_group()


def _run(world, mode):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q, mode)) for r in range(world)]
    for p in procs:
        p.start()
    out = dict(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    return [out[r] for r in range(world)]


@pytest.mark.parametrize("world", [2, 3])
def test_distributed_transport_equals_global_scheme(world):
    res = _run(world, "steps")
    u0 = np.sin(np.linspace(0, 2 * np.pi, 12 * world, endpoint=False)).astype(np.float32) + 1.5
    ref, t = _global_reference(u0, 20)
    got = np.concatenate([r["u"] for r in res])
    assert np.array_equal(got, ref)
    assert all(r["gen"] == 20 and r["time"] == t and r["reached"] is False for r in res)


def test_distributed_goal_reached_on_every_rank():
    res = _run(2, "goal")
    u0 = np.sin(np.linspace(0, 2 * np.pi, 24, endpoint=False)).astype(np.float32) + 1.5
    ref, t = _global_reference(u0, 10 ** 6, goal=0.5)
    assert all(r["reached"] for r in res)
    assert np.array_equal(np.concatenate([r["u"] for r in res]), ref)
    assert res[0]["gen"] == res[1]["gen"] and res[0]["time"] == res[1]["time"] == t


def test_distributed_timeout_and_error_stop_every_rank():
    res = _run(2, "timeout")
    assert all(r["reached"] is False for r in res)
    assert res[0]["gen"] == res[1]["gen"] == 16  # one batch, on both ranks
    res = _run(3, "error")
    assert all(r["raised"] for r in res)


@pytest.mark.parametrize("name", sorted(SLAB_CASES))
def test_distributed_mhd_step_equals_reference_ranks(name):
    """The real MHD step through DistributedSlab on as many gloo ranks as the
    reference case has (2, 3, 4; shear-periodic radial wrap, Z margins), each
    rank's slab advanced by the oracle's split-phase functions: every rank's
    state is bitwise the reference's own P-rank run (tests/golden/<name>.npz,
    written by its communicate() and MPI_Allreduce through the file-mailbox
    MPI of oracle/refshim), and every rank has the reference's clock."""
    make, steps = SLAB_CASES[name]
    cfg, states = make()
    fx = np.load(os.path.join(GOLDEN, name + ".npz"))
    assert [str(h) for h in fx["input_sha256"]] == [_digest(s) for s in states]
    res = _run(len(states), name)
    assert [_digest(r["w"]) for r in res] == [str(h) for h in fx["output_sha256"]]
    if "output" in fx:
        for r, ref in zip(res, fx["output"]):
            assert np.array_equal(r["w"], ref)
    assert all(r["gen"] == steps and r["time"] == fx["times"][-1] and r["reached"] is False for r in res)
