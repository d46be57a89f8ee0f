"""Radial slab decomposition on the GPU: SlabGroup (every slab of the box in
one process, halos read in place from the neighbours' send buffers, one CFL
minimum kernel) against the reference's own P-rank run, bitwise: the
committed fixtures (tests/golden/make_golden.py), and the host-compiled
reference itself where it is built.  A single slab with its messages looped
back is bitwise nmhd_proceed's step."""
import hashlib
import os

import numpy as np
import pytest

from nmhd_b200.problems import orszag_tang_3d, shearing_box
from nmhd_b200.slab import SlabGroup, slab_config
from nmhd_b200.solver import MHDSolver
from oracle import oracle
from test_slab import SLAB_CASES

pytestmark = pytest.mark.gpu


def _digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.mark.parametrize("name", sorted(SLAB_CASES))
def test_slab_group_matches_reference_ranks(gpu, golden_dir, name):
    make, steps = SLAB_CASES[name]
    cfg, states = make()
    fx = np.load(os.path.join(golden_dir, name + ".npz"))
    grp = SlabGroup(cfg, states)
    try:
        assert grp.step(steps) == steps
        outs = grp.get_states()
        assert grp.current_time() == fx["times"][-1]
        assert grp.generation() == steps
    finally:
        grp.close()
    if "output" in fx.files:
        for r, o in enumerate(outs):
            assert np.array_equal(o, fx["output"][r]), f"rank {r}: max diff {np.abs(o - fx['output'][r]).max()}"
    assert [_digest(o) for o in outs] == [str(h) for h in fx["output_sha256"]]
    if oracle.ref_binary(name) is not None:
        ref, times, _ = oracle.run_ref_slabs(name, states, steps)
        for o, q in zip(outs, ref):
            assert np.array_equal(o, q)


def test_slab_group_goal_time(gpu):
    make, _ = SLAB_CASES["shear32x16x8_p2"]
    cfg, states = make()
    grp = SlabGroup(cfg, states)
    try:
        assert grp.proceed(0.05) is True
        t, g = grp.current_time(), grp.generation()
        assert t == np.float32(0.05) or abs(t - float(np.float32(0.05))) < 1e-12
        # at the goal, proceed() takes one step of dt = goal - time = 0, as the
        # reference's loop does (mhd_solver.inlrb:880-884)
        assert grp.proceed(0.05) is True
        assert grp.generation() == g + 1 and grp.current_time() == t
    finally:
        grp.close()
    if oracle.ref_binary("shear32x16x8_p2") is not None:
        ref, times, infos = oracle.run_ref_slabs("shear32x16x8_p2", states, 10 ** 6, goal_time=0.05)
        assert infos[0]["steps"] == g and infos[0]["time"] == t


@pytest.mark.parametrize("case", ["shear", "shear_mz", "ot_nomargin"])
def test_single_slab_loopback_is_proceed(gpu, case):
    if case == "ot_nomargin":
        cfg, s = orszag_tang_3d(16)
    else:
        cfg, s = shearing_box(n_radial=16, n_azimuthal=32, n_vertical=8, l_azimuthal=4.0, seed=11)
        if case == "shear_mz":
            cfg.margin_z, cfg.size_z = 4, 16
            s = np.concatenate([s[:, -4:], s, s[:, :4]], axis=1)
    grp = SlabGroup(slab_config(cfg, 1), [s])
    try:
        grp.step(13)
        got, t = grp.get_states()[0], grp.current_time()
    finally:
        grp.close()
    with MHDSolver(cfg) as sol:
        sol.set_state(s)
        sol.step(13)
        assert np.array_equal(got, sol.get_state())
        assert t == sol.current_time()


def test_slab_refused_by_whole_box_entry_points(gpu):
    cfg, states = SLAB_CASES["shear32x16x8_p2"][0]()
    with MHDSolver(cfg) as sol:
        sol.set_state(states[0])
        with pytest.raises(RuntimeError, match="not supported"):
            sol.step(1)


def test_distributed_slab_one_rank_nccl(gpu):
    """DistributedSlab on a one-rank NCCL group: the solver backend's CFL slot
    (a device float of the library) all-reduced by NCCL in the solver's stream
    order; bitwise the whole-box step."""
    import datetime
    import socket

    import torch.distributed as dist
    from nmhd_b200.slab import DistributedSlab, SolverBackend
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    cfg, s = shearing_box(n_radial=16, n_azimuthal=32, n_vertical=8, l_azimuthal=4.0, seed=12)
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60))
    try:
        sol = MHDSolver(slab_config(cfg, 1))
        sol.set_state(s)
        ds = DistributedSlab(SolverBackend(sol, gpu))
        assert ds.proceed(np.inf, max_steps=21) is False
        assert ds.last_steps == 21
        got, t = sol.get_state(), sol.current_time()
        sol.close()
    finally:
        dist.destroy_process_group()
    with MHDSolver(cfg) as ref:
        ref.set_state(s)
        ref.step(21)
        assert np.array_equal(got, ref.get_state()) and t == ref.current_time()


def test_slab_snapshot_is_the_reference_snapshot(gpu, tmp_path):
    """save_state of every slab writes the reference's P-rank snapshot folder:
    the same .bin bytes as the reference's ranks after the same steps, and
    setup texts equal to theirs plus the exact-time member; the reference's
    to_gnuplot reads it like its own."""
    import subprocess
    name = "shear48x24x12_p3"
    if oracle.ref_binary(name) is None:
        pytest.skip(f"reference binary ref_{name} not built")
    cfg, states = SLAB_CASES[name][0]()
    grp = SlabGroup(cfg, states)
    try:
        grp.step(6)
        assert grp.save_state(tmp_path / "ours", "c")
    finally:
        grp.close()
    oracle.run_ref_slabs(name, states, 6, ckpt_dir=tmp_path / "ref", save_tag="c")
    for r in range(3):
        a = (tmp_path / "ours" / "c" / ("%04d.bin" % r)).read_bytes()
        b = (tmp_path / "ref" / "c" / ("%04d.bin" % r)).read_bytes()
        assert a == b, f"rank {r}"
        ours = (tmp_path / "ours" / "c" / ("%04d_setup.txt" % r)).read_text().splitlines()
        ref = (tmp_path / "ref" / "c" / ("%04d_setup.txt" % r)).read_text().splitlines()
        keep = lambda lines: [x for x in lines if not x.startswith(("current_time_exact", "output_directory"))
                              and x not in ("20", "21")]
        assert keep(ours) == keep(ref), f"rank {r}"
    tg = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref", "to_gnuplot")
    if os.path.exists(tg):
        a = subprocess.run([tg, str(tmp_path / "ours" / "c")], check=True, capture_output=True, text=True).stdout
        b = subprocess.run([tg, str(tmp_path / "ref" / "c")], check=True, capture_output=True, text=True).stdout
        assert a == b
