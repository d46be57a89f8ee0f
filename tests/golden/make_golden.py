"""Generate the golden fixtures in this directory from the reference itself.

Runs the host-compiled reference solver (oracle/_ref/ref_*, built by
``make -C oracle ref`` from the reference sources; see oracle/Makefile) on
seeded inputs and stores its outputs.  The reference ships no golden vectors
of its own, so these fixtures pin both the oracle (tests/test_oracle_pin.py)
and, through it, the CUDA path.

Usage:  python tests/golden/make_golden.py [NAME ...]   (default: every case)
"""
from __future__ import annotations

import hashlib
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from nmhd_b200.problems import orszag_tang_3d, shearing_box, shearing_box_slabs  # noqa: E402
from oracle import oracle  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))

def scheme(built, space=2, time=2):
    """A problem with generate_config.rb's scheme options (-s space, -t time)."""
    cfg, state = built
    cfg.space_order, cfg.time_order = space, time
    return cfg, state


# name -> (reference binary, problem builder, steps, goal_time, store input)
CASES = {
    "ot16": ("ot16", lambda: orszag_tang_3d(16), 10, 1.0e30, True),
    "ot16_goal": ("ot16", lambda: orszag_tang_3d(16), 100, 0.05, True),
    "ot24x20x12": ("ot24x20x12", lambda: orszag_tang_3d(24, ny=20, nz=12), 12, 1.0e30, True),
    "shear32x16x8": ("shear32x16x8",
                     lambda: shearing_box(n_radial=16, n_azimuthal=32, n_vertical=8, l_azimuthal=4.0),
                     20, 1.0e30, False),
    "shear48x20x12": ("shear48x20x12",
                      lambda: shearing_box(n_radial=20, n_azimuthal=48, n_vertical=12, l_azimuthal=2.0),
                      8, 1.0e30, False),
    # the reference's piecewiseconst1 / euler1 schemes (oracle/expand_variant.py)
    "ot24x20x12_s1": ("ot24x20x12_s1", lambda: scheme(orszag_tang_3d(24, ny=20, nz=12), space=1),
                      15, 1.0e30, False),
    "shear32x16x8_t1": ("shear32x16x8_t1",
                        lambda: scheme(shearing_box(n_radial=16, n_azimuthal=32, n_vertical=8,
                                                    l_azimuthal=4.0, seed=4), time=1), 15, 1.0e30, False),
    "shear48x20x12_s1t1": ("shear48x20x12_s1t1",
                           lambda: scheme(shearing_box(n_radial=20, n_azimuthal=48, n_vertical=12,
                                                       l_azimuthal=2.0, seed=5), space=1, time=1),
                           15, 1.0e30, False),
}


# Radial slab decompositions, run as one reference process per rank
# (oracle.run_ref_slabs).  name -> (binary, slab builder, steps, store outputs)
# Without stored outputs the fixture keeps each rank's SHA-256 (bitwise parity
# needs no more).
SLAB_CASES = {
    "shear32x16x8_p2": ("shear32x16x8_p2",
                        lambda: shearing_box_slabs(2, n_radial=16, n_azimuthal=32, n_vertical=8,
                                                   l_azimuthal=4.0, seed=3), 10, True),
    "shear32x16x8_p4": ("shear32x16x8_p4",
                        lambda: shearing_box_slabs(4, n_radial=16, n_azimuthal=32, n_vertical=8,
                                                   l_azimuthal=4.0, seed=4), 10, False),
    "shear48x24x12_p3": ("shear48x24x12_p3",
                         lambda: shearing_box_slabs(3, n_radial=24, n_azimuthal=48, n_vertical=12,
                                                    l_radial=1.5, l_azimuthal=2.0, seed=5), 8, False),
    "shear64x32x16_mz_p2": ("shear64x32x16_mz_p2", lambda: _z_margins(shearing_box_slabs(
        2, n_radial=32, n_azimuthal=64, n_vertical=16, l_azimuthal=4.0, seed=6)), 6, False),
}


def _z_margins(slabs, m=4):
    """The slabs with m periodic Z-margin planes on each side."""
    cfg, states = slabs
    cfg.margin_z, cfg.size_z = m, cfg.size_z + 2 * m
    return cfg, [np.concatenate([s[:, -m:], s, s[:, :m]], axis=1) for s in states]


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def main():
    only = set(sys.argv[1:])
    for name, (binary, make, steps, goal, keep_input) in CASES.items():
        if only and name not in only:
            continue
        cfg, state = make()
        out, times, info = oracle.run_ref(binary, state, steps, goal_time=goal)
        payload = {"output": out, "times": times, "steps": np.int64(info["steps"]),
                   "goal_time": np.float64(goal), "input_sha256": np.bytes_(digest(state)),
                   "goal_reached": np.int64(info["goal_reached"])}
        if keep_input:
            payload["input"] = state
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **payload)
        print(name, info)
    for name, (binary, make, steps, keep) in SLAB_CASES.items():
        if only and name not in only:
            continue
        cfg, states = make()
        outs, times, infos = oracle.run_ref_slabs(binary, states, steps)
        payload = {"times": times, "steps": np.int64(infos[0]["steps"]),
                   "output_sha256": np.array([digest(o) for o in outs]),
                   "input_sha256": np.array([digest(s) for s in states])}
        if keep:
            payload["output"] = np.stack(outs)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **payload)
        print(name, infos[0])


if __name__ == "__main__":
    main()
