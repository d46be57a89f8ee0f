"""L1 error of the FP32 time step against an FP64 run of the same scheme
(TEST INFRASTRUCTURE: uses the oracle).

The workload is config 5's physics on a 128 (radial) x 256 (azimuthal) x 64
subsample of the large box: MRI shearing box, beta 400, q 1.5, seeded noise
(seed 3), 200 RK2 steps.  The FP32 solution is computed on the GPU through the
C ABI when a GPU is present (and then checked bitwise against the FP32
oracle), else by the FP32 oracle, which is bitwise equal to the CUDA path.  The
FP64 solution is the FP64 build of the oracle (pinned bitwise to the
reference's Real = double build).  Prints one JSON line: relative L1 error
per field, sum |a - b| / sum |b|, and the clocks.

    python oracle/accuracy_report.py [--steps 200] [--seed 3]
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
# run as a script, this directory comes first on the path and would shadow the
# package of the same name
sys.path[:] = [p for p in sys.path if os.path.abspath(p or ".") != os.path.dirname(os.path.abspath(__file__))]
sys.path.insert(0, ROOT)

from nmhd_b200.problems import shearing_box  # noqa: E402
from oracle import oracle  # noqa: E402

FIELDS = ("density", "vx", "vy", "vz", "pressure", "Bx", "By", "Bz")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--seed", type=int, default=3)
    args = ap.parse_args()
    cfg, s32 = shearing_box(seed=args.seed)
    t0 = time.perf_counter()
    o32 = oracle.proceed(cfg, s32, args.steps)
    t32 = time.perf_counter() - t0
    gpu = None
    try:
        import torch
        if torch.cuda.is_available():
            from nmhd_b200.solver import MHDSolver
            with MHDSolver(cfg) as sol:
                sol.set_state(s32)
                sol.step(args.steps)
                g = sol.get_state()
                gpu = {"bitwise_equal_to_fp32_oracle": bool(np.array_equal(g, o32["state"])),
                       "time_equal": sol.current_time() == o32["time"]}
    except ImportError:
        pass
    t0 = time.perf_counter()
    o64 = oracle.proceed(cfg, s32.astype(np.float64), args.steps, dtype=np.float64)
    t64 = time.perf_counter() - t0
    a = o32["state"].astype(np.float64)
    b = o64["state"]
    interior = (slice(None), slice(None), slice(cfg.margin_y, cfg.size_y - cfg.margin_y), slice(None))
    l1 = {}
    for i, f in enumerate(FIELDS):
        da = a[interior][i]
        db = b[interior][i]
        l1[f] = float(np.sum(np.abs(da - db)) / max(np.sum(np.abs(db)), 1e-300))
    print(json.dumps({
        "workload": "mri_shearing_box_128x256x64 (config-5 physics, seed %d)" % args.seed,
        "steps": args.steps, "relative_l1_fp32_vs_fp64": l1,
        "time_fp32": o32["time"], "time_fp64": o64["time"],
        "gpu": gpu, "cpu_seconds": {"fp32": round(t32, 1), "fp64": round(t64, 1)},
    }))


if __name__ == "__main__":
    main()
