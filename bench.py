"""Benchmark: Mcell-updates/s of the ideal-MHD time step on B200.

Workload (default): the MRI shearing box, 128 (radial) x 256 (azimuthal) x 64
cells, FP32, gamma 5/3, CFL 0.4, q 1.5, Omega 1, beta 400, seeded velocity
noise (seed 1); reference axes X azimuthal, Y radial (+2x4 shearing margins),
Z vertical.  A "step" is one RK2 time step of the whole box (two stages,
margin fill, CFL reduction).  Metric: interior cells x steps / second
(the reference's "mesh updates per sec",
src/application/optimize_mhd/main_detail.curb:39-44, counted over interior
cells).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl nmhd|reference]
                  [--workload NAME]

N > 1 runs under torch.distributed (one rank per GPU): independent replicas of
the box, one per GPU (the time step has no data-parallel exchange on one box;
"scaling": "weak").  Rank 0 prints one JSON line: the device-timed rate
(value), the same through the C ABI with host buffers (e2e), the HBM roofline
of the step and, for the default box, its instruction-issue roofline, the
opt-in fast-arithmetic step beside the exact one, the reference's CPU path on
a bounded sample (cpu_baseline), and the SM clocks seen while timing.

Other workloads (--workload): the 512 x 1024 x 256 box, the 256^3 anchors
(mri_shearing_box_256, orszag_tang_256), the batched ensembles
(mri_ensemble_64, mri_ensemble_small_512), the adjoint (mri_adjoint_64) and
one box split into radial slabs over N GPUs (mri_slabs_*, strong scaling).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    "mri_shearing_box_128x256x64": dict(n_radial=128, n_azimuthal=256, n_vertical=64, l_radial=1.0,
                                        l_azimuthal=4.0, l_vertical=1.0, seed=1),
    "mri_shearing_box_512x1024x256": dict(n_radial=512, n_azimuthal=1024, n_vertical=256,
                                          l_radial=1.0, l_azimuthal=4.0, l_vertical=1.0, seed=3),
    # the 256^3 performance anchors: a cubic shearing box and the Orszag-Tang vortex
    "mri_shearing_box_256": dict(n_radial=256, n_azimuthal=256, n_vertical=256, l_radial=1.0,
                                 l_azimuthal=1.0, l_vertical=1.0, seed=5),
    "orszag_tang_256": dict(problem="orszag_tang", n=256),
}


def make_workload(name):
    """(config, state) of a named single-box workload."""
    kw = dict(WORKLOADS[name])
    if kw.pop("problem", "shearing_box") == "orszag_tang":
        from nmhd_b200.problems import orszag_tang_3d
        return orszag_tang_3d(**kw)
    from nmhd_b200.problems import shearing_box
    return shearing_box(**kw)
REF_BINARY = {"mri_shearing_box_128x256x64": "shear256x128x64"}
ENSEMBLES = {"mri_ensemble_64": dict(n_boxes=64, seed=0),
             # many small boxes (sides 8..16 radial/vertical, 2-4x azimuthal):
             # the regime where per-box launches are latency-bound
             "mri_ensemble_small_512": dict(n_boxes=512, seed=0, sides=(8, 12, 16))}
# Differentiation: 64^3 shearing box of the MRI physics (Lx = Ly = Lz = 1,
# seed 2), 200 FP32 steps, loss = Maxwell stress averaged over states 151..200,
# checkpoints every 20 steps; 16 central-difference directions (seeds
# 100..115) with eps = 1e-3 relative to the velocity noise.
ADJOINTS = {"mri_adjoint_64": dict(n=64, seed=2, steps=200, window=(151, 200), ckpt=20, fd_dirs=16,
                                   fd_eps=1e-3, tlm_dirs=4)}
# Radial slab decomposition of one box (strong scaling): rank r of N holds
# radial slab r of the named box, halos over NCCL point-to-point, dt by an
# NCCL all-reduce (nmhd_b200.slab.DistributedSlab).
SLABS = {"mri_slabs_128x256x64": "mri_shearing_box_128x256x64",
         "mri_slabs_512x1024x256": "mri_shearing_box_512x1024x256"}
BYTES_PER_CELL_UPDATE = 160  # 8 FP32 state words: stage 1 read+write, stage 2 2x read + write


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """SM clock and clock-event (throttle) reasons sampled while running.

    NVML is polled every 2 ms from a thread (read-only queries), so that a
    timed region of a few milliseconds still carries its own clock record;
    without NVML, nvidia-smi samples every 200 ms."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, index, period_s=0.002):
        self.index = index
        self.period = period_s
        self.proc = None
        self.out = None
        self.thread = None
        self.samples = []
        self.max_mhz = None
        self.stop = threading.Event()
        self.source = None

    def _nvml_handle(self):
        import pynvml
        pynvml.nvmlInit()
        try:
            import torch
            uuid = str(torch.cuda.get_device_properties(self.index).uuid)
            return pynvml, pynvml.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
        except Exception:
            vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
            ids = [v for v in vis.split(",") if v.strip()]
            idx = int(ids[self.index]) if self.index < len(ids) and ids[self.index].strip().isdigit() else self.index
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(idx)

    def _poll(self, nv, h):
        bits = {"hw_slowdown": nv.nvmlClocksEventReasonHwSlowdown,
                "hw_thermal_slowdown": nv.nvmlClocksEventReasonHwThermalSlowdown,
                "sw_thermal_slowdown": nv.nvmlClocksEventReasonSwThermalSlowdown,
                "sw_power_cap": nv.nvmlClocksEventReasonSwPowerCap}
        while not self.stop.is_set():
            try:
                mhz = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
            except Exception:
                break
            self.samples.append((float(mhz), [k for k, b in bits.items() if r & b]))
            self.stop.wait(self.period)

    def __enter__(self):
        try:
            nv, h = self._nvml_handle()
            self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            self.thread = threading.Thread(target=self._poll, args=(nv, h), daemon=True)
            self.thread.start()
            self.source = "nvml, %g ms period" % (1e3 * self.period)
            return self
        except Exception:
            self.thread = None
        if shutil.which("nvidia-smi"):
            self.out = tempfile.TemporaryFile(mode="w+")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.out, stderr=subprocess.DEVNULL)
            self.source = "nvidia-smi, 200 ms period"
        return self

    def __exit__(self, *exc):
        if self.thread:
            self.stop.set()
            self.thread.join(timeout=5)
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], self.max_mhz, set()
        if self.thread is not None:
            for mhz, rs in self.samples:
                sm.append(mhz)
                reasons.update(rs)
        elif self.out:
            self.out.seek(0)
            for line in self.out:
                f = [t.strip() for t in line.split(",")]
                if len(f) < 7:
                    continue
                try:
                    sm.append(float(f[0]))
                    mx = float(f[1])
                except ValueError:
                    continue
                for name, val in zip(self.NAMES, f[3:7]):
                    if val.lower() == "active":
                        reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm), "source": self.source}


def cpu_reference_run(workload, steps, threads=None):
    """Run the host-compiled reference solver (oracle/_ref) on the workload;
    returns (interior cell-updates/s, steps, seconds, threads, kind)."""
    from oracle import oracle
    cfg, state = make_workload(workload)
    name = REF_BINARY.get(workload)
    threads = threads or os.cpu_count()
    if name and oracle.ref_binary(name):
        _, _, info = oracle.run_ref(name, state, steps, threads=threads)
        secs = info["seconds"]
        kind = "reference"
    else:
        os.environ["OMP_NUM_THREADS"] = str(threads)
        t0 = time.perf_counter()
        oracle.proceed(cfg, state, steps)
        secs = time.perf_counter() - t0
        kind = "port"
    return cfg.interior_cells * steps / secs, steps, secs, threads, kind


def cpu_sample(workload, budget_s=12.0):
    """Bounded CPU sample: calibrate with one step, then run ~budget_s seconds."""
    rate, _, secs, threads, kind = cpu_reference_run(workload, 1)
    steps = max(1, min(200, int(budget_s / max(secs, 1e-3))))
    rate, steps, secs, threads, kind = cpu_reference_run(workload, steps)
    return {"value": rate / 1e6, "unit": "Mcell-updates/s", "cores": threads, "kind": kind,
            "sample": f"{steps} full RK2 steps of {workload} ({secs:.1f} s, OpenMP {threads} threads)"}


def dist_setup(n_gpus, force=False):
    import torch
    import torch.distributed as dist
    if force and "RANK" not in os.environ and n_gpus == 1:
        # a one-rank process group (the slab arm's transport needs one)
        os.environ.update(RANK="0", WORLD_SIZE="1", LOCAL_RANK="0", MASTER_ADDR="127.0.0.1")
        import socket
        with socket.socket() as so:
            so.bind(("127.0.0.1", 0))
            os.environ.setdefault("MASTER_PORT", str(so.getsockname()[1]))
    if n_gpus > 1 or "RANK" in os.environ:
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        rank = int(os.environ.get("RANK", 0))
        world = int(os.environ.get("WORLD_SIZE", 1))
        local = int(os.environ.get("LOCAL_RANK", rank))
        if torch.cuda.is_available():
            torch.cuda.set_device(local)
        from datetime import timedelta
        dist.init_process_group("nccl" if torch.cuda.is_available() else "gloo",
                                timeout=timedelta(seconds=120))
        return rank, world, local, dist
    return 0, 1, 0, None


def run_reference_arm(args):
    rank, world, _, dist = dist_setup(args.gpus)
    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return
    # a slab workload's reference arm is the whole box on the host cores
    wl = SLABS.get(args.workload, args.workload)
    if wl not in WORKLOADS:
        why = ("the reference has no batched ensemble; its sizes are compile-time constants"
               if wl in ENSEMBLES else "the reference has no differentiated step")
        print(json.dumps({"impl": "reference", "unavailable": why}), flush=True)
        if dist:
            dist.destroy_process_group()
        return
    cpu_reference_run(wl, max(1, min(args.warmup, 2)))
    # bounded: at most ~90 s of timed CPU work
    _, _, secs1, _, _ = cpu_reference_run(wl, 1)
    steps = max(1, min(args.steps, int(90.0 / max(secs1, 1e-3))))
    rate, steps, secs, threads, kind = cpu_reference_run(wl, steps)
    v = rate / 1e6
    line = {"metric": "Mcell-updates/s", "value": v, "unit": "Mcell-updates/s", "impl": "reference",
            "n_gpus": args.gpus, "steps": steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * secs / steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded shearing-box noise)",
            "config": {"workload": wl, "parallelism": "replicas"},
            "cpu_baseline": {"value": v, "unit": "Mcell-updates/s", "cores": threads, "kind": kind,
                             "sample": f"{steps} full RK2 steps ({secs:.1f} s)"},
            "e2e": {"value": v, "unit": "Mcell-updates/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


def run_gpu_arm(args):
    import torch
    from nmhd_b200.solver import MHDSolver

    rank, world, local, dist = dist_setup(args.gpus)
    dev = torch.device("cuda", local)
    wl = args.workload
    cfg, state = make_workload(wl)
    stream = torch.cuda.Stream(device=dev)
    sol = MHDSolver(cfg)
    sol.set_stream(stream.cuda_stream)
    sol.set_state(state)
    tuning = None
    if args.kernel:
        v, rows, zc = (int(t) for t in args.kernel.split(","))
        sol.set_kernel(v, rows, zc)
        choice = {"variant": v, "tile_rows": rows, "z_chunk": zc, "source": "--kernel"}
    else:
        tuning = sol.autotune(steps=5)
        best = min(tuning, key=lambda t: t[3])
        choice = {"variant": best[0], "tile_rows": best[1], "z_chunk": best[2], "source": "autotune"}
    # the timed region launches only graphs built here, before it starts
    sol.prepare(args.steps)
    sol.step(args.warmup)
    torch.cuda.synchronize(dev)

    def barrier():
        if dist:
            dist.barrier()

    def max_over_ranks(x):
        if not dist:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    # -- device-timed steps, state resident in HBM ---------------------------
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize(dev)
    with ClockSampler(dev.index) as clocks:
        start.record(stream)
        sol.step(args.steps)
        end.record(stream)
        torch.cuda.synchronize(dev)
    barrier()
    ms = max_over_ranks(start.elapsed_time(end))
    ms_per_step = ms / args.steps
    cells = cfg.interior_cells
    value = world * cells * args.steps / (ms * 1e-3) / 1e6

    # -- opt-in fast arithmetic (NMHD_FLAG_FAST_ARITHMETIC): same box, timed the
    # same way; its deviation after one step from the exact step of the same
    # state, relative to each quantity's scale ------------------------------
    fast = None
    if not args.no_fast:
        from dataclasses import replace as _replace
        from nmhd_b200.config import FLAG_FAST_ARITHMETIC
        exact1 = sol.get_state()
        t_state = sol.current_time()
        fs = MHDSolver(_replace(cfg, flags=cfg.flags | FLAG_FAST_ARITHMETIC))
        fs.set_stream(stream.cuda_stream)
        fs.set_state(exact1)
        fs.set_time(t_state, 0)
        ref_sol = MHDSolver(cfg)
        ref_sol.set_stream(stream.cuda_stream)
        ref_sol.set_state(exact1)
        ref_sol.set_time(t_state, 0)
        ref_sol.step(1)
        fs.step(1)
        ys = slice(cfg.margin_y, cfg.size_y - cfg.margin_y)  # interior rows
        a, b = fs.get_state()[:, :, ys], ref_sol.get_state()[:, :, ys]
        fdev = max(float(np.abs(a[g_].astype(np.float64) - b[g_]).max() / max(np.abs(b[g_]).max(), 1e-30))
                   for g_ in ([0], [1, 2, 3], [4], [5, 6, 7]))
        ref_sol.close()
        fs.prepare(args.steps)
        fs.step(args.warmup)
        torch.cuda.synchronize(dev)
        barrier()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        fs.step(args.steps)
        f1.record(stream)
        torch.cuda.synchronize(dev)
        fms = max_over_ranks(f0.elapsed_time(f1))
        fast = {"value": world * cells * args.steps / (fms * 1e-3) / 1e6, "unit": "Mcell-updates/s",
                "ms_per_step": fms / args.steps, "one_step_max_rel_dev": fdev,
                "note": "opt-in flag, not bitwise: contracted and approximate face-flux arithmetic; "
                        "one_step_max_rel_dev = largest |fast - exact| over the interior after one step "
                        "from the same state, relative to each quantity's scale"}
        fs.close()

    # -- per-kernel times (CUDA events around each launch, same stream) -------
    prof = sol.profile(max(3, min(20, args.steps)))
    kernel_ms_step = sum(t for t, _ in prof.values())  # device ms per step of each kernel class

    # -- end to end through the C ABI with pinned host buffers ---------------
    host_in = torch.empty((8,) + cfg.shape, dtype=torch.float32, pin_memory=True).numpy()
    host_in[...] = state
    host_out = torch.empty((8,) + cfg.shape, dtype=torch.float32, pin_memory=True).numpy()
    e2e_steps = args.steps
    barrier()
    torch.cuda.synchronize(dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    sol.set_state(host_in)
    sol.step(e2e_steps)
    sol.get_state(host_out)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    e2e_ms = max_over_ranks(e0.elapsed_time(e1))
    state_bytes = 8 * 4 * cfg.cells
    e2e = {"value": world * cells * e2e_steps / (e2e_ms * 1e-3) / 1e6, "unit": "Mcell-updates/s",
           "h2d_bytes_per_step": state_bytes / e2e_steps, "d2h_bytes_per_step": state_bytes / e2e_steps,
           "note": "set_state(pinned host) + proceed(K steps) + get_state(pinned host), per step"}

    if rank == 0:
        peak, peak_kind = load_peaks()
        # the RK2 step is the unit: 160 algorithmic bytes per cell-update
        achieved = BYTES_PER_CELL_UPDATE * cells / (kernel_ms_step * 1e-3) / 1e9
        # DRAM bytes and warp instructions per step of the chosen kernel
        # variant, from an ncu capture of the same box (not measured in this
        # run; the file says which launches)
        traffic, winst, tsrc = None, None, None
        tf = os.path.join(ROOT, "profiles", "traffic_" + wl + ".json")
        if os.path.exists(tf):
            tj = json.load(open(tf))
            tv = tj.get("by_variant", {}).get(str(choice["variant"]))
            if tv:
                traffic = tv.get("dram_bytes_per_step")
                winst = tv.get("warp_instructions_per_step")
                tsrc = "profiles/traffic_%s.json (ncu capture of kernel variant %s): %s" % (
                    wl, choice["variant"], tj.get("source", ""))
        launches_per_step = sum(k for _, k in prof.values())
        line = {
            "metric": "Mcell-updates/s", "value": value, "unit": "Mcell-updates/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded shearing-box noise)",
            "config": {"workload": wl, "cells_interior": cells, "cells_with_margins": cfg.cells,
                       "parallelism": "replicas" if world > 1 else "single",
                       "l2": "working set per step (state x3 + fluxes) > 126 MB L2",
                       "kernel": choice},
            "e2e": e2e,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "traffic_source": tsrc,
                         "peak_kind": peak_kind,
                         "unit_of_work": "one RK2 step (all kernels); 160 B per cell-update",
                         "kernels_ms_per_step": {k: round(t, 5) for k, (t, _) in prof.items()}},
            "gpu_launches": int(round(launches_per_step * args.steps)),
            "clocks": clocks.summary(),
        }
        if winst:
            # the bound the step actually meets: instruction issue (one warp
            # instruction per cycle per SM sub-partition), from the ncu count
            # of warp instructions per step at the sampled SM clock
            cs = line["clocks"] or {}
            mhz = cs.get("sm_mhz") or 1965.0
            sms = torch.cuda.get_device_properties(dev).multi_processor_count
            peak_i = sms * 4 * mhz * 1e6 / 1e9
            ach_i = winst / (ms_per_step * 1e-3) / 1e9
            line["issue_roofline"] = {"bound": "issue", "achieved": ach_i, "peak": peak_i,
                                      "unit": "G warp-instructions/s", "frac": ach_i / peak_i,
                                      "warp_instructions_per_step": winst, "sm_mhz": mhz, "sms": sms}
        if fast:
            line["fast_arithmetic"] = fast
        if tuning:
            line["autotune_ms_per_step"] = {f"v{a}_r{b}_z{c}": round(d, 4) for a, b, c, d in tuning}
        if world == 1 and not args.no_cpu:
            line["cpu_baseline"] = cpu_sample(wl)
    sol.close()
    # the other two parts of the metric (plain vs batched; adjoint/forward),
    # measured in the same run on one GPU: the 64-box ensemble batched and
    # through per-box plain launches, and the adjoint of the 64^3 box with
    # the whole tape kept and with the last segment only
    if world == 1 and not args.no_extras:
        ens = ensemble_measure("mri_ensemble_64", max(args.steps, 16), args.warmup, dev)
        line["ensemble_64"] = {k: ens[k] for k in ("value", "unit", "steps", "ms_per_step", "boxes",
                                                   "cells_interior", "plain_per_box", "batch_speedup",
                                                   "e2e", "gpu_launches", "schedule", "clocks")}
        line["ensemble_64"]["metric"] = "Mcell-updates/s, 64 uneven boxes batched (plain_per_box: same boxes, one solver each)"
        adj = {}
        for name, budget in (("whole_tape", -1), ("last_segment_only", 0)):
            m = adjoint_measure("mri_adjoint_64", dev, tape_budget=budget, warmup=1, reps=3)
            adj[name] = {k: m[k] for k in ("value", "forward_ms", "adjoint_total_ms", "adjoint_reverse_ms",
                                           "segments_kept_on_tape", "segments", "phases_ms")}
        line["adjoint_64"] = {"metric": "adjoint/forward time ratio, 64^3 shearing box, 200 steps, "
                                        "checkpoints every 20",
                              "unit": "x", "higher_is_better": False, **adj}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


def ensemble_measure(workload, steps, warmup, dev, rank=0, world=1, dist=None, n_boxes=0, plain=True):
    """Batched ensemble (e.g. 64 uneven shearing boxes): aggregate interior
    cell-updates/s of the batch (device-timed, states resident), the same end
    to end through the public API, and of the same boxes stepped one by one
    through the single-box path (plain per-box launches).  With world > 1 the
    boxes are partitioned over the ranks (no data-path collective) and times
    are the max over ranks."""
    import torch
    from nmhd_b200.batch import BatchSolver
    from nmhd_b200.problems import mri_ensemble
    from nmhd_b200.shard import my_boxes
    from nmhd_b200.solver import MHDSolver

    all_boxes, params = mri_ensemble(**ENSEMBLES[workload])
    if n_boxes:  # the first N boxes only (small profiling cases)
        all_boxes = all_boxes[:n_boxes]
    total_interior = sum(c.interior_cells for c, _ in all_boxes)
    boxes = [all_boxes[i] for i in my_boxes([c for c, _ in all_boxes], rank, world)]
    cfgs = [c for c, _ in boxes]

    def max_over_ranks(x):
        if not dist:
            return x
        tt = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        return float(tt.item())

    stream = torch.cuda.Stream(device=dev)
    batch = BatchSolver(cfgs)
    batch.set_stream(stream.cuda_stream)
    for i, (_, s) in enumerate(boxes):
        batch.set_state(i, s)
    batch.step(warmup)
    # schedule of each stage kernel (persistent or one tile per CTA), timed on these boxes
    tuning = batch.autotune(reps=3)
    names = ("flux", "ct", "update", "fused", "staged_flux")

    def sched(k, p, s):
        if k >= 3:
            return ("persistent" if p else "per_tile") if s else "off"
        return ("persistent" if p else "per_tile") + ("_split" if s else "")

    schedule = {names[k]: sched(k, p, s)
                for k, p, s, ms in tuning if ms == min(m for kk, _, _, m in tuning if kk == k)}
    batch.prepare(steps)
    batch.step(warmup)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(dev)
    if dist:
        dist.barrier()
    with ClockSampler(dev.index) as clocks:
        e0.record(stream)
        batch.step(steps)
        e1.record(stream)
        torch.cuda.synchronize(dev)
    ms = max_over_ranks(e0.elapsed_time(e1))
    value = total_interior * steps / (ms * 1e-3) / 1e6
    launches = batch.launches_per_step() * steps
    # end to end through the public API: every box's state in from pinned host
    # memory, the same steps, every box's state out to pinned host memory
    pinned = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).pin_memory().numpy()
    host_in = [pinned(s) for _, s in boxes]
    host_out = [pinned(np.empty_like(s, dtype=np.float32)) for _, s in boxes]
    torch.cuda.synchronize(dev)
    if dist:
        dist.barrier()
    e0.record(stream)
    batch.set_states(host_in)
    batch.step(steps)
    batch.get_states(out=host_out)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    e2e_ms = max_over_ranks(e0.elapsed_time(e1))
    state_bytes = sum(h.nbytes for h in host_in)
    e2e = {"value": total_interior * steps / (e2e_ms * 1e-3) / 1e6, "unit": "Mcell-updates/s",
           "h2d_bytes_per_step": state_bytes / steps, "d2h_bytes_per_step": state_bytes / steps,
           "note": "set_states (every box, pinned host) + proceed(K steps) + get_states (every box, "
                   "pinned host), per step"}
    batch.close()
    # plain: each box through its own single-box solver, one after another,
    # graphs built before the timed region
    plain_steps = max(3, steps // 4) if plain else 0
    solvers = []
    plain_wall = 0.0
    for c, s in boxes if plain_steps else []:
        sol = MHDSolver(c)
        sol.set_stream(stream.cuda_stream)
        sol.set_state(s)
        sol.prepare(plain_steps)
        sol.step(warmup)
        solvers.append(sol)
    if plain_steps:
        torch.cuda.synchronize(dev)
        if dist:
            dist.barrier()
        e0.record(stream)
        for sol in solvers:
            sol.step(plain_steps)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        plain_wall = max_over_ranks(e0.elapsed_time(e1)) * 1e-3
    plain_v = total_interior * plain_steps / plain_wall / 1e6 if plain_steps else None
    for sol in solvers:
        sol.close()
    return {"value": value, "unit": "Mcell-updates/s", "steps": steps, "ms_per_step": ms / steps,
            "boxes": len(all_boxes), "cells_interior": total_interior, "schedule": schedule,
            "autotune_ms_per_launch": {"%s_%s" % (names[k], sched(k, p, s)): round(ms_, 4)
                                       for k, p, s, ms_ in tuning},
            "plain_per_box": {"value": plain_v, "unit": "Mcell-updates/s", "steps": plain_steps,
                              "note": "same boxes, one single-box solver each, stepped one after another"},
            "batch_speedup": value / plain_v if plain_v else None,
            "e2e": e2e, "gpu_launches": launches, "clocks": clocks.summary()}


def run_ensemble_arm(args):
    """The batched ensemble as the bench line's workload (strong scaling over
    ranks: the same boxes, partitioned)."""
    import torch
    rank, world, local, dist = dist_setup(args.gpus)
    dev = torch.device("cuda", local)
    m = ensemble_measure(args.workload, args.steps, args.warmup, dev, rank, world, dist, args.boxes,
                         plain=not args.no_plain)
    if rank == 0:
        line = {
            "metric": "Mcell-updates/s", "value": m["value"], "unit": "Mcell-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": m["ms_per_step"],
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded ensemble of shearing boxes)",
            "config": {"workload": args.workload, "boxes": m["boxes"], "cells_interior": m["cells_interior"],
                       "parallelism": "boxes sharded over %d GPUs" % world if world > 1 else "single",
                       "timing": "CUDA events on the batch's stream around proceed() (graphs built "
                                 "before the timed region)",
                       "schedule": m["schedule"]},
            "autotune_ms_per_launch": m["autotune_ms_per_launch"],
            "plain_per_box": m["plain_per_box"], "batch_speedup": m["batch_speedup"],
            "e2e": m["e2e"], "gpu_launches": m["gpu_launches"], "clocks": m["clocks"],
        }
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


def run_slab_arm(args):
    """One box split into N radial slabs, one per GPU (strong scaling): the
    split-phase step with NCCL halos and dt all-reduce, interior
    cell-updates/s of the whole box."""
    import torch
    from nmhd_b200.problems import shearing_box_slabs
    from nmhd_b200.slab import DistributedSlab, SolverBackend
    from nmhd_b200.solver import MHDSolver

    rank, world, local, dist = dist_setup(args.gpus, force=True)
    dev = torch.device("cuda", local)
    wl = SLABS[args.workload]
    cfg, states = shearing_box_slabs(world, only=rank, **WORKLOADS[wl])
    sol = MHDSolver(cfg)
    backend = SolverBackend(sol, dev)
    sol.set_state(states[0])
    slab = DistributedSlab(backend)
    stream = torch.cuda.current_stream(dev)
    slab.proceed(math.inf, max_steps=args.warmup)
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    dist.barrier()
    torch.cuda.synchronize(dev)
    with ClockSampler(dev.index) as clocks:
        start.record(stream)
        slab.proceed(math.inf, max_steps=args.steps)
        end.record(stream)
        torch.cuda.synchronize(dev)
    dist.barrier()
    t = torch.tensor([start.elapsed_time(end)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms = float(t.item())
    cells = cfg.interior_cells * world
    value = cells * args.steps / (ms * 1e-3) / 1e6
    # end to end: this rank's slab in from pinned host memory, K steps, out
    host = torch.empty((8,) + cfg.shape, dtype=torch.float32, pin_memory=True).numpy()
    host[...] = states[0]
    del states
    dist.barrier()
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    sol.set_state(host)
    slab.proceed(math.inf, max_steps=args.steps)
    sol.get_state(host)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    t = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    e2e_ms = float(t.item())
    state_bytes = 8 * 4 * cfg.cells * world
    halo_bytes = 2 * 4 * backend.halo_count()
    if rank == 0:
        peak, peak_kind = load_peaks()
        achieved = BYTES_PER_CELL_UPDATE * cells / world / (ms / args.steps * 1e-3) / 1e9
        line = {
            "metric": "Mcell-updates/s", "value": value, "unit": "Mcell-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded shearing-box noise)",
            "config": {"workload": args.workload, "box": wl, "cells_interior": cells,
                       "parallelism": "radial slabs over %d GPU(s)" % world,
                       "slab": [cfg.size_x, cfg.size_y, cfg.size_z],
                       "halo_bytes_per_rank_per_step": halo_bytes,
                       "l2": "working set per step (state x3 + fluxes) > 126 MB L2"},
            "e2e": {"value": cells * args.steps / (e2e_ms * 1e-3) / 1e6, "unit": "Mcell-updates/s",
                    "h2d_bytes_per_step": state_bytes / args.steps,
                    "d2h_bytes_per_step": state_bytes / args.steps,
                    "note": "set_state(pinned host) + K slab steps + get_state(pinned host), per step"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": None, "peak_kind": peak_kind,
                         "unit_of_work": "one RK2 step of one slab (whole-step time); 160 B per cell-update"},
            # per step: halo pack, halo unpack (+ Z fill), margin CFL, and 3
            # kernels per RK stage (the CFL all-reduce and the halo transfer
            # are NCCL's)
            "gpu_launches": (2 * (cfg.margin_y > 0) + (cfg.margin_z > 0) + 1 + 6) * args.steps,
            "clocks": clocks.summary(),
        }
        print(json.dumps(line), flush=True)
    sol.close()
    dist.destroy_process_group()


def adjoint_measure(workload, dev, tape_budget=-1, warmup=3, reps=1, adjoint_steps=0, checks=False):
    """Adjoint / forward time ratio on the 64^3 shearing box (200 FP32 steps,
    checkpoints every 20): the forward is the production path (nmhd_proceed,
    its graphs built before timing), the adjoint run is nmhd_adjoint_run with
    the given tape budget (-1: as many segments as fit in half the free HBM;
    0: the last segment only, every other segment recomputed from its
    checkpoint).  Median over `reps` runs of each."""
    import torch
    from nmhd_b200.problems import shearing_box
    from nmhd_b200.solver import MHDSolver

    spec = ADJOINTS[workload]
    n = spec["n"]
    cfg, s = shearing_box(n_radial=n, n_azimuthal=n, n_vertical=n, l_radial=1.0, l_azimuthal=1.0,
                          l_vertical=1.0, seed=spec["seed"])
    steps, window, K = spec["steps"], spec["window"], spec["ckpt"]
    if adjoint_steps:  # shorter runs (profiling): the window keeps its length, at the end
        steps = adjoint_steps
        window = (max(0, steps - (window[1] - window[0])), steps)
    stream = torch.cuda.Stream(device=dev)
    sol = MHDSolver(cfg)
    sol.set_stream(stream.cuda_stream)
    sol.set_state(s)
    sol.set_adjoint_tape_budget(tape_budget)
    for _ in range(warmup):
        sol.adjoint(steps, window=window, ckpt_every=K)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    fwd = []
    with ClockSampler(dev.index) as clocks:
        for _ in range(reps):
            sol.set_state(s)
            sol.set_time(0.0, 0)
            sol.prepare(steps)
            sol.step(3)  # warm, then restart from the initial state
            sol.set_state(s)
            sol.set_time(0.0, 0)
            torch.cuda.synchronize(dev)
            e0.record(stream)
            sol.step(steps)
            e1.record(stream)
            torch.cuda.synchronize(dev)
            fwd.append(e0.elapsed_time(e1))
        sol.set_state(s)
        sol.set_time(0.0, 0)
        adj = []
        for _ in range(reps):
            J, g, dts = sol.adjoint(steps, window=window, ckpt_every=K)
            adj.append(sol.adjoint_timing())
    fwd_ms = statistics.median(fwd)
    tot = statistics.median([a["total"] for a in adj])
    rev = statistics.median([a["adjoint"] for a in adj])  # reverse sweep, recomputation overlapped
    out = {"value": tot / fwd_ms, "unit": "x", "steps": steps, "cells_interior": cfg.interior_cells,
           "cells_with_margins": cfg.cells, "loss": "Maxwell stress -<BxBy>, states %d..%d" % window,
           "ckpt_every": K, "tape_budget_bytes": tape_budget,
           "segments_kept_on_tape": sol.adjoint_kept_segments(), "segments": -(-steps // K),
           "forward_ms": fwd_ms, "adjoint_total_ms": tot, "adjoint_reverse_ms": rev,
           "reverse_over_forward": rev / fwd_ms, "phases_ms": adj[-1], "loss_value": J,
           "clocks": clocks.summary()}
    if checks:
        out["gradient_checks"] = adjoint_checks(sol, s, g, dts, steps, window, K, spec, cfg)
    sol.close()
    return out


def run_adjoint_arm(args):
    """Adjoint / forward time ratio on the 64^3 shearing box, with the
    gradient's checks: central differences of the FP32 and FP64 losses along
    16 seeded initial-velocity directions, the FP64 tangent-linear run along 4
    of them, and the FP64 adjoint-vs-tangent transpose identity."""
    import torch
    rank, world, local, dist = dist_setup(args.gpus)
    dev = torch.device("cuda", local)
    m = adjoint_measure(args.workload, dev, args.tape_budget, args.warmup, max(1, args.steps // 100),
                        args.adjoint_steps, checks=not args.no_checks)
    line = {
        "metric": "adjoint/forward time ratio", "value": m["value"], "unit": "x",
        "n_gpus": world, "steps": m["steps"], "warmup": args.warmup, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded shearing box)",
        "config": {"workload": args.workload, "cells_interior": m["cells_interior"],
                   "cells_with_margins": m["cells_with_margins"], "loss": m["loss"],
                   "ckpt_every": m["ckpt_every"], "tape_budget_bytes": args.tape_budget,
                   "segments_kept_on_tape": m["segments_kept_on_tape"], "segments": m["segments"],
                   "parallelism": "replicas" if world > 1 else "single"},
        "forward_ms": m["forward_ms"], "adjoint_total_ms": m["adjoint_total_ms"],
        "adjoint_reverse_ms": m["adjoint_reverse_ms"], "reverse_over_forward": m["reverse_over_forward"],
        "phases_ms": m["phases_ms"], "loss": m["loss_value"], "clocks": m["clocks"],
    }
    if "gradient_checks" in m:
        line["gradient_checks"] = m["gradient_checks"]
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


def adjoint_checks(sol, s, g, dts, steps, window, K, spec, cfg):
    """Gradient checks along directions dv = sigma * N(0, 1) on the three
    initial velocity fields, sigma = the noise amplitude 0.01 c_s.

    The discrete step is piecewise smooth: limiter, upwind-corner and sign(Bx)
    choices jump when a perturbation moves a decision variable across zero, and
    on the 64^3 box over 200 steps that happens for perturbations down to
    ~1e-8 sigma.  The derivative is therefore checked against FP64 central
    differences around the same float state with eps = 1e-9 sigma, accepted
    only where the two one-sided differences agree to 1% (no jump inside
    +-eps), else retried at eps/3 (twice).  Differences at the nominal
    eps = 1e-3 (FP32 and FP64) are reported beside them: they measure those
    jumps as well as the derivative."""
    gd = g.astype(np.float64)
    sigma = 0.01 * math.sqrt(cfg.gamma)
    eps = spec["fd_eps"]
    J0, _ = sol.tlm(steps, dts, None, window=window)
    _, g64 = sol.adjoint_f64(steps, dts, window=window, ckpt_every=K)
    rows = []
    for k in range(spec["fd_dirs"]):
        rng = np.random.default_rng(100 + k)
        d = np.zeros(s.shape)
        d[1:4] = sigma * rng.normal(0.0, 1.0, s[1:4].shape)
        row = {"adjoint32": float(np.sum(gd * d)), "adjoint64": float(np.sum(g64 * d))}
        e = 1e-9
        for _ in range(3):
            jp, _ = sol.tlm(steps, dts, d, window=window, shift=e)
            jm, _ = sol.tlm(steps, dts, d, window=window, shift=-e)
            sp_, sm_ = (jp - J0) / e, (J0 - jm) / e
            smooth = abs(sp_ - sm_) <= 0.01 * abs(sp_ + sm_) / 2
            if smooth:
                break
            e /= 3.0
        row["eps_used"] = e
        if smooth:
            row["fd64"] = (jp - jm) / (2 * e)
        jp, _ = sol.tlm(steps, dts, d, window=window, shift=eps)
        jm, _ = sol.tlm(steps, dts, d, window=window, shift=-eps)
        row["fd64_nominal"] = (jp - jm) / (2 * eps)
        sp = (s + eps * d).astype(np.float32)
        sm = (s - eps * d).astype(np.float32)
        d_applied = (sp.astype(np.float64) - sm.astype(np.float64)) / (2 * eps)
        sol.set_state(sp)
        jp32, _ = sol.loss_run(steps, window=window, dt=dts)
        sol.set_state(sm)
        jm32, _ = sol.loss_run(steps, window=window, dt=dts)
        sol.set_state(s)
        row["fd32_nominal"] = (jp32 - jm32) / (2 * eps)
        row["adjoint32_applied"] = float(np.sum(gd * d_applied))
        if k < spec["tlm_dirs"]:
            row["tlm64"] = sol.tlm(steps, dts, d, window=window)[1]
        rows.append(row)

    def rel(a, b):
        v = np.array([abs(r[a] - r[b]) / abs(r[b]) for r in rows if a in r and b in r])
        return {"median": float(np.median(v)), "max": float(np.max(v)), "n": int(len(v)),
                "within_1e-3": int(np.sum(v < 1e-3))}
    rng = np.random.default_rng(99)
    d = np.zeros(s.shape)
    d[1:4] = sigma * rng.normal(0.0, 1.0, s[1:4].shape)
    _, dJ64 = sol.tlm(steps, dts, d, window=window)
    return {"directions": spec["fd_dirs"], "noise_sigma": sigma, "eps_nominal": eps,
            "fd64_flip_free_directions": int(sum("fd64" in r for r in rows)),
            "eps_used": sorted({r["eps_used"] for r in rows}),
            "adjoint64_vs_fd64": rel("adjoint64", "fd64"),
            "adjoint32_vs_fd64": rel("adjoint32", "fd64"),
            "tlm64_vs_fd64": rel("tlm64", "fd64"),
            "adjoint32_vs_tlm64": rel("adjoint32", "tlm64"),
            "adjoint32_vs_adjoint64": rel("adjoint32", "adjoint64"),
            "fd64_nominal_vs_fd64": rel("fd64_nominal", "fd64"),
            "adjoint32_vs_fd32_nominal": rel("adjoint32_applied", "fd32_nominal"),
            "fp64_adjoint_transpose_rel": abs(float(np.sum(g64 * d)) - dJ64) / abs(dJ64)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="nmhd", choices=["nmhd", "reference"])
    ap.add_argument("--workload", default="mri_shearing_box_128x256x64",
                    choices=sorted(WORKLOADS) + sorted(ENSEMBLES) + sorted(ADJOINTS) + sorted(SLABS))
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--no-fast", action="store_true", help="skip the fast-arithmetic measurement")
    ap.add_argument("--no-extras", action="store_true",
                    help="default workload: skip the ensemble and adjoint measurements")
    ap.add_argument("--kernel", default="", help="variant,tile_rows,z_chunk (skip autotuning)")
    ap.add_argument("--no-checks", action="store_true", help="adjoint workload: timing only")
    ap.add_argument("--adjoint-steps", type=int, default=0, help="adjoint workload: steps per run (default 200)")
    ap.add_argument("--boxes", type=int, default=0, help="ensemble workloads: the first N boxes only")
    ap.add_argument("--no-plain", action="store_true", help="ensemble workloads: skip the per-box plain arm")
    ap.add_argument("--tape-budget", type=int, default=-1,
                    help="adjoint workload: bytes of tape beyond the last segment (-1: half the free HBM)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        run_reference_arm(args)
    elif args.workload in ENSEMBLES:
        run_ensemble_arm(args)
    elif args.workload in ADJOINTS:
        run_adjoint_arm(args)
    elif args.workload in SLABS:
        run_slab_arm(args)
    else:
        run_gpu_arm(args)


if __name__ == "__main__":
    main()
