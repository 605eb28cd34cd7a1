"""Benchmark of the exterior Burton-Miller solve on B200.

Workload (dense plain FP64 form): pulsating rigid sphere of radius 0.1 m as an
icosphere with 3 subdivisions (642 vertices / 1280 triangles), uniform normal
velocity 1 m/s, c = 343 m/s, rho = 1.205 kg/m^3, 32 log-spaced frequencies
100 Hz - 5 kHz, observers (0,0,.3), (1,0,0), (0,0,3). One step = one sweep of
the 32 frequency points through a solver session whose interaction plan is
cached across steps (the reference's sweep usage). Metric: frequency-point
solves per second (higher is better).

Multi-GPU: one process per GPU, each rank solves its own replica of the sweep
(frequency points are independent; no collective on the data path); value is
the total over ranks divided by the slowest rank's device time.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
"""
from __future__ import annotations

import argparse
import json
import math
import os
import pathlib
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

FREQUENCIES = [float(f) for f in __import__("numpy").geomspace(100.0, 5000.0, 32)]
OBSERVERS = [(0.0, 0.0, 0.3), (1.0, 0.0, 0.0), (0.0, 0.0, 3.0)]
DENSITY, SOUND_SPEED = 1.205, 343.0
METRIC = "freq-point solves/s (dense plain FP64 form, C1 sphere sweep)"
# Algorithmic FP64 operations per regular-pair sample (one Green-kernel
# evaluation shared by both orientations of an unordered pair), counted from
# the regular-pair kernel source: displacement 15, |d|^2 5, 1/r 1, r and kr 2,
# sincos 1, weight 2, g 2, g(1+ikr) 4, 1/r^2 1, two normal projections 12,
# P and Q 4, three basis contractions 36.
FLOPS_PER_REGULAR_SAMPLE = 85
CONFIG = {"workload": "C1 icosphere s3 (642 v / 1280 t), 32 log freqs 100 Hz-5 kHz, 3 observers, dense FP64",
          "mesh": "icosphere-3 r=0.1 m", "frequencies": 32, "observers": 3, "excitations": 1,
          "l2": "per-sweep working set 10 GB (pair records) > 126 MB L2; L2 also flushed between steps"}


def env_rank():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def request(hs):
    return hs.BemRequest(frequencies=FREQUENCIES, observers=OBSERVERS,
                         excitations=[hs.BemExcitation("uniform", [hs.FaceVelocity(1, 1.0)])],
                         medium=hs.AcousticMedium(DENSITY, SOUND_SPEED))


def cpu_reference(samples: int, frequencies_per_sample: int):
    """The FP64 CPU restatement of the reference's dense path (plan, FP64
    assembly, LU, fields) on this host's cores, over a bounded sample of the
    sweep's frequencies."""
    from hornsculpt_b200 import meshes
    from oracle import oracle as O

    mesh = meshes.icosphere(3)
    picks = [FREQUENCIES[int(i)] for i in __import__("numpy").linspace(0, 31, frequencies_per_sample)]
    times = []
    for _ in range(samples):
        t0 = time.perf_counter()
        O.solve(mesh, picks, [[(1, 1.0)]], OBSERVERS, density=DENSITY, sound_speed=SOUND_SPEED,
                plan_frequencies=FREQUENCIES)
        times.append(time.perf_counter() - t0)
    return times, picks


class ClockSampler:
    """nvidia-smi clock and throttle-reason samples during the timed region."""

    FIELDS = "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown," \
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown," \
             "clocks_event_reasons.sw_power_cap"

    def __init__(self, device_index: int):
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.device = device_index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.file,
                                         stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            self.proc.wait(timeout=10)

    def summary(self):
        self.file.flush()
        rows = [line.split(",") for line in open(self.file.name).read().splitlines() if line.strip()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        sm, mx, reasons = [], 0.0, set()
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = max(mx, float(r[2]))
                for name, v in zip(names, r[5:9]):
                    if v.strip() == "Active":
                        reasons.add(name)
            except (ValueError, IndexError):
                continue
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    path = ROOT / "MEASURED_PEAKS.json"
    return json.loads(path.read_text()) if path.exists() else {}


def fp64_peak_tflops(torch):
    """FP64 dense throughput of cuBLAS DGEMM (4096^3, best of 5) on this GPU."""
    n = 4096
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    torch.matmul(a, b)
    torch.cuda.synchronize()
    best = math.inf
    for _ in range(5):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        e.synchronize()
        best = min(best, s.elapsed_time(e) / 1e3)
    return 2 * n ** 3 / best / 1e12


def run_reference(args, rank, world):
    if rank != 0:
        return
    from oracle import oracle as O  # noqa: F401  (built by build())
    per_step = 2
    for _ in range(args.warmup):
        cpu_reference(1, per_step)
    times = []
    for _ in range(args.steps):
        t, picks = cpu_reference(1, per_step)
        times += t
    value = per_step * len(times) / sum(times)
    cores = os.cpu_count()
    line = {"metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * sum(times) / len(times), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": CONFIG,
            "impl": "reference",
            "cpu_baseline": {"value": value, "unit": "solves/s", "cores": cores, "kind": "port",
                             "sample": f"{per_step} of the 32 sweep frequencies per step ({picks[0]:.0f} and "
                                       f"{picks[-1]:.0f} Hz), plan at 5 kHz each step, FP64 assembly on {cores} "
                                       "threads, dense LU, observer fields"},
            "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)  # >= 3 for reported numbers
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--sweep-frequencies", type=int, default=32,
                    help="solve only the first n sweep frequencies (small profiling cases)")
    args = ap.parse_args()
    rank, world, local = env_rank()
    if args.impl == "reference":
        return run_reference(args, rank, world)

    import numpy as np
    import torch
    import torch.distributed as dist

    import hornsculpt_b200 as hs

    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    stream = torch.cuda.Stream()
    mesh = hs.icosphere(3)
    req = request(hs)
    req.frequencies = FREQUENCIES[: args.sweep_frequencies]
    req.interaction_plan_frequencies = FREQUENCIES
    solver = hs.CudaBemSolver(mesh)
    solver.set_stream(stream.cuda_stream)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()

    for _ in range(args.warmup):
        solver.solve(req)
    peaks = measured_peaks()
    fp64 = fp64_peak_tflops(torch)
    solver.set_profiling(True)
    device_s, wall_s = 0.0, 0.0
    barrier()
    with ClockSampler(local) as clocks:
        for _ in range(args.steps):
            with torch.cuda.stream(stream):
                flush.zero_()
            start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            start.record(stream)
            t0 = time.perf_counter()
            result = solver.solve(req)
            wall_s += time.perf_counter() - t0
            end.record(stream)
            end.synchronize()
            device_s += start.elapsed_time(end) / 1e3
    barrier()
    times = torch.tensor([device_s, wall_s], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(times, op=dist.ReduceOp.MAX)
    device_s, wall_s = times.tolist()
    profile, work = solver.profile(), solver.work()
    points = len(req.frequencies) * args.steps * world
    if rank == 0:
        regular = [k for k in profile if k.startswith("regular_")]
        regular_ms = sum(profile[k][0] for k in regular)
        regular_launches = sum(profile[k][1] for k in regular)
        total_ms = sum(v[0] for v in profile.values())
        flops = work["regular_samples"] * FLOPS_PER_REGULAR_SAMPLE
        achieved = flops / (regular_ms / 1e3) / 1e12
        ex = result.frequencies[0].excitations[0]
        T, N, O = mesh.triangle_count, mesh.vertex_count, len(OBSERVERS)
        h2d = len(FREQUENCIES) * (T * 16 + 8) + O * 24
        d2h = len(FREQUENCIES) * (N * 16 + O * 16 + 32)
        line = {
            "metric": METRIC, "value": points / device_s, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * device_s / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": CONFIG,
            "e2e": {"value": points / wall_s, "unit": "solves/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "gpu_launches": int(sum(v[1] for v in profile.values())),
            "roofline": {"kernel": "regularPairsKernel (4 rule sizes)", "bound": "fp64", "achieved": achieved,
                         "peak": fp64, "unit": "TFLOP/s", "frac": achieved / fp64,
                         "peak_source": "cuBLAS DGEMM 4096^3 measured in this run (MEASURED_PEAKS.json has no FP64 figure)",
                         "traffic": None, "share_of_device_time": regular_ms / total_ms,
                         "algorithmic": f"{work['regular_samples']} regular samples x {FLOPS_PER_REGULAR_SAMPLE} FLOP"},
            "kernel_ms": {k: round(v[0] / args.steps, 4) for k, v in sorted(profile.items())},
            "clocks": clocks.summary(), "peaks": {"hbm_gbs": peaks.get("hbm_gbs"), "fp64_tflops_dgemm": fp64},
            "residual_max": max(e.boundary_residual for f in result.frequencies for e in f.excitations),
        }
        if world == 1 and not args.no_cpu_baseline:
            times_cpu, picks = cpu_reference(1, 2)
            line["cpu_baseline"] = {"value": len(picks) / times_cpu[0], "unit": "solves/s", "cores": os.cpu_count(),
                                    "kind": "port",
                                    "sample": f"2 of the 32 frequencies ({picks[0]:.0f}, {picks[-1]:.0f} Hz) with "
                                              "planning, FP64 assembly, LU and fields by the FP64 CPU restatement"}
        print(json.dumps(line), flush=True)
    solver.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
