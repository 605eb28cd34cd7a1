"""Benchmark of the exterior Burton-Miller solve on B200.

Workload (dense form): pulsating rigid sphere of radius 0.1 m as an
icosphere with 3 subdivisions (642 vertices / 1280 triangles), uniform normal
velocity 1 m/s, c = 343 m/s, rho = 1.205 kg/m^3, 32 log-spaced frequencies
100 Hz - 5 kHz, observers (0,0,.3), (1,0,0), (0,0,3). One step = one sweep of
the 32 frequency points through a solver session whose interaction plan is
cached across steps (the reference's sweep usage). Metric: frequency-point
solves per second (higher is better) of the mixed-precision form, whose
surface-pressure error against the plain FP64 form is measured in the same
run; the plain FP64 form is timed beside it.

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
METRIC = "freq-point solves/s (dense mixed-precision form at <=1e-5 surface-pressure error vs the plain FP64 form, C1 sphere sweep)"
# Algorithmic FP64 operations per regular-pair sample (one Green-kernel
# evaluation shared by both orientations of an unordered pair), counted from
# the regular-pair kernel source: displacement 15, |d|^2 5, 1/r 1, r and kr 2,
# sincos 1, weight 2, g 2, g(1+ikr) 4, 1/r^2 1, two normal projections 12,
# P and Q 4, three basis contractions 36.
FLOPS_PER_REGULAR_SAMPLE = 85
# Mixed-form regular sample (all FP32), counted from its kernel source:
# r^2 - r0^2 polynomial 10, r^2 1, 1/r 1, r 1, r + r0 1, quotient 2, phase 2,
# turns 3, reduction 4, sin and cos 2, k*r 1, weight 2, g 2, g(1+ikr) 4,
# 1/r^2 1, P 2, adjoint projection 4, Q 2, trial contractions 36.
MIXED_FP32_FLOPS_PER_SAMPLE = 81
# Per test point of a pair: the test-side contraction of the three kinds
# (54 FMA) and the double-layer projection factor (6).
MIXED_FP32_FLOPS_PER_TEST_POINT = 114
# DRAM bytes per unordered q12 pair of regularMixedKernel<12> (reads of panel
# data and bins, the two FP32 records' writes), from the ncu capture of
# regularMixedKernel<12> (ncu summary in profiles/); scaled by the pairs of a
# launch for the roofline's traffic figure.
REGULAR_Q12_DRAM_BYTES_PER_PAIR = 325
# Column gather: per ordered panel pair the three FP32 record entries of a
# column (72 B), per matrix entry the FP64 complex write (16 B).
GATHER_BYTES_PER_ORDERED_PAIR = 72
CONFIG = {"workload": "C1 icosphere s3 (642 v / 1280 t), 32 log freqs 100 Hz-5 kHz, 3 observers, dense; "
                      "mixed form timed, plain FP64 form timed beside it",
          "mesh": "icosphere-3 r=0.1 m", "frequencies": 32, "observers": 3, "excitations": 1,
          "l2": "per-sweep working set 10 GB (pair records) > 126 MB L2; L2 also flushed between steps"}


def env_rank():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def max_over_ranks(values, world, dist, torch, device):
    """Each value's maximum over the ranks (one collective of all values; the
    job's time is its slowest rank's). Identity for one rank."""
    t = torch.tensor(list(values), dtype=torch.float64, device=device)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.tolist()


def request(hs):
    return hs.BemRequest(frequencies=FREQUENCIES, observers=OBSERVERS,
                         excitations=[hs.BemExcitation("uniform", [hs.FaceVelocity(1, 1.0)])],
                         medium=hs.AcousticMedium(DENSITY, SOUND_SPEED))


def cpu_model() -> str:
    try:
        for line in pathlib.Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


_CPU_PLAN_S = None


def cpu_reference(samples: int, frequencies_per_sample: int):
    """The FP64 CPU restatement of the reference's dense path on this host's
    cores, over a bounded sample of the sweep's frequencies: FP64 assembly on
    every core, LAPACK zgetrf/zgetrs (scipy's OpenBLAS, all cores), FP64
    refinement and observer fields. Like the GPU session, the interaction plan
    (planned for the sweep's highest frequency) is built once and cached; its
    one-off time is reported separately."""
    global _CPU_PLAN_S
    from hornsculpt_b200 import meshes
    from oracle import oracle as O

    np = __import__("numpy")
    mesh = meshes.icosphere(3)
    lapack = O.use_lapack()
    if _CPU_PLAN_S is None:  # plan once for the sweep (untimed, reported beside the value)
        t0 = time.perf_counter()
        O.solve(mesh, [FREQUENCIES[0]], [[(1, 1.0)]], (), density=DENSITY, sound_speed=SOUND_SPEED,
                plan_frequencies=FREQUENCIES)
        _CPU_PLAN_S = time.perf_counter() - t0
    picks = [FREQUENCIES[int(i)] for i in np.linspace(0, 31, frequencies_per_sample)]
    times = []
    for _ in range(samples):
        t0 = time.perf_counter()
        O.solve(mesh, picks, [[(1, 1.0)]], OBSERVERS, density=DENSITY, sound_speed=SOUND_SPEED,
                plan_frequencies=FREQUENCIES)
        times.append(time.perf_counter() - t0)
    info = {"cores": os.cpu_count(), "cpu_model": cpu_model(), "lu": lapack,
            "plan_s_once": round(_CPU_PLAN_S, 3)}
    return times, picks, info


class ClockSampler:
    """SM clock, power and throttle reasons sampled during the timed region by
    an in-process NVML thread (read-only queries; one light query set per
    period, which perturbs the host's CUDA calls far less than a polling
    nvidia-smi process). Falls back to `nvidia-smi -lms` when NVML is absent."""

    REASONS = {"hw_slowdown": 0x8, "hw_thermal_slowdown": 0x40, "sw_thermal_slowdown": 0x20, "sw_power_cap": 0x4}

    def __init__(self, device_index: int, enabled: bool = True, period_s: float = 0.02):
        self.device = device_index
        self.enabled = enabled
        self.period = period_s
        self.samples = []
        self.thread = None
        self.stop = None
        self.proc = None
        self.file = None

    def __enter__(self):
        if not self.enabled:
            return self
        import threading
        try:
            import pynvml
            pynvml.nvmlInit()
            handle = pynvml.nvmlDeviceGetHandleByIndex(self.device)
        except Exception:
            self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            fields = "clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active"
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={fields}",
                                          "--format=csv,noheader,nounits", "-lms", "500"], stdout=self.file,
                                         stderr=subprocess.DEVNULL)
            return self
        self.stop = threading.Event()

        def run():
            while True:
                try:
                    sm = pynvml.nvmlDeviceGetClockInfo(handle, pynvml.NVML_CLOCK_SM)
                    mx = pynvml.nvmlDeviceGetMaxClockInfo(handle, pynvml.NVML_CLOCK_SM)
                    reasons = pynvml.nvmlDeviceGetCurrentClocksEventReasons(handle)
                    self.samples.append((sm, mx, reasons))
                except Exception:
                    pass
                if self.stop.wait(self.period):
                    return

        self.thread = threading.Thread(target=run, daemon=True)
        self.thread.start()
        return self

    def __exit__(self, *exc):
        if self.thread:
            self.stop.set()
            self.thread.join(timeout=5)
        if self.proc:
            self.proc.terminate()
            self.proc.wait(timeout=10)

    def summary(self):
        if self.file is not None:
            self.file.flush()
            for line in open(self.file.name).read().splitlines():
                parts = line.split(",")
                try:
                    self.samples.append((float(parts[0]), float(parts[1]), int(parts[3], 16)))
                except (ValueError, IndexError):
                    continue
        sm = [x[0] for x in self.samples]
        reasons = sorted({name for _, _, bits in self.samples for name, mask in self.REASONS.items() if bits & mask})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max((x[1] for x in self.samples), default=None), "reasons": reasons,
                "samples": len(sm), "source": "nvml" if self.file is None else "nvidia-smi"}


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


def fp32_peak_tflops(torch):
    """FP32 dense throughput of cuBLAS SGEMM with TF32 disabled (4096^3, best of 5)."""
    previous = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    try:
        n = 4096
        a = torch.randn(n, n, dtype=torch.float32, device="cuda")
        b = torch.randn(n, n, dtype=torch.float32, device="cuda")
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
    finally:
        torch.backends.cuda.matmul.allow_tf32 = previous


def run_reference(args, rank, world):
    if rank != 0:
        return
    from oracle import oracle as O  # noqa: F401  (built by build())
    per_step = 4
    for _ in range(args.warmup):
        cpu_reference(1, per_step)
    times = []
    for _ in range(args.steps):
        t, picks, info = cpu_reference(1, per_step)
        times += t
    value = per_step * len(times) / sum(times)
    cores = info["cores"]
    line = {"metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * sum(times) / len(times), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": CONFIG,
            "impl": "reference",
            "cpu_baseline": {"value": value, "unit": "solves/s", "cores": cores, "kind": "port",
                             "sample": f"{per_step} of the 32 sweep frequencies per step "
                                       f"({', '.join(f'{f:.0f}' for f in picks)} Hz); plan for 5 kHz built once "
                                       f"and cached like the GPU session's; FP64 assembly on {cores} threads, "
                                       f"{info['lu']}, FP64 refinement, observer fields",
                             **info},
            "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


C3_FREQUENCIES = [250.0, 1000.0, 2500.0]


def c3_cases(hs):
    """Mixed dense sizes (N = 2k, 4k, 8k, 16k complex DOFs) of the sphere and horn
    families: icosphere / octahedral sphere refinements and the seeded horn
    shell at the edge length that gives the size. A fourth element limits the
    forms run for that case."""
    m = hs.meshes
    return [("sphere", "icosphere-4 r=0.1 m", lambda: m.icosphere(4)),
            ("sphere", "octahedral-5 r=0.1 m", lambda: m.octahedral_sphere(5)),
            ("sphere", "ring-meshed sphere h=4 mm r=0.1 m seed 0", lambda: m.revolved_sphere(h=0.004)),
            ("horn", "exponential horn h=12.8 mm seed 0", lambda: m.exponential_horn(h=0.0128)),
            ("horn", "exponential horn h=9.0 mm seed 0", lambda: m.exponential_horn(h=0.0090)),
            ("horn", "exponential horn h=6.4 mm seed 0", lambda: m.exponential_horn(h=0.0064)),
            # N = 16k: the plain form's FP64 pair records alone would be 206 GB; the FP64
            # fast-multipole form at tolerance 1e-7 (the reference's tightest) is the FP64 comparison
            ("sphere", "octahedral-6 r=0.1 m", lambda: m.octahedral_sphere(6), ("mixed", "fmm64"))]


def run_c3(args):
    """Per mesh: the plain FP64 form and the mixed form (FP32 samples and LU,
    FP64 GMRES-IR to 1e-10) on the same frequencies; one JSON line each with
    the per-frequency device time of both forms and the mixed form's
    surface-pressure error against the plain form."""
    import numpy as np
    import torch

    import hornsculpt_b200 as hs

    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    cases = c3_cases(hs)
    chosen = [int(c) for c in args.c3_cases.split(",")] if args.c3_cases else range(len(cases))
    forms = tuple(args.c3_forms.split(","))
    for case in (cases[c] for c in chosen):
        if len(case) >= 4:
            forms_here = case[3]
        else:
            forms_here = forms
        family, name, make = case[:3]
        case_forms = tuple(forms_here)
        mesh = make()
        if family == "horn":
            exc = [hs.BemExcitation("throat", [hs.FaceVelocity(hs.meshes.HORN_THROAT, 1.0)])]
            obs = [(0.0, 0.0, 1.0), (0.5, 0.0, 0.8), (0.0, 0.0, -1.0)]
        else:
            exc = [hs.BemExcitation("uniform", [hs.FaceVelocity(1, 1.0)])]
            obs = OBSERVERS
        v = mesh.vertices[mesh.triangles]
        area = 0.5 * np.linalg.norm(np.cross(v[:, 1] - v[:, 0], v[:, 2] - v[:, 0]), axis=1)
        line = {"workload": "C3 mixed dense size", "family": family, "mesh": name, "N": mesh.vertex_count,
                "T": mesh.triangle_count, "frequencies": C3_FREQUENCIES}
        results = {}
        with hs.CudaBemSolver(mesh) as solver:
            solver.set_stream(stream.cuda_stream)
            for form in case_forms:
                numerics = (hs.BemNumerics(precision="fp64", acceleration="fast_multipole",
                                           relative_residual_tolerance=1e-7,
                                           fast_multipole=hs.FastMultipoleSettings(restart_length=50))
                            if form == "fmm64" else hs.BemNumerics(precision=form))
                req = hs.BemRequest(frequencies=C3_FREQUENCIES, observers=obs, excitations=exc,
                                    medium=hs.AcousticMedium(DENSITY, SOUND_SPEED), numerics=numerics)
                solver.solve(req)  # plan, workspace and warm-up
                solver.set_profiling(True)
                t0 = time.perf_counter()
                res = solver.solve(req)
                wall = time.perf_counter() - t0
                prof = solver.profile()
                solver.set_profiling(False)
                span = prof.pop("solve_span", (0.0, 0))[0]
                results[form] = res
                line[form] = {"ms_per_frequency": span / len(C3_FREQUENCIES),
                              "wall_ms_per_frequency": 1e3 * wall / len(C3_FREQUENCIES),
                              "solves_per_s": 1e3 * len(C3_FREQUENCIES) / span if span else None,
                              "kernel_ms": {k: round(v[0], 3) for k, v in sorted(prof.items(), key=lambda t: -t[1][0])[:8]},
                              "residual_max": max(e.boundary_residual for f in res.frequencies for e in f.excitations)}
                if form == "mixed":
                    line[form]["gmres_iterations"] = [e.iterations for f in res.frequencies for e in f.excitations]
        base = "fp64" if "fp64" in results else "fmm64" if "fmm64" in results else None
        if base and "mixed" in results:
            err = 0.0
            for fp, fm in zip(results[base].frequencies, results["mixed"].frequencies):
                a, b = fp.excitations[0].boundary.surface_pressure, fm.excitations[0].boundary.surface_pressure
                err = max(err, float(np.sqrt((area * np.abs(b - a) ** 2).sum() / (area * np.abs(a) ** 2).sum())))
            line[f"max_rel_err_surface_mixed_vs_{base}"] = err
            line[f"mixed_over_{base}"] = line[base]["ms_per_frequency"] / line["mixed"]["ms_per_frequency"]
        print(json.dumps(line), flush=True)
        del results
        torch.cuda.empty_cache()


C2_FREQUENCIES = [float(f) for f in __import__("numpy").geomspace(200.0, 8000.0, 16)]


def run_c2(args):
    """The C2 horn: exponential horn r(x) = r_t exp(m x), r_t = 25 mm, r_m = 150 mm,
    L = 300 mm, 3 mm wall, rear cap, throat disc driven at 1 m/s, isotropic
    h = lambda(8 kHz)/6 = 7.15 mm with +-5 % tangential jitter (seed 0); 16 log
    frequencies 200 Hz-8 kHz. The reference solves this configuration with its
    FMM; here both dense forms run (one session each, one interaction plan for
    the raster). One JSON line; the actual triangle count is in it."""
    import numpy as np
    import torch

    import hornsculpt_b200 as hs

    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    mesh = hs.meshes.exponential_horn(h=args.c2_h) if args.c2_h else hs.meshes.exponential_horn()
    v = mesh.vertices[mesh.triangles]
    area = 0.5 * np.linalg.norm(np.cross(v[:, 1] - v[:, 0], v[:, 2] - v[:, 0]), axis=1)
    exc = [hs.BemExcitation("throat", [hs.FaceVelocity(hs.meshes.HORN_THROAT, 1.0)])]
    obs = [(0.0, 0.0, 1.0), (0.5, 0.0, 0.8), (0.0, 0.0, -1.0)]
    line = {"workload": "C2 horn sweep", "mesh": "exponential horn r_t 25 mm, r_m 150 mm, L 300 mm, "
            f"wall 3 mm, h {1e3 * (args.c2_h or 0.00715):.2f} mm, seed 0", "N": mesh.vertex_count, "T": mesh.triangle_count,
            "frequencies": len(C2_FREQUENCIES), "range_hz": [200.0, 8000.0]}
    results = {}
    forms = [f for f in args.c2_forms.split(",") if f]
    for form in forms:
        with hs.CudaBemSolver(mesh) as solver:
            solver.set_stream(stream.cuda_stream)

            def request(fs):
                if form in ("fmm64", "fmm32"):  # C2 GMRES settings: restart 50, tolerance 1e-6
                    numerics = hs.BemNumerics(precision="fp64" if form == "fmm64" else "mixed",
                                              acceleration="fast_multipole", relative_residual_tolerance=1e-6,
                                              fast_multipole=hs.FastMultipoleSettings(restart_length=50))
                else:
                    numerics = hs.BemNumerics(precision=form)
                return hs.BemRequest(frequencies=fs, observers=obs, excitations=exc,
                                     medium=hs.AcousticMedium(DENSITY, SOUND_SPEED), numerics=numerics,
                                     interaction_plan_frequencies=C2_FREQUENCIES)
            t0 = time.perf_counter()
            solver.solve(request(C2_FREQUENCIES[-1:]))  # plan, workspace and warm-up
            first = time.perf_counter() - t0
            solver.set_profiling(True)
            t0 = time.perf_counter()
            res = solver.solve(request(C2_FREQUENCIES))
            wall = time.perf_counter() - t0
            prof = solver.profile()
            solver.set_profiling(False)
            span = prof.pop("solve_span", (0.0, 0))[0]
            results[form] = res
            line[form] = {"ms_per_frequency": span / len(C2_FREQUENCIES),
                          "wall_ms_per_frequency": 1e3 * wall / len(C2_FREQUENCIES),
                          "solves_per_s": 1e3 * len(C2_FREQUENCIES) / span if span else None,
                          "first_call_s_with_planning": round(first, 2),
                          "kernel_ms": {k: round(v[0], 3) for k, v in sorted(prof.items(), key=lambda t: -t[1][0])[:12]},
                          "residual_max": max(e.boundary_residual for f in res.frequencies for e in f.excitations),
                          "gmres_iterations": [f.excitations[0].iterations for f in res.frequencies]}
    # Far-field apply of the FP64 fast-multipole operator at 2 and 8 kHz: the rotational
    # M2L against its algorithmic FLOP (per link and channel 2 rotations of
    # 2 sum_n (2n+1)^2 real x complex products and the coaxial sum_m (p-m+1)^2 complex
    # products, six channels), and the same apply with the plane-wave levels.
    if "fmm64" in forms:
        apply_rows = []
        rng = np.random.default_rng(3)
        pvec = rng.normal(size=mesh.vertex_count) + 1j * rng.normal(size=mesh.vertex_count)
        fp64_peak = fp64_peak_tflops(torch)
        with hs.CudaBemSolver(mesh) as solver:
            solver.set_stream(stream.cuda_stream)
            numerics = hs.BemNumerics(precision="fp64", acceleration="fast_multipole")
            for freq in (2000.0, 8000.0):
                k = 2 * np.pi * freq / SOUND_SPEED
                row = {"frequency": freq}
                for mode, threshold in (("rotational", 1e12), ("plane_wave", 8.0)):
                    solver.set_plane_wave_threshold(threshold)
                    solver.debug_fmm_far(numerics, k, 1e-8, pvec)  # prepare, warm-up
                    solver.set_profiling(True)
                    solver.debug_fmm_far(numerics, k, 1e-8, pvec)
                    prof = solver.profile()
                    solver.set_profiling(False)
                    _, _, _, levels = solver.debug_fmm_far(numerics, k, 1e-8, pvec)
                    m2l_ms = prof.get("fmm_m2l", (0.0, 0))[0]
                    entry = {"m2l_ms": round(m2l_ms, 3),
                             "apply_ms": round(sum(v[0] for kk, v in prof.items() if kk.startswith("fmm_")), 3),
                             "levels": levels.tolist()}
                    if mode == "rotational":
                        flop = 0.0
                        for lv, p_, _nodes, links, _pw in levels.tolist():
                            rot = 2 * sum((2 * n + 1) ** 2 for n in range(p_ + 1)) * 2
                            coax = sum((p_ - m + 1) ** 2 for m in range(p_ + 1)) * 8
                            flop += links * 6 * (2 * rot + coax)
                        entry["m2l_gflop"] = round(flop / 1e9, 3)
                        entry["m2l_tflops"] = round(flop / (m2l_ms / 1e3) / 1e12, 3) if m2l_ms else None
                        entry["frac_of_dgemm"] = (round(flop / (m2l_ms / 1e3) / 1e12 / fp64_peak, 4)
                                                  if m2l_ms else None)
                    row[mode] = entry
                apply_rows.append(row)
            solver.set_plane_wave_threshold(8.0)
        line["fmm_far_apply"] = {"rows": apply_rows, "fp64_dgemm_tflops": fp64_peak,
                                 "note": "one far-field apply (P2M, M2M, M2L, L2L, L2P) at expansion tolerance 1e-8; "
                                         "CUDA events per kernel family"}
    base = "fp64" if "fp64" in results else "fmm64" if "fmm64" in results else None
    for other in [f for f in forms if f != base and base]:
        err = 0.0
        for fp, fm in zip(results[base].frequencies, results[other].frequencies):
            a, b = fp.excitations[0].boundary.surface_pressure, fm.excitations[0].boundary.surface_pressure
            err = max(err, float(np.sqrt((area * np.abs(b - a) ** 2).sum() / (area * np.abs(a) ** 2).sum())))
        line[f"max_rel_err_surface_{other}_vs_{base}"] = err
        line[f"{other}_over_{base}"] = line[base]["ms_per_frequency"] / line[other]["ms_per_frequency"]
    print(json.dumps(line), flush=True)


def run_fmm_apply(args):
    """Far-field applies of the FP64 fast-multipole operator on the C2 horn
    (the kernel-profiling case): expansion tolerance 1e-8, every level
    rotational, grouped M2L; a preparing apply, then two timed applies with
    per-kernel CUDA events. One JSON line with the levels (level, order,
    nodes, M2L links, plane wave) and the M2L milliseconds."""
    import numpy as np
    import torch

    import hornsculpt_b200 as hs

    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    mesh = hs.meshes.exponential_horn(h=args.c2_h) if args.c2_h else hs.meshes.exponential_horn()
    freq = args.apply_frequency
    k = 2 * np.pi * freq / SOUND_SPEED
    rng = np.random.default_rng(3)
    pvec = rng.normal(size=mesh.vertex_count) + 1j * rng.normal(size=mesh.vertex_count)
    numerics = hs.BemNumerics(precision="fp64", acceleration="fast_multipole")
    with hs.CudaBemSolver(mesh) as solver:
        solver.set_stream(stream.cuda_stream)
        solver.set_plane_wave_threshold(1e12)
        solver.set_fmm_grouped_m2l(True)
        _, _, _, levels = solver.debug_fmm_far(numerics, k, 1e-8, pvec)  # prepare
        solver.set_profiling(True)
        for _ in range(2):
            solver.debug_fmm_far(numerics, k, 1e-8, pvec)
        prof = solver.profile()
        solver.set_profiling(False)
    print(json.dumps({"workload": "fast-multipole far-field apply (C2 horn, all levels rotational, grouped M2L)",
                      "T": mesh.triangle_count, "frequency_hz": freq, "levels": levels.tolist(),
                      "m2l_ms_two_applies": round(prof.get("fmm_m2l", (0.0, 0))[0], 3),
                      "kernel_ms_two_applies": {kk: round(v[0], 3) for kk, v in prof.items() if kk.startswith("fmm_")}}),
          flush=True)


def run_refgpu(args):
    """C1 through HornSculpt's own GPU CudaBemSolver (compiled from the reference
    sources into oracle/_ref/reference_solve) and through the adapter over this
    library (hornsculpt_b200/adapter/adapter_solve): the same driver program and
    request, default numerics (the reference's FP32 LU with FP64 refinement; the
    adapter's plain FP64 form), 32 frequencies, one solver object per program.
    Wall-clock milliseconds of each sweep after the first (plan cached), and the
    surface-pressure difference of the two. One JSON line."""
    import numpy as np
    import struct
    from hornsculpt_b200 import meshes
    from hornsculpt_b200.build import ADAPTER_BINARY

    mesh = meshes.icosphere(3)
    work = pathlib.Path(tempfile.mkdtemp())
    with open(work / "in.bin", "wb") as f:
        f.write(struct.pack("<4Q", mesh.vertex_count, mesh.triangle_count, len(FREQUENCIES), len(OBSERVERS)))
        f.write(np.ascontiguousarray(mesh.vertices, np.float64).tobytes())
        f.write(np.ascontiguousarray(mesh.triangles, np.uint32).tobytes())
        f.write(np.ascontiguousarray(mesh.face_ids, np.uint32).tobytes())
        f.write(np.ascontiguousarray(mesh.boundary, np.uint8).tobytes())
        f.write(np.asarray(FREQUENCIES, np.float64).tobytes())
        f.write(np.asarray(OBSERVERS, np.float64).tobytes())
        f.write(np.array([DENSITY, SOUND_SPEED, 5e-5], np.float64).tobytes())
        f.write(struct.pack("<Q", args.steps + 1))
    line = {"workload": "C1 through CudaBemSolver::solve (same driver): the reference's GPU build vs the adapter "
                        "over this library", "frequencies": len(FREQUENCIES), "sweeps": args.steps}
    outputs = {}
    for name, binary in (("reference_gpu", ROOT / "oracle" / "_ref" / "reference_solve"),
                         ("this_library_adapter", ADAPTER_BINARY)):
        if not binary.exists():
            line[name] = {"unavailable": f"{binary.name} not built"}
            continue
        run = subprocess.run([str(binary), str(work / "in.bin"), str(work / f"{name}.bin")], capture_output=True,
                             text=True, timeout=1800)
        if run.returncode != 0:
            line[name] = {"failed": run.stderr.strip()[-300:]}
            continue
        info = json.loads(run.stdout.strip().splitlines()[-1])
        wall = info["wall_ms"][1:]
        line[name] = {"ms_per_sweep_median": statistics.median(wall), "ms_per_sweep": wall,
                      "first_call_ms": info["wall_ms"][0],
                      "solves_per_s": 1e3 * len(FREQUENCIES) / statistics.median(wall), "device": info["device"]}
        outputs[name] = np.fromfile(work / f"{name}.bin", np.float64)
    if len(outputs) == 2:
        N, O = mesh.vertex_count, len(OBSERVERS)
        per = 2 * N + 2 * O + 1
        v = mesh.vertices[mesh.triangles]
        area = 0.5 * np.linalg.norm(np.cross(v[:, 1] - v[:, 0], v[:, 2] - v[:, 0]), axis=1)
        worst = 0.0
        for i in range(len(FREQUENCIES)):
            a, b = (outputs[n][i * per:i * per + 2 * N].view(np.complex128)[mesh.triangles].mean(axis=1)
                    for n in ("reference_gpu", "this_library_adapter"))
            worst = max(worst, float(np.sqrt(np.sum(area * np.abs(a - b) ** 2) / np.sum(area * np.abs(b) ** 2))))
        line["max_rel_err_surface_reference_gpu_vs_plain_fp64"] = worst
        line["speedup_plain_fp64_over_reference_gpu"] = (line["reference_gpu"]["ms_per_sweep_median"] /
                                                         line["this_library_adapter"]["ms_per_sweep_median"])
    print(json.dumps(line), flush=True)


C4_FREQUENCIES = [float(f) for f in __import__("numpy").geomspace(100.0, 12000.0, 64)]


def run_c4(args):
    """Batched sweeps on larger meshes: icospheres s4 / s5 (2562 / 10242 vertices),
    64 log frequencies 100 Hz-12 kHz, one interaction plan per mesh (the raster's
    planning frequency). The mixed form solves all 64 frequencies; the plain FP64
    form solves every 8th of them (8 points, the comparison set). One JSON line per
    mesh; the third mesh is the C2 horn (12.8k triangles), driven at its throat;
    the fourth the same horn at h = 4 mm (39 776 triangles), where the dense
    forms do not fit and the fast-multipole forms run (FP64 every 8th point,
    FP32 + FP64 GMRES-IR all 64; restart 50, tolerance 1e-6)."""
    import numpy as np
    import torch

    import hornsculpt_b200 as hs

    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    sphere = [hs.BemExcitation("uniform", [hs.FaceVelocity(1, 1.0)])]
    throat = [hs.BemExcitation("throat", [hs.FaceVelocity(hs.meshes.HORN_THROAT, 1.0)])]
    plain_freqs = C4_FREQUENCIES[::8]
    only = [int(c) for c in args.c3_cases.split(",")] if args.c3_cases else None
    cases = (("icosphere-4 r=0.1 m", lambda: hs.meshes.icosphere(4), sphere),
             ("icosphere-5 r=0.1 m", lambda: hs.meshes.icosphere(5), sphere),
             ("C2 horn h=7.15 mm seed 0", lambda: hs.meshes.exponential_horn(), throat),
             ("C2 horn h=4 mm seed 0 (fast multipole)", lambda: hs.meshes.exponential_horn(h=0.004), throat))
    for c, (name, make, exc) in enumerate(cases):
        if only is not None and c not in only:
            continue
        mesh = make()
        v = mesh.vertices[mesh.triangles]
        area = 0.5 * np.linalg.norm(np.cross(v[:, 1] - v[:, 0], v[:, 2] - v[:, 0]), axis=1)
        line = {"workload": "C4 batched sweep", "mesh": name, "N": mesh.vertex_count, "T": mesh.triangle_count,
                "frequencies": {"mixed": len(C4_FREQUENCIES), "fp64": len(plain_freqs), "range_hz": [100.0, 12000.0]}}
        results = {}
        fmm = c == 3
        for form, freqs in (("fp64", plain_freqs), ("mixed", C4_FREQUENCIES)):
            # one session per form: at s5 each form's workspace alone takes over half the device
            torch.cuda.synchronize()
            line.setdefault("device_free_gib_before", {})[form] = round(torch.cuda.mem_get_info()[0] / 2**30, 1)
            with hs.CudaBemSolver(mesh) as solver:
                solver.set_stream(stream.cuda_stream)

                def request(fs):
                    numerics = (hs.BemNumerics(precision=form, acceleration="fast_multipole",
                                               relative_residual_tolerance=1e-6,
                                               fast_multipole=hs.FastMultipoleSettings(restart_length=50))
                                if fmm else hs.BemNumerics(precision=form))
                    return hs.BemRequest(frequencies=fs, observers=OBSERVERS, excitations=exc,
                                         medium=hs.AcousticMedium(DENSITY, SOUND_SPEED), numerics=numerics,
                                         interaction_plan_frequencies=C4_FREQUENCIES)
                t0 = time.perf_counter()
                solver.solve(request(freqs[-1:]))  # plan, workspace and warm-up
                first = time.perf_counter() - t0
                plan_stats = solver.plan_stats()
                solver.set_profiling(True)
                t0 = time.perf_counter()
                res = solver.solve(request(freqs))
                wall = time.perf_counter() - t0
                prof = solver.profile()
                solver.set_profiling(False)
                span = prof.pop("solve_span", (0.0, 0))[0]
                results[form] = res
                line[form] = {"ms_per_frequency": span / len(freqs), "wall_ms_per_frequency": 1e3 * wall / len(freqs),
                              "solves_per_s": 1e3 * len(freqs) / span if span else None,
                              "first_call_s_with_planning": round(first, 2),
                              "plan_device_ms": round(plan_stats["device_ms"] + plan_stats["host_ms"], 1),
                              "kernel_ms": {k: round(v[0], 3) for k, v in sorted(prof.items(), key=lambda t: -t[1][0])[:8]},
                              "residual_max": max(e.boundary_residual for f in res.frequencies for e in f.excitations)}
                if fmm:
                    line[form]["gmres_iterations"] = [f.excitations[0].iterations for f in res.frequencies]
        err = 0.0
        mixed_at = {f.frequency: f for f in results["mixed"].frequencies}
        for fp in results["fp64"].frequencies:
            a = fp.excitations[0].boundary.surface_pressure
            b = mixed_at[fp.frequency].excitations[0].boundary.surface_pressure
            err = max(err, float(np.sqrt((area * np.abs(b - a) ** 2).sum() / (area * np.abs(a) ** 2).sum())))
        line["max_rel_err_surface_mixed_vs_fp64"] = err
        line["mixed_over_fp64"] = line["fp64"]["ms_per_frequency"] / line["mixed"]["ms_per_frequency"]
        print(json.dumps(line), flush=True)
        del results
        torch.cuda.empty_cache()


def serve_stream(hs, count: int, seed: int, rate: float, distinct: int = 0, triangles=(2000, 4000), kh=1.9):
    """Seeded Poisson stream of horn requests: throat U[15, 50] mm, mouth
    U[80, 300] mm, length U[100, 600] mm, flare exponent U[1, 4], triangle
    count log-uniform in `triangles` (default [2k, 4k]), wall max(3 mm, 1.2 h)
    so the mouth rim meshes with angles >= 20 degrees, 1-16 frequencies
    log-uniform in 200 Hz-20 kHz kept where k * (longest edge) <= kh (default
    1.9, below the plan's all-pairs switch at 2; the reference's limit is
    3.25). Returns [(arrival_s, mesh, frequencies)] and the number of rejected
    frequencies."""
    import numpy as np

    rng = np.random.default_rng(seed)
    stream, t, rejected = [], 0.0, 0
    if distinct:
        # a design-iteration stream: `distinct` horns, each request a random subset of
        # its mesh's 16-point raster (passed as the planning raster, so plans are reused)
        designs, _ = serve_stream(hs, distinct, seed + 1, rate, 0, triangles, kh)
        rasters = []
        for _, mesh, _, _ in designs:
            fmax = min(20000.0, kh / mesh.max_edge() * SOUND_SPEED / (2 * math.pi))
            rasters.append([float(f) for f in np.round(np.geomspace(200.0, fmax, 16), 3)])
        while len(stream) < count:
            d = int(rng.integers(distinct))
            n = int(rng.integers(1, 17))
            freqs = sorted(rng.choice(rasters[d], size=n, replace=False).tolist())
            t += rng.exponential(1.0 / rate)
            stream.append((t, designs[d][1], freqs, rasters[d]))
        return stream, 0
    while len(stream) < count:
        throat, mouth = rng.uniform(0.015, 0.050), rng.uniform(0.080, 0.300)
        length, flare = rng.uniform(0.100, 0.600), rng.uniform(1.0, 4.0)
        target = math.exp(rng.uniform(math.log(triangles[0]), math.log(triangles[1])))
        z = np.linspace(0, length, 400)
        r = throat * np.exp(math.log(mouth / throat) * (z / length) ** flare)
        lateral = float(np.sum(np.pi * (r[1:] + r[:-1]) * np.hypot(np.diff(z), np.diff(r))))
        h = math.sqrt(2.1 * lateral / (0.433 * target))
        wall = max(0.003, 1.2 * h)
        mesh = hs.meshes.exponential_horn(throat, mouth, length, wall=wall, rear=wall, h=h,
                                          seed=int(rng.integers(1 << 31)), flare=flare)
        kmax = kh / mesh.max_edge()
        freqs = sorted(set(np.round(np.exp(rng.uniform(math.log(200), math.log(20000), int(rng.integers(1, 17)))), 3)))
        kept = [float(f) for f in freqs if 2 * math.pi * f / SOUND_SPEED <= kmax]
        rejected += len(freqs) - len(kept)
        t += rng.exponential(1.0 / rate)
        if kept:
            stream.append((t, mesh, kept, None))
    return stream, rejected


def run_serve(args):
    """Serving form on the stream above, mixed form and plain FP64 form back to
    back on the same B200: freq-point solves/s over the makespan and p50/p99
    request latency (arrival to result, measured inside the library)."""
    import threading

    import numpy as np

    import hornsculpt_b200 as hs

    stream, rejected = serve_stream(hs, args.serve_requests, args.serve_seed, args.serve_rate, args.serve_distinct,
                                    (args.serve_min_triangles, args.serve_max_triangles), args.serve_kh)
    line = {"workload": "C5 serving loop (seeded Poisson horn stream" +
                        (f", {args.serve_distinct} designs revisited" if args.serve_distinct else ", every mesh new") + ")",
            "requests": len(stream),
            "rate_per_s": args.serve_rate, "seed": args.serve_seed, "rejected_frequencies": rejected,
            "kh_limit": args.serve_kh,
            "frequency_points": sum(len(f) for _, _, f, _ in stream),
            "triangles": [min(m.triangle_count for _, m, _, _ in stream), max(m.triangle_count for _, m, _, _ in stream)]}
    for form in ("mixed", "fp64"):
        latencies, errors = [None] * len(stream), []
        runs, plans = [None] * len(stream), [None] * len(stream)
        with hs.BemServer(hs.ServeOptions(workers=args.serve_workers)) as server:
            # warm the library (CUDA context, rule tables) outside the timed stream
            warm = stream[0]
            server.wait(server.submit(meshes_warm := hs.meshes.icosphere(2), hs.BemRequest(
                frequencies=[500.0], excitations=[hs.BemExcitation("u", [hs.FaceVelocity(1, 1.0)])],
                numerics=hs.BemNumerics(precision=form))))
            del warm, meshes_warm
            tickets = [None] * len(stream)
            done = threading.Event()
            abandon = threading.Event()

            def collect():
                for i in range(len(stream)):
                    while tickets[i] is None:
                        if abandon.is_set():
                            return
                        time.sleep(0.0005)
                    if tickets[i] < 0:
                        continue
                    try:
                        result, timing = server.wait(tickets[i])
                        latencies[i] = timing.latency_ms
                        runs[i] = timing.run_ms
                        plans[i] = sum(f.interaction_plan_milliseconds for f in result.frequencies)
                    except Exception as e:  # recorded, not fatal
                        errors.append(f"{type(e).__name__}: {e}")
                done.set()

            waiter = threading.Thread(target=collect, daemon=True)
            waiter.start()
            t0 = time.perf_counter()
            try:
                for i, (arrival, mesh, freqs, raster) in enumerate(stream):
                    delay = arrival - (time.perf_counter() - t0)
                    if delay > 0:
                        time.sleep(delay)
                    req = hs.BemRequest(frequencies=freqs, observers=[(0.0, 0.0, 1.0)],
                                        excitations=[hs.BemExcitation("throat",
                                                                      [hs.FaceVelocity(hs.meshes.HORN_THROAT, 1.0)])],
                                        numerics=hs.BemNumerics(precision=form),
                                        interaction_plan_frequencies=raster or [])
                    try:
                        tickets[i] = server.submit(mesh, req)
                    except Exception as e:  # recorded, not fatal
                        errors.append(f"submit {type(e).__name__}: {e}")
                        tickets[i] = -1
            finally:
                if not done.wait(timeout=args.serve_timeout):
                    abandon.set()
                    errors.append("stream did not finish within the serving timeout")
            makespan = time.perf_counter() - t0
        ok = [x for x in latencies if x is not None]
        points = sum(len(f) for (_, _, f, _), x in zip(stream, latencies) if x is not None)
        run_ok = [x for x in runs if x is not None]
        plan_ok = [x for x in plans if x is not None]
        line[form] = {"solves_per_s": points / makespan, "makespan_s": makespan,
                      "p50_ms": float(np.percentile(ok, 50)) if ok else None,
                      "p99_ms": float(np.percentile(ok, 99)) if ok else None,
                      "run_ms_mean": float(np.mean(run_ok)) if run_ok else None,
                      "plan_ms_mean": float(np.mean(plan_ok)) if plan_ok else None,
                      "completed": len(ok), "errors": errors[:5]}
    line["mixed_over_fp64_solves_per_s"] = line["mixed"]["solves_per_s"] / line["fp64"]["solves_per_s"]
    print(json.dumps(line), flush=True)


PLAN_CASES = [
    ("C1 icosphere s3", lambda hs: hs.meshes.icosphere(3), 5000.0, {}),
    ("C2 horn h 7.15 mm", lambda hs: hs.meshes.exponential_horn(), 8000.0, {}),
    ("horn h 12.8 mm (all-pairs mode)", lambda hs: hs.meshes.exponential_horn(h=0.0128), 8000.0, {}),
    ("short horn h 12.8 mm, tol 1e-5 (all-pairs mode)",
     lambda hs: hs.meshes.exponential_horn(length=0.1, mouth_radius=0.05, h=0.0128), 1000.0,
     {"near_relative_tolerance": 1e-5}),
]


def run_plan(args):
    """Interaction planning (makeInteractionPlan) on the GPU against the host
    planner on all host threads, same mesh and planning wavenumber; wall
    clock of each, the device planner's statistics and whether the two plans
    are equal bit for bit. One JSON line per mesh."""
    import os

    import numpy as np
    import torch

    import hornsculpt_b200 as hs

    torch.cuda.set_device(0)
    cases = [c for i, c in enumerate(PLAN_CASES) if not args.c3_cases or str(i) in args.c3_cases.split(",")]
    hs.device_plan(hs.meshes.icosphere(2), hs.BemNumerics(), 10.0)  # context and module load
    for name, make, f, kw in cases:
        mesh = make(hs)
        k = 2 * np.pi * f / SOUND_SPEED
        numerics = hs.BemNumerics(**kw)
        t0 = time.perf_counter()
        d = hs.device_plan(mesh, numerics, k)
        t1 = time.perf_counter()
        h = hs.host_plan(mesh, numerics, k)
        t2 = time.perf_counter()
        equal = all(np.array_equal(d[key], h[key]) for key in ("touching", "near", "patches", "whole", "trials",
                                                                 "offsets"))
        st = d["stats"]
        # refinement kernel against the FP64 roofline: 97 FLOP per kernel sample (displacement 6,
        # distance 5 + sqrt, phase 2 + sincos, 1/r and factors 5, derivative kernel 12, weight 1,
        # 12 complex multiply-adds into the row sums 51, magnitude sums 12; sqrt, division and
        # sincos counted as 1)
        fp64 = fp64_peak_tflops(torch)
        achieved = st["samples"] * 97 / (st["refine_kernel_ms"] / 1e3) / 1e12 if st["refine_kernel_ms"] else None
        line = {"workload": "interaction planning", "mesh": name, "T": mesh.triangle_count, "frequency_hz": f,
                "numerics": kw, "device_planner_s": round(t1 - t0, 3), "host_planner_s": round(t2 - t1, 3),
                "speedup": round((t2 - t1) / (t1 - t0), 2), "host_threads": os.cpu_count(),
                "plans_equal_bit_for_bit": equal, "near_jobs": int(len(h["near"])), "patches": int(len(h["patches"])),
                "whole_panel_bytes": int(len(h["whole"])), "stats": {k2: round(v, 3) for k2, v in d["stats"].items()},
                "roofline_refine": {"bound": "fp64", "achieved": achieved, "peak": fp64, "unit": "TFLOP/s",
                                    "frac": achieved / fp64 if achieved else None,
                                    "algorithmic": f"{st['samples']:.0f} kernel samples x 97 FP64 FLOP",
                                    "peak_source": "cuBLAS DGEMM measured in this run"}}
        print(json.dumps(line), flush=True)


def roofline_components(form, mesh, frequencies, steps, fp32_tflops, hbm_gbs):
    """Per kernel family of the mixed C1 sweep: share of device time, bound,
    algorithmic work per sweep, achieved rate and fraction of its peak, and the
    time-weighted sum of the fractions (families without a roofline, the
    latency-bound ones, count with fraction 0). Work per sweep: regular pairs
    from the library's pair counters (samples x 81 + test points x 114 FP32
    FLOP), touching and near pairs from its sample counters at the regular
    sample's 85 FLOP (the same integrand), the column gather 72 B per ordered
    panel pair and 16 B per matrix entry written, the LU 8 N^3 / 3 real FLOP
    per matrix, the FP64 residual 16 B per matrix entry per evaluation."""
    prof, work = form["profile"], form["work"]
    T, N, F = mesh.triangle_count, mesh.vertex_count, frequencies
    total = sum(v[0] for v in prof.values()) / steps
    ms = lambda *keys: sum(prof[k][0] for k in prof if any(k.startswith(p) for p in keys)) / steps  # noqa: E731
    launches = lambda key: prof.get(key, (0.0, 0))[1] / steps  # noqa: E731
    reg_flop = sum(work.get(f"pairs_q{n}", 0) * (n * n * MIXED_FP32_FLOPS_PER_SAMPLE + n * MIXED_FP32_FLOPS_PER_TEST_POINT)
                   for n in (6, 12, 16, 64)) / steps
    rows = [
        ("regular pairs", ms("regular_mixed_q"), "fp32", reg_flop, "FLOP"),
        ("touching pairs", ms("singular_mixed"), "fp32", work.get("singular_samples", 0) / steps * 85, "FLOP"),
        ("near pairs", ms("near"), "fp32", work.get("near_samples", 0) / steps * 85, "FLOP"),
        ("column gather", ms("gather_column"), "hbm", F * (T * T * GATHER_BYTES_PER_ORDERED_PAIR + N * N * 16), "B"),
        ("LU factorisation", ms("lu_panel", "lu_gemm", "lu_pack", "lu_swap", "lu_trsm"), "fp32", F * 8 * N ** 3 / 3,
         "FLOP"),
        ("FP64 residual", ms("residual"), "hbm", launches("residual") * F * N * N * 16, "B"),
    ]
    comps, weighted, covered = [], 0.0, 0.0
    for name, t_ms, bound, amount, unit in rows:
        if t_ms <= 0:
            continue
        rate = amount / (t_ms / 1e3)
        peak = fp32_tflops * 1e12 if bound == "fp32" else (hbm_gbs or 0) * 1e9
        frac = rate / peak if peak else None
        share = t_ms / total
        comps.append({"family": name, "ms_per_sweep": round(t_ms, 4), "share": round(share, 4), "bound": bound,
                      "work_per_sweep": amount, "unit": unit, "achieved": rate, "frac": frac})
        weighted += share * (frac or 0.0)
        covered += share
    return {"components": comps, "time_weighted_frac": weighted, "share_with_roofline": covered,
            "peaks": {"fp32_tflops_sgemm": fp32_tflops, "hbm_gbs": hbm_gbs},
            "note": "kernels outside these families (pair classification, right-hand sides, triangular solves, "
                    "GMRES-IR orthogonalisation, fields) are latency-bound and count with fraction 0"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)  # >= 3 for reported numbers
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-clock-sampler", action="store_true", help="skip nvidia-smi sampling (diagnostics)")
    ap.add_argument("--sweep-frequencies", type=int, default=32,
                    help="solve only n sweep frequencies (small profiling cases)")
    ap.add_argument("--first-frequency", type=int, default=0,
                    help="index of the first sweep frequency solved (small profiling cases)")
    ap.add_argument("--workload", default="c1",
                    choices=["c1", "c2", "c3", "c4", "serve", "refgpu", "plan", "fmm-apply"],
                    help="c1: the headline sweep; c2: the 12.8k-triangle horn sweep (dense forms); "
                         "c3: mixed dense sizes N = 2k-16k (one line per mesh); "
                         "c4: 64-frequency sweeps on icospheres s4/s5; "
                         "serve: the serving loop on a seeded Poisson horn stream; "
                         "plan: interaction planning on the device against the host planner; "
                         "fmm-apply: far-field applies of the fast-multipole operator (kernel profiling)")
    ap.add_argument("--apply-frequency", type=float, default=2000.0, help="fmm-apply: frequency in Hz")
    ap.add_argument("--c3-cases", default="", help="c3/c4: comma-separated case indices (default: all)")
    ap.add_argument("--c2-h", type=float, default=0.0,
                    help="C2 edge length in metres (0: 7.15 mm, the spec's lambda(8 kHz)/6)")
    ap.add_argument("--c2-forms", default="fp64,mixed,fmm64,fmm32",
                    help="C2 forms: fp64 and mixed dense, fmm64 the FP64 fast-multipole form")
    ap.add_argument("--c3-forms", default="fp64,mixed", help="c3: forms to run (the error needs both)")
    ap.add_argument("--serve-requests", type=int, default=60)
    ap.add_argument("--serve-rate", type=float, default=1.0, help="mean arrivals per second")
    ap.add_argument("--serve-timeout", type=float, default=400.0, help="seconds to wait for a stream to drain")
    ap.add_argument("--serve-seed", type=int, default=2026)
    ap.add_argument("--serve-workers", type=int, default=4)
    ap.add_argument("--serve-min-triangles", type=int, default=2000)
    ap.add_argument("--serve-max-triangles", type=int, default=4000)
    ap.add_argument("--serve-kh", type=float, default=1.9,
                    help="frequencies kept where k x longest edge <= this (the reference's limit is 3.25)")
    ap.add_argument("--serve-distinct", type=int, default=0,
                    help="> 0: requests revisit this many horn designs (planning rasters reused)")
    args = ap.parse_args()
    rank, world, local = env_rank()
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.workload == "c3":
        return run_c3(args)
    if args.workload == "c4":
        return run_c4(args)
    if args.workload == "c2":
        return run_c2(args)
    if args.workload == "serve":
        return run_serve(args)
    if args.workload == "refgpu":
        return run_refgpu(args)
    if args.workload == "plan":
        return run_plan(args)
    if args.workload == "fmm-apply":
        return run_fmm_apply(args)

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
    req.frequencies = FREQUENCIES[args.first_frequency: args.first_frequency + args.sweep_frequencies]
    req.interaction_plan_frequencies = FREQUENCIES
    solver = hs.CudaBemSolver(mesh)
    solver.set_stream(stream.cuda_stream)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()

    peaks = measured_peaks()
    fp64 = fp64_peak_tflops(torch)
    fp32 = fp32_peak_tflops(torch)

    def run_form(precision):
        """Warm-up, then the timed steps of one precision form; device and wall seconds (max over ranks)."""
        req.numerics = hs.BemNumerics(precision=precision)
        for _ in range(args.warmup):
            solver.solve(req)
        solver.set_profiling(True)
        device_s, wall_s, result = 0.0, 0.0, None
        step_ms, phase_ms, e2e_ms = [], [], []
        barrier()
        with ClockSampler(local, enabled=not args.no_clock_sampler) as clocks:
            for _ in range(args.steps):
                with torch.cuda.stream(stream):
                    flush.zero_()
                start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                start.record(stream)
                result = solver.solve(req)
                end.record(stream)
                end.synchronize()
                device_s += start.elapsed_time(end) / 1e3
                step_ms.append(round(start.elapsed_time(end), 2))
                phase_ms.append(round(sum(f.assembly_milliseconds + f.solve_milliseconds + f.field_milliseconds
                                          for f in result.frequencies), 2))
            # e2e: the same steps through the public API with the library's kernel
            # profiling off (its per-family event records are instrumentation, not work)
            profile, work = solver.profile(), solver.work()
            solver.set_profiling(False)
            launches0 = solver.graph_launches()
            plain_s = 0.0
            for _ in range(args.steps):
                with torch.cuda.stream(stream):
                    flush.zero_()
                stream.synchronize()
                start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                t0 = time.perf_counter()
                start.record(stream)
                solver.solve(req)
                end.record(stream)
                wall_s += time.perf_counter() - t0
                e2e_ms.append(round(1e3 * (time.perf_counter() - t0), 2))
                end.synchronize()
                plain_s += start.elapsed_time(end) / 1e3
            graph_replays = solver.graph_launches() - launches0
        barrier()
        span = profile.pop("solve_span", (0.0, 0))[0] / 1e3
        device_s, wall_s, plain_s, span = max_over_ranks([device_s, wall_s, plain_s, span], world, dist, torch, "cuda")
        return dict(device_s=device_s, wall_s=wall_s, span_s=span, result=result, profile=profile, work=work,
                    clocks=clocks.summary(), step_ms=step_ms, phase_ms=phase_ms, e2e_ms=e2e_ms, plain_s=plain_s,
                    graph_replays=graph_replays)

    plain = run_form("fp64")
    mixed = run_form("mixed")
    points = len(req.frequencies) * args.steps * world
    if rank == 0:
        def regular_stats(form, prefix):
            prof = form["profile"]
            keys = [k for k in prof if k.startswith(prefix)]
            ms = sum(prof[k][0] for k in keys)
            return ms, sum(v[0] for v in prof.values())

        p_ms, p_total = regular_stats(plain, "regular_q")
        m_ms, m_total = regular_stats(mixed, "regular_mixed_q")
        p_samples = plain["work"]["regular_samples"]
        p_achieved = p_samples * FLOPS_PER_REGULAR_SAMPLE / (p_ms / 1e3) / 1e12
        # the mixed form's single largest launch: regularMixedKernel<12>, one launch per step
        q12_ms = mixed["profile"].get("regular_mixed_q12", (0.0, 0))[0] / args.steps
        q12_pairs = mixed["work"]["pairs_q12"] / args.steps
        q12_flop = q12_pairs * (144 * MIXED_FP32_FLOPS_PER_SAMPLE + 12 * MIXED_FP32_FLOPS_PER_TEST_POINT)
        m32 = q12_flop / (q12_ms / 1e3) / 1e12 if q12_ms > 0 else 0.0
        # area-weighted relative L2 of DP0 surface pressure, mixed vs plain, worst frequency
        v = mesh.vertices[mesh.triangles]
        area = 0.5 * np.linalg.norm(np.cross(v[:, 1] - v[:, 0], v[:, 2] - v[:, 0]), axis=1)
        err = 0.0
        for fp, fm in zip(plain["result"].frequencies, mixed["result"].frequencies):
            a, b = fp.excitations[0].boundary.surface_pressure, fm.excitations[0].boundary.surface_pressure
            err = max(err, float(np.sqrt((area * np.abs(b - a) ** 2).sum() / (area * np.abs(a) ** 2).sum())))
        T, N, O = mesh.triangle_count, mesh.vertex_count, len(OBSERVERS)
        F = len(req.frequencies)
        h2d = F * (T * 16 + 8) + O * 24
        d2h = F * (N * 16 + O * 16 + 32)
        # value: CUDA events on the session stream around each sweep with kernel profiling
        # off (the production configuration: dense chains replayed as graphs)
        value = points / mixed["plain_s"]
        line = {
            "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * mixed["plain_s"] / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64 (mixed form)", "data": "synthetic",
            "config": CONFIG,
            "e2e": {"value": points / mixed["wall_s"], "unit": "solves/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "gpu_launches": int(sum(v[1] for v in mixed["profile"].values())),
            "forms": {
                "fp64_plain": {"value": points / plain["plain_s"], "e2e": points / plain["wall_s"],
                               "ms_per_step": 1e3 * plain["plain_s"] / args.steps,
                               "value_profiled": points / plain["span_s"], "graph_replays": plain["graph_replays"],
                               "step_ms": plain["step_ms"], "phase_ms": plain["phase_ms"], "e2e_ms": plain["e2e_ms"],
                               "residual_max": max(e.boundary_residual for f in plain["result"].frequencies
                                                   for e in f.excitations)},
                "mixed": {"value": value, "e2e": points / mixed["wall_s"],
                          "ms_per_step": 1e3 * mixed["plain_s"] / args.steps,
                          "value_profiled": points / mixed["span_s"], "graph_replays": mixed["graph_replays"],
                          "step_ms": mixed["step_ms"], "phase_ms": mixed["phase_ms"], "e2e_ms": mixed["e2e_ms"],
                          "residual_max": max(e.boundary_residual for f in mixed["result"].frequencies
                                              for e in f.excitations),
                          "max_rel_err_surface_vs_fp64": err},
                "mixed_over_fp64": plain["plain_s"] / mixed["plain_s"],
                "timing": "value: CUDA events on the session stream around each sweep (first upload to last "
                          "result download, host control included) with kernel profiling off, so the dense batch "
                          "chain replays as a CUDA graph; value_profiled: the library's in-sweep span over steps "
                          "run with per-kernel CUDA-event profiling on (plain launches), the source of kernel_ms "
                          "and the roofline; e2e: wall clock of the same unprofiled Python API calls with host "
                          "request and result buffers",
            },
            "roofline": {"kernel": "regularMixedKernel<12> (mixed form, largest launch)", "bound": "fp32",
                         "achieved": m32, "peak": fp32, "unit": "TFLOP/s", "frac": m32 / fp32,
                         "peak_source": "cuBLAS SGEMM (TF32 off) 4096^3 measured in this run; MEASURED_PEAKS.json "
                                        "has no FP32 figure",
                         "traffic": (REGULAR_Q12_DRAM_BYTES_PER_PAIR * q12_pairs
                                     if REGULAR_Q12_DRAM_BYTES_PER_PAIR else None),
                         "traffic_note": "DRAM bytes per launch: ncu bytes per q12 pair x pairs of the launch",
                         "launch_ms": q12_ms, "pairs_per_launch": q12_pairs,
                         "share_of_device_time": q12_ms * args.steps / m_total,
                         "algorithmic": f"per q12 pair 144 samples x {MIXED_FP32_FLOPS_PER_SAMPLE} + 12 test points "
                                        f"x {MIXED_FP32_FLOPS_PER_TEST_POINT} FP32 FLOP"},
            "roofline_fp64_plain": {"kernel": "regularPairsKernel (4 rule sizes)", "bound": "fp64",
                                    "achieved": p_achieved, "peak": fp64, "unit": "TFLOP/s", "frac": p_achieved / fp64,
                                    "share_of_device_time": p_ms / p_total,
                                    "algorithmic": f"{p_samples} samples x {FLOPS_PER_REGULAR_SAMPLE} FLOP"},
            "kernel_ms": {"mixed": {k: round(v[0] / args.steps, 4) for k, v in sorted(mixed["profile"].items())},
                          "fp64_plain": {k: round(v[0] / args.steps, 4) for k, v in sorted(plain["profile"].items())}},
            "clocks": mixed["clocks"], "clocks_fp64_plain": plain["clocks"],
            "peaks": {"hbm_gbs": peaks.get("hbm_gbs"), "fp64_tflops_dgemm": fp64, "fp32_tflops_sgemm": fp32},
        }
        line["roofline_components"] = roofline_components(mixed, mesh, len(req.frequencies), args.steps, fp32,
                                                          peaks.get("hbm_gbs"))
        if world == 1 and not args.no_cpu_baseline:
            times_cpu, picks, info = cpu_reference(2, 4)
            line["cpu_baseline"] = {"value": len(picks) * len(times_cpu) / sum(times_cpu), "unit": "solves/s",
                                    "kind": "port",
                                    "sample": f"4 of the 32 frequencies ({', '.join(f'{f:.0f}' for f in picks)} Hz), "
                                              "2 repeats; plan for 5 kHz built once and cached like the GPU session's; "
                                              f"FP64 assembly on {info['cores']} threads, {info['lu']}, FP64 "
                                              "refinement and observer fields by the FP64 CPU restatement",
                                    **info}
        print(json.dumps(line), flush=True)
    solver.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
