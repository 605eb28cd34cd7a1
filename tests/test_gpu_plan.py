"""The interaction planner on the GPU (needs a B200): its plans equal the
reference's makeInteractionPlan fixtures and the host planner bit for bit,
from the sphere meshes to a thin-walled horn whose near pairs refine to
hundreds of patches, and a session planned on the device solves bit for bit
like one planned on the host."""
import time

import numpy as np
import pytest

import hornsculpt_b200 as hs
from hornsculpt_b200 import meshes

pytestmark = pytest.mark.gpu

KEYS = ("touching", "near", "patches", "whole", "trials", "offsets")
FIXTURES = {"octa2_1715": (lambda: meshes.octahedral_sphere(2), {}),
            "octa3_1000": (lambda: meshes.octahedral_sphere(3), {}),
            "ico2_3000": (lambda: meshes.icosphere(2), {}),
            "octa2_tight": (lambda: meshes.octahedral_sphere(2), {"near_relative_tolerance": 1e-6}),
            "tetra_400": (meshes.scalene_tetrahedron, {"singular_order": 12})}


@pytest.mark.parametrize("name", list(FIXTURES))
def test_device_plan_equals_reference_plan(golden, name):
    make, kw = FIXTURES[name]
    plans = golden["plans"]
    p = hs.device_plan(make(), hs.BemNumerics(**kw), float(plans[f"{name}/k"][0]))
    for key in KEYS:
        assert np.array_equal(p[key], plans[f"{name}/{key}"]), key


CASES = [
    # C1 icosphere at its 5 kHz planning frequency
    ("c1_5khz", lambda: meshes.icosphere(3), 5000.0, {}),
    # jittered ring mesh: no symmetric ties
    ("ring_sphere", lambda: meshes.revolved_sphere(h=0.012), 4000.0, {}),
    # thin-walled horn (3 mm wall, h = 12.8 mm): all-pairs mode, near pairs
    # across the wall refined to hundreds of patches at depth 6
    ("short_horn", lambda: meshes.exponential_horn(length=0.1, mouth_radius=0.05, h=0.0128), 3000.0, {}),
    ("short_horn_tight", lambda: meshes.exponential_horn(length=0.1, mouth_radius=0.05, h=0.0128), 1000.0,
     {"near_relative_tolerance": 1e-5}),
    # 0.2 mm thin box: pairs across the gap on projected patches (refined by the host's code)
    ("thin_box", lambda: meshes.thin_box(0.02, 0.02, 0.0002, 2), 1000.0, {}),
]


@pytest.mark.parametrize("name,make,f,kw", CASES, ids=[c[0] for c in CASES])
def test_device_plan_equals_host_plan(name, make, f, kw):
    mesh = make()
    k = 2 * np.pi * f / 343.0
    t0 = time.perf_counter()
    d = hs.device_plan(mesh, hs.BemNumerics(**kw), k)
    t1 = time.perf_counter()
    h = hs.host_plan(mesh, hs.BemNumerics(**kw), k)
    t2 = time.perf_counter()
    for key in KEYS:
        assert np.array_equal(d[key], h[key]), key
    s = d["stats"]
    print(f"{name}: T={mesh.triangle_count} device plan {1e3 * (t1 - t0):.1f} ms (device {s['device_ms']:.1f}, host "
          f"{s['host_ms']:.1f}), host planner {1e3 * (t2 - t1):.1f} ms; pairs {s['device_pairs']:.0f} on the device, "
          f"{s['flagged_pairs']:.0f} handed back, {s['resolved_pairs']:.0f} ordered by the host, "
          f"{s['projected_pairs']:.0f} projected")
    assert s["device_pairs"] > 0
    if name == "thin_box":
        assert s["projected_pairs"] > 0
    else:
        assert s["flagged_pairs"] <= 0.01 * s["device_pairs"]


def test_session_planned_on_the_device_solves_like_the_host_planner():
    mesh = meshes.icosphere(3)
    freqs = [300.0, 2000.0, 5000.0]
    req = hs.BemRequest(frequencies=freqs, excitations=[hs.BemExcitation("unit", [hs.FaceVelocity(1, 1.0)])],
                        observers=[(0, 0, .3), (1, 0, 0)])
    results = {}
    for planner in ("device", "host"):
        with hs.CudaBemSolver(mesh) as solver:
            solver.set_planner(planner)
            results[planner] = solver.solve(req)
            if planner == "device":
                assert solver.plan_stats()["device_pairs"] > 10000
    for a, b in zip(results["device"].frequencies, results["host"].frequencies):
        ea, eb = a.excitations[0], b.excitations[0]
        assert np.array_equal(ea.boundary.pressure_trace, eb.boundary.pressure_trace)
        assert np.array_equal(ea.observer_pressure, eb.observer_pressure)
