"""The device interaction planner's algorithm, run on the host with one lane
per warp (hs_bem_debug_plan_device mode 1): its plans equal the reference's
makeInteractionPlan fixtures and the host planner bit for bit. The same
template code runs with 32 lanes on the GPU (tests/test_gpu_plan.py)."""
import numpy as np
import pytest

import hornsculpt_b200 as hs
from hornsculpt_b200 import meshes

KEYS = ("touching", "near", "patches", "whole", "trials", "offsets")
CASES = {"octa2_1715": (lambda: meshes.octahedral_sphere(2), {}),
         "octa3_1000": (lambda: meshes.octahedral_sphere(3), {}),
         "ico2_3000": (lambda: meshes.icosphere(2), {}),
         "octa2_tight": (lambda: meshes.octahedral_sphere(2), {"near_relative_tolerance": 1e-6}),
         "tetra_400": (meshes.scalene_tetrahedron, {"singular_order": 12})}


@pytest.mark.parametrize("name", list(CASES))
def test_emulated_device_plan_equals_reference_plan(golden, name):
    make, kw = CASES[name]
    plans = golden["plans"]
    p = hs.device_plan(make(), hs.BemNumerics(**kw), float(plans[f"{name}/k"][0]), emulate=True)
    for key in KEYS:
        assert np.array_equal(p[key], plans[f"{name}/{key}"]), key
    s = p["stats"]
    # ties of the octahedral meshes' mirror-image leaves go to the host; the
    # rest is refined by the device algorithm
    assert s["flagged_pairs"] <= 0.05 * max(s["device_pairs"], 1)


def test_emulated_device_plan_equals_host_plan_on_a_jittered_mesh():
    """A ring-meshed sphere with node jitter: no symmetric ties."""
    mesh = meshes.revolved_sphere(h=0.012)
    k = 2 * np.pi * 4000 / 343
    d = hs.device_plan(mesh, hs.BemNumerics(), k, emulate=True)
    h = hs.host_plan(mesh, hs.BemNumerics(), k)
    for key in KEYS:
        assert np.array_equal(d[key], h[key]), key
    assert d["stats"]["device_pairs"] > 10000 and d["stats"]["flagged_pairs"] == 0


def test_device_plan_validates_like_the_host_plan():
    mesh = meshes.octahedral_sphere(1)
    with pytest.raises(ValueError, match="interaction-plan input"):
        hs.device_plan(mesh, hs.BemNumerics(near_maximum_depth=17), 10.0, emulate=True)


def test_emulated_device_plan_hands_projected_pairs_to_the_host():
    """A 0.2 mm thin box: panels facing each other across the gap are integrated on
    projected patches by the host planner's code; the merged plan is the host's."""
    mesh = meshes.thin_box(0.02, 0.02, 0.0002, 2)
    k = 2 * np.pi * 1000 / 343
    d = hs.device_plan(mesh, hs.BemNumerics(), k, emulate=True)
    h = hs.host_plan(mesh, hs.BemNumerics(), k)
    for key in KEYS:
        assert np.array_equal(d[key], h[key]), key
    assert d["stats"]["projected_pairs"] > 0 and (h["patches"][:, 20] == 1).any()
