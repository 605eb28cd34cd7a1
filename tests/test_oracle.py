"""The FP64 CPU oracle pinned against the reference's golden data, closed
forms and the reference's own compiled planner (no GPU)."""
from math import factorial

import numpy as np
import pytest

from conftest import analytic_sphere, rel_l2
from hornsculpt_b200 import meshes
from oracle import oracle as O


def test_reference_rules_are_exact(golden):
    """The reference's triangle rules (pair_quadrature.cpp:715-769), as pinned
    in the fixture, have unit measure 1/2 and their documented polynomial
    exactness; its Gauss-Legendre rules integrate x^(2n-1) exactly."""
    for d, pts in golden["rules"]["triangle"].items():
        pts, d = np.array(pts), int(d)
        assert abs(pts[:, 3].sum() - .5) < 3e-15
        for a in range(d + 1):
            for b in range(d + 1 - a):
                exact = factorial(a) * factorial(b) / factorial(a + b + 2)
                assert abs((pts[:, 3] * pts[:, 1] ** a * pts[:, 2] ** b).sum() - exact) < 4e-15
    for n, g in golden["rules"]["gauss"].items():
        g, n = np.array(g), int(n)
        assert abs((g[:, 1] * g[:, 0] ** (2 * n - 1)).sum() - 1 / (2 * n)) < 1e-14


def test_beat_sphere_observer_pressure(golden):
    """Observer pressure on the 512-triangle sphere agrees with the external
    BEAT FP64 reference below 1e-6 relative L2 (docs/BURTON-MILLER.md:202-204)."""
    g = golden["sphere"]
    freqs = [row["frequency"] for row in g["rows"]]
    r = O.solve(meshes.octahedral_sphere(3), freqs, [[(1, 1.0)]], g["observers"], density=g["density"])
    for i, row in enumerate(g["rows"]):
        ref = np.array([complex(*p) for p in row["pressure"]])
        assert rel_l2(r["observer"][i, 0], ref) < 1e-6
        assert r["residual"][i, 0] < 1e-12


def test_beat_tetra_singular_ports(golden):
    """Port mean pressures of the scalene tetrahedron (every pair touching:
    Sauter-Schwab order 12 only) match BEAT's FP64 LU to 1e-8."""
    g = golden["tetra"]
    m = meshes.scalene_tetrahedron()
    names = list(g["excitations"])
    exc = [[(f, v) for f, v in g["excitations"][n]] for n in names]
    r = O.solve(m, [g["frequency"]], exc, [], density=g["density"],
                numerics=O.Numerics.default(singular_order=g["singular_order"]))
    v = m.vertices[m.triangles]
    area = 0.5 * np.linalg.norm(np.cross(v[:, 1] - v[:, 0], v[:, 2] - v[:, 0]), axis=1)
    for port in g["ports"]:
        e = names.index(port["excitation"])
        sel = m.face_ids == port["face"]
        assert abs(area[sel].sum() - port["area"]) < 1e-15
        mean = (r["surface"][0, e][sel] * area[sel]).sum() / area[sel].sum()
        ref = complex(*port["mean_pressure"])
        assert abs(mean - ref) / abs(ref) < 1e-8


def test_analytic_sphere_discretisation():
    """Pulsating sphere within the discretisation error of 512 triangles
    (analytic p(a) = rho c v ika/(1+ika)); the reference's own 512-triangle
    level is 2.5% (docs/BURTON-MILLER.md:101-105)."""
    obs = [(0, 0, .3), (1, 0, 0), (0, 0, 3)]
    r = O.solve(meshes.octahedral_sphere(3), [100.0, 1000.0], [[(1, 1.0)]], obs)
    for i, f in enumerate([100.0, 1000.0]):
        for j, rad in enumerate([.3, 1.0, 3.0]):
            assert abs(r["observer"][i, 0, j] / analytic_sphere(f, rad) - 1) < 0.03


@pytest.mark.parametrize("order,tol", [(4, 2e-4), (8, 2e-6), (16, 2e-12)])
def test_coincident_laplace_closed_form(order, tol):
    """int_T int_T 1/|x-y| on the unit right triangle = (2+sqrt 2) asinh(1)/3
    (tests/pair_quadrature_tests.cpp:225-243)."""
    tri = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], float)
    value = O.laplace_pair(tri, [0, 1, 2], tri, [0, 1, 2], order)
    assert abs(value - (2 + np.sqrt(2)) * np.arcsinh(1) / 3) < tol


def test_oracle_plan_matches_reference_fixtures(golden):
    """The oracle's restated plan equals the reference's own makeInteractionPlan."""
    plans = golden["plans"]
    cases = {"octa2_1715": (meshes.octahedral_sphere(2), {}), "ico2_3000": (meshes.icosphere(2), {}),
             "octa2_tight": (meshes.octahedral_sphere(2), {"near_tol": 1e-6}),
             "tetra_400": (meshes.scalene_tetrahedron(), {"singular_order": 12})}
    for name, (mesh, kw) in cases.items():
        p = O.oracle_plan(mesh, O.Numerics.default(**kw), float(plans[f"{name}/k"][0]))
        for key in ("touching", "near", "patches", "whole", "trials", "offsets"):
            assert np.array_equal(p[key], plans[f"{name}/{key}"]), (name, key)


@pytest.mark.skipif(not O.reference_available(), reason="oracle/_ref not built (reference tree absent)")
def test_patch_estimates_match_reference():
    """Embedded 6/8 and 12/14 estimates, including a projected patch, agree with
    the reference's estimatePairPatchCpu."""
    a = np.array([[0, 0, 0], [.01, 0, 0], [0, .01, 0]], float)
    b = np.array([[.002, .002, .0004], [.012, .002, .0004], [.002, .012, .0002]], float)
    for proj, deg, iv in [(0, 8, 1), (0, 14, 1), (1, 8, 1), (1, 8, 2)]:
        patch = np.zeros(22)
        patch[0:9] = [1, 0, 0, 0, 1, 0, 0, 0, 1]
        patch[9:18] = [1, 0, 0, 0, 1, 0, 0, 0, 1]
        patch[18:22] = [1.0, deg, proj, iv]
        mo, eo = O.estimate_patch("oracle", a, b, [0, 1, 2], [3, 4, 5], patch, 30.0)
        mr, er = O.estimate_patch("ref", a, b, [0, 1, 2], [3, 4, 5], patch, 30.0)
        assert np.max(np.abs(mo - mr)) <= 1e-13 * np.max(np.abs(mr))
        assert np.allclose(eo, er, rtol=1e-9, atol=1e-18)


@pytest.mark.skipif(not O.reference_available(), reason="oracle/_ref not built (reference tree absent)")
def test_reference_pressure_field_pulsating_sphere():
    """HornSculpt's own evaluatePressureField (compiled into oracle/_ref), fed
    the analytic pulsating-sphere traces on icosphere s3: points inside are
    excluded, a point 0.1 um off the surface is boundary, air points (one
    0.5 mm off the surface, which needs adaptive subdivision) agree with the
    analytic field to the mesh's discretisation error."""
    mesh = meshes.icosphere(3)
    a, c, rho, f, v = 0.1, 343.0, 1.21, 500.0, 1.0
    k = 2 * np.pi * f / c

    def exact(r):
        return rho * c * v * (1j * k * a / (1 + 1j * k * a)) * (a / r) * np.exp(-1j * k * (r - a))

    trace = exact(np.linalg.norm(mesh.vertices, axis=1))
    q = np.full(mesh.triangle_count, -1j * rho * 2 * np.pi * f * v)
    pts = np.array([(0, 0, .3), (.2, .1, 0), (0, 0, 0), (.1000001, 0, 0), (0, 0, .1005)])
    p, status = O.reference_pressure_field(mesh, f, c, trace, q, pts)
    assert list(status) == [0, 0, 2, 1, 0]
    for i in (0, 1, 4):
        r = np.linalg.norm(pts[i])
        assert abs(p[i] - exact(r)) <= 1e-2 * abs(exact(r))
    assert p[2] == 0 and p[3] == 0
    with pytest.raises(ValueError, match="Invalid pressure field settings"):
        O.reference_pressure_field(mesh, f, c, trace, q, pts, tolerance=0.5)
