"""Mixed-precision form (FP32 regular/near samples with FP64 displacement and
phase, FP64 touching pairs, FP32 LU, FP64 refinement) against the FP64
oracle and the plain FP64 form (needs a B200). Contract: relative surface
pressure error <= 1e-5 and relative residual <= 1e-10."""
import numpy as np
import pytest

import hornsculpt_b200 as hs
from conftest import rel_l2
from hornsculpt_b200 import meshes
from oracle import oracle as O

pytestmark = pytest.mark.gpu

MIXED_TOL = 1e-5
MIXED = hs.BemNumerics(precision="mixed")
# The plain form solves with an FP64 LU: its relative residual sits near FP64
# round-off (about 1e-13), far below the reference's refinement target.
PLAIN_RESIDUAL = 1e-12


def test_mixed_assembly_against_oracle():
    """Entry-wise error of the mixed-form matrix: FP32 sample arithmetic only
    (a few 1e-7 of the largest entry), well inside the 1e-5 budget."""
    mesh = meshes.octahedral_sphere(3)
    rng = np.random.default_rng(3)
    q = rng.standard_normal(mesh.triangle_count) + 1j * rng.standard_normal(mesh.triangle_count)
    plan_k = 2 * np.pi * 1715 / 343
    with hs.CudaBemSolver(mesh) as solver:
        for f in (150.0, 1715.0):
            k = 2 * np.pi * f / 343
            A, b = solver.debug_assemble(MIXED, plan_k, k, q)
            Ao, bo = O.assemble(mesh, O.Numerics.default(), plan_k, k, q)
            assert np.max(np.abs(A - Ao)) <= 1e-6 * np.max(np.abs(Ao))
            assert np.max(np.abs(b - bo)) <= 1e-6 * np.max(np.abs(bo))


@pytest.mark.parametrize("make,freqs", [(lambda: meshes.octahedral_sphere(3), [100.0, 500.0, 1000.0, 1715.0]),
                                        (lambda: meshes.icosphere(3), list(np.geomspace(100, 5000, 32)))],
                         ids=["sphere512", "c1_sweep"])
def test_mixed_solve_matches_plain_form(make, freqs):
    mesh = make()
    obs = [(0, 0, .3), (1, 0, 0), (0, 0, 3)]
    exc = [hs.BemExcitation("unit", [hs.FaceVelocity(1, 1.0)])]
    with hs.CudaBemSolver(mesh) as solver:
        plain = solver.solve(hs.BemRequest(frequencies=freqs, excitations=exc, observers=obs))
        mixed = solver.solve(hs.BemRequest(frequencies=freqs, excitations=exc, observers=obs, numerics=MIXED))
    v = mesh.vertices[mesh.triangles]
    area = 0.5 * np.linalg.norm(np.cross(v[:, 1] - v[:, 0], v[:, 2] - v[:, 0]), axis=1)
    for fp, fm in zip(plain.frequencies, mixed.frequencies):
        p, m = fp.excitations[0], fm.excitations[0]
        # area-weighted relative L2 of DP0 surface pressure (tests/bem_small_mesh_parity_tests.cpp:60-76)
        err = np.sqrt((area * np.abs(m.boundary.surface_pressure - p.boundary.surface_pressure) ** 2).sum() /
                      (area * np.abs(p.boundary.surface_pressure) ** 2).sum())
        assert err <= MIXED_TOL
        assert m.boundary_residual <= 1e-10
        assert rel_l2(m.observer_pressure, p.observer_pressure) <= MIXED_TOL


@pytest.mark.parametrize("restart", [40, 2], ids=["restart40", "restart2"])
def test_mixed_gmres_ir(restart):
    """GMRES-IR: FP64 GMRES cycles preconditioned by the FP32 LU drive every
    system to <= 1e-10 relative residual; Krylov steps are reported and a short
    restart only adds outer steps. The result equals the plain form within the
    mixed-form tolerance, and repeats bit for bit."""
    mesh = meshes.octahedral_sphere(3)
    freqs = [150.0, 900.0, 1715.0]
    exc = [hs.BemExcitation("unit", [hs.FaceVelocity(1, 1.0)]),
           hs.BemExcitation("half", [hs.FaceVelocity(1, 0.5 - 0.25j)])]
    numerics = hs.BemNumerics(precision="mixed", fast_multipole=hs.FastMultipoleSettings(restart_length=restart))
    with hs.CudaBemSolver(mesh) as solver:
        plain = solver.solve(hs.BemRequest(frequencies=freqs, excitations=exc))
        first = solver.solve(hs.BemRequest(frequencies=freqs, excitations=exc, numerics=numerics))
        again = solver.solve(hs.BemRequest(frequencies=freqs, excitations=exc, numerics=numerics))
    for fp, fm, fa in zip(plain.frequencies, first.frequencies, again.frequencies):
        for p, m, a in zip(fp.excitations, fm.excitations, fa.excitations):
            assert m.boundary_residual <= 1e-10
            assert m.refinement_steps >= 1 and m.iterations >= m.refinement_steps
            assert m.iterations <= m.refinement_steps * restart
            assert rel_l2(m.boundary.pressure_trace, p.boundary.pressure_trace) <= MIXED_TOL
            assert np.array_equal(m.boundary.pressure_trace, a.boundary.pressure_trace)


def test_mixed_rejects_bad_gmres_settings():
    mesh = meshes.octahedral_sphere(2)
    numerics = hs.BemNumerics(precision="mixed", fast_multipole=hs.FastMultipoleSettings(restart_length=1))
    with hs.CudaBemSolver(mesh) as solver:
        with pytest.raises(ValueError, match="GMRES settings"):
            solver.solve(hs.BemRequest(frequencies=[500.0], excitations=[hs.BemExcitation("u", [hs.FaceVelocity(1, 1.0)])],
                                       numerics=numerics))


def test_tall_panels_on_a_cluster():
    """N = 1026 puts the first LU panels above one CTA's shared memory in both
    forms (FP64 beyond 430 rows, FP32 beyond 860): they are factored by a
    thread-block cluster. Both forms converge (the plain form within its
    reference refinement budget) and agree within the mixed tolerance."""
    mesh = meshes.octahedral_sphere(4)
    freqs = [400.0, 1300.0]
    exc = [hs.BemExcitation("unit", [hs.FaceVelocity(1, 1.0)])]
    with hs.CudaBemSolver(mesh) as solver:
        plain = solver.solve(hs.BemRequest(frequencies=freqs, excitations=exc))
        mixed = solver.solve(hs.BemRequest(frequencies=freqs, excitations=exc, numerics=MIXED))
    for fp, fm in zip(plain.frequencies, mixed.frequencies):
        p, m = fp.excitations[0], fm.excitations[0]
        assert p.boundary_residual <= PLAIN_RESIDUAL and m.boundary_residual <= 1e-10
        assert rel_l2(m.boundary.pressure_trace, p.boundary.pressure_trace) <= MIXED_TOL


@pytest.mark.parametrize("make", [lambda: meshes.octahedral_sphere(5), lambda: meshes.revolved_sphere(h=0.004)],
                         ids=["N4098", "N7899"])
def test_panels_beyond_cluster_shared_memory(make):
    """Panels taller than a full cluster's shared memory (FP64 above 8 x 384
    rows at N = 4098, FP32 above 8 x 768 rows at N = 7899) keep their extra
    rows in global memory. Both forms converge and agree within the mixed
    tolerance, so both LU paths (FP64 one-level, FP32 two-level with the
    tensor-core update) and the blocked triangular solves are exercised at
    these sizes."""
    mesh = make()
    exc = [hs.BemExcitation("unit", [hs.FaceVelocity(1, 1.0)])]
    with hs.CudaBemSolver(mesh) as solver:
        plain = solver.solve(hs.BemRequest(frequencies=[700.0], excitations=exc))
        mixed = solver.solve(hs.BemRequest(frequencies=[700.0], excitations=exc, numerics=MIXED))
    p, m = plain.frequencies[0].excitations[0], mixed.frequencies[0].excitations[0]
    assert p.boundary_residual <= PLAIN_RESIDUAL and m.boundary_residual <= 1e-10
    assert rel_l2(m.boundary.pressure_trace, p.boundary.pressure_trace) <= MIXED_TOL


def test_exactly_packed_bins_above_ten_thousand_triangles():
    """Above 10k triangles the regular pairs are binned exactly (count pass,
    on-device scan, fill pass) and the mixed form's trial-gathered columns are
    FP32. At T = 10090 both forms run that path and agree within the mixed
    tolerance; the plain form's residual meets its reference budget."""
    mesh = meshes.revolved_sphere(h=0.005)
    assert mesh.triangle_count > 10000
    exc = [hs.BemExcitation("unit", [hs.FaceVelocity(1, 1.0)])]
    with hs.CudaBemSolver(mesh) as solver:
        plain = solver.solve(hs.BemRequest(frequencies=[900.0], excitations=exc))
    with hs.CudaBemSolver(mesh) as solver:
        mixed = solver.solve(hs.BemRequest(frequencies=[900.0], excitations=exc, numerics=MIXED))
    p, m = plain.frequencies[0].excitations[0], mixed.frequencies[0].excitations[0]
    assert p.boundary_residual <= PLAIN_RESIDUAL and m.boundary_residual <= 1e-10
    assert rel_l2(m.boundary.pressure_trace, p.boundary.pressure_trace) <= MIXED_TOL
