"""CUDA plain-form parity through the C ABI against the FP64 CPU oracle, the
reference's golden data and the analytic sphere (needs a B200)."""
import numpy as np
import pytest

import hornsculpt_b200 as hs
from conftest import analytic_sphere, rel_l2
from hornsculpt_b200 import meshes
from oracle import oracle as O

pytestmark = pytest.mark.gpu

# Plain FP64 form: entry-wise assembly parity relative to the largest entry,
# solution parity in relative L2 (1e-9 for the FP64 form).
ASSEMBLY_TOL = 1e-12
SOLVE_TOL = 1e-9


def _oracle_numerics(n: hs.BemNumerics):
    return O.Numerics.default(quadrature_order=n.quadrature_order, singular_order=n.singular_order,
                              near_ratio=n.near_distance_ratio, near_tol=n.near_relative_tolerance,
                              near_depth=n.near_maximum_depth, residual_tol=n.relative_residual_tolerance,
                              max_refine=n.maximum_refinement_steps)


ASSEMBLY_CASES = [
    ("octa2", lambda: meshes.octahedral_sphere(2), hs.BemNumerics(), 1715.0, [100.0, 1000.0, 1715.0]),
    ("ico2", lambda: meshes.icosphere(2), hs.BemNumerics(), 3000.0, [250.0, 3000.0]),
    ("octa2_allpairs", lambda: meshes.octahedral_sphere(2), hs.BemNumerics(near_relative_tolerance=1e-6), 2000.0,
     [2000.0]),
    ("tetra_s12", meshes.scalene_tetrahedron, hs.BemNumerics(singular_order=12), 400.0, [400.0]),
    ("octa3_s6", lambda: meshes.octahedral_sphere(3), hs.BemNumerics(singular_order=6), 1000.0, [700.0]),
]


@pytest.mark.parametrize("name,make,numerics,plan_f,freqs", ASSEMBLY_CASES, ids=[c[0] for c in ASSEMBLY_CASES])
def test_assembly_matches_oracle(name, make, numerics, plan_f, freqs):
    """Row-equilibrated A and B q, entry by entry, against the oracle's FP64
    assembly with the identical plan."""
    mesh = make()
    rng = np.random.default_rng(7)
    q = (rng.standard_normal(mesh.triangle_count) + 1j * rng.standard_normal(mesh.triangle_count)) * 100
    plan_k = 2 * np.pi * plan_f / 343.0
    with hs.CudaBemSolver(mesh) as solver:
        for f in freqs:
            k = 2 * np.pi * f / 343.0
            A, b = solver.debug_assemble(numerics, plan_k, k, q)
            Ao, bo = O.assemble(mesh, _oracle_numerics(numerics), plan_k, k, q)
            assert np.max(np.abs(A - Ao)) <= ASSEMBLY_TOL * np.max(np.abs(Ao)), (name, f)
            assert np.max(np.abs(b - bo)) <= ASSEMBLY_TOL * np.max(np.abs(bo)), (name, f)


def _request(freqs, obs, excitations=None, **kw):
    excitations = excitations or [hs.BemExcitation("unit", [hs.FaceVelocity(1, 1.0)])]
    return hs.BemRequest(frequencies=freqs, excitations=excitations, observers=obs, **kw)


def test_solve_matches_oracle_and_beat(golden):
    """512-triangle sphere: traces, DP0 pressure and observer pressure equal the
    oracle to 1e-9 and the external BEAT FP64 reference below 1e-6."""
    g = golden["sphere"]
    mesh = meshes.octahedral_sphere(3)
    freqs = [row["frequency"] for row in g["rows"]]
    with hs.CudaBemSolver(mesh) as solver:
        res = solver.solve(_request(freqs, g["observers"]))
    ref = O.solve(mesh, freqs, [[(1, 1.0)]], g["observers"], density=1.21)
    for i, row in enumerate(g["rows"]):
        ex = res.frequencies[i].excitations[0]
        assert rel_l2(ex.boundary.pressure_trace, ref["trace"][i, 0]) < SOLVE_TOL
        assert rel_l2(ex.boundary.surface_pressure, ref["surface"][i, 0]) < SOLVE_TOL
        assert rel_l2(ex.observer_pressure, ref["observer"][i, 0]) < SOLVE_TOL
        assert ex.boundary_residual < 1e-12 and ex.refinement_steps == 0
        assert (ex.field_quadrature_comparison_degree, ex.field_quadrature_verification_degree) == \
            tuple(ref["field_degrees"][i, 0])
        beat = np.array([complex(*p) for p in row["pressure"]])
        assert rel_l2(ex.observer_pressure, beat) < 1e-6
        z = ex.impedances[0]
        assert abs(z.mean_pressure / z.volume_velocity - z.volume_impedance) < 1e-8 * abs(z.volume_impedance)


def test_singular_ports_match_beat(golden):
    """Scalene tetrahedron, every panel pair touching, singular order 12:
    port mean pressures against BEAT's FP64 LU."""
    g = golden["tetra"]
    mesh = meshes.scalene_tetrahedron()
    excitations = [hs.BemExcitation(n, [hs.FaceVelocity(f, v) for f, v in faces]) for n, faces in
                   g["excitations"].items()]
    with hs.CudaBemSolver(mesh) as solver:
        res = solver.solve(hs.BemRequest(frequencies=[g["frequency"]], excitations=excitations,
                                         numerics=hs.BemNumerics(singular_order=12)))
    names = list(g["excitations"])
    for port in g["ports"]:
        ex = res.frequencies[0].excitations[names.index(port["excitation"])]
        imp = {z.face_id: z for z in ex.impedances}[port["face"]]
        ref = complex(*port["mean_pressure"])
        assert abs(imp.mean_pressure - ref) / abs(ref) < 1e-8
        assert abs(imp.volume_velocity - complex(*port["volume_velocity"])) < 1e-15


def test_c1_sweep_against_oracle_and_analytic():
    """C1 workload (icosphere s3, 642 vertices / 1280 triangles, 32 log-spaced
    frequencies 100 Hz-5 kHz, rho 1.205): the whole sweep solves, every
    residual is FP64-tight, the analytic sphere holds within discretisation
    error, repeated solves are bitwise identical, and sampled frequencies
    equal the oracle to 1e-9."""
    mesh = meshes.icosphere(3)
    freqs = list(np.geomspace(100, 5000, 32))
    obs = [(0, 0, .3), (1, 0, 0), (0, 0, 3)]
    req = _request(freqs, obs, medium=hs.AcousticMedium(1.205, 343.0))
    with hs.CudaBemSolver(mesh) as solver:
        first = solver.solve(req)
        second = solver.solve(req)
    for fa, fb in zip(first.frequencies, second.frequencies):
        a, b = fa.excitations[0], fb.excitations[0]
        assert np.array_equal(a.boundary.pressure_trace, b.boundary.pressure_trace)
        assert np.array_equal(a.observer_pressure, b.observer_pressure)
        assert a.boundary_residual < 1e-10
        for j, r in enumerate([.3, 1.0, 3.0]):
            expected = analytic_sphere(fa.frequency, r, density=1.205)
            # 1280 flat triangles: discretisation error grows to ~2.2 % at ka = 9.2 (5 kHz)
            assert abs(a.observer_pressure[j] / expected - 1) < 0.03
    for i in (0, 31):
        ref = O.solve(mesh, [freqs[i]], [[(1, 1.0)]], obs, density=1.205, plan_frequencies=freqs)
        ex = first.frequencies[i].excitations[0]
        assert rel_l2(ex.boundary.pressure_trace, ref["trace"][0, 0]) < SOLVE_TOL
        assert rel_l2(ex.observer_pressure, ref["observer"][0, 0]) < SOLVE_TOL


def test_far_field_and_superposition():
    """Far-field observation normalised at R equals the oracle and, for the
    pulsating sphere (an exact monopole), the analytic pressure at R; a second
    excitation scaled by a complex factor scales every output linearly."""
    mesh = meshes.octahedral_sphere(3)
    dirs = [(0, 0, 1), (1, 0, 0), (0, -1, 0)]
    alpha = 0.6 * np.exp(0.71j)
    exc = [hs.BemExcitation("unit", [hs.FaceVelocity(1, 1.0)]), hs.BemExcitation("phase", [hs.FaceVelocity(1, alpha)])]
    req = hs.BemRequest(frequencies=[500.0, 1715.0], excitations=exc, observers=dirs,
                        far_field=hs.FarFieldObservation((0.0, 0.0, 0.0), 2.0))
    with hs.CudaBemSolver(mesh) as solver:
        res = solver.solve(req)
    ref = O.solve(mesh, [500.0, 1715.0], [[(1, 1.0)], [(1, alpha)]], dirs, far_field=((0, 0, 0), 2.0))
    for i, f in enumerate([500.0, 1715.0]):
        unit, phase = res.frequencies[i].excitations
        assert rel_l2(unit.observer_pressure, ref["observer"][i, 0]) < SOLVE_TOL
        assert np.allclose(phase.observer_pressure, alpha * unit.observer_pressure, rtol=1e-12)
        assert np.allclose(phase.boundary.pressure_trace, alpha * unit.boundary.pressure_trace, rtol=1e-12)
        assert np.all(np.abs(unit.observer_pressure / analytic_sphere(f, 2.0) - 1) < 0.03)
