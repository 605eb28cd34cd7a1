"""Request validation, error classes and cancellation of the CUDA solver,
matching the reference's behaviour (cuda_solver.cu:1054-1137, 1165-1212)."""
import dataclasses

import numpy as np
import pytest

import hornsculpt_b200 as hs
from hornsculpt_b200 import meshes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def solver():
    s = hs.CudaBemSolver(meshes.octahedral_sphere(2))
    yield s
    s.close()


def req(**kw):
    base = dict(frequencies=[500.0], excitations=[hs.BemExcitation("u", [hs.FaceVelocity(1, 1.0)])],
                observers=[(0, 0, .5)])
    base.update(kw)
    return hs.BemRequest(**base)


def test_device_description():
    assert "B200" in hs.CudaBemSolver.device_description()


@pytest.mark.parametrize("kw,match", [
    (dict(frequencies=[]), "Invalid BEM medium"),
    (dict(frequencies=[-5.0]), "Invalid BEM medium|Solved frequency is invalid"),
    (dict(medium=hs.AcousticMedium(-1.0, 343.0)), "Invalid BEM medium"),
    (dict(numerics=hs.BemNumerics(quadrature_order=3)), "Invalid BEM medium"),
    (dict(numerics=hs.BemNumerics(singular_order=21)), "Invalid BEM medium"),
    (dict(numerics=hs.BemNumerics(relative_residual_tolerance=1e-9)), "Invalid BEM medium"),
    (dict(excitations=[hs.BemExcitation("x", [hs.FaceVelocity(7, 1.0)])]), "known Driven face"),
    (dict(excitations=[hs.BemExcitation("x", [hs.FaceVelocity(1, 1.0), hs.FaceVelocity(1, 2.0)])]),
     "known Driven face"),
    (dict(excitations=[hs.BemExcitation("x", [])]), "at least one assigned Driven face"),
    (dict(observers=[(0, 0, 0.01)]), "outside the solid"),
    (dict(frequencies=[500.0], interaction_plan_frequencies=[400.0, 600.0]), "planning raster"),
    (dict(far_field=hs.FarFieldObservation((0, 0, 0), 1.0), observers=[(0, 0, 0)]), "differ from its origin"),
])
def test_invalid_requests(solver, kw, match):
    with pytest.raises(ValueError, match=match):
        solver.solve(req(**kw))


def test_electrically_coarse_mesh_rejected():
    """k*h > 3.25 (regular_qualification.hpp:360-368) stops the observer field
    (tetrahedron: every pair touches, so planning is trivial)."""
    with hs.CudaBemSolver(meshes.scalene_tetrahedron()) as tetra:
        with pytest.raises(hs.BemError, match="qualified electrical range"):
            tetra.solve(req(frequencies=[2000.0], excitations=[hs.BemExcitation("u", [hs.FaceVelocity(50, 1.0)])],
                            observers=[(0, 0, 1.0)]))


def test_cancellation(solver):
    stop = hs.StopToken()
    stop.request_stop()
    with pytest.raises(hs.BemCancelled, match="BEM calculation cancelled."):
        solver.solve(req(), stop=stop)
    # the session stays usable after a cancelled call
    assert solver.solve(req()).frequencies[0].excitations[0].boundary_residual < 1e-12


def test_zero_excitation_gives_zero_field(solver):
    res = solver.solve(req(excitations=[hs.BemExcitation("z", [hs.FaceVelocity(1, 0.0)])]))
    ex = res.frequencies[0].excitations[0]
    assert np.all(ex.observer_pressure == 0) and np.all(ex.boundary.pressure_trace == 0)
    assert ex.impedances == []


def test_progress_and_plan_reuse(solver):
    phases = []
    r1 = solver.solve(req(frequencies=[300.0, 500.0], interaction_plan_frequencies=[300.0, 500.0]),
                      progress=lambda p: phases.append(p.phase))
    r2 = solver.solve(req(frequencies=[300.0], interaction_plan_frequencies=[300.0, 500.0]))
    assert phases[0] == 0 and phases.count(6) == 2
    assert r2.frequencies[0].interaction_plan_reused
    a, b = r1.frequencies[0].excitations[0], r2.frequencies[0].excitations[0]
    assert np.array_equal(a.boundary.pressure_trace, b.boundary.pressure_trace)


def test_lem_coupled_solve_equals_direct_solve_of_coupled_velocities():
    """BEM side of LEM coupling: the superposed unit-port solves equal one direct solve
    with the coupled face velocities, and the port pressures close with the network's."""
    m = meshes.icosphere(2)
    c = m.vertices[m.triangles].mean(axis=1)
    faces = np.where(c[:, 2] > 0.06, 17, np.where(c[:, 0] < -0.06, 29, 90)).astype(np.uint32)
    kind = np.where(faces == 90, meshes.WALL, meshes.DRIVEN).astype(np.uint8)
    mesh = hs.SurfaceMesh(m.vertices, m.triangles, faces, kind)
    flows = np.array([2e-4 + 1e-5j, -5e-5j])

    def network(f, Z):
        return [hs.PortSolution(q, p) for q, p in zip(flows, Z @ flows)]
    request = hs.BemRequest(frequencies=[600.0], excitations=[], observers=[(0, 0, 0.5)],
                            numerics=hs.BemNumerics(relative_residual_tolerance=1e-7))
    ports = [hs.BemPort("front", [17]), hs.BemPort("side", [29])]
    with hs.CudaBemSolver(mesh) as solver:
        coupled = hs.coupled_solve(solver, mesh, ports, request, network)[0]
        direct = solver.solve(hs.BemRequest(frequencies=[600.0], observers=[(0, 0, 0.5)],
                                            excitations=[hs.BemExcitation("lem", coupled.face_velocities)],
                                            numerics=request.numerics))
    d = direct.frequencies[0].excitations[0]
    assert np.linalg.norm(coupled.pressure_trace - d.boundary.pressure_trace) <= 1e-6 * np.linalg.norm(
        d.boundary.pressure_trace)
    assert abs(coupled.observer_pressure[0] - d.observer_pressure[0]) <= 1e-6 * abs(d.observer_pressure[0])


def test_mapped_host_patch_residency_equals_device():
    """CudaStorageOptions.quadrature_patches = mapped_host (cuda_solver.cu:112-160):
    the near-pair quadrature patches stay in mapped pinned host memory that the
    kernels read over the bus. The result equals the device-resident one bit for
    bit, and the session holds the patches' bytes less device memory."""
    mesh = meshes.octahedral_sphere(3)
    request = req(frequencies=[400.0, 1700.0], observers=[(0, 0, 0.3)],
                  numerics=hs.BemNumerics(near_relative_tolerance=1e-6))
    plan = hs.host_plan(mesh, request.numerics, 2 * np.pi * 1700.0 / 343.0)
    assert len(plan["patches"]) > 0
    results = {}
    for where in ("device", "mapped_host"):
        with hs.CudaBemSolver(mesh, hs.CudaStorageOptions(quadrature_patches=where)) as solver:
            results[where] = solver.solve(request)
    for fd, fm in zip(results["device"].frequencies, results["mapped_host"].frequencies):
        assert np.array_equal(fd.excitations[0].boundary.pressure_trace, fm.excitations[0].boundary.pressure_trace)
        assert np.array_equal(fd.excitations[0].observer_pressure, fm.excitations[0].observer_pressure)
    saved = results["device"].peak_device_bytes - results["mapped_host"].peak_device_bytes
    assert saved >= len(plan["patches"]) * 22 * 8 * 0.9


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_library_coupled_solve(precision):
    """The coupled solve inside the library (hs_bem_solve_coupled): the port
    impedance from the basis solves, a network that depends on it (each port a
    pressure source behind an internal impedance: (Z + Zs) Q = U), the superposed
    coupled field refined as its own equation, the closure check, and one coupled
    excitation per frequency. It equals the host-side superposition of the same
    basis and a direct solve with the coupled face velocities."""
    m = meshes.icosphere(2)
    c = m.vertices[m.triangles].mean(axis=1)
    faces = np.where(c[:, 2] > 0.06, 17, np.where(c[:, 0] < -0.06, 29, 90)).astype(np.uint32)
    kind = np.where(faces == 90, meshes.WALL, meshes.DRIVEN).astype(np.uint8)
    mesh = hs.SurfaceMesh(m.vertices, m.triangles, faces, kind)
    U = np.array([1.0, 0.3j])
    Zs = np.diag([2e4 + 1e3j, 5e4])

    def flows_of(Z):
        q = np.linalg.solve(Z + Zs, U)
        return q, Z @ q
    numerics = hs.BemNumerics(precision=precision, relative_residual_tolerance=1e-7)
    ports = [hs.BemPort("front", [17]), hs.BemPort("side", [29])]
    basis = hs.make_coupling_basis(ports, mesh)
    request = hs.BemRequest(frequencies=[600.0, 1500.0], excitations=basis.excitations, observers=[(0, 0, 0.5)],
                            numerics=numerics)
    with hs.CudaBemSolver(mesh) as solver:
        lib_result, extra = solver.solve_coupled(request, lambda f, Z: flows_of(Z))
        host = hs.coupled_solve(solver, mesh, ports, dataclasses.replace(request, excitations=[]),
                                lambda f, Z: [hs.PortSolution(q, p) for q, p in zip(*flows_of(Z))])
        for frame, (Z, q, p), h in zip(lib_result.frequencies, extra, host):
            assert len(frame.excitations) == 1
            e = frame.excitations[0]
            assert np.allclose(Z, h.impedance, rtol=1e-9, atol=0)
            assert np.allclose(q, [s.volume_velocity for s in h.ports], rtol=1e-9, atol=0)
            assert np.linalg.norm(e.boundary.pressure_trace - h.pressure_trace) <= 1e-6 * np.linalg.norm(
                h.pressure_trace)
            assert e.boundary_residual <= (1e-10 if precision == "mixed" else 1e-7)
            direct = solver.solve(hs.BemRequest(frequencies=[frame.frequency], observers=[(0, 0, 0.5)],
                                                excitations=[hs.BemExcitation("lem", h.face_velocities)],
                                                numerics=numerics)).frequencies[0].excitations[0]
            assert np.linalg.norm(e.boundary.pressure_trace - direct.boundary.pressure_trace) <= 1e-6 * np.linalg.norm(
                direct.boundary.pressure_trace)
            assert abs(e.observer_pressure[0] - direct.observer_pressure[0]) <= 1e-6 * abs(direct.observer_pressure[0])
            assert np.allclose(e.boundary.normal_derivative, direct.boundary.normal_derivative, rtol=1e-12, atol=0)
