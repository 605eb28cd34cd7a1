"""BEM side of LEM coupling (lem_coupling.cpp, cuda_solver.cu:1584-1630): unit-port
basis, port impedance, superposition and the pressure-closure check, on synthetic
basis solutions (host only; the solves themselves are the tested multi-excitation
path)."""
import numpy as np
import pytest

import hornsculpt_b200 as hs
from hornsculpt_b200 import meshes


def _mesh():
    m = meshes.icosphere(1)
    c = m.vertices[m.triangles].mean(axis=1)
    faces = np.where(c[:, 2] > 0.06, 17, np.where(c[:, 0] < -0.06, 29, 90)).astype(np.uint32)
    kind = np.where(faces == 90, meshes.WALL, meshes.DRIVEN).astype(np.uint8)
    return hs.SurfaceMesh(m.vertices, m.triangles, faces, kind)


def _areas(mesh):
    v = mesh.vertices[mesh.triangles]
    return 0.5 * np.linalg.norm(np.cross(v[:, 1] - v[:, 0], v[:, 2] - v[:, 0]), axis=1)


def test_basis_has_unit_flow():
    mesh = _mesh()
    basis = hs.make_coupling_basis([hs.BemPort("a", [17]), hs.BemPort("b", [29])], mesh)
    areas = _areas(mesh)
    for j, fid in enumerate([17, 29]):
        S = areas[mesh.face_ids == fid].sum()
        assert np.isclose(basis.areas[j], S)
        # Q = sum A_f v_f = 1
        assert np.isclose(sum(areas[t] * basis.panel_velocities[t] for t in np.nonzero(basis.panel_ports == j)[0]), 1.0)
        assert basis.excitations[j].faces[0].normal_velocity == pytest.approx(1 / S)
    assert (basis.panel_ports[mesh.face_ids == 90] == -1).all()


@pytest.mark.parametrize("ports, message", [
    ([hs.BemPort("a", [17])], "Every Driven face needs a BEM port"),
    ([hs.BemPort("a", [17, 90]), hs.BemPort("b", [29])], "Coupled faces must exist"),
    ([hs.BemPort("a", [17]), hs.BemPort("b", [17, 29])], "Coupled faces must exist"),
    ([], "between one and 1024"),
])
def test_basis_errors(ports, message):
    with pytest.raises(ValueError, match=message):
        hs.make_coupling_basis(ports, _mesh())


class _FakeSolver:
    """Basis solutions with surface pressure linear in the port of each panel."""

    def __init__(self, mesh, Zsurf):
        self.mesh, self.Zsurf = mesh, Zsurf

    def solve(self, request):
        T, N = self.mesh.triangle_count, self.mesh.vertex_count
        frames = []
        for f in request.frequencies:
            exc = []
            for j, e in enumerate(request.excitations):
                surface = np.array([self.Zsurf[j] * (1 + 0.01 * t) * f / 1000 for t in range(T)])
                bd = hs.BemBoundaryData(surface, np.full(N, surface.mean()), np.zeros(T, complex))
                exc.append(hs.BemExcitationResult(e.name, np.array([surface[0]]), [], 0, 1e-10, 6, 8, 0, bd))
            frames.append(hs.BemFrequencyResult(f, exc, 0, 0, 0, 0, 0, 0, 0, True))
        return hs.BemResult("test", T, N, 0, frames)


def test_coupled_superposition_and_closure():
    mesh = _mesh()
    ports = [hs.BemPort("a", [17]), hs.BemPort("b", [29], {29: 2.0})]
    solver = _FakeSolver(mesh, [3 + 1j, -1 + 2j])
    flows = np.array([1e-4 + 2e-5j, -3e-5j])

    def network(f, Z):  # prescribed flows; the port pressures the network sees
        p = Z @ flows
        return [hs.PortSolution(q, pi) for q, pi in zip(flows, p)]
    req = hs.BemRequest(frequencies=[500.0, 900.0], excitations=[], observers=[(0, 0, 1)])
    out = hs.coupled_solve(solver, mesh, ports, req, network)
    assert len(out) == 2
    basis = hs.make_coupling_basis(ports, mesh)
    r = solver.solve(hs.BemRequest(frequencies=[500.0], excitations=basis.excitations, observers=[(0, 0, 1)]))
    expect = sum(e.boundary.surface_pressure * q for e, q in zip(r.frequencies[0].excitations, flows))
    assert np.allclose(out[0].surface_pressure, expect)
    assert out[0].impedance.shape == (2, 2)
    # coupled face velocities: unit-flow velocity times the port flow
    v17 = [fv.normal_velocity for fv in out[0].face_velocities if fv.face_id == 17][0]
    assert np.isclose(v17, basis.excitations[0].faces[0].normal_velocity * flows[0])

    def wrong(f, Z):
        p = Z @ flows
        return [hs.PortSolution(q, 1.01 * pi) for q, pi in zip(flows, p)]
    with pytest.raises(RuntimeError, match="feedback consistency"):
        hs.coupled_solve(solver, mesh, ports, req, wrong)
