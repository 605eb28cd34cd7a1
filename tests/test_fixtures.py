"""The reference's solver-input fixture format (hornsculpt-solver-input-1):
read_fixture restates tests/solver_benchmark.cpp:80-174, write_fixture the keys
of tests/export_bem_fixture.cpp:75-92. Host only."""
import json
import math

import numpy as np
import pytest

import hornsculpt_b200 as hs
from hornsculpt_b200 import meshes


def _split_sphere():
    """icosphere s2 with its driven faces split into tags 50 / 51 by the sign of
    the centroid's z, as the reference's exporter does for its sphere case."""
    m = meshes.icosphere(2)
    z = m.vertices[m.triangles][:, :, 2].sum(axis=1)
    tags = np.where(z >= 0, 50, 51).astype(np.uint32)
    return meshes.SurfaceMesh(m.vertices, m.triangles, tags, np.full(m.triangle_count, meshes.DRIVEN, np.uint8))


def _request():
    return hs.BemRequest(
        frequencies=[100.0, 500.0, 1000.0, 1715.0],
        excitations=[hs.BemExcitation("uniform", [hs.FaceVelocity(50, 1.0), hs.FaceVelocity(51, 1.0)]),
                     hs.BemExcitation("antisymmetric", [hs.FaceVelocity(50, 1.0), hs.FaceVelocity(51, -1.0)])],
        observers=[(0.0, 0.0, 1.0), (0.5, 0.0, 0.0)], medium=hs.AcousticMedium(1.21, 343.0))


def test_round_trip():
    mesh, req = _split_sphere(), _request()
    text = json.dumps(hs.write_fixture(mesh, req, "sphere")).encode()
    m2, r2, digest = hs.read_fixture(text)
    assert len(digest) == 64
    assert np.array_equal(m2.vertices, mesh.vertices) and np.array_equal(m2.triangles, mesh.triangles)
    assert np.array_equal(m2.face_ids, mesh.face_ids) and np.array_equal(m2.boundary, mesh.boundary)
    assert r2.frequencies == req.frequencies and [tuple(o) for o in r2.observers] == list(req.observers)
    assert r2.medium == req.medium
    assert [(e.name, [(f.face_id, f.normal_velocity) for f in e.faces]) for e in r2.excitations] == \
        [(e.name, [(f.face_id, complex(f.normal_velocity)) for f in e.faces]) for e in req.excitations]


def test_legacy_driven_velocity():
    """Without "excitations": a uniform and a proportional-phase (0.6 at 0.71 rad)
    excitation on every driven tag (solver_benchmark.cpp:141-153)."""
    root = hs.write_fixture(_split_sphere(), _request())
    del root["excitations"], root["normal_velocities_m_s"]
    root["driven_velocity"] = [1, 0]
    _, req, digest = hs.read_fixture(root)
    assert digest is None
    assert [e.name for e in req.excitations] == ["uniform", "proportional-phase"]
    phase = req.excitations[1].faces[0].normal_velocity
    assert abs(abs(phase) - 0.6) < 1e-15 and abs(math.atan2(phase.imag, phase.real) - 0.71) < 1e-15
    assert [f.face_id for f in req.excitations[0].faces] == [50, 51]


@pytest.mark.parametrize("edit, message", [
    (lambda r: r.update(phasor="exp(-iwt)"), "positive-time phasor"),
    (lambda r: r.update(rho="x"), "Missing or invalid scalar"),
    (lambda r: r["triangles0"][0].__setitem__(0, 1e9), "out of range"),
    (lambda r: r["triangles0"][0].__setitem__(0, 1.5), "Invalid unsigned fixture index"),
    (lambda r: r["tags"].pop(), "Triangle and tag counts differ"),
    (lambda r: r["frequencies_hz"].__setitem__(0, -5), "Frequency must be positive"),
    (lambda r: r["normal_velocities_m_s"][0][0].__setitem__(0, 2.0), "does not reproduce fixture DP0"),
    (lambda r: r["normal_velocities_m_s"].pop(), "DP0 RHS count mismatch"),
    (lambda r: r["vertices_m"][0].pop(), "three coordinates"),
])
def test_reader_errors(edit, message):
    root = hs.write_fixture(_split_sphere(), _request())
    edit(root)
    with pytest.raises(ValueError, match=message):
        hs.read_fixture(root)


def test_wall_velocity_is_rejected():
    mesh, req = _split_sphere(), _request()
    boundary = mesh.boundary.copy()
    boundary[0] = meshes.WALL
    root = hs.write_fixture(meshes.SurfaceMesh(mesh.vertices, mesh.triangles, mesh.face_ids, boundary), req)
    root["driven_tags"] = [51]
    root["tags"][0] = 60.0
    root["normal_velocities_m_s"][0][0] = [1.0, 0.0]
    with pytest.raises(ValueError, match="does not reproduce|Nonzero Wall velocity"):
        hs.read_fixture(root)


def test_invalid_json():
    with pytest.raises(ValueError, match="Invalid fixture JSON"):
        hs.read_fixture(b"{not json")
