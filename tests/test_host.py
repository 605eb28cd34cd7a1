"""Host-side product code without a GPU: the C ABI loads and exports every
declared symbol, the library's host planner equals the reference planner,
mesh validation rejects what the reference rejects."""
import numpy as np
import pytest

import hornsculpt_b200 as hs
from hornsculpt_b200 import _lib, meshes
from oracle import oracle as O


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    declared = _lib.declared_symbols()
    assert len(declared) >= 20
    missing = [s for s in declared if not hasattr(lib, s)]
    assert not missing


def test_numerics_defaults_match_reference():
    """BemNumerics{} defaults (bem.hpp:113-123) through hs_numerics_default."""
    n = _lib.hs_numerics()
    _lib.load().hs_numerics_default(n)
    assert (n.quadrature_order, n.singular_order, n.near_maximum_depth, n.maximum_refinement_steps) == (4, 4, 6, 3)
    assert (n.near_distance_ratio, n.near_relative_tolerance, n.relative_residual_tolerance) == (1.0, 1e-4, 5e-5)
    assert (n.fmm_leaf_support_capacity, n.fmm_restart_length, n.fmm_preconditioner_block_width) == (16, 40, 32)
    d = hs.BemNumerics().to_c()
    assert d.quadrature_order == 4 and d.relative_residual_tolerance == 5e-5


CASES = {"octa2_1715": (lambda: meshes.octahedral_sphere(2), {}),
         "octa3_1000": (lambda: meshes.octahedral_sphere(3), {}),
         "ico2_3000": (lambda: meshes.icosphere(2), {}),
         "octa2_tight": (lambda: meshes.octahedral_sphere(2), {"near_relative_tolerance": 1e-6}),
         "tetra_400": (meshes.scalene_tetrahedron, {"singular_order": 12})}


@pytest.mark.parametrize("name", list(CASES))
def test_host_plan_equals_reference_plan(golden, name):
    """Touching jobs, near jobs, patches (bit-exact doubles), whole-panel
    degrees and the near CSR equal the reference's makeInteractionPlan."""
    make, kw = CASES[name]
    plans = golden["plans"]
    p = hs.host_plan(make(), hs.BemNumerics(**kw), float(plans[f"{name}/k"][0]))
    for key in ("touching", "near", "patches", "whole", "trials", "offsets"):
        assert np.array_equal(p[key], plans[f"{name}/{key}"]), key


@pytest.mark.skipif(not O.reference_available(), reason="oracle/_ref not built (reference tree absent)")
def test_host_plan_equals_reference_plan_c1():
    """The full C1 icosphere (1280 triangles) at the 5 kHz planning wavenumber."""
    mesh = meshes.icosphere(3)
    k = 2 * np.pi * 5000 / 343
    p = hs.host_plan(mesh, hs.BemNumerics(), k)
    r = O.reference_plan(mesh, O.Numerics.default(), k)
    for key in ("touching", "near", "patches", "whole", "trials", "offsets"):
        assert np.array_equal(p[key], r[key]), key


def test_meshes():
    for n, (v, t) in enumerate([(6, 8), (18, 32), (66, 128), (258, 512)]):
        m = meshes.octahedral_sphere(n)
        assert (m.vertex_count, m.triangle_count) == (v, t)
        assert meshes.signed_volume(m) > 0
    for n, (v, t) in enumerate([(12, 20), (42, 80), (162, 320), (642, 1280)]):
        m = meshes.icosphere(n)
        assert (m.vertex_count, m.triangle_count) == (v, t)
        assert meshes.signed_volume(m) > 0
    assert meshes.signed_volume(meshes.scalene_tetrahedron()) > 0


def _session(mesh):
    return hs.CudaBemSolver(mesh)


def test_open_mesh_rejected():
    m = meshes.octahedral_sphere(1)
    open_mesh = meshes.SurfaceMesh(m.vertices, m.triangles[1:], m.face_ids[1:], m.boundary[1:])
    with pytest.raises(ValueError, match="closed, outward-oriented"):
        _session(open_mesh)


def test_inverted_mesh_rejected():
    m = meshes.octahedral_sphere(1)
    flipped = meshes.SurfaceMesh(m.vertices, m.triangles[:, ::-1], m.face_ids, m.boundary)
    with pytest.raises(ValueError, match="outward winding"):
        _session(flipped)


def test_nested_components_rejected():
    a = meshes.octahedral_sphere(1, radius=0.2)
    b = meshes.octahedral_sphere(1, radius=0.05)
    both = meshes.SurfaceMesh(np.vstack([a.vertices, b.vertices]),
                              np.vstack([a.triangles, b.triangles + a.vertex_count]),
                              np.concatenate([a.face_ids, b.face_ids]), np.concatenate([a.boundary, b.boundary]))
    with pytest.raises(ValueError, match="Nested surface components"):
        _session(both)


def test_self_intersecting_mesh_rejected():
    a = meshes.octahedral_sphere(1)
    b = meshes.octahedral_sphere(1)
    shifted = b.vertices + np.array([0.05, 0, 0])
    both = meshes.SurfaceMesh(np.vstack([a.vertices, shifted]), np.vstack([a.triangles, b.triangles + a.vertex_count]),
                              np.concatenate([a.face_ids, b.face_ids]), np.concatenate([a.boundary, b.boundary]))
    with pytest.raises(ValueError, match="non-intersecting"):
        _session(both)


def test_non_finite_mesh_rejected():
    m = meshes.octahedral_sphere(1)
    v = m.vertices.copy()
    v[3, 1] = np.nan
    with pytest.raises(ValueError, match="not finite"):
        _session(meshes.SurfaceMesh(v, m.triangles, m.face_ids, m.boundary))


def _passes_host_validation(mesh):
    """Session creation validates the mesh on the host before it looks for a
    device: with a GPU the session opens; without one the only error is the
    missing device."""
    try:
        hs.CudaBemSolver(mesh).close()
    except ValueError:
        return False
    except hs.BemError as e:
        assert "CUDA device" in str(e)
    return True


@pytest.mark.parametrize("h,triangles", [(None, 12756), (0.004, 39776)])
def test_exponential_horn(h, triangles):
    """The horn shell of the precision-form workload: watertight, every
    directed edge paired with its reverse, outward (positive volume), all
    triangle angles >= 20 degrees (qualified for the regular rules), the throat
    disc its own Driven face, seeded and reproducible, accepted by the
    library's exterior-surface validation."""
    m = meshes.exponential_horn(h=h, seed=7)
    assert abs(m.triangle_count - triangles) <= 0.01 * triangles  # ring counts follow the jittered meridian
    edges = {}
    for t in m.triangles:
        for a, b in ((t[0], t[1]), (t[1], t[2]), (t[2], t[0])):
            edges[(a, b)] = edges.get((a, b), 0) + 1
    assert all(c == 1 and edges.get((b, a)) == 1 for (a, b), c in edges.items())
    assert meshes.signed_volume(m) > 0
    v = m.vertices[m.triangles]
    for i in range(3):
        u, w = v[:, (i + 1) % 3] - v[:, i], v[:, (i + 2) % 3] - v[:, i]
        cos = (u * w).sum(-1) / np.linalg.norm(u, axis=-1) / np.linalg.norm(w, axis=-1)
        assert np.degrees(np.arccos(np.clip(cos, -1, 1))).min() >= 20
    throat = m.face_ids == meshes.HORN_THROAT
    assert throat.any() and (m.boundary[throat] == meshes.DRIVEN).all() and (m.boundary[~throat] == meshes.WALL).all()
    # the throat disc lies in z = 0 inside the throat radius
    tv = m.vertices[m.triangles[throat]]
    assert np.allclose(tv[..., 2], 0) and np.hypot(tv[..., 0], tv[..., 1]).max() <= 0.025 + 1e-12
    again = meshes.exponential_horn(h=h, seed=7)
    assert np.array_equal(again.vertices, m.vertices) and np.array_equal(again.triangles, m.triangles)
    assert not np.array_equal(meshes.exponential_horn(h=h, seed=8).vertices, m.vertices)
    if h is None:
        assert _passes_host_validation(m)


def _box(n: int, size: float = 0.1) -> meshes.SurfaceMesh:
    """Closed outward box with an n x n grid of quads per side (flat faces)."""
    verts, index, tris = [], {}, []

    def vid(p):
        key = tuple(np.round(p, 12))
        if key not in index:
            index[key] = len(verts)
            verts.append(p)
        return index[key]

    g = np.linspace(-size / 2, size / 2, n + 1)
    for axis in range(3):
        for sign in (-1, 1):
            u, w = [(axis + 1) % 3, (axis + 2) % 3][:: sign]
            for i in range(n):
                for j in range(n):
                    corners = []
                    for di, dj in ((0, 0), (1, 0), (1, 1), (0, 1)):
                        p = np.zeros(3)
                        p[axis] = sign * size / 2
                        p[u], p[w] = g[i + di], g[j + dj]
                        corners.append(vid(p))
                    a, b, c, d = corners
                    tris += [(a, b, c), (a, c, d)]
    m = meshes.SurfaceMesh(np.asarray(verts), np.asarray(tris), np.ones(len(tris)), np.ones(len(tris)))
    if meshes.signed_volume(m) < 0:
        m = meshes.SurfaceMesh(m.vertices, m.triangles[:, ::-1], m.face_ids, m.boundary)
    return m


def test_flat_faces_accepted():
    """Coplanar triangles without a common vertex are separated by in-plane
    axes: a box with flat gridded sides is a valid exterior surface."""
    assert _passes_host_validation(_box(4))


def test_revolved_sphere():
    s = meshes.revolved_sphere(radius=0.1, h=0.004, seed=3)
    assert 7500 < s.vertex_count < 8300
    assert abs(meshes.signed_volume(s) - 4 / 3 * np.pi * 0.1 ** 3) < 2e-3 * 4 / 3 * np.pi * 0.1 ** 3
    assert np.allclose(np.linalg.norm(s.vertices, axis=1), 0.1)
    assert _passes_host_validation(meshes.revolved_sphere(radius=0.1, h=0.02))


def test_horn_too_coarse_for_its_wall():
    with pytest.raises(ValueError, match="too coarse"):
        meshes.exponential_horn(h=0.03)
