"""Synthetic closed surface meshes for the exterior solve.

Mesh generation is outside this library's scope (the reference meshes with its
own frontal-Delaunay/CGAL tool chain, ``modules/meshing``); these generators
produce the seeded benchmark and test geometries: octahedral and icosahedral
spheres, the scalene tetrahedron of the singular-port test, and an
exponential horn shell.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

WALL = 0
DRIVEN = 1


@dataclasses.dataclass
class SurfaceMesh:
    """Closed, outward-oriented triangle mesh (``modules/core/include/hornsculpt/mesh.hpp:10-33``).

    vertices: (N, 3) float64 metres; triangles: (T, 3) uint32 vertex indices;
    face_ids: (T,) uint32 physical face ids; boundary: (T,) uint8, 0 wall / 1 driven.
    """

    vertices: np.ndarray
    triangles: np.ndarray
    face_ids: np.ndarray
    boundary: np.ndarray

    def __post_init__(self):
        self.vertices = np.ascontiguousarray(self.vertices, dtype=np.float64).reshape(-1, 3)
        self.triangles = np.ascontiguousarray(self.triangles, dtype=np.uint32).reshape(-1, 3)
        self.face_ids = np.ascontiguousarray(self.face_ids, dtype=np.uint32).reshape(-1)
        self.boundary = np.ascontiguousarray(self.boundary, dtype=np.uint8).reshape(-1)
        if len(self.face_ids) != len(self.triangles) or len(self.boundary) != len(self.triangles):
            raise ValueError("face_ids and boundary need one entry per triangle")

    @property
    def vertex_count(self) -> int:
        return len(self.vertices)

    @property
    def triangle_count(self) -> int:
        return len(self.triangles)

    def max_edge(self) -> float:
        v = self.vertices[self.triangles]
        e = np.stack([v[:, 1] - v[:, 0], v[:, 2] - v[:, 1], v[:, 0] - v[:, 2]], 1)
        return float(np.sqrt((e * e).sum(-1)).max())


def _refine_on_sphere(vertices, triangles, refinements, radius):
    verts = [tuple(v) for v in vertices]
    tris = [tuple(t) for t in triangles]
    for _ in range(refinements):
        edges = {}
        out = []

        def mid(i, j):
            key = (min(i, j), max(i, j))
            found = edges.get(key)
            if found is not None:
                return found
            a, b = verts[i], verts[j]
            p = (a[0] + b[0], a[1] + b[1], a[2] + b[2])
            f = radius / math.sqrt(p[0] ** 2 + p[1] ** 2 + p[2] ** 2)
            verts.append((p[0] * f, p[1] * f, p[2] * f))
            edges[key] = len(verts) - 1
            return edges[key]

        for a, b, c in tris:
            ab, bc, ac = mid(a, b), mid(b, c), mid(a, c)
            out += [(a, ab, ac), (ab, b, bc), (ac, bc, c), (ab, bc, ac)]
        tris = out
    return np.array(verts), np.array(tris, dtype=np.uint32)


def octahedral_sphere(refinements: int, radius: float = 0.1, face_id: int = 1) -> SurfaceMesh:
    """Octahedron refined by edge midpoints projected to the sphere; 8*4^n triangles,
    all one driven face (the geometry of ``tests/fixture_geometry.hpp:11-51``)."""
    r = radius
    v = [(r, 0, 0), (0, r, 0), (-r, 0, 0), (0, -r, 0), (0, 0, r), (0, 0, -r)]
    t = [(4, 0, 1), (4, 1, 2), (4, 2, 3), (4, 3, 0), (5, 1, 0), (5, 2, 1), (5, 3, 2), (5, 0, 3)]
    verts, tris = _refine_on_sphere(v, t, refinements, radius)
    n = len(tris)
    return SurfaceMesh(verts, tris, np.full(n, face_id), np.full(n, DRIVEN))


def icosphere(subdivisions: int, radius: float = 0.1, face_id: int = 1) -> SurfaceMesh:
    """Icosahedron refined by projected edge midpoints: 10*4^n+2 vertices, 20*4^n
    flat triangles (s3: 642 / 1280), outward winding, all one driven face."""
    g = (1 + math.sqrt(5)) / 2
    base = [(-1, g, 0), (1, g, 0), (-1, -g, 0), (1, -g, 0), (0, -1, g), (0, 1, g), (0, -1, -g), (0, 1, -g),
            (g, 0, -1), (g, 0, 1), (-g, 0, -1), (-g, 0, 1)]
    s = radius / math.sqrt(1 + g * g)
    v = [(x * s, y * s, z * s) for x, y, z in base]
    t = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
         (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11),
         (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    verts, tris = _refine_on_sphere(v, t, subdivisions, radius)
    n = len(tris)
    return SurfaceMesh(verts, tris, np.full(n, face_id), np.full(n, DRIVEN))


def scalene_tetrahedron() -> SurfaceMesh:
    """Closed outward scalene tetrahedron of the singular-port fixture: faces 50/51
    driven, 52/53 wall (``tests/bem_singular_port_tests.cpp:72-81``)."""
    v = [(0, 0, 0), (.2, 0, 0), (.03, .14, 0), (.02, .025, .09)]
    t = [(0, 2, 1), (0, 1, 3), (0, 3, 2), (1, 2, 3)]
    return SurfaceMesh(v, t, [50, 51, 52, 53], [DRIVEN, DRIVEN, WALL, WALL])


def signed_volume(mesh: SurfaceMesh) -> float:
    v = mesh.vertices[mesh.triangles] - mesh.vertices.min(0)
    return float(np.einsum("ij,ij->i", v[:, 0], np.cross(v[:, 1], v[:, 2])).sum() / 6)
