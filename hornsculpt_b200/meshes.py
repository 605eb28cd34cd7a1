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


def thin_box(lx: float, ly: float, lz: float, n: int, face_id: int = 1) -> SurfaceMesh:
    """Closed outward cuboid [0, lx] x [0, ly] x [0, lz]: n x n squares (two triangles
    each) on the top and bottom faces, one layer of n squares on each side. With lz much
    smaller than lx / n the top and bottom panels face each other across a gap the
    interaction plan integrates on projected patches (like the reference's thin closed
    box, ``docs/BURTON-MILLER.md:277-283``). All faces driven."""
    index, verts, tris = {}, [], []

    def vid(p):
        key = tuple(round(c, 12) for c in p)
        if key not in index:
            index[key] = len(verts)
            verts.append(p)
        return index[key]

    def quad(a, b, c, d):  # counter-clockwise seen from outside
        tris.append((vid(a), vid(b), vid(c)))
        tris.append((vid(a), vid(c), vid(d)))

    xs, ys = np.linspace(0, lx, n + 1), np.linspace(0, ly, n + 1)
    for i in range(n):
        for j in range(n):
            x0, x1, y0, y1 = xs[i], xs[i + 1], ys[j], ys[j + 1]
            quad((x0, y0, lz), (x1, y0, lz), (x1, y1, lz), (x0, y1, lz))
            quad((x0, y0, 0), (x0, y1, 0), (x1, y1, 0), (x1, y0, 0))
    for i in range(n):
        x0, x1, y0, y1 = xs[i], xs[i + 1], ys[i], ys[i + 1]
        quad((x0, 0, 0), (x1, 0, 0), (x1, 0, lz), (x0, 0, lz))
        quad((x0, ly, 0), (x0, ly, lz), (x1, ly, lz), (x1, ly, 0))
        quad((0, y0, 0), (0, y0, lz), (0, y1, lz), (0, y1, 0))
        quad((lx, y0, 0), (lx, y1, 0), (lx, y1, lz), (lx, y0, lz))
    T = len(tris)
    return SurfaceMesh(np.array(verts, float), np.array(tris, np.uint32), np.full(T, face_id, np.uint32),
                       np.full(T, DRIVEN, np.uint8))


def signed_volume(mesh: SurfaceMesh) -> float:
    v = mesh.vertices[mesh.triangles] - mesh.vertices.min(0)
    return float(np.einsum("ij,ij->i", v[:, 0], np.cross(v[:, 1], v[:, 2])).sum() / 6)


# Face ids of the horn: the driven throat disc and the rigid rest of the shell.
HORN_THROAT = 1
HORN_SHELL = 2


def _meridian_piece(curve, length: float, h: float, interior_jitter, rng, jitter: float):
    """Points of one meridian piece at equal arc-length steps of at most h.

    curve(t) -> (z, r) for t in [0, 1]; the end points are kept exactly (sharp
    corners between pieces); interior points move along the meridian by up to
    jitter * h when interior_jitter is set."""
    n = max(1, int(math.ceil(length / h - 1e-9)))
    t_fine = np.linspace(0.0, 1.0, 4097)
    p_fine = np.array([curve(t) for t in t_fine])
    s_fine = np.concatenate([[0.0], np.cumsum(np.hypot(*np.diff(p_fine, axis=0).T))])
    targets = np.linspace(0.0, s_fine[-1], n + 1)
    if interior_jitter and n > 1:
        targets[1:-1] += rng.uniform(-jitter, jitter, n - 1) * h
    t = np.interp(targets, s_fine, t_fine)
    return [curve(x) for x in t]


def _surface_of_revolution(pieces, h: float, rng, jitter: float, face_of_piece) -> SurfaceMesh:
    """Mesh of the surface swept by a closed meridian about the z axis.

    pieces: (curve(t) -> (z, r), arc length or None, jitter interior points)
    traversed so that the solid lies to the right in the (z, r) half-plane and
    starting and ending on the axis. Each meridian node becomes a ring of
    max(3, round(2 pi r / h)) nodes (a single vertex on the axis); adjacent
    rings are zipped by angle. Ring nodes move by up to jitter * h along the
    ring except on corner rings (piece ends)."""
    meridian, corner, piece_of = [], [], []
    for index, (curve, plen, interior) in enumerate(pieces):
        if plen is None:
            zs = np.linspace(0.0, 1.0, 2001)
            p = np.array([curve(x) for x in zs])
            plen = float(np.hypot(*np.diff(p, axis=0).T).sum())
        pts = _meridian_piece(curve, plen, h, interior, rng, jitter)
        start = 0 if index == 0 else 1  # the first point of a piece is the last of the previous
        for k in range(start, len(pts)):
            meridian.append(pts[k])
            corner.append(k == 0 or k == len(pts) - 1)
            piece_of.append(index)
    vertices, rings = [], []
    for i, (z, r) in enumerate(meridian):
        if r <= 1e-12:
            rings.append([len(vertices)])
            vertices.append((0.0, 0.0, z))
            continue
        n = max(3, int(round(2 * math.pi * r / h)))
        offset = 0.5 * (i % 2)
        angles = 2 * math.pi * (np.arange(n) + offset) / n
        if not corner[i]:
            angles = angles + rng.uniform(-jitter, jitter, n) * h / r
        ring = []
        for a in angles:
            ring.append(len(vertices))
            vertices.append((r * math.cos(a), r * math.sin(a), z))
        rings.append(ring)

    def ring_angles(ring):
        v = np.asarray([vertices[q] for q in ring])
        return np.mod(np.arctan2(v[:, 1], v[:, 0]), 2 * math.pi)

    triangles, faces = [], []
    for i in range(len(rings) - 1):
        A, B = rings[i], rings[i + 1]
        face = face_of_piece(piece_of[i + 1])  # the strip belongs to its outer node's piece
        if len(A) == 1 or len(B) == 1:
            if len(A) == 1:
                for j in range(len(B)):
                    triangles.append((A[0], B[(j + 1) % len(B)], B[j]))
            else:
                for j in range(len(A)):
                    triangles.append((A[j], A[(j + 1) % len(A)], B[0]))
            faces += [face] * (len(B) if len(A) == 1 else len(A))
            continue
        # zip the two rings by angle, starting at each ring's smallest angle
        aa, ab = ring_angles(A), ring_angles(B)
        oa, ob = np.argsort(aa), np.argsort(ab)
        A = [A[q] for q in oa]
        B = [B[q] for q in ob]
        ta = np.concatenate([aa[oa], aa[oa][:1] + 2 * math.pi])
        tb = np.concatenate([ab[ob], ab[ob][:1] + 2 * math.pi])
        ia = ib = 0
        while ia < len(A) or ib < len(B):
            if ib == len(B) or (ia < len(A) and ta[ia + 1] <= tb[ib + 1]):
                triangles.append((A[ia % len(A)], A[(ia + 1) % len(A)], B[ib % len(B)]))
                ia += 1
            else:
                triangles.append((A[ia % len(A)], B[(ib + 1) % len(B)], B[ib % len(B)]))
                ib += 1
            faces.append(face)
    verts = np.asarray(vertices)
    tris = np.asarray(triangles, dtype=np.int64)
    faces = np.asarray(faces)
    mesh = SurfaceMesh(verts, tris, faces, np.where(faces == HORN_THROAT, DRIVEN, WALL))
    if signed_volume(mesh) < 0:
        mesh = SurfaceMesh(verts, tris[:, ::-1], mesh.face_ids, mesh.boundary)
    return mesh


def exponential_horn(throat_radius: float = 0.025, mouth_radius: float = 0.15, length: float = 0.3,
                     wall: float = 0.003, rear: float = 0.003, h: float | None = None, frequency: float = 8000.0,
                     sound_speed: float = 343.0, seed: int = 0, jitter: float = 0.05,
                     flare: float = 1.0) -> SurfaceMesh:
    """Closed exponential-horn shell, meshed isotropically at edge length h.

    Inner skin r(z) = r_t exp(m (z/L)^flare) with m = ln(r_mouth / r_t), from
    the throat (z = 0) to the mouth (z = L); outer skin at r(z) + wall; an
    annular mouth rim; a rigid rear cap body of thickness `rear` behind the
    throat; the throat disc (face HORN_THROAT, Driven) closes the inner skin,
    everything else is face HORN_SHELL (wall). flare = 1 is the plain
    exponential; larger values bend the flare towards the mouth. Default h is
    lambda/6 at `frequency`. Nodes move tangentially by up to jitter * h
    (uniform, numpy Generator seeded with `seed`), except on the axis and the
    corner rings. A solid of revolution about z: genus 0, watertight,
    outward-oriented."""
    if h is None:
        h = sound_speed / frequency / 6.0
    if not (0 < throat_radius < mouth_radius and length > 0 and wall > 0 and rear > 0 and h > 0):
        raise ValueError("invalid horn dimensions")
    # ring facets bulge by about h^2 / (8 r) towards the axis: keep that below half
    # the wall at the throat, or the inner and outer skins cross
    if h * h / (8 * throat_radius) > 0.5 * wall:
        raise ValueError(f"edge length {h} m is too coarse for a {wall} m wall at a {throat_radius} m throat")
    rng = np.random.default_rng(seed)
    m = math.log(mouth_radius / throat_radius)

    def inner(z):
        return throat_radius * math.exp(m * (z / length) ** flare)

    ro0 = throat_radius + wall
    rim_outer = inner(length) + wall
    pieces = [
        (lambda t: (-rear, t * ro0), ro0, False),                                   # rear cap disc
        (lambda t: (-rear + t * rear, ro0), rear, False),                            # rear cap side
        (lambda t: (t * length, inner(t * length) + wall), None, True),              # outer skin
        (lambda t: (length, rim_outer - t * wall), wall, False),                     # mouth rim
        (lambda t: ((1 - t) * length, inner((1 - t) * length)), None, True),         # inner skin
        (lambda t: (0.0, throat_radius * (1 - t)), throat_radius, False),            # throat disc
    ]
    return _surface_of_revolution(pieces, h, rng, jitter, lambda p: HORN_THROAT if p == 5 else HORN_SHELL)


def revolved_sphere(radius: float = 0.1, h: float = 0.01, seed: int = 0, jitter: float = 0.05,
                    face_id: int = 1) -> SurfaceMesh:
    """Sphere meshed by rings at edge length h (any size between the
    icosahedral levels), all one Driven face; seeded tangential jitter."""
    rng = np.random.default_rng(seed)
    pieces = [(lambda t: (-radius * math.cos(math.pi * t), radius * math.sin(math.pi * t)), math.pi * radius, True)]
    mesh = _surface_of_revolution(pieces, h, rng, jitter, lambda p: HORN_THROAT)
    return SurfaceMesh(mesh.vertices, mesh.triangles, np.full(mesh.triangle_count, face_id),
                       np.full(mesh.triangle_count, DRIVEN))
