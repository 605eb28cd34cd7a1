"""HornSculpt's solver-input fixture format ("hornsculpt-solver-input-1").

The reference exports a solve as JSON (``tests/export_bem_fixture.cpp:41-93``)
and reads it back in its benchmark harness (``tests/solver_benchmark.cpp:80-174``).
``read_fixture`` restates that reader: the same keys, the same legacy form
(``driven_velocity`` without ``excitations`` gives a "uniform" and a
"proportional-phase" excitation on every driven tag), the same consistency
check of the per-triangle ``normal_velocities_m_s`` columns and the same
messages, raised as ValueError (the reference's std::invalid_argument).
``write_fixture`` produces the schema from a mesh and a request, so a request
served here can be replayed by the reference and the other way round.
"""
from __future__ import annotations

import hashlib
import json
import math
import pathlib
from typing import Union

import numpy as np

from .bem import AcousticMedium, BemExcitation, BemRequest, FaceVelocity
from .meshes import DRIVEN, WALL, SurfaceMesh

SCHEMA = "hornsculpt-solver-input-1"
_U32_MAX = 2 ** 32 - 1


def _require(condition: bool, message: str) -> None:
    if not condition:
        raise ValueError(message)


def _is_number(value) -> bool:
    return isinstance(value, (int, float)) and not isinstance(value, bool)


def _number(root: dict, name: str) -> float:
    value = root.get(name)
    _require(_is_number(value) and math.isfinite(value), "Missing or invalid scalar fixture value.")
    return float(value)


def _array(root: dict, name: str) -> list:
    _require(isinstance(root.get(name), list), "Missing fixture array.")
    return root[name]


def _position(value) -> tuple:
    _require(isinstance(value, list) and len(value) == 3, "Position must contain three coordinates.")
    for c in value:
        _require(_is_number(c) and math.isfinite(c), "Invalid position coordinate.")
    return float(value[0]), float(value[1]), float(value[2])


def _index(value) -> int:
    _require(_is_number(value) and 0 <= value <= _U32_MAX and math.floor(value) == value,
             "Invalid unsigned fixture index.")
    return int(value)


def read_fixture(source: Union[str, pathlib.Path, bytes, dict]):
    """(SurfaceMesh, BemRequest, sha256 hex of the input bytes or None) from a fixture
    file, its bytes or its parsed object (solver_benchmark.cpp:80-174)."""
    digest = None
    if isinstance(source, dict):
        root = source
    else:
        data = source if isinstance(source, bytes) else pathlib.Path(source).read_bytes()
        digest = hashlib.sha256(data).hexdigest()
        try:
            root = json.loads(data)
        except ValueError:
            root = None
        _require(isinstance(root, dict), "Invalid fixture JSON.")
    _require(root.get("phasor") == "exp(+iwt)", "Expected positive-time phasor fixture.")
    medium = AcousticMedium(density=_number(root, "rho"), sound_speed=_number(root, "c"))
    vertices = [_position(v) for v in _array(root, "vertices_m")]
    driven = {_index(t) for t in root["driven_tags"]} if "driven_tags" in root else set()
    tags, triangles = _array(root, "tags"), _array(root, "triangles0")
    _require(len(tags) == len(triangles), "Triangle and tag counts differ.")
    if not driven:
        driven = {_index(t) for t in tags}
    tris, face_ids, boundary = [], [], []
    for tri, tag in zip(triangles, tags):
        _require(isinstance(tri, list) and len(tri) == 3, "Triangle must contain three indices.")
        idx = [_index(v) for v in tri]
        for v in idx:
            _require(v < len(vertices), "Triangle index is out of range.")
        tag = _index(tag)
        tris.append(idx)
        face_ids.append(tag)
        boundary.append(DRIVEN if tag in driven else WALL)
    observers = [_position(p) for p in _array(root, "observations_m")]
    frequencies = []
    for f in _array(root, "frequencies_hz"):
        _require(_is_number(f) and f > 0, "Frequency must be positive.")
        frequencies.append(float(f))
    excitations = []
    if "excitations" in root:
        for definition in _array(root, "excitations"):
            faces = [FaceVelocity(_index(face.get("face_id")), complex(_number(face, "real"), _number(face, "imag")))
                     for face in _array(definition, "face_velocities")]
            excitations.append(BemExcitation(str(definition.get("name", "")), faces))
    else:
        velocity = _array(root, "driven_velocity")
        _require(len(velocity) == 2, "Invalid legacy complex velocity.")
        unit = complex(float(velocity[0]), float(velocity[1]))
        for factor in (1.0 + 0j, 0.6 * complex(math.cos(0.71), math.sin(0.71))):
            name = "uniform" if not excitations else "proportional-phase"
            excitations.append(BemExcitation(name, [FaceVelocity(tag, unit * factor) for tag in sorted(driven)]))
    _require(bool(excitations), "Fixture has no excitation.")
    if "normal_velocities_m_s" in root:
        columns = _array(root, "normal_velocities_m_s")
        _require(len(columns) == len(excitations), "DP0 RHS count mismatch.")
        for column, excitation in zip(columns, excitations):
            _require(isinstance(column, list) and len(column) == len(triangles), "DP0 column length mismatch.")
            by_face = {}
            for fv in excitation.faces:
                by_face.setdefault(fv.face_id, complex(fv.normal_velocity))
            for row, value in enumerate(column):
                _require(isinstance(value, list) and len(value) == 2, "Invalid DP0 velocity.")
                expected = complex(float(value[0]), float(value[1]))
                actual = by_face.get(face_ids[row], 0j)
                _require(abs(expected - actual) < 1e-12, "Face excitation does not reproduce fixture DP0 data.")
                _require(boundary[row] == DRIVEN or abs(expected) == 0, "Nonzero Wall velocity.")
    mesh = SurfaceMesh(np.asarray(vertices, np.float64).reshape(-1, 3), np.asarray(tris, np.uint32).reshape(-1, 3),
                       np.asarray(face_ids, np.uint32), np.asarray(boundary, np.uint8))
    request = BemRequest(frequencies=frequencies, excitations=excitations, observers=observers, medium=medium)
    return mesh, request, digest


def write_fixture(mesh: SurfaceMesh, request: BemRequest, case: str = "b200") -> dict:
    """The fixture object of a mesh and request (the keys of
    export_bem_fixture.cpp:75-92); ``json.dumps`` it to write a file."""
    driven = sorted({int(t) for t, b in zip(mesh.face_ids, mesh.boundary) if b == DRIVEN})
    columns = []
    for excitation in request.excitations:
        by_face = {}
        for fv in excitation.faces:
            by_face.setdefault(int(fv.face_id), complex(fv.normal_velocity))
        columns.append([[by_face.get(int(t), 0j).real, by_face.get(int(t), 0j).imag] if b == DRIVEN else [0.0, 0.0]
                        for t, b in zip(mesh.face_ids, mesh.boundary)])
    return {
        "schema": SCHEMA, "case": case, "phasor": "exp(+iwt)", "amplitude": "RMS", "normal": "outward into fluid",
        "rho": request.medium.density, "c": request.medium.sound_speed,
        "vertices_m": mesh.vertices.tolist(), "triangles0": mesh.triangles.astype(float).tolist(),
        "tags": mesh.face_ids.astype(float).tolist(), "driven_tags": driven,
        "normal_velocities_m_s": columns,
        "excitations": [{"name": e.name, "face_velocities": [
            {"face_id": int(fv.face_id), "real": complex(fv.normal_velocity).real,
             "imag": complex(fv.normal_velocity).imag} for fv in e.faces]} for e in request.excitations],
        "frequencies_hz": [float(f) for f in request.frequencies],
        "observations_m": [list(map(float, p)) for p in request.observers],
    }
