"""HornSculpt's study request and complex result document (the MCP study adapter).

The reference's MCP server accepts a simulation study as JSON, checks it against
the open project and turns it into a BemRequest (``parseStudyRequest``,
``apps/mcp/simulation_api.cpp:160-295``). After the solve it packs the complex
results into a ``hornsculpt.complex-study`` document (``complexResultDocument``,
``:317-466``). ``describeStudyCapabilities`` (``:297-315``) publishes the input
schema. This module restates the three for this solver. The project's part is
passed in explicitly: its checked mesh (face ids and boundary kinds), medium, and
the numerics the project sets (acceleration, fast-multipole settings, near-field
depth). The project-state refusals (active LEM coupling, infinite baffle,
axisymmetric mode, stale mesh) do not apply, because this solver only has the
exterior 3-D form.

Validation follows the reference: the same limits, key rules, order of checks and
messages, in German as in the reference. The messages are raised as ValueError
with the reference's prefixes: "MCP-Studie: " for study checks, "Ungültige
Projektdatei: " for the JSON value helpers (``apps/desktop/project_json.cpp:11-98``).
Qt's JSON objects iterate keys in sorted order, so unknown keys are reported the
same way.
"""
from __future__ import annotations

import dataclasses
import json
import math
from typing import Optional, Union

from .bem import AcousticMedium, BemExcitation, BemNumerics, BemRequest, BemResult, FarFieldObservation, FaceVelocity
from .meshes import DRIVEN, WALL, SurfaceMesh

MAXIMUM_FREQUENCIES = 8192
MAXIMUM_OBSERVERS = 4096
MAXIMUM_EXCITATIONS = 16
_U32 = 4294967295


def _study(message: str):
    raise ValueError("MCP-Studie: " + message)


def _require(condition: bool, message: str) -> None:
    if not condition:
        _study(message)


def _project(message: str):
    raise ValueError("Ungültige Projektdatei: " + message)


# ---- the JSON value helpers (project_json.cpp:15-98) ----

def _keys(value: dict, expected) -> None:
    missing = sorted(k for k in expected if k not in value)
    unexpected = sorted(k for k in value if k not in expected)
    if missing or unexpected:
        _project(f"Felder fehlen: {', '.join(missing)}; unbekannte Felder: {', '.join(unexpected)}.")


def _object(value) -> dict:
    if not isinstance(value, dict):
        _project("Objekt erwartet.")
    return value


def _array(value, maximum: int, minimum: int = 0) -> list:
    if not isinstance(value, list):
        _project("Liste erwartet.")
    if len(value) < minimum or len(value) > maximum:
        _project("Listenlänge außerhalb des erlaubten Bereichs.")
    return value


def _number(value) -> float:
    if isinstance(value, bool) or not isinstance(value, (int, float)):
        _project("Endliche Zahl erwartet.")
    try:  # an integer literal beyond double range reads as infinity in the reference's parser
        result = float(value)
    except OverflowError:
        result = math.inf
    if not math.isfinite(result):
        _project("Endliche Zahl erwartet.")
    return result


def _positive(value) -> float:
    result = _number(value)
    if result <= 0:
        _project("Positive Zahl erwartet.")
    return result


def _text(value, allow_empty: bool = False) -> str:
    if not isinstance(value, str) or len(value) > 4096 or (not allow_empty and not value):
        _project("Ungültiger Text.")
    return value


def _integer(value, maximum: int = _U32) -> int:
    result = _number(value)
    if result < 0 or result > maximum or result != math.floor(result):
        _project("Ungültige Ganzzahl oder ID.")
    return int(result)


def _vector(value) -> tuple:
    v = _array(value, 3, 3)
    return _number(v[0]), _number(v[1]), _number(v[2])


def _complex(value) -> complex:
    v = _array(value, 2, 2)
    return complex(_number(v[0]), _number(v[1]))


# ---- study checks (simulation_api.cpp:26-55) ----

def _allowed_keys(value: dict, allowed) -> None:
    for key in sorted(value):
        if key not in allowed:
            _study("Unbekanntes Feld: " + key)


def _in_range(value, minimum: float, maximum: float) -> float:
    result = _number(value)
    _require(minimum <= result <= maximum, "Numerikwert außerhalb des unterstützten Bereichs.")
    return result


def _identifier(value) -> str:
    result = _text(value)
    _require(bool(result.strip()), "Leere ID oder Anregungsbezeichnung.")
    return result


def _mesh_faces(mesh: SurfaceMesh) -> dict:
    """Face id -> boundary kind of the project mesh (project_json.cpp meshFaces)."""
    faces = {}
    for face, kind in zip(mesh.face_ids.tolist(), mesh.boundary.tolist()):
        if not face or kind not in (WALL, DRIVEN):
            _project("Ungültige Netzfläche oder Randbedingung.")
        if faces.setdefault(face, kind) != kind:
            _project("Widersprüchliche Randbedingungen einer Fläche.")
    return faces


@dataclasses.dataclass
class StudyRequest:
    """The parsed study: the solver request, the observers' metadata (id, role,
    position) in input order, and the reference excitation and face of the transfer."""
    request: BemRequest
    observer_metadata: list
    reference_excitation: str
    reference_face_id: int


def parse_study_request(study: Union[dict, str, bytes], mesh: SurfaceMesh,
                        medium: Optional[AcousticMedium] = None,
                        numerics: Optional[BemNumerics] = None) -> StudyRequest:
    """A study JSON (object, or its text) against a project with this mesh, medium and
    numerics (simulation_api.cpp:160-295)."""
    if not isinstance(study, dict):
        study = json.loads(study)
    _object(study)
    _allowed_keys(study, {"frequenciesHz", "observers", "observation", "excitations", "reference", "medium",
                          "numerics"})
    faces_of_mesh = _mesh_faces(mesh)
    project = numerics or BemNumerics()
    n = BemNumerics(acceleration=project.acceleration, fast_multipole=dataclasses.replace(project.fast_multipole),
                    near_maximum_depth=project.near_maximum_depth)
    request = BemRequest(frequencies=[], excitations=[], observers=[], medium=medium or AcousticMedium(),
                         numerics=n)
    for value in _array(study.get("frequenciesHz"), MAXIMUM_FREQUENCIES, 1):
        frequency = _positive(value)
        _require(not request.frequencies or frequency > request.frequencies[-1],
                 "Frequenzen müssen streng aufsteigend sein.")
        request.frequencies.append(frequency)
    request.interaction_plan_frequencies = list(request.frequencies)
    ids, metadata, references = set(), [], 0
    for value in _array(study.get("observers"), MAXIMUM_OBSERVERS, 1):
        observer = _object(value)
        _keys(observer, ("id", "role", "positionMetres"))
        oid, role = _identifier(observer["id"]), _text(observer["role"])
        _require(oid not in ids, "Doppelte Beobachter-ID: " + oid)
        ids.add(oid)
        _require(role in ("reference", "validation", "sample"), "Unbekannte Beobachterrolle.")
        references += role == "reference"
        request.observers.append(_vector(observer["positionMetres"]))
        metadata.append(observer)
    _require(references == 1, "Genau ein Beobachter benötigt die Rolle reference.")
    if "observation" in study:
        observation = _object(study["observation"])
        mode = _text(observation.get("mode"))
        if mode == "finite":
            _keys(observation, ("mode",))
        elif mode == "far_field":
            _allowed_keys(observation, {"mode", "originMetres", "referenceDistanceMetres"})
            far = FarFieldObservation()
            if "originMetres" in observation:
                far.origin = _vector(observation["originMetres"])
            if "referenceDistanceMetres" in observation:
                far.reference_distance = _positive(observation["referenceDistanceMetres"])
            for point in request.observers:
                d = math.hypot(point[0] - far.origin[0], point[1] - far.origin[1], point[2] - far.origin[2])
                _require(math.isfinite(d) and d > 0, "Fernfeldrichtung muss endlich und vom Ursprung verschieden sein.")
            request.far_field = far
        else:
            _study("Beobachtungsmodus muss finite oder far_field sein.")
    names = set()
    for value in _array(study.get("excitations"), MAXIMUM_EXCITATIONS, 1):
        excitation = _object(value)
        _keys(excitation, ("name", "faces"))
        name = _identifier(excitation["name"])
        _require(name not in names, "Doppelte Anregung: " + name)
        names.add(name)
        seen, velocities, has_velocity = set(), [], False
        for face_value in _array(excitation["faces"], 65536, 1):
            face = _object(face_value)
            _keys(face, ("faceId", "normalVelocity"))
            fid = _integer(face["faceId"])
            _require(bool(fid) and faces_of_mesh.get(fid) == DRIVEN and fid not in seen,
                     "Jede Anregung darf vorhandene Driven-Flächen höchstens einmal zuweisen.")
            seen.add(fid)
            velocity = _complex(face["normalVelocity"])
            has_velocity = has_velocity or velocity != 0
            velocities.append(FaceVelocity(fid, velocity))
        _require(has_velocity, "Jede Anregung benötigt mindestens eine Geschwindigkeit != 0.")
        request.excitations.append(BemExcitation(name, velocities))
    reference = _object(study.get("reference"))
    _keys(reference, ("excitation", "faceId"))
    ref_name, ref_face = _identifier(reference["excitation"]), _integer(reference["faceId"])
    match = [e for e in request.excitations if e.name == ref_name]
    _require(bool(match), "Bezugsanregung fehlt.")
    _reference_velocity(match[0].faces, ref_face)
    if "medium" in study:
        m = _object(study["medium"])
        _keys(m, ("densityKgM3", "soundSpeedMetresPerSecond"))
        request.medium = AcousticMedium(_positive(m["densityKgM3"]), _positive(m["soundSpeedMetresPerSecond"]))
    _require(math.isfinite(request.medium.density) and request.medium.density > 0 and
             math.isfinite(request.medium.sound_speed) and request.medium.sound_speed > 0,
             "Das Medium benötigt positive endliche Dichte und Schallgeschwindigkeit.")
    if "numerics" in study:
        given = _object(study["numerics"])
        _allowed_keys(given, {"acceleration", "nearRelativeTolerance", "nearMaximumDepth", "relativeResidualTolerance"})
        if "acceleration" in given:
            mode = _text(given["acceleration"])
            _require(mode in ("dense", "fastMultipole"), "Unbekannter Beschleunigungsmodus.")
            n.acceleration = "dense" if mode == "dense" else "fast_multipole"
        if "nearRelativeTolerance" in given:
            n.near_relative_tolerance = _in_range(given["nearRelativeTolerance"], 1e-10, .01)
        if "nearMaximumDepth" in given:
            n.near_maximum_depth = _integer(given["nearMaximumDepth"], 10)
        if "relativeResidualTolerance" in given:
            n.relative_residual_tolerance = _in_range(given["relativeResidualTolerance"], 1e-7, .01)
    _acceleration_name(n.acceleration)
    _require(n.near_maximum_depth <= 10, "Maximale Nahquadraturtiefe muss zwischen 0 und 10 liegen.")
    return StudyRequest(request, metadata, ref_name, ref_face)


def _reference_velocity(faces, face_id: int) -> complex:
    for f in faces:
        if f.face_id == face_id:
            _require(complex(f.normal_velocity) != 0, "Die Bezugsfläche muss tatsächlich mit v != 0 angeregt werden.")
            return complex(f.normal_velocity)
    _study("Die Bezugsfläche muss tatsächlich mit v != 0 angeregt werden.")


def _acceleration_name(value: str) -> str:
    _require(value in ("dense", "fast_multipole"), "Unbekannter Beschleunigungsmodus.")
    return "dense" if value == "dense" else "fastMultipole"


def _encode_complex(value: complex) -> list:
    value = complex(value)
    _require(math.isfinite(value.real) and math.isfinite(value.imag), "Nicht endlicher komplexer Ergebniswert.")
    return [value.real, value.imag]


def _nonnegative(value: float) -> float:
    _require(math.isfinite(value) and value >= 0, "Nicht endlicher oder negativer Ergebniswert.")
    return float(value)


def describe_study_capabilities() -> dict:
    """The capabilities document with the input schema (simulation_api.cpp:108-159, 297-315)."""
    number = {"type": "number"}
    positive = {"type": "number", "exclusiveMinimum": 0}
    text = {"type": "string", "minLength": 1, "maxLength": 4096}
    face_id = {"type": "integer", "minimum": 1, "maximum": 4294967295.0}

    def obj(properties, required):
        return {"type": "object", "properties": properties, "required": required, "additionalProperties": False}

    def arr(items, lo, hi):
        return {"type": "array", "items": items, "minItems": lo, "maxItems": hi}

    frequencies = dict(arr(positive, 1, MAXIMUM_FREQUENCIES),
                       description="Explicit strictly ascending positive frequencies in Hz.")
    observers = dict(arr(obj({"id": text, "role": {"type": "string", "enum": ["reference", "validation", "sample"]},
                              "positionMetres": arr(number, 3, 3)}, ["id", "role", "positionMetres"]),
                         1, MAXIMUM_OBSERVERS),
                     description="Unique IDs; exactly one reference role. World SI coordinates.")
    excitation = obj({"name": text, "faces": arr(obj({"faceId": face_id, "normalVelocity": arr(number, 2, 2)},
                                                     ["faceId", "normalVelocity"]), 1, 65536)}, ["name", "faces"])
    finite = obj({"mode": {"const": "finite"}}, ["mode"])
    far = obj({"mode": {"const": "far_field"}, "originMetres": arr(number, 3, 3), "referenceDistanceMetres": positive},
              ["mode"])
    schema = obj({
        "frequenciesHz": frequencies, "observers": observers,
        "observation": {"oneOf": [finite, far],
                        "description": "Default: finite. Far-field defaults: origin [0,0,0], distance 1 m."},
        "excitations": arr(excitation, 1, MAXIMUM_EXCITATIONS),
        "reference": obj({"excitation": text, "faceId": face_id}, ["excitation", "faceId"]),
        "medium": obj({"densityKgM3": positive, "soundSpeedMetresPerSecond": positive},
                      ["densityKgM3", "soundSpeedMetresPerSecond"]),
        "numerics": obj({"acceleration": {"enum": ["dense", "fastMultipole"]},
                         "nearRelativeTolerance": {"type": "number", "minimum": 1e-10, "maximum": .01},
                         "nearMaximumDepth": {"type": "integer", "minimum": 0, "maximum": 10},
                         "relativeResidualTolerance": {"type": "number", "minimum": 1e-7, "maximum": .01}}, [])},
        ["frequenciesHz", "observers", "excitations", "reference"])
    return {"schemaVersion": 1, "inputSchema": schema, "geometryMode": "threeDimensional",
            "sourceModel": "prescribed_normal_velocity", "observations": ["finite", "far_field"],
            "acceleration": ["dense", "fastMultipole"], "maximumFrequencies": MAXIMUM_FREQUENCIES,
            "maximumObservers": MAXIMUM_OBSERVERS, "maximumExcitations": MAXIMUM_EXCITATIONS,
            "unsupportedActiveProjectPhysics": ["LEM", "infinite_baffle", "axisymmetric_m0"],
            "excitationConvention": "Complex RMS m/s into the BEM air domain; omitted Driven faces have zero "
                                    "velocity.",
            "transferDefinition": "p / actual reference-face normal velocity, in Pa/(m/s), for every observer of "
                                  "the selected excitation.",
            "modalDecomposition": False, "impulseResponse": False, "firDesign": False}


def complex_result_document(study: StudyRequest, result: BemResult) -> dict:
    """The ``hornsculpt.complex-study`` document of a solved study (simulation_api.cpp:317-466).
    The actual face velocities are the requested ones (the velocities are prescribed).
    Fields of the reference's fast-multipole audit that this solver does not report
    (operator discrepancy, accuracy seeds, far-quadrature discrepancy) are 0."""
    bem = study.request
    _require(len(result.frequencies) == len(bem.frequencies) and result.frequencies and
             len(study.observer_metadata) == len(bem.observers) and result.acceleration == bem.numerics.acceleration
             and bool(result.device) and result.triangle_count and result.pressure_dof_count,
             "Ergebnis und Studienauftrag passen nicht zusammen.")
    requested = [{"name": e.name, "faces": [{"faceId": float(f.face_id), "normalVelocity": _encode_complex(f.normal_velocity)}
                                             for f in e.faces]} for e in bem.excitations]
    reference_observer = next((m["id"] for m in study.observer_metadata if m.get("role") == "reference"), "")
    _require(bool(reference_observer), "Referenzbeobachter fehlt.")
    frequencies = []
    for f, frame in enumerate(result.frequencies):
        _require(math.isfinite(frame.frequency) and frame.frequency == bem.frequencies[f] and
                 len(frame.excitations) == len(bem.excitations),
                 "Frequenz- oder Anregungszuordnung des Ergebnisses stimmt nicht.")
        excitations, selected = [], None
        for ex, given in zip(frame.excitations, bem.excitations):
            _require(ex.name == given.name and len(ex.observer_pressure) == len(bem.observers),
                     "Komplexe Beobachter- oder Quellendaten sind unvollständig.")
            velocities = [{"faceId": float(v.face_id), "normalVelocity": _encode_complex(v.normal_velocity)}
                          for v in given.faces]
            impedances = [{"faceId": float(z.face_id), "areaSquareMetres": z.area,
                           "meanPressurePaRms": _encode_complex(z.mean_pressure),
                           "volumeVelocityCubicMetresPerSecondRms": _encode_complex(z.volume_velocity),
                           "volumeImpedancePascalSecondsPerCubicMetre": _encode_complex(z.volume_impedance)}
                          for z in ex.impedances]
            residual = _nonnegative(ex.boundary_residual)
            _require(residual <= bem.numerics.relative_residual_tolerance,
                     "Gleichungs-Auditrest überschreitet die angeforderte Toleranz.")
            fmm = bem.numerics.acceleration == "fast_multipole"
            excitations.append({
                "name": ex.name, "pressurePaRms": [_encode_complex(p) for p in ex.observer_pressure],
                "actualFaceVelocitiesMetresPerSecondRms": velocities, "sourceImpedances": impedances,
                "relativeBoundaryResidual": residual,
                "residualEvaluation": "higherOrderFastMultipole" if fmm else "directGalerkin",
                "fastMultipoleKrylovResidual": residual if fmm else 0.0,
                "fastMultipoleKrylovTarget": bem.numerics.relative_residual_tolerance if fmm else 0.0,
                "fastMultipoleOperatorDiscrepancy": 0.0, "fastMultipoleAccuracySeed": 0.0,
                "fastMultipoleComparisonAccuracySeed": 0.0, "fastMultipoleVerificationAccuracySeed": 0.0,
                "farQuadratureDiscrepancy": 0.0,
                "fieldQuadratureDiscrepancy": _nonnegative(ex.field_quadrature_discrepancy),
                "refinementSteps": int(ex.refinement_steps), "iterations": int(ex.iterations)})
            if ex.name == study.reference_excitation:
                v = _reference_velocity(given.faces, study.reference_face_id)
                selected = {"excitation": study.reference_excitation, "referenceFaceId": float(study.reference_face_id),
                            "referenceVelocity": _encode_complex(v), "unit": "Pa/(m/s)",
                            "pressureOverReferenceVelocity": [_encode_complex(p / v) for p in ex.observer_pressure]}
        _require(selected is not None, "Komplexe Bezugsübertragung fehlt.")
        frequencies.append({
            "frequencyHz": frame.frequency, "excitations": excitations, "selectedTransfer": selected,
            "timingMilliseconds": {"assembly": _nonnegative(frame.assembly_milliseconds),
                                   "solve": _nonnegative(frame.solve_milliseconds),
                                   "factorization": _nonnegative(frame.factorization_milliseconds),
                                   "triangularSolve": _nonnegative(frame.triangular_solve_milliseconds),
                                   "field": _nonnegative(frame.field_milliseconds),
                                   "residualCheck": _nonnegative(frame.residual_check_milliseconds),
                                   "interactionPlan": _nonnegative(frame.interaction_plan_milliseconds)},
            "interactionPlanReused": bool(frame.interaction_plan_reused)})
    n = bem.numerics
    if bem.far_field is not None:
        observation = {"mode": "far_field", "originMetres": list(map(float, bem.far_field.origin)),
                       "referenceDistanceMetres": bem.far_field.reference_distance,
                       "coordinateMeaning": "directions_from_origin",
                       "pressureMeaning": "asymptotic_outgoing_pressure_at_reference_distance"}
    else:
        observation = {"mode": "finite", "originMetres": None, "referenceDistanceMetres": None,
                       "coordinateMeaning": "physical_world_points", "pressureMeaning": "finite_distance_pressure"}
    fm = n.fast_multipole
    return {
        "schema": "hornsculpt.complex-study", "schemaVersion": 1,
        "conventions": {"time": "exp(+i*omega*t)", "outgoingWave": "exp(-i*k*r)", "amplitude": "RMS",
                        "complexEncoding": "[real,imaginary]", "lengthUnit": "m", "frequencyUnit": "Hz",
                        "pressureUnit": "Pa", "positiveNormalVelocity": "into_the_BEM_air_domain"},
        "medium": {"densityKgM3": bem.medium.density, "soundSpeedMetresPerSecond": bem.medium.sound_speed},
        "observation": observation, "observers": study.observer_metadata,
        "reference": {"excitation": study.reference_excitation, "faceId": float(study.reference_face_id),
                      "observerId": reference_observer},
        "requestedExcitations": requested,
        "numerics": {"quadratureOrder": n.quadrature_order, "singularOrder": n.singular_order,
                     "nearDistanceRatio": n.near_distance_ratio, "nearRelativeTolerance": n.near_relative_tolerance,
                     "nearMaximumDepth": n.near_maximum_depth,
                     "relativeResidualTolerance": n.relative_residual_tolerance,
                     "maximumRefinementSteps": n.maximum_refinement_steps,
                     "acceleration": _acceleration_name(n.acceleration),
                     "fastMultipole": {"leafSupportCapacity": fm.leaf_support_capacity,
                                       "preconditionerBlockWidth": fm.preconditioner_block_width,
                                       "orderSelection": "automatic_per_level",
                                       "separationRatio": fm.separation_ratio,
                                       "maximumIterations": fm.maximum_iterations,
                                       "restartLength": fm.restart_length}},
        "solver": {"device": result.device, "triangleCount": float(result.triangle_count),
                   "pressureDofCount": float(result.pressure_dof_count),
                   "peakDeviceBytes": float(result.peak_device_bytes),
                   "acceleration": _acceleration_name(result.acceleration), "geometryMode": "threeDimensional",
                   "method": "Burton-Miller Galerkin P1/DP0"},
        "frequencies": frequencies,
        "audioInterpretation": "Finite positive-frequency acoustic samples; no IR, FIR or modal decomposition has "
                               "been computed."}
