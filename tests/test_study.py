"""The MCP study adapter restated (apps/mcp/simulation_api.cpp): the study JSON
parser with the reference's checks, order and messages, the capabilities document
and the complex result document. Host only."""
import copy

import numpy as np
import pytest

import hornsculpt_b200 as hs
from hornsculpt_b200 import meshes


def _mesh():
    """icosphere s1 with faces 17 and 29 driven, the rest wall face 90."""
    m = meshes.icosphere(1)
    z = m.vertices[m.triangles][:, :, 2].mean(axis=1)
    x = m.vertices[m.triangles][:, :, 0].mean(axis=1)
    faces = np.where(z > 0.06, 17, np.where(x < -0.06, 29, 90)).astype(np.uint32)
    kind = np.where(faces == 90, meshes.WALL, meshes.DRIVEN).astype(np.uint8)
    return meshes.SurfaceMesh(m.vertices, m.triangles, faces, kind)


STUDY = {
    "frequenciesHz": [200, 500.5, 1000],
    "observers": [{"id": "on-axis", "role": "reference", "positionMetres": [0, 0, 1]},
                  {"id": "side", "role": "sample", "positionMetres": [1, 0, 0]}],
    "excitations": [{"name": "drive", "faces": [{"faceId": 17, "normalVelocity": [1, 0]},
                                                {"faceId": 29, "normalVelocity": [0, 0.5]}]},
                    {"name": "port2", "faces": [{"faceId": 29, "normalVelocity": [2, 0]}]}],
    "reference": {"excitation": "drive", "faceId": 17},
    "medium": {"densityKgM3": 1.2, "soundSpeedMetresPerSecond": 340},
    "numerics": {"acceleration": "fastMultipole", "relativeResidualTolerance": 1e-6},
}


def test_valid_study():
    s = hs.parse_study_request(STUDY, _mesh(), numerics=hs.BemNumerics(near_maximum_depth=5))
    r = s.request
    assert r.frequencies == [200.0, 500.5, 1000.0] and r.interaction_plan_frequencies == r.frequencies
    assert r.observers == [(0.0, 0.0, 1.0), (1.0, 0.0, 0.0)] and r.far_field is None
    assert [e.name for e in r.excitations] == ["drive", "port2"]
    assert r.excitations[0].faces[1].normal_velocity == 0.5j
    assert (r.medium.density, r.medium.sound_speed) == (1.2, 340.0)
    assert r.numerics.acceleration == "fast_multipole" and r.numerics.relative_residual_tolerance == 1e-6
    assert r.numerics.near_maximum_depth == 5  # from the project
    assert (s.reference_excitation, s.reference_face_id) == ("drive", 17)
    assert [m["id"] for m in s.observer_metadata] == ["on-axis", "side"]
    # the text form parses the same
    import json
    assert hs.parse_study_request(json.dumps(STUDY), _mesh()).request.frequencies == r.frequencies


def test_far_field_observation_defaults():
    study = dict(STUDY, observation={"mode": "far_field"})
    r = hs.parse_study_request(study, _mesh()).request
    assert r.far_field.origin == (0.0, 0.0, 0.0) and r.far_field.reference_distance == 1.0


def _edit(path, value=None, delete=False):
    study = copy.deepcopy(STUDY)
    target = study
    for key in path[:-1]:
        target = target[key]
    if delete:
        del target[path[-1]]
    else:
        target[path[-1]] = value
    return study


@pytest.mark.parametrize("study, message", [
    (_edit(["extra"], 1), "MCP-Studie: Unbekanntes Feld: extra"),
    (_edit(["frequenciesHz"], [500, 200]), "Frequenzen müssen streng aufsteigend sein."),
    (_edit(["frequenciesHz"], [0]), "Ungültige Projektdatei: Positive Zahl erwartet."),
    (_edit(["frequenciesHz"], []), "Listenlänge außerhalb des erlaubten Bereichs."),
    (_edit(["frequenciesHz"], delete=True), "Ungültige Projektdatei: Liste erwartet."),
    (_edit(["observers", 1, "id"], "on-axis"), "Doppelte Beobachter-ID: on-axis"),
    (_edit(["observers", 1, "role"], "reference"), "Genau ein Beobachter benötigt die Rolle reference."),
    (_edit(["observers", 1, "role"], "probe"), "Unbekannte Beobachterrolle."),
    (_edit(["observers", 0, "rolle"], "x"), "Felder fehlen: ; unbekannte Felder: rolle."),
    (_edit(["observers", 0, "id"], "  "), "Leere ID oder Anregungsbezeichnung."),
    (_edit(["observation"], {"mode": "near"}), "Beobachtungsmodus muss finite oder far_field sein."),
    (_edit(["observation"], {"mode": "far_field", "originMetres": [0, 0, 1]}),
     "Fernfeldrichtung muss endlich und vom Ursprung verschieden sein."),
    (_edit(["excitations", 0, "faces", 0, "faceId"], 90),
     "Jede Anregung darf vorhandene Driven-Flächen höchstens einmal zuweisen."),
    (_edit(["excitations", 0, "faces", 1, "faceId"], 17),
     "Jede Anregung darf vorhandene Driven-Flächen höchstens einmal zuweisen."),
    (_edit(["excitations", 1, "faces", 0, "normalVelocity"], [0, 0]),
     "Jede Anregung benötigt mindestens eine Geschwindigkeit != 0."),
    (_edit(["excitations", 1, "name"], "drive"), "Doppelte Anregung: drive"),
    (_edit(["reference", "excitation"], "none"), "Bezugsanregung fehlt."),
    (_edit(["reference", "faceId"], 29), None),
    (_edit(["reference"], {"excitation": "port2", "faceId": 17}),
     "Die Bezugsfläche muss tatsächlich mit v != 0 angeregt werden."),
    (_edit(["numerics", "relativeResidualTolerance"], 1.0), "Numerikwert außerhalb des unterstützten Bereichs."),
    (_edit(["numerics", "acceleration"], "tree"), "Unbekannter Beschleunigungsmodus."),
    (_edit(["numerics", "nearMaximumDepth"], 11), "Ungültige Ganzzahl oder ID."),
    (_edit(["numerics", "quadratureOrder"], 4), "Unbekanntes Feld: quadratureOrder"),
    (_edit(["medium", "densityKgM3"], -1), "Positive Zahl erwartet."),
    # an integer literal beyond double range (JSON digits, not a float) is rejected as not finite
    (_edit(["medium", "densityKgM3"], 10 ** 400), "Endliche Zahl erwartet."),
    (_edit(["frequenciesHz"], [200, 10 ** 400]), "Endliche Zahl erwartet."),
])
def test_study_errors(study, message):
    if message is None:  # a valid variant
        hs.parse_study_request(study, _mesh())
        return
    with pytest.raises(ValueError) as err:
        hs.parse_study_request(study, _mesh())
    assert message in str(err.value)


def test_capabilities_document():
    doc = hs.describe_study_capabilities()
    schema = doc["inputSchema"]
    assert schema["required"] == ["frequenciesHz", "observers", "excitations", "reference"]
    assert schema["properties"]["excitations"]["maxItems"] == 16
    assert doc["maximumFrequencies"] == 8192 and doc["acceleration"] == ["dense", "fastMultipole"]


def _result(study, residual=1e-8):
    r = study.request
    frames = []
    for f in r.frequencies:
        exc = []
        for e, ex in enumerate(r.excitations):
            p = np.array([1 + 2j, 3 - 1j]) * (e + 1) * f / 1000
            imp = [hs.FaceImpedance(fv.face_id, 0.01, 1 + 1j, 0.01 * fv.normal_velocity, (1 + 1j) / (0.01 * fv.normal_velocity))
                   for fv in ex.faces if fv.normal_velocity != 0]
            bd = hs.BemBoundaryData(np.zeros(3, complex), np.zeros(3, complex), np.zeros(3, complex))
            exc.append(hs.BemExcitationResult(ex.name, p, imp, 1, residual, 6, 8, 1e-9, bd, 12))
        frames.append(hs.BemFrequencyResult(f, exc, 1, 2, 0.5, 0.5, 0.1, 0.2, 0, True))
    return hs.BemResult("NVIDIA B200", 80, 42, 1 << 20, frames, acceleration=r.numerics.acceleration)


def test_complex_result_document():
    study = hs.parse_study_request(STUDY, _mesh())
    doc = hs.complex_result_document(study, _result(study))
    assert doc["schema"] == "hornsculpt.complex-study" and len(doc["frequencies"]) == 3
    t = doc["frequencies"][1]["selectedTransfer"]
    assert t["excitation"] == "drive" and t["referenceVelocity"] == [1.0, 0.0]
    p = study and np.array([1 + 2j, 3 - 1j]) * 500.5 / 1000
    assert np.allclose([complex(*v) for v in t["pressureOverReferenceVelocity"]], p)
    assert doc["reference"]["observerId"] == "on-axis"
    assert doc["numerics"]["acceleration"] == "fastMultipole"
    assert doc["frequencies"][0]["excitations"][0]["residualEvaluation"] == "higherOrderFastMultipole"
    with pytest.raises(ValueError, match="Auditrest"):
        hs.complex_result_document(study, _result(study, residual=1e-3))
