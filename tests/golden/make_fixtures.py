"""Regenerates the golden fixtures of this directory from the reference tree.

Run where the reference tree is mounted, after `make -C oracle
REFERENCE=<reference root>` has compiled oracle/_ref/libhsref.so:

    python tests/golden/make_fixtures.py <reference root>

Writes
  beat_sphere_512.json       external BEAT CPU FP64 observer pressures on the
                             512-triangle octahedral sphere (reference
                             tests/data/beat-sphere-512.csv)
  beat_tetra_singular12.json external BEAT CUDA FP64 port means of the scalene
                             tetrahedron, singular order 12 (reference
                             tests/data/beat-scalene-tetra-singular12.csv)
  reference_rules.json       the reference's own triangle and Gauss rules
  reference_plans.npz        interaction plans computed by the reference's
                             own makeInteractionPlan on small meshes
"""
from __future__ import annotations

import json
import pathlib
import sys

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

from hornsculpt_b200 import meshes  # noqa: E402
from oracle import oracle  # noqa: E402

# Meshes and planning wavenumbers of the plan fixtures.
PLAN_CASES = [
    ("octa2_1715", lambda: meshes.octahedral_sphere(2), 1715.0, {}),
    ("octa3_1000", lambda: meshes.octahedral_sphere(3), 1000.0, {}),
    ("ico2_3000", lambda: meshes.icosphere(2), 3000.0, {}),
    ("octa2_tight", lambda: meshes.octahedral_sphere(2), 2000.0, {"near_tol": 1e-6}),
    ("tetra_400", meshes.scalene_tetrahedron, 400.0, {"singular_order": 12}),
]


def csv_rows(path):
    return [line.strip() for line in open(path) if line.strip() and not line.startswith("#")]


def main(reference: str) -> None:
    ref = pathlib.Path(reference)
    sphere = []
    for row in csv_rows(ref / "tests/data/beat-sphere-512.csv"):
        v = [float(x) for x in row.split(",")]
        sphere.append({"frequency": v[0], "pressure": [[v[1], v[2]], [v[3], v[4]], [v[5], v[6]]]})
    (HERE / "beat_sphere_512.json").write_text(json.dumps({
        "mesh": "octahedral sphere, 3 refinements, radius 0.1 m, all faces driven 1 m/s RMS",
        "density": 1.21, "sound_speed": 343.0,
        "observers": [[0, 0, .3], [1, 0, 0], [0, 0, 3]],
        "rows": sphere}, indent=1))
    ports = []
    for row in csv_rows(ref / "tests/data/beat-scalene-tetra-singular12.csv"):
        ex, face, area, qr, qi, pr, pi, zr, zi = row.split(",")
        ports.append({"excitation": ex, "face": int(face), "area": float(area), "volume_velocity": [float(qr), float(qi)],
                      "mean_pressure": [float(pr), float(pi)], "impedance": [float(zr), float(zi)]})
    (HERE / "beat_tetra_singular12.json").write_text(json.dumps({
        "frequency": 400.0, "density": 1.21, "sound_speed": 343.0, "singular_order": 12,
        "excitations": {"uniform": [[50, 1.0], [51, 1.0]], "antisymmetric": [[50, 1.0], [51, -1.0]]},
        "ports": ports}, indent=1))
    rules = {"triangle": {d: oracle.reference_triangle_rule(d).tolist() for d in (2, 4, 6, 8, 12, 14)},
             "gauss": {n: oracle.reference_gauss(n).tolist() for n in range(2, 21)}}
    (HERE / "reference_rules.json").write_text(json.dumps(rules))
    arrays = {}
    for name, make, freq, overrides in PLAN_CASES:
        mesh = make()
        k = 2 * np.pi * freq / 343.0
        plan = oracle.reference_plan(mesh, oracle.Numerics.default(**overrides), k)
        for key in ("touching", "near", "patches", "whole", "trials", "offsets"):
            arrays[f"{name}/{key}"] = plan[key]
        arrays[f"{name}/k"] = np.array([k])
    np.savez_compressed(HERE / "reference_plans.npz", **arrays)
    print("fixtures written to", HERE)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_fixtures.py <reference root>")
    main(sys.argv[1])
