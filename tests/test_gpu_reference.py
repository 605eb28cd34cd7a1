"""The reference's own GPU implementation on the same inputs: HornSculpt's
CudaBemSolver compiled from its sources (oracle/refgpu.mk, CUDA 12.9 for
sm_100a, with two link stubs for CGAL-backed meshing) and driven by the same
caller as the adapter over this library (hornsculpt_b200/adapter/adapter_solve.cpp).
Its FP32 LU with FP64 refinement to a 1e-7 residual against this library's plain
FP64 and mixed forms on the C1 sphere: surface pressure within the FP32 forms'
1e-5 bar."""
import pathlib
import subprocess

import numpy as np
import pytest

import hornsculpt_b200 as hs
from hornsculpt_b200 import meshes
from test_adapter import _write_input

pytestmark = pytest.mark.gpu

REFERENCE_SOLVE = pathlib.Path(__file__).resolve().parent.parent / "oracle" / "_ref" / "reference_solve"


@pytest.mark.skipif(not REFERENCE_SOLVE.exists(), reason="reference GPU harness not built")
def test_reference_gpu_solver_matches_ours_on_c1(tmp_path):
    mesh = meshes.icosphere(3)
    freqs = [100.0, 1200.0, 5000.0]
    obs = [(0.0, 0.0, 0.3), (1.0, 0.0, 0.0), (0.0, 0.0, 3.0)]
    density, c = 1.205, 343.0
    _write_input(tmp_path / "in.bin", mesh, freqs, obs, density, c, tolerance=1e-7)
    run = subprocess.run([str(REFERENCE_SOLVE), str(tmp_path / "in.bin"), str(tmp_path / "out.bin")],
                         capture_output=True, text=True, timeout=900)
    assert run.returncode == 0, run.stderr
    raw = np.fromfile(tmp_path / "out.bin", np.float64)
    N, O = mesh.vertex_count, len(obs)
    per = 2 * N + 2 * O + 1
    v = mesh.vertices[mesh.triangles]
    area = 0.5 * np.linalg.norm(np.cross(v[:, 1] - v[:, 0], v[:, 2] - v[:, 0]), axis=1)
    for precision in ("fp64", "mixed"):
        request = hs.BemRequest(frequencies=freqs, observers=obs, medium=hs.AcousticMedium(density, c),
                                excitations=[hs.BemExcitation("unit", [hs.FaceVelocity(1, 1.0)])],
                                numerics=hs.BemNumerics(precision=precision, relative_residual_tolerance=1e-7))
        with hs.CudaBemSolver(mesh) as solver:
            ours = solver.solve(request)
        for i, frame in enumerate(ours.frequencies):
            chunk = raw[i * per:(i + 1) * per]
            trace = chunk[:2 * N].view(np.complex128)
            observer = chunk[2 * N:2 * N + 2 * O].view(np.complex128)
            surf_ref = trace[mesh.triangles].mean(axis=1)
            e = frame.excitations[0]
            d = e.boundary.surface_pressure - surf_ref
            err = np.sqrt(np.sum(area * np.abs(d) ** 2) / np.sum(area * np.abs(surf_ref) ** 2))
            ferr = np.linalg.norm(e.observer_pressure - observer) / np.linalg.norm(observer)
            print(precision, freqs[i], "surface vs reference GPU", err, "observer", ferr, "reference residual",
                  chunk[-1])
            assert chunk[-1] <= 1e-7
            assert err < 1e-5 and ferr < 1e-5
