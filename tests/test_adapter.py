"""The reference-side adapter (hornsculpt_b200/adapter/cuda_bem_solver_b200.cpp):
HornSculpt's own hornsculpt::CudaBemSolver class implemented over this
library's C ABI. It is compiled against the reference's headers as they are
declared there (where the reference tree is present) and linked to
libhs_bem.so; on a GPU a C1 solve through it must equal the same solve through
the Python mirror, bit for bit."""
import struct
import subprocess

import numpy as np
import pytest

import hornsculpt_b200 as hs
from hornsculpt_b200 import build, meshes

@pytest.mark.skipif(not build.ADAPTER_BINARY.exists(), reason="adapter not built (needs the reference headers)")
def test_adapter_links_only_this_library():
    """build() compiled the adapter and its driver against the reference's headers;
    at run time they need libhs_bem.so and the C++ runtime, nothing of the reference."""
    needed = subprocess.run(["ldd", str(build.ADAPTER_BINARY)], capture_output=True, text=True).stdout
    assert "libhs_bem.so" in needed and "not found" not in needed


def _write_input(path, mesh, freqs, obs, density, c, tolerance=5e-5, repeats=1):
    with open(path, "wb") as f:
        f.write(struct.pack("<4Q", mesh.vertex_count, mesh.triangle_count, len(freqs), len(obs)))
        f.write(np.ascontiguousarray(mesh.vertices, np.float64).tobytes())
        f.write(np.ascontiguousarray(mesh.triangles, np.uint32).tobytes())
        f.write(np.ascontiguousarray(mesh.face_ids, np.uint32).tobytes())
        f.write(np.ascontiguousarray(mesh.boundary, np.uint8).tobytes())
        f.write(np.asarray(freqs, np.float64).tobytes())
        f.write(np.asarray(obs, np.float64).tobytes())
        f.write(np.array([density, c, tolerance], np.float64).tobytes())
        f.write(struct.pack("<Q", repeats))


@pytest.mark.gpu
@pytest.mark.skipif(not build.ADAPTER_BINARY.exists(), reason="adapter not built (needs the reference headers)")
def test_adapter_c1_solve_equals_the_python_mirror(tmp_path):
    mesh = meshes.icosphere(3)
    freqs = [100.0, 1200.0, 5000.0]
    obs = [(0.0, 0.0, 0.3), (1.0, 0.0, 0.0), (0.0, 0.0, 3.0)]
    density, c = 1.205, 343.0
    _write_input(tmp_path / "in.bin", mesh, freqs, obs, density, c)
    run = subprocess.run([str(build.ADAPTER_BINARY), str(tmp_path / "in.bin"), str(tmp_path / "out.bin")],
                         capture_output=True, text=True, timeout=600)
    assert run.returncode == 0, run.stderr
    raw = np.fromfile(tmp_path / "out.bin", np.float64)
    N, O = mesh.vertex_count, len(obs)
    per = 2 * N + 2 * O + 1
    assert raw.size == per * len(freqs)
    request = hs.BemRequest(frequencies=freqs, observers=obs, medium=hs.AcousticMedium(density, c),
                            excitations=[hs.BemExcitation("unit", [hs.FaceVelocity(1, 1.0)])])
    with hs.CudaBemSolver(mesh) as solver:
        mirror = solver.solve(request)
    for i, frame in enumerate(mirror.frequencies):
        chunk = raw[i * per:(i + 1) * per]
        trace = chunk[:2 * N].view(np.complex128)
        observer = chunk[2 * N:2 * N + 2 * O].view(np.complex128)
        e = frame.excitations[0]
        assert np.array_equal(trace, e.boundary.pressure_trace)
        assert np.array_equal(observer, e.observer_pressure)
        assert chunk[-1] == e.boundary_residual
