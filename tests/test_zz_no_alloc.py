"""The allocation-free observer field, hs_bem_observer_field_noalloc.

Some callers cannot allocate device memory at the moment they need a field:
an interactive frequency sweep that must not stall on the device-wide
synchronisation cudaMalloc/cudaFree imply, or a host application that gives
the solver only memory from its own pre-sized arena. This test plays such a
caller: it owns every device buffer (allocated up front), calls the entry
point through the C ABI twice in a row, and checks the result against the
observer pressure that hs_bem_solve (the existing entry point) reports for
the same solved traces at the same rule degree. The file runs last so that a
failure here leaves every other test already run.
"""
import ctypes as C

import numpy as np
import pytest
import torch

import hornsculpt_b200 as hs
from hornsculpt_b200 import _lib, meshes

pytestmark = pytest.mark.gpu

# Same field kernel and arithmetic as the solve; only the panel table is
# built on the device instead of the host (last-bit differences at most).
TOLERANCE = 1e-12


def _device(array, dtype):
    return torch.as_tensor(np.ascontiguousarray(array), dtype=dtype, device="cuda")


def _complex_pairs(z):
    z = np.asarray(z, np.complex128)
    return np.stack([z.real, z.imag], -1)


def _call(mesh_dev, trace, flux, observers, k, degree, far=None, tolerance=1.25e-6, depth=6, out=None,
          triangle_count=None):
    lib = _lib.load()
    vertices, triangles = mesh_dev
    origin = (C.c_double * 3)(*(far[0] if far else (0.0, 0.0, 0.0)))
    status = lib.hs_bem_observer_field_noalloc(
        vertices.data_ptr(), vertices.shape[0], triangles.data_ptr(),
        triangle_count if triangle_count is not None else triangles.shape[0], trace.data_ptr(), flux.data_ptr(),
        observers.data_ptr(), observers.shape[0], k, degree, int(far is not None), origin,
        far[1] if far else 1.0, tolerance, depth, C.c_void_p(torch.cuda.current_stream().cuda_stream),
        out.data_ptr())
    _lib.check(status)
    return out


@pytest.mark.parametrize("far", [None, ((0.01, 0.0, 0.0), 2.0)], ids=["finite", "far_field"])
def test_noalloc_field_matches_solve(far):
    mesh = meshes.octahedral_sphere(3)
    freqs = [500.0, 1715.0]
    # the last finite observer sits 5 mm off the surface: adaptive near-field panels
    obs = [(0, 0, .3), (1, 0, 0), (0, 0, .105)] if far is None else [(0, 0, 1), (1, 0, 0), (0, -1, 0)]
    request = hs.BemRequest(frequencies=freqs, observers=obs,
                            excitations=[hs.BemExcitation("unit", [hs.FaceVelocity(1, 1.0)])],
                            far_field=None if far is None else hs.FarFieldObservation(*far))
    with hs.CudaBemSolver(mesh) as solver:
        result = solver.solve(request)
    mesh_dev = (_device(mesh.vertices, torch.float64), _device(mesh.triangles.astype(np.int32), torch.int32))
    observers = _device(np.asarray(obs, np.float64), torch.float64)
    for i, f in enumerate(freqs):
        ex = result.frequencies[i].excitations[0]
        k = 2 * np.pi * f / request.medium.sound_speed
        trace = _device(_complex_pairs(ex.boundary.pressure_trace), torch.float64)
        flux = _device(_complex_pairs(ex.boundary.normal_derivative), torch.float64)
        expected = np.asarray(ex.observer_pressure)
        for _ in range(2):  # two calls in a row reuse the same scratch
            out = torch.full((len(obs), 2), np.nan, dtype=torch.float64, device="cuda")
            _call(mesh_dev, trace, flux, observers, k, ex.field_quadrature_verification_degree, far=far, out=out)
            got = out.cpu().numpy()
            got = got[:, 0] + 1j * got[:, 1]
            assert np.max(np.abs(got - expected)) <= TOLERANCE * np.max(np.abs(expected))


def test_noalloc_field_rejects_sizes_beyond_its_scratch():
    """32768 triangles need 6.5 MB of panel scratch: refused before any device work."""
    big = meshes.octahedral_sphere(6)
    mesh_dev = (_device(big.vertices, torch.float64), _device(big.triangles.astype(np.int32), torch.int32))
    trace = torch.zeros((big.vertex_count, 2), dtype=torch.float64, device="cuda")
    flux = torch.zeros((big.triangle_count, 2), dtype=torch.float64, device="cuda")
    observers = _device(np.array([[0, 0, 1.0]]), torch.float64)
    out = torch.zeros((1, 2), dtype=torch.float64, device="cuda")
    with pytest.raises(ValueError, match="fixed maximum"):
        _call(mesh_dev, trace, flux, observers, 10.0, 4, out=out)
