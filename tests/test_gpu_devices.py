"""Sessions on two devices of one process. Constant-memory quadrature tables,
kernel attributes and cluster limits are per device: a solve on device 1 after
one on device 0 must find its own tables uploaded, and give the same result
bit for bit. Skipped when fewer than two devices are visible."""
import numpy as np
import pytest
import torch

import hornsculpt_b200 as hs
from hornsculpt_b200 import meshes

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(torch.cuda.device_count() < 2, reason="needs two visible CUDA devices")]


def _solve(device, numerics):
    mesh = meshes.octahedral_sphere(3)
    request = hs.BemRequest(frequencies=[500.0, 2000.0], observers=[(0, 0, 0.3), (1, 0, 0)],
                            excitations=[hs.BemExcitation("unit", [hs.FaceVelocity(1, 1.0)])], numerics=numerics)
    with torch.cuda.device(device):
        with hs.CudaBemSolver(mesh) as solver:
            return solver.solve(request)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_second_device_matches_first(precision):
    numerics = hs.BemNumerics(precision=precision)
    first, second = _solve(0, numerics), _solve(1, numerics)
    for f0, f1 in zip(first.frequencies, second.frequencies):
        e0, e1 = f0.excitations[0], f1.excitations[0]
        assert np.array_equal(e0.boundary.pressure_trace, e1.boundary.pressure_trace)
        assert np.array_equal(e0.observer_pressure, e1.observer_pressure)
        assert np.all(np.abs(e1.observer_pressure) > 0)
