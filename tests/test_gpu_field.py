"""Post-solve pressure samples at arbitrary points (hs_bem_pressure_field,
the GPU form of HornSculpt's evaluatePressureField for the exterior closed
surface). Parity is against the reference's own field_evaluation.cpp compiled
into oracle/_ref, on the traces of a solved sphere: the same status for every
point and the same pressure to FP64 rounding (the per-panel sums are added in
another order)."""
import numpy as np
import pytest

import hornsculpt_b200 as hs
from hornsculpt_b200 import meshes
from oracle import oracle as O

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not O.reference_available(), reason="oracle/_ref not built (reference tree absent)")]

# air far and near (0.5 mm and 2 mm off the surface: adaptive subdivision),
# inside (excluded), on the surface within 0.1 mm (boundary)
POINTS = np.array([(0, 0, .3), (.2, .1, -.05), (1, 0, 0), (0, 0, .1005), (.0712, .0712, .0020),
                   (0, 0, 0), (.03, -.02, .01), (.1000001, 0, 0), (0, .09995, 0)])


def _solve(mesh, f):
    req = hs.BemRequest(frequencies=[f], observers=[tuple(p) for p in POINTS[:3]],
                        excitations=[hs.BemExcitation("u", [hs.FaceVelocity(1, 1.0)])])
    solver = hs.CudaBemSolver(mesh)
    return solver, solver.solve(req).frequencies[0].excitations[0]


@pytest.mark.parametrize("freq", [300.0, 2500.0])
def test_pressure_field_matches_reference(freq):
    mesh = meshes.icosphere(3)
    solver, sol = _solve(mesh, freq)
    with solver:
        samples = solver.pressure_field(freq, sol, POINTS)
    ref_p, ref_status = O.reference_pressure_field(mesh, freq, 343.0, sol.boundary.pressure_trace,
                                                   sol.boundary.normal_derivative, POINTS)
    status = np.array([int(s.status) for s in samples])
    p = np.array([s.pressure for s in samples])
    assert list(status) == list(ref_status)
    assert list(status[:5]) == [0] * 5 and status[5] == 2 and status[6] == 2 and status[7] == 1 and status[8] == 1
    assert np.max(np.abs(p - ref_p)) <= 1e-9 * np.max(np.abs(ref_p))
    # the solve's own observer pressure (degree loop, a different quadrature) agrees closely
    assert np.max(np.abs(p[:3] - sol.observer_pressure[:3])) <= 1e-3 * np.max(np.abs(p[:3]))


def test_pressure_field_settings_and_depth():
    mesh = meshes.icosphere(2)
    solver, sol = _solve(mesh, 800.0)
    with solver:
        with pytest.raises(ValueError, match="Invalid pressure field settings"):
            solver.pressure_field(800.0, sol, POINTS, hs.PressureFieldSettings(relative_quadrature_tolerance=0.5))
        with pytest.raises(ValueError, match="Invalid pressure field settings"):
            solver.pressure_field(800.0, sol, POINTS, hs.PressureFieldSettings(maximum_quadrature_depth=13))
        with pytest.raises(ValueError, match="Invalid pressure field point"):
            solver.pressure_field(800.0, sol, [(np.nan, 0, 0)])
        # a tight tolerance with no subdivision allowed leaves the near points unconverged, as in the reference
        tight = hs.PressureFieldSettings(relative_quadrature_tolerance=1e-8, maximum_quadrature_depth=0)
        samples = solver.pressure_field(800.0, sol, POINTS, tight)
        ref_p, ref_status = O.reference_pressure_field(mesh, 800.0, 343.0, sol.boundary.pressure_trace,
                                                       sol.boundary.normal_derivative, POINTS, tolerance=1e-8,
                                                       depth=0)
        assert [int(s.status) for s in samples] == list(ref_status)
        assert 3 in ref_status
        p = np.array([s.pressure for s in samples])
        assert np.max(np.abs(p - ref_p)) <= 1e-9 * np.max(np.abs(ref_p))
