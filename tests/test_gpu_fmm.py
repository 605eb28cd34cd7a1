"""Fast-multipole form on the GPU: the far-field operator (P2M, rotation-based
M2M/M2L/L2L, L2P on the reference's support-tree partition) against the far
support pairs of the dense FP64 matrix of the same discretisation."""
import numpy as np
import pytest

import hornsculpt_b200 as hs
from hornsculpt_b200 import meshes

pytestmark = pytest.mark.gpu

FP64 = hs.BemNumerics(precision="fp64")


def _far_mask(N, row, cols):
    mask = np.ones((N, N), bool)
    for i in range(N):
        mask[i, cols[row[i]:row[i + 1]]] = False
    return mask


@pytest.mark.parametrize("case, freq", [("icosphere3", 500.0), ("icosphere3", 3000.0), ("horn", 2000.0)])
def test_far_operator_matches_dense_far_part(case, freq):
    mesh = {"icosphere3": lambda: meshes.icosphere(3),
            "horn": lambda: meshes.exponential_horn(h=0.0128, seed=5)}[case]()
    N, T = mesh.vertex_count, mesh.triangle_count
    k = 2 * np.pi * freq / 343.0
    rng = np.random.default_rng(11)
    p = rng.normal(size=N) + 1j * rng.normal(size=N)
    with hs.CudaBemSolver(mesh) as solver:
        A, _ = solver.debug_assemble(FP64, k, k, np.zeros(T, complex))
        far, row, cols, levels = solver.debug_fmm_far(FP64, k, 1e-8, p)
    mask = _far_mask(N, row, cols)
    expected = (A * mask) @ p
    full = A @ p
    assert len(levels) > 0 and mask.sum() > 0
    far_rel = np.linalg.norm(far - expected) / np.linalg.norm(expected)
    full_rel = np.linalg.norm(far - expected) / np.linalg.norm(full)
    print(case, freq, "levels", levels.tolist(), "far rel", far_rel, "of full", full_rel)
    assert full_rel < 1e-6
    assert far_rel < 1e-4


@pytest.mark.parametrize("case, freqs", [("icosphere3", [500.0, 2500.0]), ("horn", [1500.0])])
def test_fast_multipole_solve_matches_dense(case, freqs):
    """acceleration = fast_multipole (FP64): GMRES on near + expansion far field with
    block-Jacobi, against the dense FP64 LU solve of the same discretisation."""
    mesh, face = {"icosphere3": (meshes.icosphere(3), 1),
                  "horn": (meshes.exponential_horn(h=0.0128, seed=5), meshes.HORN_THROAT)}[case]
    obs = [(0.0, 0.0, 0.4), (0.5, 0.1, 0.0)]

    def request(acc):
        return hs.BemRequest(frequencies=freqs, observers=obs,
                             excitations=[hs.BemExcitation("drive", [hs.FaceVelocity(face, 1.0)])],
                             numerics=hs.BemNumerics(precision="fp64", acceleration=acc,
                                                     relative_residual_tolerance=1e-7))
    with hs.CudaBemSolver(mesh) as solver:
        dense = solver.solve(request("dense"))
        fmm = solver.solve(request("fast_multipole"))
    for fd, ff in zip(dense.frequencies, fmm.frequencies):
        ed, ef = fd.excitations[0], ff.excitations[0]
        trace = np.linalg.norm(ef.boundary.pressure_trace - ed.boundary.pressure_trace) / np.linalg.norm(
            ed.boundary.pressure_trace)
        field = np.linalg.norm(ef.observer_pressure - ed.observer_pressure) / np.linalg.norm(ed.observer_pressure)
        print(case, ff.frequency, "trace", trace, "field", field, "iterations", ef.iterations,
              "residual", ef.boundary_residual)
        assert ef.iterations > 0
        assert ef.boundary_residual <= 1e-6
        assert trace < 1e-5 and field < 1e-5
