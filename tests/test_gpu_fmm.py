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
