"""The batched dense LU kernels checked directly, not only through solves.

Both factorisations the solver uses are run through the C ABI test hook
hs_bem_debug_lu and compared with LAPACK (scipy's zgetrf / cgetrf, the
algorithm behind the reference's cusolverDnCgetrf, cuda_solver.cu:1485-1513):

* FP64 (the plain form): the interchange sequence equals LAPACK zgetrf's, and
  the factorisation passes LAPACK's own acceptance test xGET01,
  ||P A - L U||_1 / (n ||A||_1 eps) < 30, with a Frobenius residual within
  twice LAPACK's on the same matrix.
* FP32 (the mixed form; tensor-core trailing updates): the same xGET01 ratio
  with FP32 eps, and a Frobenius residual within eight times cgetrf's. Its
  pivots are its own (near ties break differently in FP32).

Sizes cover every panel kernel: N = 642 (shared-memory panels; FP64 cluster
panels at the start), 1026 (cluster panels), 4098 and 7899 (FP64 cluster panels
with rows kept in global memory; FP32 cluster panels, global rows at 7899).
"""
import numpy as np
import pytest
import scipy.linalg.lapack as lapack
import torch

import hornsculpt_b200 as hs
from hornsculpt_b200 import meshes

pytestmark = pytest.mark.gpu

# LAPACK's acceptance threshold for the factorisation ratio (TESTING/LIN xGET01, THRESH = 30).
XGET01_THRESHOLD = 30.0
EPS64 = np.finfo(np.float64).eps / 2  # LAPACK's dlamch('Epsilon'): unit roundoff 2^-53
EPS32 = np.finfo(np.float32).eps / 2


def _random(n, batch, seed):
    rng = np.random.default_rng(seed)
    return rng.standard_normal((batch, n, n)) + 1j * rng.standard_normal((batch, n, n))


def _permutation(piv):
    """Row order P A from a 0-based interchange sequence."""
    p = np.arange(len(piv))
    for i, q in enumerate(piv):
        p[i], p[q] = p[q], p[i]
    return p


def _residuals(a, factors, piv):
    """(xGET01 numerator ||PA - LU||_1 / (n ||A||_1), Frobenius ||PA - LU|| / ||A||) on the GPU."""
    n = a.shape[0]
    dev = torch.device("cuda")
    lu = torch.as_tensor(factors, device=dev)
    lower = torch.tril(lu, -1) + torch.eye(n, dtype=lu.dtype, device=dev)
    upper = torch.triu(lu)
    pa = torch.as_tensor(a[_permutation(piv)], device=dev)
    r = pa - lower @ upper
    one = torch.linalg.matrix_norm(r, ord=1).item() / (n * torch.linalg.matrix_norm(pa, ord=1).item())
    fro = (torch.linalg.matrix_norm(r).item() / torch.linalg.matrix_norm(pa).item())
    return one, fro


def _lapack(a, fp32):
    lu, piv, info = (lapack.cgetrf if fp32 else lapack.zgetrf)(a.astype(np.complex64 if fp32 else np.complex128))
    assert info == 0
    return lu.astype(np.complex128), piv


@pytest.mark.parametrize("n,batch", [(642, 3), (1026, 2), (4098, 1), (7899, 1)])
def test_fp64_lu_matches_lapack(n, batch):
    a = _random(n, batch, seed=n)
    factors, piv, info = hs.debug_lu_factor(a)
    assert info == 0
    for b in range(batch):
        ref_lu, ref_piv = _lapack(a[b], fp32=False)
        assert np.array_equal(piv[b], ref_piv), f"pivot sequence differs from zgetrf at N={n}"
        one, fro = _residuals(a[b], factors[b], piv[b])
        _, ref_fro = _residuals(a[b], ref_lu, ref_piv)
        assert one / EPS64 < XGET01_THRESHOLD, (n, one / EPS64)
        assert fro <= 2 * ref_fro + 1e-16, (n, fro, ref_fro)


@pytest.mark.parametrize("n,batch", [(642, 3), (1026, 2), (4098, 1), (7899, 1)])
def test_fp32_tensor_core_lu_passes_lapack_acceptance(n, batch):
    a = _random(n, batch, seed=n + 1)
    factors, piv, info = hs.debug_lu_factor(a, fp32=True)
    assert info == 0
    for b in range(batch):
        a32 = a[b].astype(np.complex64).astype(np.complex128)  # the input the FP32 kernels factor
        one, fro = _residuals(a32, factors[b], piv[b])
        ref_lu, ref_piv = _lapack(a[b], fp32=True)
        _, ref_fro = _residuals(a32, ref_lu, ref_piv)
        assert one / EPS32 < XGET01_THRESHOLD, (n, one / EPS32)
        # 3xTF32 trailing products drop the lo*lo term (about 2^-22 relative each),
        # so the FP32 factors sit a few times above LAPACK's cgetrf, not at it
        assert fro <= 8 * ref_fro, (n, fro, ref_fro)
        # a permutation: every row chosen once
        assert np.array_equal(np.sort(_permutation(piv[b])), np.arange(n))


def test_lu_of_burton_miller_matrix():
    """The C1 matrix (icosphere s3, 5 kHz): FP64 pivots equal zgetrf's, and both
    factorisations reproduce P A to the precision of their arithmetic."""
    mesh = meshes.icosphere(3)
    k = 2 * np.pi * 5000.0 / 343.0
    q = np.ones(mesh.triangle_count, np.complex128)
    with hs.CudaBemSolver(mesh) as solver:
        a, _ = solver.debug_assemble(hs.BemNumerics(), k, k, q)
    factors, piv, info = hs.debug_lu_factor(a)
    assert info == 0
    _, ref_piv = _lapack(a, fp32=False)
    assert np.array_equal(piv[0], ref_piv)
    one, fro = _residuals(a, factors[0], piv[0])
    assert one / EPS64 < XGET01_THRESHOLD and fro < 1e-14, (one / EPS64, fro)
    factors32, piv32, info32 = hs.debug_lu_factor(a, fp32=True)
    assert info32 == 0
    one32, fro32 = _residuals(a.astype(np.complex64).astype(np.complex128), factors32[0], piv32[0])
    assert one32 / EPS32 < XGET01_THRESHOLD and fro32 < 1e-6, (one32 / EPS32, fro32)


def test_lu_reports_a_zero_pivot():
    """A singular matrix (a zero column) is reported through the status word, as
    cusolverDnCgetrf's devInfo is (column + 1)."""
    a = _random(96, 1, seed=3)
    a[0, :, 40] = 0
    _, _, info = hs.debug_lu_factor(a)
    assert info == 41
    # the FP32 factorisation (its panels of at most 512 rows are factored in registers)
    _, _, info32 = hs.debug_lu_factor(a, fp32=True)
    assert info32 == 41


@pytest.mark.parametrize("n", [96, 642])
def test_pivot_ties_take_the_lowest_row(n):
    """Entries of equal |re| + |im| in the first column: both factorisations choose the
    lowest row, as zgetrf (izamax) does, in the register, shared-memory and cluster panels."""
    rng = np.random.default_rng(n + 7)
    a = rng.standard_normal((1, n, n)) + 1j * rng.standard_normal((1, n, n))
    a[0, :, 0] = rng.choice([1 + 1j, 1 - 1j, -1 + 1j, -1 - 1j, 2, -2j], n)  # |re| + |im| = 2 throughout
    for fp32 in (False, True):
        factors, piv, info = hs.debug_lu_factor(a, fp32=fp32)
        assert info == 0
        assert piv[0][0] == 0, (fp32, piv[0][:4])
    _, ref_piv = _lapack(a[0], fp32=False)
    assert ref_piv[0] == 0
