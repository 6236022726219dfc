"""GPU parity of the FP64 LU and solve (dgetrf/dgetrs semantics, best/best.f:444,
best/besolve.f90:133) against LAPACK (scipy's OpenBLAS, the reference's LAPACK), and of the DMMA
trailing-update GEMM against numpy.  Tolerances: backward error ||PA - LU|| / ||A|| <= 1e-13 and the
same pivots as LAPACK; solutions within 1e-11 relative of LAPACK's on well-conditioned systems."""
import numpy as np
import pytest
import scipy.linalg as sla

import best_hydro_b200 as bh
from oracle import best as ob
from best_hydro_b200 import meshes

pytestmark = pytest.mark.gpu


def _torch():
    import torch
    assert torch.cuda.is_available()
    return torch


def to_dev(a, ld=None):
    """Column-major host matrix -> device buffer with leading dimension ld (even)."""
    torch = _torch()
    m, n = a.shape
    ld = ld or (m + (m & 1))
    t = torch.zeros((n, ld), dtype=torch.float64)
    t[:, :m] = torch.from_numpy(np.ascontiguousarray(a.T))
    t = t.cuda()
    torch.cuda.synchronize()  # the library's stream does not wait for torch's
    return t, ld


def from_dev(t, m):
    return np.asfortranarray(t[:, :m].cpu().numpy().T)


@pytest.mark.parametrize("m,n,k", [(1, 1, 1), (7, 5, 3), (64, 64, 16), (130, 129, 17), (1000, 300, 256),
                                   (2048, 2048, 256), (4097, 96, 32)])
def test_dgemm_minus(m, n, k):
    rng = np.random.default_rng(m * 7 + n * 3 + k)
    A = np.asfortranarray(rng.standard_normal((m, k)))
    B = np.asfortranarray(rng.standard_normal((k, n)))
    C = np.asfortranarray(rng.standard_normal((m, n)))
    dA, lda = to_dev(A)
    dB, ldb = to_dev(B)
    dC, ldc = to_dev(C)
    bh.dgemm_minus_device(m, n, k, dA.data_ptr(), lda, dB.data_ptr(), ldb, dC.data_ptr(), ldc)
    got = from_dev(dC, m)
    want = C - A @ B
    err = np.max(np.abs(got - want)) / (np.max(np.abs(A)) * np.max(np.abs(B)) * k)
    assert err < 1e-15, err


def lu_check(A, expect_same_pivots=True):
    torch = _torch()
    n = A.shape[0]
    dA, lda = to_dev(A, ld=(n + 31) // 32 * 32)
    ipiv = torch.zeros(n, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    info = bh.dgetrf_device(n, dA.data_ptr(), lda, ipiv.data_ptr())
    LU = from_dev(dA, n)
    piv = ipiv.cpu().numpy()
    lu_ref, piv_ref, info_ref = sla.lapack.dgetrf(A)
    if expect_same_pivots:
        assert np.array_equal(piv, piv_ref + 1)
    L = np.tril(LU, -1) + np.eye(n)
    U = np.triu(LU)
    PA = A.copy()
    for i in range(n):
        p = piv[i] - 1
        PA[[i, p]] = PA[[p, i]]
    berr = np.max(np.abs(PA - L @ U)) / np.max(np.abs(A))
    return info, berr, dA, lda, ipiv


@pytest.mark.parametrize("n", [1, 2, 7, 33, 100, 257, 600, 1031, 3001])
def test_dgetrf_random(n):
    rng = np.random.default_rng(n)
    A = np.asfortranarray(rng.standard_normal((n, n)))
    info, berr, *_ = lu_check(A)
    assert info == 0
    assert berr < 1e-12 * max(1, np.log2(n)), berr


def test_dgetrf_zero_pivot_info():
    """dgetrf's info: the first exactly-zero pivot (1-based), factorisation completed."""
    rng = np.random.default_rng(5)
    n = 300
    A = np.asfortranarray(rng.standard_normal((n, n)))
    A[:, 77] = 0.0
    info, berr, *_ = lu_check(A)
    lu_ref, piv_ref, info_ref = sla.lapack.dgetrf(A)
    assert info == info_ref == 78


def test_dgetrs_matches_lapack():
    torch = _torch()
    rng = np.random.default_rng(11)
    n = 1500
    A = np.asfortranarray(rng.standard_normal((n, n)) + n ** 0.5 * np.eye(n))
    info, berr, dA, lda, ipiv = lu_check(A)
    B = np.asfortranarray(rng.standard_normal((n, 6)))
    dB, ldb = to_dev(B)
    bh.dgetrs_device(n, 6, dA.data_ptr(), lda, ipiv.data_ptr(), dB.data_ptr(), ldb)
    X = from_dev(dB, n)
    Xr = sla.lu_solve(sla.lu_factor(A), B)
    assert np.max(np.abs(X - Xr)) / np.max(np.abs(Xr)) < 1e-11


def test_lu_of_best_matrix_matches_lapack():
    """The deflated GR of a closed surface: LU + 11-RHS solve against dgetrf/dgetrs."""
    torch = _torch()
    tri, ta, tv = meshes.ellipsoid(8)
    s = ob.setup(tri, 1, ta)
    gr, x, self9 = ob.assemble(s)
    xmu, gdef = ob.deflation_vectors(s, ob.diag_mean(self9, s.n))
    ob.deflate(s, gr, xmu, gdef)
    n = gr.shape[0]
    info, berr, dA, lda, ipiv = lu_check(gr, expect_same_pivots=False)
    assert info == 0 and berr < 1e-13
    B = np.asfortranarray(np.concatenate([ob.rhs6(x, s.n), ob.strain5(x, s.n)], axis=1))
    dB, ldb = to_dev(B)
    bh.dgetrs_device(n, 11, dA.data_ptr(), lda, ipiv.data_ptr(), dB.data_ptr(), ldb)
    X = from_dev(dB, n)
    lu, piv, _ = ob.getrf(gr.copy(order="F"))
    Xr, _ = ob.getrs(lu, piv, B)
    assert np.max(np.abs(X - Xr)) / np.max(np.abs(Xr)) < 1e-11
