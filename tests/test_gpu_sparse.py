"""ShiftedMat mul! (src/types/RLSMatrices.jl:24-66) on the device against SciPy.

Y = C X + s·X[1:min(m,n), :] and its adjoint Cᴴ X + conj(s)·X[1:min(m,n), :], FP64
complex; tolerance 1e-13 relative to |C|·|X| (row sums in a different order).
"""
import ctypes as C

import numpy as np
import pytest
import scipy.sparse as sp

import rls_b200 as R
from rls_b200._lib import lib, check, ptr, c64, DimensionMismatch
from rls_b200.examples import sprand, skewlap3d

pytestmark = pytest.mark.gpu


def _ref(Cm, s, X, adj):
    m, n = Cm.shape
    A = Cm.conj().T if adj else Cm
    Y = A @ X
    k = min(m, n)
    Y[:k] += (np.conj(s) if adj else s) * X[:k]
    return Y


def _crand(rng, *shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


@pytest.mark.parametrize("b", [1, 6, 12])
@pytest.mark.parametrize("adj", [False, True])
def test_spmm_shifted_matches_scipy(cuda_device, b, adj):
    rng = np.random.default_rng(b + 10 * adj)
    Cm = sprand(600).astype(np.complex128)
    Cm = Cm + 1j * sp.random(600, 600, density=0.004, random_state=3, format="csc")
    e = R.Engine(cuda_device)
    A = R.ShiftedMat(Cm, -0.5 + 0.02j, e)
    X = _crand(rng, 600, b)
    Y = (A.adjoint() if adj else A) @ X
    ref = _ref(Cm, -0.5 + 0.02j, X, adj)
    scale = abs(Cm).max() * np.abs(X).max() * max(Cm.getnnz(axis=1).max(), 1)
    assert np.max(np.abs(Y - ref)) <= 1e-13 * scale
    e.close()


@pytest.mark.parametrize("shape", [(300, 200), (150, 420)])
def test_spmm_shifted_rectangular_and_one_based(cuda_device, shape):
    m, n = shape
    rng = np.random.default_rng(m)
    Cm = sp.random(m, n, density=0.05, random_state=m, format="csc") * (1 + 0.5j)
    Cm = sp.csc_matrix(Cm)
    e = R.Engine(cuda_device)
    colptr = (Cm.indptr + 1).astype(np.int64)           # Julia's 1-based SparseMatrixCSC layout
    rowval = (Cm.indices + 1).astype(np.int64)
    nzval = np.ascontiguousarray(Cm.data, dtype=np.complex128)
    check(lib().rls_sparse_upload_csc(e._h, m, n, ptr(colptr), ptr(rowval), ptr(nzval), 1), e._h)
    e.sparse_shape = (m, n)
    for adj in (False, True):
        X = _crand(rng, m if adj else n, 3)
        Y = e.spmm_shifted(0.3 - 0.1j, X, adj=adj)
        assert np.allclose(Y, _ref(Cm, 0.3 - 0.1j, X, adj), rtol=0, atol=1e-13 * np.abs(X).max() * 10)
    e.close()


def test_spmm_shifted_skewlap3d_vector(cuda_device):
    """The 3-D skew Laplacian (7-point stencil) with a vector right-hand side."""
    Cm = skewlap3d(10).astype(np.complex128)
    n = Cm.shape[0]
    e = R.Engine(cuda_device)
    A = R.ShiftedMat(Cm, 12.5 - 3j, e)
    x = _crand(np.random.default_rng(1), n)
    y = A @ x
    ref = _ref(Cm, 12.5 - 3j, x.reshape(-1, 1), False)[:, 0]
    assert np.max(np.abs(y - ref)) <= 1e-13 * abs(Cm).max() * np.abs(x).max() * 8
    e.close()


def test_sparse_upload_rejects_bad_indices(cuda_device):
    e = R.Engine(cuda_device)
    colptr = np.array([0, 1, 2], dtype=np.int64)
    rowval = np.array([0, 5], dtype=np.int64)          # row 5 of a 3 × 2 matrix
    nzval = np.ones(2, dtype=np.complex128)
    with pytest.raises(DimensionMismatch):
        check(lib().rls_sparse_upload_csc(e._h, 3, 2, ptr(colptr), ptr(rowval), ptr(nzval), 0), e._h)
    X, Y = np.ones(2, dtype=np.complex128), np.ones(3, dtype=np.complex128)
    with pytest.raises(R.RLSError):
        check(lib().rls_spmm_shifted(e._h, c64(0, 0), 0, 1, ptr(X), 2, ptr(Y), 3), e._h)
    e.close()
