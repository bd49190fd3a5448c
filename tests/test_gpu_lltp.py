"""SparseLLTP ldiv! (src/preconditioner/RLSPreconditioner.jl:79-116) on the device against the
CPU restatement (oracle/precond.py: SciPy forward and backward substitution, FP64).

The block-row solve sums a row's terms in a different order from SciPy's substitution, so
the bar is relative: ‖X − X_ref‖ ≤ 1e-12 ‖X_ref‖ (the factors here have condition numbers
of a few units, as the reference's scaled IC factors do).
"""
import ctypes as C

import numpy as np
import pytest
import scipy.sparse as sp
import torch

import rls_b200 as R
from oracle.precond import lltp_ldiv
from rls_b200._lib import lib, check, ptr, DimensionMismatch, SingularException
from rls_b200.examples import ic_factor_banded

pytestmark = pytest.mark.gpu
RTOL = 1e-12


def _crand(rng, *shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


def _rel(X, ref):
    return np.linalg.norm(X - ref) / np.linalg.norm(ref)


def _perm(n, seed):
    p = np.random.default_rng(seed).permutation(n)
    return p, np.argsort(p)


@pytest.mark.parametrize("n,band,fill", [(777, 40, 0.4), (3000, 120, 0.66), (32, 31, 1.0), (1, 1, 1.0)])
@pytest.mark.parametrize("b", [1, 6, 13])
def test_ldiv_matches_oracle(cuda_device, n, band, fill, b):
    L = ic_factor_banded(n, band, fill, seed=n + b)
    p, invp = _perm(n, n)
    B = _crand(np.random.default_rng(b), n, b)
    K = R.SparseLLTP(L, p, invp, R.Engine(cuda_device))
    X = K.ldiv(B)
    assert _rel(X, lltp_ldiv(L, p, invp, B)) <= RTOL
    X2 = K.ldiv(B)                                    # a second call (next epoch) gives the same bits
    assert np.array_equal(X, X2)
    K.engine.close()


def test_ldiv_forty_columns_real_factor_and_stored_invp(cuda_device):
    """The pred-stage block width (r_pred = 40: five 8-column chunks), a real factor, and an
    invp that is not p's inverse: it is used as stored, as the reference does."""
    n = 2000
    L = ic_factor_banded(n, 90, 0.5, seed=9, complex_values=False)
    p, _ = _perm(n, 4)
    invp = np.random.default_rng(5).permutation(n)
    B = _crand(np.random.default_rng(6), n, 40)
    K = R.SparseLLTP(L, p, invp, R.Engine(cuda_device))
    assert _rel(K.ldiv(B), lltp_ldiv(L, p, invp, B)) <= RTOL
    K.engine.close()


def test_ldiv_in_place_one_based_and_upper_entries_ignored(cuda_device):
    """ldiv!(K, B) through the C ABI with X == B, Julia's 1-based CSC and permutation, and
    entries above the diagonal that LowerTriangular(L) does not see."""
    n = 500
    L = ic_factor_banded(n, 60, 0.5, seed=11)
    U = sp.triu(sp.random(n, n, density=0.01, random_state=2), k=1) * (3 + 1j)
    A = sp.csc_matrix(L + U)
    A.sort_indices()
    p, invp = _perm(n, 12)
    B = np.asfortranarray(_crand(np.random.default_rng(13), n, 6))
    ref = lltp_ldiv(L, p, invp, B)
    e = R.Engine(cuda_device)
    colptr = np.ascontiguousarray(A.indptr + 1, dtype=np.int64)
    rowval = np.ascontiguousarray(A.indices + 1, dtype=np.int64)
    nzval = np.ascontiguousarray(A.data, dtype=np.complex128)
    p1 = np.ascontiguousarray(p + 1, dtype=np.int64)
    ip1 = np.ascontiguousarray(invp + 1, dtype=np.int64)
    check(lib().rls_lltp_upload(e._h, n, ptr(colptr), ptr(rowval), ptr(nzval), ptr(p1), ptr(ip1), 1), e._h)
    check(lib().rls_lltp_ldiv(e._h, 6, ptr(B), n, ptr(B), n), e._h)
    assert _rel(B, ref) <= RTOL
    e.close()


def test_ldiv_device_pointers(cuda_device):
    n, b = 1500, 6
    L = ic_factor_banded(n, 100, 0.6, seed=21)
    p, invp = _perm(n, 22)
    B = _crand(np.random.default_rng(23), n, b)
    e = R.Engine(cuda_device)
    K = R.SparseLLTP(L, p, invp, e)
    dev = torch.device("cuda", cuda_device)
    # column-major n × b on the device: a (b, n) row-major tensor
    dB = torch.from_numpy(np.ascontiguousarray(B.T)).to(dev)
    dX = torch.zeros_like(dB)
    torch.cuda.synchronize()                          # the library works on its own stream
    check(lib().rls_lltp_ldiv_dev(e._h, b, C.c_void_p(dB.data_ptr()), n, C.c_void_p(dX.data_ptr()), n), e._h)
    X = dX.cpu().numpy().T
    assert _rel(X, lltp_ldiv(L, p, invp, B)) <= RTOL
    with pytest.raises(R.ArgumentError):
        check(lib().rls_lltp_ldiv_dev(e._h, b, C.c_void_p(dB.data_ptr()), n, C.c_void_p(dB.data_ptr()), n), e._h)
    e.close()


def test_ldiv_errors(cuda_device):
    n = 100
    L = ic_factor_banded(n, 10, 0.5, seed=31).tolil()
    L[40, 40] = 0.0
    L[70, 70] = 0.0
    p, invp = _perm(n, 32)
    e = R.Engine(cuda_device)
    B = np.ones((n, 2), dtype=np.complex128)
    with pytest.raises(R.RLSError):                    # no factor uploaded yet
        check(lib().rls_lltp_ldiv(e._h, 2, ptr(B), n, ptr(B), n), e._h)
    K = R.SparseLLTP(L.tocsc(), p, invp, e)
    with pytest.raises(SingularException) as ex:
        K.ldiv(B)
    assert "SingularException(41)" in str(ex.value)
    with pytest.raises(DimensionMismatch):
        K.ldiv(np.ones((n + 1, 2)))
    bad = p.copy()
    bad[3] = n
    with pytest.raises(DimensionMismatch):
        R.SparseLLTP(ic_factor_banded(n, 10, 0.5, seed=33), bad, invp, e)
    e.close()
