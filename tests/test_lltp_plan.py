"""SparseLLTP ldiv! (src/preconditioner/RLSPreconditioner.jl:79-116) on the CPU: the oracle
against the dense definition, and the block-row plan that the device solve runs
(rls_test_lltp_plan_dense, host only) against tril(L) and its adjoint.
"""
import ctypes as C

import numpy as np
import pytest
import scipy.sparse as sp

from oracle.precond import lltp_ldiv, SingularException as OSingular
from rls_b200.examples import ic_factor_banded as random_ic_factor
from rls_b200._lib import lib, check, ptr, DimensionMismatch


def _csc_arrays(L, base=0):
    A = sp.csc_matrix(L, dtype=np.complex128)
    return (np.ascontiguousarray(A.indptr + base, dtype=np.int64), np.ascontiguousarray(A.indices + base, dtype=np.int64),
            np.ascontiguousarray(A.data, dtype=np.complex128))


def plan_dense(L, op, base=0):
    n = L.shape[0]
    colptr, rowval, nzval = _csc_arrays(L, base)
    D = np.zeros((n, n), dtype=np.complex128, order="F")
    sing = C.c_int64()
    lev = C.c_int()
    check(lib().rls_test_lltp_plan_dense(n, ptr(colptr), ptr(rowval), ptr(nzval), base, op, ptr(D), C.byref(sing),
                                         C.byref(lev)), None)
    return D, sing.value, lev.value


def _messy_factor(n, seed):
    """Lower factor plus entries above the diagonal (ignored, as LowerTriangular ignores them)
    and a duplicated entry (added up), unsorted within columns."""
    rng = np.random.default_rng(seed)
    L = random_ic_factor(n, band=min(n, 70), fill=0.3, seed=seed).tocoo()
    r, c, v = list(L.row), list(L.col), list(L.data)
    for _ in range(max(1, n // 4)):
        i, j = sorted(rng.integers(0, n, 2))
        if i < j:
            r.append(i); c.append(j); v.append(5.0 + 1j)            # above the diagonal
    if n > 3:
        r.append(n - 1); c.append(1); v.append(0.25 - 0.5j)         # may duplicate an entry
    perm = rng.permutation(len(r))
    return sp.coo_matrix((np.array(v)[perm], (np.array(r)[perm], np.array(c)[perm])), shape=(n, n)).tocsc()


def test_oracle_matches_dense_definition():
    n = 90
    L = random_ic_factor(n, band=20, fill=0.5, seed=1)
    rng = np.random.default_rng(2)
    p = rng.permutation(n)
    invp = np.argsort(p)
    B = rng.standard_normal((n, 5)) + 1j * rng.standard_normal((n, 5))
    Ld = np.tril(L.toarray())
    ref = np.linalg.solve(Ld.conj().T, np.linalg.solve(Ld, B[p]))[invp]
    assert np.allclose(lltp_ldiv(L, p, invp, B), ref, rtol=0, atol=1e-12 * np.abs(ref).max())
    # invp is used as stored, not recomputed from p
    ref2 = np.linalg.solve(Ld.conj().T, np.linalg.solve(Ld, B[p]))[p]
    assert np.allclose(lltp_ldiv(L, p, p, B), ref2, rtol=0, atol=1e-12 * np.abs(ref2).max())
    L2 = L.tolil()
    L2[7, 7] = 0.0
    with pytest.raises(OSingular) as e:
        lltp_ldiv(L2.tocsc(), p, invp, B)
    assert e.value.j == 8


@pytest.mark.parametrize("n", [1, 31, 32, 33, 100, 257])
@pytest.mark.parametrize("base", [0, 1])
def test_plan_reconstructs_lower_triangle_and_adjoint(n, base):
    L = _messy_factor(n, seed=n)
    Lt = np.tril(L.toarray())
    scale = np.abs(Lt).max()
    D0, sing, lev0 = plan_dense(L, 0, base)
    D1, _, lev1 = plan_dense(L, 1, base)
    assert sing == 0
    assert np.max(np.abs(D0 - Lt)) <= 1e-14 * scale
    assert np.max(np.abs(D1 - Lt.conj().T)) <= 1e-14 * scale
    nblk = -(-n // 32)
    assert 1 <= lev0 <= nblk and 1 <= lev1 <= nblk


def test_plan_levels():
    n = 100
    assert plan_dense(sp.identity(n, format="csc") * (2 + 1j), 0)[2] == 1      # no dependencies
    bidiag = (sp.identity(n) + sp.diags(np.full(n - 1, 0.5), -1)).tocsc()
    assert plan_dense(bidiag, 0)[2] == 4 and plan_dense(bidiag, 1)[2] == 4     # one chain of 4 block rows
    blockdiag = sp.block_diag([sp.csr_matrix(np.tril(np.ones((32, 32))))] * 3 +
                              [sp.csr_matrix(np.tril(np.ones((4, 4))))]).tocsc()
    assert plan_dense(blockdiag, 0)[2] == 1                                      # in-block terms only


def test_plan_reports_first_zero_diagonal():
    n = 50
    L = random_ic_factor(n, band=10, fill=0.5, seed=3).tolil()
    L[9, 9] = 0.0                       # explicit zero
    L = L.tocsc()
    L.eliminate_zeros()                 # and absent at 9 (0-based) ...
    L = L.tolil()
    L[5, 5] = 0.0                       # ... with an explicit zero earlier at 5
    _, sing, _ = plan_dense(L.tocsc(), 0)
    assert sing == 6


def test_plan_rejects_bad_indices():
    colptr = np.array([0, 1, 2], dtype=np.int64)
    rowval = np.array([0, 5], dtype=np.int64)
    nzval = np.ones(2, dtype=np.complex128)
    D = np.zeros((2, 2), dtype=np.complex128)
    with pytest.raises(DimensionMismatch):
        check(lib().rls_test_lltp_plan_dense(2, ptr(colptr), ptr(rowval), ptr(nzval), 0, 0, ptr(D), None, None), None)


def test_plan_invariants_on_the_af23560_shaped_factor():
    """The full-size factor of the benchmark (n = 23,560, 4.7·10⁶ nonzeros): plan checks only."""
    from rls_b200.examples import ic_factor_banded
    L = ic_factor_banded(23560, 300, 2.0 / 3.0, seed=20260318, complex_values=False)
    colptr, rowval, nzval = _csc_arrays(L)
    for op in (0, 1):
        sing = C.c_int64()
        lev = C.c_int()
        check(lib().rls_test_lltp_plan_dense(23560, ptr(colptr), ptr(rowval), ptr(nzval), 0, op, None,
                                             C.byref(sing), C.byref(lev)), None)
        assert sing.value == 0 and lev.value == -(-23560 // 32)      # one chain through every block row


def test_plan_rejects_non_finite_entries():
    """The checks rls_lltp_upload shares with the plan: a non-finite factor entry is an error."""
    from rls_b200._lib import ArgumentError
    colptr = np.array([0, 2, 3], dtype=np.int64)
    rowval = np.array([0, 1, 1], dtype=np.int64)
    nzval = np.array([1.0, np.nan, 2.0], dtype=np.complex128)
    D = np.zeros((2, 2), dtype=np.complex128)
    with pytest.raises(ArgumentError):
        check(lib().rls_test_lltp_plan_dense(2, ptr(colptr), ptr(rowval), ptr(nzval), 0, 0, ptr(D), None, None), None)
