"""get_hsl_LLTP's incomplete-Cholesky factorisation on the host (rls_ic_factor) against the CPU
restatement (oracle/icfact.py, bit for bit), and the restatement against the definition: with
no dropping the factor is the exact Cholesky factor of the permuted normal matrix.
"""
import ctypes as C

import numpy as np
import pytest
import scipy.sparse as sp

import rls_b200 as R
from oracle.icfact import ic_factor as oracle_ic_factor
from rls_b200._lib import lib, check, ptr, c64, ArgumentError, DimensionMismatch
from rls_b200.examples import skewlap3d, sprand


def _case(kind, n, seed):
    if kind == "random":
        dens = 0.08 if n < 200 else 6.0 / n
        return (sp.random(n, n, density=dens, random_state=seed, format="csc") + sp.identity(n) * 0.3).tocsc()
    if kind == "complex":
        A = sp.random(n, n, density=0.06, random_state=seed, format="csc")
        B = sp.random(n, n, density=0.03, random_state=seed + 1, format="csc")
        return (A + 1j * B + sp.identity(n) * (0.2 - 0.1j)).tocsc()
    if kind == "stencil":                         # many equal magnitudes: ties in the selection
        return skewlap3d(round(n ** (1 / 3))).tocsc()
    if kind == "sprand":
        return sprand(n).tocsc()
    raise ValueError(kind)


CASES = [
    ("random", 60, 0.2 + 0.1j, 1e-2, 1e-3, 0.0, 3, 2),
    ("random", 80, -0.5, 1e-3, 1e-4, 0.0, 10, 5),
    ("random", 50, 0.1j, 1e-3, 0.0, 0.0, 4, 3),        # τ₂ = 0: every R candidate kept
    ("complex", 70, 0.3 - 0.2j, 5e-3, 5e-4, 0.0, 6, 6),
    ("complex", 40, 0.0, 1e-2, 1e-3, 0.05, 2, 0),     # caller's α
    ("stencil", 64, 12.5 - 3j, 1e-3, 1e-4, 0.0, 8, 4),
    ("stencil", 125, -40.0, 1e-2, 1e-3, 0.0, 5, 5),
    ("sprand", 120, 0.5 + 0.05j, 1e-3, 1e-4, 0.0, 20, 10),
    ("random", 600, 0.1 - 0.2j, 1e-2, 1e-3, 0.0, 6, 4),     # the normal product on several threads
]


@pytest.mark.parametrize("kind,n,z,tau1,tau2,alpha,lsize,rsize", CASES)
def test_host_factor_matches_oracle_bit_for_bit(kind, n, z, tau1, tau2, alpha, lsize, rsize):
    Cm = _case(kind, n, seed=n)
    n = Cm.shape[0]
    p = np.random.default_rng(n).permutation(n)
    L1, ip1, a1 = R.ic_factor(Cm, z, tau1, tau2, alpha, lsize, rsize, p)
    L2, ip2, a2 = oracle_ic_factor(Cm, z, tau1, tau2, alpha, lsize, rsize, p)
    assert a1 == a2
    assert np.array_equal(ip1, ip2) and np.array_equal(ip1[p], np.arange(n))
    assert np.array_equal(L1.indptr, L2.indptr) and np.array_equal(L1.indices, L2.indices)
    assert np.array_equal(L1.data, L2.data)
    # each column: the diagonal first, then rows ascending below it; in all at most n·(1 + lsize)
    for j in range(n):
        rows = L1.indices[L1.indptr[j]:L1.indptr[j + 1]]
        assert rows[0] == j and np.all(np.diff(rows) > 0)
    assert L1.nnz <= n * (1 + min(lsize, n - 1))


@pytest.mark.parametrize("kind,n,z", [("random", 60, 0.2 + 0.1j), ("complex", 50, -0.3j), ("stencil", 64, 12.5 - 3j)])
def test_no_dropping_gives_the_cholesky_factor(kind, n, z):
    Cm = _case(kind, n, seed=3)
    n = Cm.shape[0]
    p = np.random.default_rng(4).permutation(n)
    L, invp, a = R.ic_factor(Cm, z, 0.0, 0.0, 0.0, n - 1, 0, p)
    assert a == 0.0
    Cz = Cm.toarray() - z * np.eye(n)
    N = (Cz.conj().T @ Cz)[np.ix_(p, p)]
    Ld = L.toarray()
    assert np.allclose(np.triu(Ld, 1), 0)
    assert np.max(np.abs(Ld @ Ld.conj().T - N)) <= 1e-13 * np.abs(N).max()


def test_shift_grows_on_breakdown_and_factor_feeds_the_device_plan():
    """Heavy dropping breaks the factorisation down; the retried factor with α > 0 has a
    positive diagonal and passes every check of the block-row plan the device solve runs."""
    Cm = _case("random", 60, seed=60)
    p = np.random.default_rng(60).permutation(60)
    L, invp, a = R.ic_factor(Cm, 0.2 + 0.1j, 1e-2, 1e-3, 0.0, 3, 2, p)
    assert a > 0.0
    assert np.all(L.diagonal().real > 0)
    A = sp.csc_matrix(L)
    colptr = np.ascontiguousarray(A.indptr, dtype=np.int64)
    rowval = np.ascontiguousarray(A.indices, dtype=np.int64)
    nzval = np.ascontiguousarray(A.data, dtype=np.complex128)
    sing = C.c_int64()
    lev = C.c_int()
    D = np.zeros((60, 60), dtype=np.complex128, order="F")
    check(lib().rls_test_lltp_plan_dense(60, ptr(colptr), ptr(rowval), ptr(nzval), 0, 0, ptr(D), C.byref(sing),
                                         C.byref(lev)), None)
    assert sing.value == 0
    Ld = L.toarray()                                  # the plan keeps 1/diagonal: two reciprocals
    assert np.max(np.abs(D - Ld)) <= 1e-14 * np.abs(Ld).max()


def _raw(Cm, p, base=0, lsize=3, rsize=2, cap=None, rows=None):
    A = sp.csc_matrix(Cm, dtype=np.complex128)
    A.sort_indices()
    n = A.shape[0]
    colptr = np.ascontiguousarray(A.indptr + base, dtype=np.int64)
    rowval = np.ascontiguousarray((A.indices if rows is None else rows) + base, dtype=np.int64)
    nzval = np.ascontiguousarray(A.data, dtype=np.complex128)
    lsz = min(max(0, lsize), n - 1)
    cap = n + lsz * n if cap is None else cap
    out = (np.zeros(n + 1, dtype=np.int64), np.zeros(max(cap, 1), dtype=np.int64),
           np.zeros(max(cap, 1), dtype=np.complex128), np.zeros(n, dtype=np.int64))
    pb = np.ascontiguousarray(p, dtype=np.int64) + base       # named: the library reads it
    st = lib().rls_ic_factor(n, ptr(colptr), ptr(rowval), ptr(nzval), base, c64(0.1, 0.0), 1e-3, 1e-4, 0.0, lsize,
                             rsize, ptr(pb), cap, ptr(out[0]), ptr(out[1]), ptr(out[2]), ptr(out[3]), None)
    return st, out


def test_one_based_input_gives_the_same_factor():
    Cm = _case("complex", 40, seed=9)
    p = np.random.default_rng(9).permutation(40)
    st0, o0 = _raw(Cm, p, 0)
    st1, o1 = _raw(Cm, p, 1)
    assert st0 == 0 and st1 == 0
    assert np.array_equal(o0[0] + 1, o1[0]) and np.array_equal(o0[3] + 1, o1[3])
    nl = o0[0][-1]
    assert np.array_equal(o0[1][:nl] + 1, o1[1][:nl]) and np.array_equal(o0[2][:nl], o1[2][:nl])


def test_errors():
    Cm = _case("random", 30, seed=2)
    p = np.random.default_rng(2).permutation(30)
    with pytest.raises(ArgumentError):                       # the reference cannot run lsize = 0
        check(_raw(Cm, p, lsize=0)[0], None)
    with pytest.raises(ArgumentError):
        check(_raw(Cm, p, rsize=-1)[0], None)
    bad = p.copy()
    bad[1] = bad[0]
    with pytest.raises(ArgumentError):                       # not a permutation
        check(_raw(Cm, bad)[0], None)
    with pytest.raises(DimensionMismatch):                   # output capacity below n·(1 + lsize)
        check(_raw(Cm, p, cap=30)[0], None)
    A = sp.csc_matrix(Cm)
    A.sort_indices()
    rows = A.indices.copy()
    j = int(np.argmax(np.diff(A.indptr) >= 2))
    a0 = A.indptr[j]
    rows[a0], rows[a0 + 1] = rows[a0 + 1], rows[a0]
    with pytest.raises(ArgumentError):                       # rows not increasing in a column
        check(_raw(Cm, p, rows=rows)[0], None)
    with pytest.raises(DimensionMismatch):
        R.ic_factor(sp.random(5, 6, density=0.5, format="csc"), 0.0, 1e-3, 1e-4, 0.0, 2, 1, np.arange(5))


def test_small_and_clamped_sizes():
    """n = 1; lsize beyond n − 1 (clamped as ichsd does) equals lsize = n − 1; the factor's
    pattern alone (NULL entry outputs) comes back from the pointers."""
    one = sp.csc_matrix(np.array([[2.0 + 1.0j]]))
    L, invp, a = R.ic_factor(one, 0.5, 1e-3, 1e-4, 0.0, 5, 0, [0])
    assert L.shape == (1, 1) and invp.tolist() == [0] and a == 0.0
    assert np.isclose(L[0, 0], abs(2.0 + 1.0j - 0.5))
    Cm = _case("random", 40, seed=5)
    p = np.random.default_rng(5).permutation(40)
    La = R.ic_factor(Cm, 0.1, 1e-3, 1e-4, 0.0, 39, 3, p)[0]
    Lb = R.ic_factor(Cm, 0.1, 1e-3, 1e-4, 0.0, 500, 3, p)[0]
    assert np.array_equal(La.indptr, Lb.indptr) and np.array_equal(La.data, Lb.data)
    A = sp.csc_matrix(Cm, dtype=np.complex128)
    A.sort_indices()
    lp = np.zeros(41, dtype=np.int64)
    ip = np.zeros(40, dtype=np.int64)
    colptr = np.ascontiguousarray(A.indptr, dtype=np.int64)   # named: the library reads them
    rowval = np.ascontiguousarray(A.indices, dtype=np.int64)
    nzval = np.ascontiguousarray(A.data)
    p64 = np.ascontiguousarray(p, dtype=np.int64)
    check(lib().rls_ic_factor(40, ptr(colptr), ptr(rowval), ptr(nzval), 0, c64(0.1, 0.0), 1e-3, 1e-4, 0.0, 39, 3,
                              ptr(p64), 40 * 40, ptr(lp), None, None, ptr(ip), None), None)
    assert np.array_equal(lp, La.indptr)


@pytest.mark.parametrize("bad", ["z", "alpha", "tau1", "entry"])
def test_non_finite_inputs_are_argument_errors(bad):
    """A non-finite shift, tolerance or matrix entry is rejected before any work."""
    Cm = _case("random", 30, seed=7).tolil()
    z, alpha, tau1 = 0.1 + 0.0j, 0.0, 1e-3
    if bad == "z":
        z = complex(np.nan, 0.0)
    elif bad == "alpha":
        alpha = np.inf
    elif bad == "tau1":
        tau1 = np.nan
    else:
        Cm[3, 3] = np.nan
    with pytest.raises(ArgumentError):
        R.ic_factor(Cm.tocsc(), z, tau1, 1e-4, alpha, 3, 2, np.arange(30))
