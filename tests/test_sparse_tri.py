"""Host side of psTriRecy's sparse branch (psTriRecy.jl:47-61, :222-234): the band order the
library picks, and the CPU restatement of the branch.

The restatement runs the reference's form — M = C[:, p], S = I[:, p], R = qr(M − zS).R — and
the form the device runs — B = PᵀCP with S = I — to show they take the same decisions and
give the same σ (the recycled space on (M, S) is a unitary image of the one on (B, I)).
"""
import numpy as np
import pytest
import scipy.sparse as sp

import oracle.pstrirecy as OP
from oracle import recugrid as G
import rls_b200 as R
from rls_b200.examples import skewlap3d, af23560_shaped


def _bandwidths(C, p):
    B = sp.coo_matrix(sp.csc_matrix(C)[p][:, p])
    d = B.row - B.col
    return int(max(d.max(), 0)), int(max((-d).max(), 0))


@pytest.mark.parametrize("make", [lambda: skewlap3d(9), lambda: skewlap3d(25), lambda: af23560_shaped(3000)])
def test_band_order_is_a_permutation_with_the_stated_bandwidths(make):
    C = make()
    p, l, u = R.band_order(C)
    n = C.shape[0]
    assert np.array_equal(np.sort(p), np.arange(n))
    assert (l, u) == _bandwidths(C, p)
    # never wider work than the natural order
    l0, u0 = _bandwidths(C, np.arange(n))
    assert l * (l + u + 1) + l + u <= l0 * (l0 + u0 + 1) + l0 + u0


def test_band_order_narrows_the_3d_stencil():
    C = skewlap3d(25)                       # n = 13824, natural bandwidths 576
    p, l, u = R.band_order(C)
    assert _bandwidths(C, np.arange(C.shape[0])) == (576, 576)
    assert l < 576 and u < 576


def test_band_order_rejects_bad_csc():
    from rls_b200._lib import lib, ArgumentError, DimensionMismatch, check
    import ctypes as C_
    colptr = np.array([0, 2, 1], dtype=np.int64)      # decreasing
    rowval = np.array([0, 1], dtype=np.int64)
    perm = np.zeros(2, dtype=np.int64)
    with pytest.raises(DimensionMismatch):
        check(lib().rls_band_order(2, colptr.ctypes.data, rowval.ctypes.data, 0, perm.ctypes.data, None, None))
    colptr = np.array([0, 1, 2], dtype=np.int64)
    rowval = np.array([0, 5], dtype=np.int64)         # row out of range
    with pytest.raises(DimensionMismatch):
        check(lib().rls_band_order(2, colptr.ctypes.data, rowval.ctypes.data, 0, perm.ctypes.data, None, None))
    with pytest.raises(ArgumentError):
        check(lib().rls_band_order(2, colptr.ctypes.data, rowval.ctypes.data, 2, perm.ctypes.data, None, None))


def _skew_case(N=7, nx=8, k=4):
    C = skewlap3d(N).astype(np.complex128)
    s = (N / 25) ** 2
    grid = (-550 * s, 100 * s, -200 * s, 200 * s, nx, nx, k)
    normC = float(np.linalg.norm(C.toarray(), 2))
    return C, normC, grid


def test_sparse_branch_restatement_matches_dense_svd_and_the_device_frame():
    C, normC, grid = _skew_case()
    n = C.shape[0]
    p, l, u = R.band_order(C)
    rec = G.recursion_grid(*grid)
    ctl = OP.PsTriRecyControl(normC=normC, tol=1e-4, p=10, p_min=1, recy_tau=1.6)
    rng = np.random.default_rng(3)
    X0 = rng.random((n, ctl.r)) + 1j * rng.random((n, ctl.r))
    s_ms, st_ms = OP.ps_tri_recy_sparse(C, p, rec, ctl, X0=X0)          # the reference's (M, S)
    B = sp.csc_matrix(C)[p][:, p]
    s_b, st_b = OP.ps_tri_recy_sparse(B, np.arange(n), rec, ctl, X0=X0)  # the device's (B, I)
    truth = np.array([OP.dense_sigma_min(C.toarray(), z) for z in rec.Z])
    assert np.max(np.abs(s_ms - truth)) <= 1e-4 * normC
    assert np.max(np.abs(s_ms - truth) / truth) <= 1e-6
    assert np.max(np.abs(s_ms - s_b) / s_ms) <= 1e-12
    assert np.array_equal(st_ms.refine_it, st_b.refine_it)
    assert np.array_equal(st_ms.r_recy, st_b.r_recy)
    assert np.array_equal(st_ms.p_count, st_b.p_count)
    assert 0 < int(np.sum(st_ms.refine_it > 0)) < len(rec.Z)


def test_sparse_lu_operator_gives_the_qr_operators_results():
    """The CPU baseline's sparse-LU operator (M − zS)⁻ᴴ and the reference's InvMat(Rᴴ) give the
    same σ and the same decisions on the restatement."""
    C, normC, grid = _skew_case(N=6, nx=6, k=3)
    n = C.shape[0]
    p, l, u = R.band_order(C)
    rec = G.recursion_grid(*grid)
    ctl = OP.PsTriRecyControl(normC=normC, tol=1e-4, p=10, p_min=1, recy_tau=1.6)
    rng = np.random.default_rng(4)
    X0 = rng.random((n, ctl.r)) + 1j * rng.random((n, ctl.r))
    s_qr, st_qr = OP.ps_tri_recy_sparse(C, p, rec, ctl, X0=X0)
    s_lu, st_lu = OP.ps_tri_recy_sparse(C, p, rec, ctl, X0=X0, factor="lu")
    assert np.max(np.abs(s_qr - s_lu) / s_qr) <= 1e-8
    assert np.array_equal(st_qr.refine_it > 0, st_lu.refine_it > 0)


@pytest.mark.parametrize("case", ["n1", "diagonal", "empty_columns", "two_blocks", "upper_only"])
def test_band_order_edge_patterns(case):
    """Degenerate patterns: the order is still a permutation, the stated bandwidths are those of
    PᵀCP, and it is never wider than the natural order."""
    rng = np.random.default_rng(3)
    if case == "n1":
        C = sp.csc_matrix(np.array([[2.0 + 1j]]))
    elif case == "diagonal":
        C = sp.diags(rng.standard_normal(50) + 3).tocsc().astype(np.complex128)
    elif case == "empty_columns":
        A = sp.random(40, 40, density=0.05, random_state=4, format="lil")
        A[:, 7] = 0
        A[:, 21] = 0
        C = (A + sp.eye(40)).tocsc().astype(np.complex128)
        C[7, 7] = 0                                   # stored zero on the diagonal
        C.eliminate_zeros()
    elif case == "two_blocks":
        B1 = sp.random(30, 30, density=0.1, random_state=5) + sp.eye(30)
        B2 = sp.random(25, 25, density=0.1, random_state=6) + sp.eye(25)
        C = sp.block_diag([B1, B2]).tocsc().astype(np.complex128)
        q = rng.permutation(55)
        C = C[q][:, q].tocsc()
    else:
        C = sp.triu(sp.random(60, 60, density=0.08, random_state=7) + sp.eye(60)).tocsc().astype(np.complex128)
    C.sort_indices()
    n = C.shape[0]
    p, l, u = R.band_order(C)
    assert np.array_equal(np.sort(p), np.arange(n))
    assert (l, u) == _bandwidths(C, p)
    l0, u0 = _bandwidths(C, np.arange(n))
    assert l * (l + u + 1) + l + u <= l0 * (l0 + u0 + 1) + l0 + u0
    if case in ("n1", "diagonal"):
        assert (l, u) == (0, 0)
