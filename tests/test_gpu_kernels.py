"""Kernel-level parity on the GPU: each device routine against the LAPACK/BLAS routine
the reference calls at that point (SciPy/NumPy FP64 on the same inputs).

Floating-point tolerances are relative to the operand norms (FP64 throughout).
"""
import ctypes as C

import numpy as np
import pytest
import scipy.linalg as sla

from oracle.linalg import svd_inplace, lq_rows_inplace
from oracle.recycle import find_rr_dim, affine_combine
from rls_b200._lib import lib, check, ptr, c64, ArgumentError
from rls_b200.solvers import Engine

pytestmark = pytest.mark.gpu


def crand(rng, *shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


@pytest.fixture(scope="module")
def eng_T(cuda_device):
    rng = np.random.default_rng(7)
    n = 300
    A = crand(rng, n, n) / np.sqrt(n)
    T = np.triu(sla.schur(A, output="complex")[0])
    e = Engine(cuda_device)
    e.set_schur(T)
    check(lib().rls_test_setup(e._h, 6, 20), e._h)
    return e, T


@pytest.mark.parametrize("adj", [0, 1])
@pytest.mark.parametrize("k", [1, 6, 18])
def test_trsm_matches_ztrsm(eng_T, adj, k):
    e, T = eng_T
    n = T.shape[0]
    rng = np.random.default_rng(k + 10 * adj)
    B = np.asfortranarray(crand(rng, n, k))
    z = 0.3 - 0.2j
    X = np.zeros((n, k), dtype=np.complex128, order="F")
    check(lib().rls_test_trsm(e._h, c64(z.real, z.imag), adj, k, ptr(B), ptr(X)), e._h)
    R = T - z * np.eye(n)
    ref = sla.solve_triangular(R, B, lower=False, trans="C" if adj else "N")
    err = np.linalg.norm(X - ref) / np.linalg.norm(ref)
    assert err < 1e-12, err


@pytest.mark.parametrize("adj", [0, 1])
@pytest.mark.parametrize("ctas", [1, 5, 64])
def test_trsm_on_fewer_ctas_matches_ztrsm(eng_T, adj, ctas):
    """rls_set_trsm_ctas: CTAs that solve several half block rows each, down to a single
    CTA walking all of them in dependency order, give the same solution."""
    e, T = eng_T
    n = T.shape[0]
    rng = np.random.default_rng(7 + adj)
    B = np.asfortranarray(crand(rng, n, 6))
    z = -0.1 + 0.25j
    X = np.zeros((n, 6), dtype=np.complex128, order="F")
    X0 = np.zeros_like(X)
    check(lib().rls_test_trsm(e._h, c64(z.real, z.imag), adj, 6, ptr(B), ptr(X0)), e._h)
    check(lib().rls_set_trsm_ctas(e._h, ctas), e._h)
    try:
        check(lib().rls_test_trsm(e._h, c64(z.real, z.imag), adj, 6, ptr(B), ptr(X)), e._h)
    finally:
        check(lib().rls_set_trsm_ctas(e._h, 0), e._h)
    ref = sla.solve_triangular(T - z * np.eye(n), B, lower=False, trans="C" if adj else "N")
    assert np.linalg.norm(X - ref) / np.linalg.norm(ref) < 1e-12
    assert np.array_equal(X, X0)             # same products in the same order per row


def test_set_trsm_ctas_rejects_negative(eng_T):
    e, _ = eng_T
    with pytest.raises(ArgumentError):
        check(lib().rls_set_trsm_ctas(e._h, -1), e._h)


@pytest.mark.parametrize("adj", [0, 1])
@pytest.mark.parametrize("k", [1, 6, 12])
def test_trmm_matches_ztrmm(eng_T, adj, k):
    e, T = eng_T
    n = T.shape[0]
    rng = np.random.default_rng(100 + k)
    X = np.asfortranarray(crand(rng, n, k))
    Y = np.zeros((n, k), dtype=np.complex128, order="F")
    check(lib().rls_test_trmm(e._h, adj, k, ptr(X), ptr(Y)), e._h)
    ref = (T.conj().T if adj else T) @ X
    assert np.linalg.norm(Y - ref) / np.linalg.norm(ref) < 1e-13


@pytest.mark.parametrize("m,k", [(300, 1), (300, 6), (257, 18), (300, 40), (200, 64), (300, 70)])
def test_qr_factor(eng_T, m, k):
    e, _ = eng_T
    rng = np.random.default_rng(m * 1000 + k)
    A = np.asfortranarray(crand(rng, m, k))
    # graded columns to exercise stability
    A *= np.logspace(0, -6, k)[None, :]
    R = np.zeros((k, k), dtype=np.complex128, order="F")
    check(lib().rls_test_qr(e._h, m, k, ptr(A), ptr(R), None), e._h)
    Rref = np.linalg.qr(A, mode="r")
    # R is unique up to a unit-modulus scaling of its rows: compare RᴴR and |diag|
    assert np.allclose(np.abs(np.diag(R)), np.abs(np.diag(Rref)), rtol=1e-10, atol=0)
    G = R.conj().T @ R
    assert np.linalg.norm(G - A.conj().T @ A) <= 1e-12 * np.linalg.norm(A) ** 2
    assert np.allclose(np.tril(R, -1), 0)
    if k <= 64:
        Q = np.zeros((m, k), dtype=np.complex128, order="F")
        R2 = np.zeros((k, k), dtype=np.complex128, order="F")
        check(lib().rls_test_qr(e._h, m, k, ptr(A), ptr(R2), ptr(Q)), e._h)
        assert np.linalg.norm(Q.conj().T @ Q - np.eye(k)) < 1e-13
        assert np.linalg.norm(Q @ R2 - A) <= 1e-13 * np.linalg.norm(A)


@pytest.mark.parametrize("nS,r,sideL,lq", [(6, 6, 1, 1), (12, 6, 1, 1), (18, 6, 1, 1), (18, 6, 0, 1),
                                            (9, 6, 0, 0), (40, 6, 0, 0), (3, 1, 1, 1)])
def test_svd_rr_matches_zgesdd(eng_T, nS, r, sideL, lq):
    e, _ = eng_T
    rng = np.random.default_rng(nS * 7 + r)
    Rin = np.asfortranarray(np.triu(crand(rng, nS, nS)) * np.logspace(0, -4, nS)[None, :])
    sig = np.zeros(nS)
    lam = np.zeros(r)
    G = np.zeros((nS, nS), dtype=np.complex128, order="F")
    check(lib().rls_test_svd_rr(e._h, nS, r, sideL, lq, ptr(Rin), ptr(sig), ptr(lam), ptr(G)), e._h)
    s_ref = np.zeros(nS)
    V_ref = np.zeros((nS, nS), dtype=np.complex128)
    svd_inplace(Rin.copy(), s_ref, V_ref, ascending=not sideL)
    if sideL:
        s_ref[:r] = 1.0 / s_ref[:r]
    assert np.allclose(sig, s_ref, rtol=1e-11, atol=1e-15 * np.abs(s_ref).max())
    assert np.allclose(lam, s_ref[:r] ** 2, rtol=1e-11)
    # Ritz vectors: columns agree up to unit phases
    for j in range(r):
        ov = abs(np.vdot(G[:, j], V_ref[:, j]))
        assert ov > 1 - 1e-9, (j, ov)
    if lq and nS > r:
        Q_mat = V_ref[:r, r:nS].copy()
        lq_rows_inplace(Q_mat)
        GP_ref = V_ref[:, r:nS] @ Q_mat.conj().T
        GP = G[:, r:2 * r]
        Pr = GP_ref @ GP_ref.conj().T
        Pg = GP @ GP.conj().T
        assert np.linalg.norm(Pr - Pg) < 1e-9


def _hz_pair(rng, pr):
    B = crand(rng, 3 * pr, pr)
    H1 = B.conj().T @ B
    H2 = crand(rng, pr, pr) * 0.3
    return np.asfortranarray(H1), np.asfortranarray(H2)


@pytest.mark.parametrize("pr,r,tau", [(12, 6, 1e-10), (36, 6, 1e-10), (90, 6, 1e-12), (120, 6, 1e-10),
                                      (6, 6, 1e-10), (18, 6, 1e10)])
def test_heev_rr_matches_zheevr(eng_T, pr, r, tau):
    e, _ = eng_T
    rng = np.random.default_rng(pr + 3)
    H1, H2 = _hz_pair(rng, pr)
    z = 0.4 + 0.1j
    shift = 1e-13
    rr = C.c_int(0)
    lam = np.zeros(pr)
    G = np.zeros((pr, pr), dtype=np.complex128, order="F")
    clk = np.zeros(6, dtype=np.int64)
    check(lib().rls_test_heev_rr(e._h, pr, r, ptr(H1), ptr(H2), c64(z.real, z.imag), shift, tau, C.byref(rr),
                                 ptr(lam), ptr(G), ptr(clk)), e._h)
    ph = np.diff(clk)
    print(f"heev pr={pr}: cycles build+tridiag {ph[0]}, eigenvalues {ph[1]}, inverse iteration {ph[2]}, "
          f"orthogonalisation {ph[3]}, back-transform {ph[4]}")
    Hz = affine_combine(z, H1, H2, H2.conj().T, np.eye(pr), shift=shift)
    Hz = np.triu(Hz) + np.triu(Hz, 1).conj().T
    Hz[np.diag_indices(pr)] = Hz.diagonal().real
    rr_ref, G_ref = find_rr_dim(Hz, r, tau)
    assert rr.value == rr_ref
    w = np.linalg.eigvalsh(Hz)
    scale = abs(w).max()
    assert abs(lam[pr - 1] - w[-1]) <= 1e-12 * scale
    k = rr.value
    assert np.allclose(lam[:min(k, pr - 1)], w[:min(k, pr - 1)], atol=1e-12 * scale, rtol=0)
    Gk = G[:, :k]
    assert np.linalg.norm(Gk.conj().T @ Gk - np.eye(k)) < 1e-10
    # invariant subspace: projector equality (eigenvectors are unique only up to phase / within clusters)
    Pg = Gk @ Gk.conj().T
    Pr = G_ref[:, :k] @ G_ref[:, :k].conj().T
    assert np.linalg.norm(Pg - Pr) < 1e-8
    # residual of the Ritz pairs
    res = np.linalg.norm(Hz @ Gk - Gk * w[:k][None, :]) / scale
    assert res < 1e-10


@pytest.fixture(scope="module")
def eng_T60(cuda_device):
    """A space of up to 60 blocks of 6 columns: the projected problem reaches pr = 360, the
    size psTriRecy's p = 60, r = 6 allow."""
    rng = np.random.default_rng(17)
    n = 400
    T = np.triu(crand(rng, n, n)) / np.sqrt(n) + np.eye(n)
    e = Engine(cuda_device)
    e.set_schur(T)
    check(lib().rls_test_setup(e._h, 6, 60), e._h)
    yield e
    e.close()


@pytest.mark.parametrize("pr,tau", [(180, 1e-10), (240, 1e-12), (360, 1e-10), (360, 1e10)])
def test_heev_rr_full_size_matches_zheevr(eng_T60, pr, tau):
    """find_rr_dim! at the sizes the p = 60 space reaches (the eigensolver keeps Hz in global
    memory beyond its shared-memory limit).  τ = 1e10 makes the gap rule run through several
    growing index ranges."""
    e = eng_T60
    r = 6
    rng = np.random.default_rng(pr + 11)
    H1, H2 = _hz_pair(rng, pr)
    z = -0.3 + 0.2j
    shift = 1e-13
    rr = C.c_int(0)
    lam = np.zeros(pr)
    G = np.zeros((pr, pr), dtype=np.complex128, order="F")
    check(lib().rls_test_heev_rr(e._h, pr, r, ptr(H1), ptr(H2), c64(z.real, z.imag), shift, tau, C.byref(rr),
                                 ptr(lam), ptr(G), None), e._h)
    Hz = affine_combine(z, H1, H2, H2.conj().T, np.eye(pr), shift=shift)
    Hz = np.triu(Hz) + np.triu(Hz, 1).conj().T
    Hz[np.diag_indices(pr)] = Hz.diagonal().real
    rr_ref, G_ref = find_rr_dim(Hz, r, tau)
    assert rr.value == rr_ref
    w = np.linalg.eigvalsh(Hz)
    scale = abs(w).max()
    assert abs(lam[pr - 1] - w[-1]) <= 1e-12 * scale
    k = rr.value
    assert np.allclose(lam[:min(k, pr - 1)], w[:min(k, pr - 1)], atol=1e-12 * scale, rtol=0)
    Gk = G[:, :k]
    assert np.linalg.norm(Gk.conj().T @ Gk - np.eye(k)) < 1e-10
    res = np.linalg.norm(Hz @ Gk - Gk * w[:k][None, :]) / scale
    assert res < 1e-10


def test_recip_nr_against_cuda_division(cuda_device):
    """The eigensolver's Sturm counts divide by the pivot through recip_nr (rcp.approx.ftz.f64
    estimate + two Newton–Raphson steps).  Its stated bound: within 2 ulp (relative error
    ≤ 2⁻⁵¹) of CUDA's correctly rounded 1.0/q for normal q whose reciprocal is normal, both
    signs, across the exponent range."""
    rng = np.random.default_rng(3)
    mant = 1.0 + rng.random(20000)
    expo = rng.integers(-1000, 1000, size=20000)
    q = np.ldexp(mant, expo) * np.where(rng.random(20000) < 0.5, -1.0, 1.0)
    q = np.concatenate([q, [1.0, -1.0, 3.0, 0.1, 1e-300, -1e300, 2.0 ** -1020, 2.0 ** 1020]])
    n = q.size
    r_nr = np.zeros(n)
    r_div = np.zeros(n)
    e = Engine(cuda_device)
    check(lib().rls_test_recip(e._h, n, ptr(q), ptr(r_nr), ptr(r_div)), e._h)
    e.close()
    assert np.array_equal(r_div, 1.0 / q)           # CUDA's division is IEEE round-to-nearest
    rel = np.abs(r_nr - r_div) / np.abs(r_div)
    assert np.all(np.isfinite(r_nr))
    assert rel.max() <= 2.0 ** -51, rel.max()
