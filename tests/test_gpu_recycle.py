"""Recycled-space update and recycle step on the GPU against the CPU restatement,
replayed on identical inputs (same X blocks, same shifts), so the two paths see the
same recycled space at every step.

Bases are compared through basis-invariant quantities (projector VVᴴ, spectrum of
the projected Hz), since an orthonormal basis is only unique up to a unitary.
"""
import ctypes as C

import numpy as np
import pytest
import scipy.linalg as sla

from oracle.pstrirecy import TriOp, IdentityOp, residual_norm_ok
from oracle.recycle import RecycledSpace, update_recycled_space, fast_svd_rayl_ritz_implicit, affine_combine
from rls_b200._lib import lib, check, ptr, c64
from rls_b200.solvers import Engine, pre_process
from rls_b200.examples import sprand

pytestmark = pytest.mark.gpu

N, R_, P_MAX = 240, 6, 8
SHIFT = 3.2 ** 2 * np.finfo(float).eps * 100


def right_sv(T, z, r):
    _, _, vh = np.linalg.svd(T - z * np.eye(T.shape[0]))
    return vh.conj().T[:, ::-1][:, :r].copy()


@pytest.fixture(scope="module")
def setup(cuda_device):
    T = pre_process(sprand(N).toarray())
    e = Engine(cuda_device)
    e.set_schur(T)
    check(lib().rls_test_setup(e._h, R_, P_MAX), e._h)
    zs = [0.45 + 0.0j + 0.01 * k + 0.004j * k for k in range(14)]
    return e, T, zs


def gpu_space(e, n):
    p = C.c_int(0)
    check(lib().rls_test_space_get(e._h, C.byref(p), None, None, None, None, None, None, None), e._h)
    pr = p.value * R_
    V = np.zeros((n, pr), dtype=np.complex128, order="F")
    J1, J2, J5 = (np.zeros_like(V) for _ in range(3))
    L, H1, H2 = (np.zeros((pr, pr), dtype=np.complex128, order="F") for _ in range(3))
    check(lib().rls_test_space_get(e._h, C.byref(p), ptr(V), ptr(J1), ptr(J2), ptr(J5), ptr(L), ptr(H1), ptr(H2)),
          e._h)
    return p.value, V, J1, J2, J5, L, H1, H2


def test_space_updates_and_recycle_match(setup):
    e, T, zs = setup
    n = T.shape[0]
    rs = RecycledSpace(n, n, P_MAX, R_, p_min=1)
    M, S = TriOp(T), IdentityOp()
    for k, z in enumerate(zs):
        X = right_sv(T, z, R_)
        update_recycled_space(M, S, z, rs, X, tau=1.6, r_sub=1, force_add=(k % 5 == 4))
        Xf = np.asfortranarray(X)
        check(lib().rls_test_space_update(e._h, c64(z.real, z.imag), ptr(Xf), 1.6, int(k % 5 == 4), 1), e._h)
        p, V, J1, J2, J5, L, H1, H2 = gpu_space(e, n)
        assert p == rs.p, (k, p, rs.p)
        pr = p * R_
        Vo = rs.V[:, :pr]
        # same subspace, orthonormal basis, consistent cached products
        assert np.linalg.norm(V.conj().T @ V - np.eye(pr)) < 1e-11
        assert np.linalg.norm(V @ V.conj().T - Vo @ Vo.conj().T) < 1e-7 * np.sqrt(pr)
        assert np.linalg.norm(J5 - T @ V) <= 1e-12 * np.linalg.norm(T) * np.sqrt(pr)
        assert np.linalg.norm(J2 - T.conj().T @ V) <= 1e-12 * np.linalg.norm(T) * np.sqrt(pr)
        assert np.linalg.norm(J1 - T.conj().T @ (T @ V)) <= 1e-11 * np.linalg.norm(T) ** 2 * np.sqrt(pr)
        assert np.linalg.norm(H1 - V.conj().T @ J1) <= 1e-11 * np.linalg.norm(T) ** 2 * np.sqrt(pr)
        assert np.linalg.norm(H2 - V.conj().T @ J2) <= 1e-11 * np.linalg.norm(T) * np.sqrt(pr)
        # L keeps the inserted block: the newest block of V spans the last X (block rotations)
        Vp = V[:, (p - 1) * R_:pr]
        Qx = np.linalg.qr(X)[0]
        assert np.linalg.norm(Vp @ Vp.conj().T - Qx @ Qx.conj().T) < 1e-8
        assert np.linalg.norm(L[:(p - 1) * R_, (p - 1) * R_:pr]) < 1e-12 * max(1.0, np.linalg.norm(L))
        # spectrum of the projected normal matrix at a probe shift
        zp = 0.5 + 0.05j
        Hg = affine_combine(zp, H1, H2, H2.conj().T, np.eye(pr), shift=SHIFT)
        Ho = affine_combine(zp, rs.H1[:pr, :pr], rs.H2[:pr, :pr], rs.H2[:pr, :pr].conj().T, np.eye(pr), shift=SHIFT)
        wg = np.linalg.eigvalsh((Hg + Hg.conj().T) / 2)
        wo = np.linalg.eigvalsh((Ho + Ho.conj().T) / 2)
        assert np.allclose(wg, wo, atol=1e-10 * np.abs(wo).max())
    # recycle step at probe points between the update shifts
    n_cmp = 0
    for zp in [0.455 + 0.002j, 0.505 + 0.021j, 0.53 + 0.04j, 0.58 + 0.05j, 0.8 + 0.3j, 1.5 + 0.5j, 0.2 - 0.1j]:
        rr = C.c_int(0)
        sig = np.zeros(R_)
        Xg = np.zeros((n, R_), dtype=np.complex128, order="F")
        Wg = np.zeros_like(Xg)
        w0 = C.c_double(0)
        check(lib().rls_test_recycle(e._h, c64(zp.real, zp.imag), SHIFT, 1e-10, C.byref(rr), ptr(sig), ptr(Xg),
                                     ptr(Wg), C.byref(w0)), e._h)
        Xo = np.zeros((n, R_), dtype=np.complex128)
        Wo = np.zeros_like(Xo)
        so = np.zeros(R_)
        rr_o = fast_svd_rayl_ritz_implicit(rs, zp, Xo, Wo, so, complex(SHIFT), 1e-10, ritz_g1_always=True)
        assert rr.value == rr_o, (zp, rr.value, rr_o)
        assert np.allclose(sig, so, rtol=1e-9, atol=1e-14), (sig, so)
        assert abs(w0.value - np.linalg.norm(Wg[:, 0])) <= 1e-12 * max(1.0, w0.value)
        n_cmp += 1
        w0o = np.linalg.norm(Wo[:, 0])
        assert abs(w0.value - w0o) <= 1e-6 * max(w0o, 1e-14) + 1e-13, (zp, w0.value, w0o)
        # X spans the same Ritz directions (column phases are free)
        for j in range(R_):
            ov = abs(np.vdot(Xg[:, j], Xo[:, j])) / (np.linalg.norm(Xg[:, j]) * np.linalg.norm(Xo[:, j]))
            assert ov > 1 - 1e-8, (zp, j, ov)
        assert residual_norm_ok(Wg, sig[0], 1e-4, 3.2) == residual_norm_ok(Wo, so[0], 1e-4, 3.2)
    assert n_cmp == 7
