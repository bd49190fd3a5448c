"""psTriRecy's sparse branch on the GPU (psTriRecy.jl:47-61 pre_process, :222-234 the shifted
sparse QR): the device band QR against LAPACK's QR, and the loop against the CPU restatement of
the reference's (M, S) form and against the dense SVD.

R of a QR is unique up to unit-modulus row phases, so R_gpu is compared as D·R_gpu with
D = diag(R_lapack) / diag(R_gpu).
"""
import numpy as np
import pytest
import scipy.sparse as sp

import oracle.pstrirecy as OP
from oracle import recugrid as G
from oracle.gradient import dense_sigma_grad
import rls_b200 as R
from rls_b200.examples import skewlap3d, af23560_shaped

pytestmark = pytest.mark.gpu


def _banded(n, l, u, seed):
    """Random complex band matrix made well conditioned by its diagonal (a random band with
    l ≫ u is numerically singular, and R's trailing phases are then noise)."""
    rng = np.random.default_rng(seed)
    diags, offs = [], []
    for d in range(-l, u + 1):
        m = n - abs(d)
        v = rng.standard_normal(m) + 1j * rng.standard_normal(m)
        if d == 0:
            v = v + 4.0 * np.sqrt(l + u + 1)
        diags.append(v)
        offs.append(d)
    return sp.diags(diags, offs, shape=(n, n), format="csc")


CASES = {
    "skew7_rcm": lambda: (skewlap3d(7).astype(np.complex128), None),
    "banded_l5_u9": lambda: (_banded(300, 5, 9, 1), np.arange(300)),
    "tridiag": lambda: (_banded(200, 1, 1, 2), np.arange(200)),
    "banded_l40_u3": lambda: (_banded(500, 40, 3, 3), np.arange(500)),
    "af_shaped_rcm": lambda: (af23560_shaped(1500).astype(np.complex128), None),
}


@pytest.mark.parametrize("name", list(CASES))
def test_band_qr_matches_lapack_r(cuda_device, name):
    C, perm = CASES[name]()
    S = R.SparseTri(C, perm)
    eng = R.Engine(0)
    try:
        eng.set_sparse_tri(S)
        B = sp.csc_matrix(C)[S.perm][:, S.perm].toarray()
        n = B.shape[0]
        scale = np.linalg.norm(B, 2) + 1.0
        for z in (0.3 - 0.2j, -1.5 + 2.0j, 0.5 * complex(B[0, 0]) + 0.1j):
            Rg, l, u = eng.band_r(z)
            A = B - z * np.eye(n)
            Rl = np.linalg.qr(A, mode="r")
            assert np.min(np.abs(np.diag(Rl))) > 1e-6 * scale     # well conditioned: phases determined
            d = np.diag(Rl) / np.diag(Rg)
            assert np.allclose(np.abs(d), 1.0, atol=1e-9)
            err = np.max(np.abs(d[:, None] * Rg - Rl))
            assert err <= 1e-12 * scale * np.sqrt(n), (name, z, err)
            # zero outside the band of width l + u, and upper triangular
            i, j = np.nonzero(Rg)
            assert np.all(j >= i) and np.all(j - i <= l + u)
            assert np.all(np.isreal(np.diag(Rg)))
    finally:
        eng.close()


def _skew_case(N=7, nx=8, k=4):
    C = skewlap3d(N).astype(np.complex128)
    s = (N / 25) ** 2
    grid = (-550 * s, 100 * s, -200 * s, 200 * s, nx, nx, k)
    normC = float(np.linalg.norm(C.toarray(), 2))
    return C, normC, grid


def test_sparse_pstrirecy_matches_restatement_and_dense_svd(cuda_device):
    C, normC, grid = _skew_case()
    n = C.shape[0]
    S = R.SparseTri(C)
    rec = R.recursion_grid(*grid)
    r, p = 6, 10
    rng = np.random.default_rng(3)
    X0 = rng.random((n, r)) + 1j * rng.random((n, r))
    ctl = R.PsTriRecyControl(normC=normC, tol=1e-4, p=p, p_min=1, recy_tau=1.6)
    sig, st = R.psTriRecy(S, rec, ctl, verbose=0, X0=X0)
    octl = OP.PsTriRecyControl(normC=normC, tol=1e-4, p=p, p_min=1, recy_tau=1.6)
    orec = G.recursion_grid(*grid)
    sig_o, st_o = OP.ps_tri_recy_sparse(C, S.perm, orec, octl, X0=X0, ritz_g1_always=True)
    truth = np.array([OP.dense_sigma_min(C.toarray(), z) for z in rec.Z])
    assert np.all(np.isfinite(sig))
    assert np.max(np.abs(sig - truth)) <= 1e-4 * normC
    assert np.max(np.abs(sig - truth) / truth) <= 1e-5
    assert np.max(np.abs(sig - sig_o)) <= 1e-4 * normC
    lead = 24
    assert np.array_equal(st.p_count[:lead], st_o.p_count[:lead])
    assert np.array_equal(st.refine_it[:lead] > 0, st_o.refine_it[:lead] > 0)
    assert np.array_equal(st.r_recy[:lead], st_o.r_recy[:lead])
    assert np.mean((st.refine_it > 0) == (st_o.refine_it > 0)) >= 0.9
    assert st.n_pts == int(np.sum(st.refine_it > 0)) > 0


def test_sparse_pstrirecy_af_shaped_lanes_and_gradient(cuda_device):
    """An af23560-shaped matrix (band ±300 at full size; here n = 1500) on 2 lanes with ∂σ/∂z
    at every point, against the dense SVD and its gradient; QR time is reported apart."""
    C = af23560_shaped(1500).astype(np.complex128)
    Cd = C.toarray()
    normC = float(np.linalg.norm(Cd, 2))
    grid = (-1.6, 0.8, -1.55, 1.55, 6, 6, 3)
    rec = R.recursion_grid(*grid)
    n = C.shape[0]
    rng = np.random.default_rng(5)
    X0 = rng.random((n, 6)) + 1j * rng.random((n, 6))
    ctl = R.PsTriRecyControl(normC=normC, tol=1e-4, p=20, p_min=1, recy_tau=1.6, collect_timing=True)
    sig, st = R.psTriRecy(C, rec, ctl, verbose=0, X0=X0, lanes=2, grad=True)
    ref = np.array([dense_sigma_grad(Cd, z)[:3] for z in rec.Z])
    assert np.max(np.abs(sig - ref[:, 0])) <= 1e-4 * normC
    assert np.max(np.abs(sig - ref[:, 0]) / ref[:, 0]) <= 1e-5
    err = np.maximum(np.abs(st.dsdx - ref[:, 1]), np.abs(st.dsdy - ref[:, 2]))
    assert err.max() <= 1e-3, err.max()
    assert st.qr_time_ns > 0 and st.n_pts > 0


def test_sparse_operator_is_dropped_by_a_schur_upload(cuda_device):
    C, normC, grid = _skew_case(N=5, nx=4, k=2)
    eng = R.Engine(0)
    try:
        eng.set_sparse_tri(R.SparseTri(C))
        T = R.pre_process(C)
        eng.set_schur(T)                      # back to the dense operator: no band left behind
        rec = R.recursion_grid(*grid)
        ctl = R.PsTriRecyControl(normC=normC, tol=1e-4, p=10)
        sig, st = eng.pstrirecy(rec, ctl)
        truth = np.array([OP.dense_sigma_min(C.toarray(), z) for z in rec.Z])
        assert np.max(np.abs(sig - truth)) <= 1e-4 * normC
        with pytest.raises(R.RLSError):
            eng.band_r(0.1)                   # no sparse operator any more
    finally:
        eng.close()


@pytest.mark.parametrize("name", ["skew7_rcm", "af_shaped_rcm"])
def test_band_qr_panel_widths_agree(cuda_device, name):
    """8- and 16-column panels (forced) give LAPACK's R up to row phases; the timed choice picks
    one of them and reports both timings."""
    C, perm = CASES[name]()
    S = R.SparseTri(C, perm)
    eng = R.Engine(0)
    try:
        eng.set_sparse_tri(S)
        B = sp.csc_matrix(C)[S.perm][:, S.perm].toarray()
        n = B.shape[0]
        z = 0.3 - 0.2j
        Rl = np.linalg.qr(B - z * np.eye(n), mode="r")
        scale = np.linalg.norm(B, 2) + 1.0
        for w in (8, 16, 0):
            eng.band_set_panel(w)
            Rg, l, u = eng.band_r(z)
            d = np.diag(Rl) / np.diag(Rg)
            assert np.allclose(np.abs(d), 1.0, atol=1e-9)
            assert np.max(np.abs(d[:, None] * Rg - Rl)) <= 1e-12 * scale * np.sqrt(n)
            _, _, wsel, m8, m16 = eng.band_info()
            if w:
                assert wsel == w
            else:
                assert wsel in (8, 16)
    finally:
        eng.close()
