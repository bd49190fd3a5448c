"""The CPU restatement of psPrecRecy (oracle/psprecrecy.py) and the pieces it adds to the
oracle: shifted Cholesky-QR, the general recycled space (orth_S = false, implict_update =
true) and fastRaylRitz!.  No device: these pin the checker the GPU parity tests use.

Bars: σ against LAPACK's dense SVD within 1e-4·normC on every grid point;
factorisation identities to 1e-12 of the operand norms.
"""
import numpy as np
import pytest
import scipy.linalg as sla
import scipy.sparse as sp

from oracle import recugrid as ogrid
from oracle.linalg import qr_shiftchol_inplace, orth_typed
from oracle.psprecrecy import PsPrecRecyControl, PsPrecRecyRun, SparseOp, InvF, Chain, LowerFactor
from oracle.recyspace import RecycledSpaceGen, update_recycled_space, fast_rayl_ritz
from oracle.icfact import ic_factor
from rls_b200.examples import af23560_shaped


def crand(rng, *shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


def small_case(n=240, seed=3):
    normC = 645.74 * n / 23560 * 10
    C = af23560_shaped(n, per_row=10, half_width=20, normC=normC, seed=seed)
    from scipy.sparse.csgraph import reverse_cuthill_mckee
    p = np.ascontiguousarray(reverse_cuthill_mckee((abs(C) + abs(C.T)).tocsr(), symmetric_mode=True), dtype=np.int64)
    return C, normC, p


def test_shiftchol_qr_factorises():
    rng = np.random.default_rng(1)
    X = crand(rng, 300, 24) * np.logspace(0, -7, 24)[None, :]     # ill-conditioned: CholQR needs 2 sweeps
    A = X.copy()
    R = np.zeros((24, 24), dtype=np.complex128)
    assert qr_shiftchol_inplace(X, R)
    assert np.linalg.norm(X.conj().T @ X - np.eye(24)) < 1e-13
    assert np.linalg.norm(X @ R - A) <= 1e-12 * np.linalg.norm(A)
    assert np.allclose(np.tril(R, -1), 0)


def test_shiftchol_qr_shift_retry_on_rank_deficiency():
    """A numerically rank-deficient block makes the first Cholesky fail: the reference's shift
    rule retries, and the result is still orthonormal to working accuracy in its range."""
    rng = np.random.default_rng(2)
    B = crand(rng, 200, 6)
    X = np.hstack([B, B[:, :2] + 1e-17 * crand(rng, 200, 2)])
    qr_shiftchol_inplace(X)
    G = X.conj().T @ X
    assert np.all(np.isfinite(G))
    assert np.linalg.norm(G[:6, :6] - np.eye(6)) < 1e-8


def test_orth_typed_shiftchol():
    rng = np.random.default_rng(3)
    V, _ = np.linalg.qr(crand(rng, 150, 10))
    X = crand(rng, 150, 4)
    orth_typed(V, X, typ="shiftchol")
    assert np.linalg.norm(V.conj().T @ X) < 1e-13
    assert np.linalg.norm(X.conj().T @ X - np.eye(4)) < 1e-13


def test_general_space_caches_match_definitions():
    """recySpace.jl's comment block (:1-20): H1 = (MV)ᴴMV, H2 = (MV)ᴴSV, H3 = (SV)ᴴSV, J1 = MᴴMV,
    J2 = MᴴSV, J3 = SᴴMV, J4 = SᴴSV, J5 = MV, J6 = SV — after several updates with block
    rotations, shifts and the implicit-update rule, for the prediction stage's M = C·invF,
    S = invF (orth_S = false)."""
    C, normC, p = small_case(160)
    L, invp, _ = ic_factor(C, -0.3 + 0.2j, 1e-3, 1e-6, 1e-6, 40, 60, p)
    F = LowerFactor(L, p, invp)
    M = Chain(SparseOp(C), InvF(F))
    S = InvF(F)
    n, r = 160, 5
    rs = RecycledSpaceGen(n, 4, r, 1, orth_S=False, implict_update=True, implict_recycle=True)
    rng = np.random.default_rng(4)
    for k in range(6):
        X = crand(rng, n, r)
        update_recycled_space(M, S, 0.1 * k + 0.05j, rs, X, tau=1.6, r_sub=3, force_add=(k % 2 == 1))
    pr = rs.p * r
    V = rs.V[:, :pr]
    MV, SV = M.mul(V), S.mul(V)
    scale = np.linalg.norm(MV) ** 2
    assert np.linalg.norm(V.conj().T @ V - np.eye(pr)) < 1e-12
    for got, ref in ((rs.J5[:, :pr], MV), (rs.J6[:, :pr], SV)):
        assert np.linalg.norm(got - ref) <= 1e-10 * np.linalg.norm(ref)
    for got, ref in ((rs.J1[:, :pr], M.mul_adj(MV)), (rs.J2[:, :pr], M.mul_adj(SV)), (rs.J3[:, :pr], S.mul_adj(MV)),
                     (rs.J4[:, :pr], S.mul_adj(SV))):
        assert np.linalg.norm(got - ref) <= 1e-10 * np.linalg.norm(ref)
    for got, ref in ((rs.H1[:pr, :pr], MV.conj().T @ MV), (rs.H2[:pr, :pr], MV.conj().T @ SV),
                     (rs.H3[:pr, :pr], SV.conj().T @ SV)):
        assert np.linalg.norm(got - ref) <= 1e-10 * scale
    # the rotations triangularise L's last block column (recySpace.jl:226-286): blocks 1..p-1
    # of it vanish and block p is upper triangular
    last = rs.L[:pr, pr - r:pr]
    assert np.linalg.norm(last[:pr - r]) <= 1e-12 * np.linalg.norm(last)
    assert np.linalg.norm(np.tril(last[pr - r:], -1)) <= 1e-12 * np.linalg.norm(last)


def test_fast_rayl_ritz_residual_definition():
    """fastRaylRitz!: W = (M − zS)ᴴ(M − zS)X − XΛ with X = V·G, E = S·X; λ the smallest
    eigenvalues of the projected normal operator."""
    C, normC, p = small_case(160)
    L, invp, _ = ic_factor(C, 0.1 + 0.1j, 1e-3, 1e-6, 1e-6, 40, 60, p)
    F = LowerFactor(L, p, invp)
    M = Chain(SparseOp(C), InvF(F))
    S = InvF(F)
    n, r = 160, 4
    rs = RecycledSpaceGen(n, 3, r, 1, orth_S=False, implict_update=True, implict_recycle=True)
    rng = np.random.default_rng(5)
    for k in range(3):
        update_recycled_space(M, S, 0.2 * k + 0j, rs, crand(rng, n, r), tau=1.6, r_sub=r)
    z = 0.15 + 0.05j
    X = np.zeros((n, r), dtype=np.complex128)
    E = np.zeros_like(X)
    W = np.zeros_like(X)
    lam = np.zeros(r)
    fast_rayl_ritz(rs, z, X, E, W, lam)
    Cz = Chain(SparseOp(C, -z), InvF(F))
    Wref = Cz.mul_adj(Cz.mul(X)) - X * lam[None, :]
    assert np.linalg.norm(W - Wref) <= 1e-10 * np.linalg.norm(Cz.mul(X)) ** 2
    assert np.linalg.norm(E - S.mul(X)) <= 1e-10 * np.linalg.norm(E)
    V = rs.V[:, :rs.p * r]
    CV = Cz.mul(V)
    w = np.linalg.eigvalsh(CV.conj().T @ CV)
    assert np.allclose(lam, w[:r], rtol=1e-9, atol=1e-12 * w[-1])


@pytest.mark.parametrize("rp,orth", [(4, "shiftchol"), (6, "lapack")])
def test_oracle_psprecrecy_matches_dense_svd(rp, orth):
    C, normC, p = small_case(240)
    n = 240
    rng = np.random.default_rng(6)
    ctl = PsPrecRecyControl(tol=1e-4, main_normC=normC, main_tau=1.6, tol_pred=1e-3, pred_tau=1.6,
                            idx_cutoff_pred=0.01, pred_orth_type=orth, pred_conv_thresh_type=1,
                            lambda_lower_min=0.01, lambda_upper_max=30.0, r_main=6, p_main=30,
                            main_implict_recycle=True, r_pred=rp, p_pred=6, hsl_tol=1e-3, hsl_cntl_1=1e-6,
                            hsl_cntl_2=1e-6, hsl_icntl_1=40, hsl_icntl_2=60)
    rec = ogrid.recursion_grid(-1.6, 0.8, -1.55, 1.55, 6, 6, 3)
    run = PsPrecRecyRun(C, rec, ctl, p, crand(rng, n, 6).real + 0j, crand(rng, n, rp), bound_x0=crand(rng, n, 1))
    sig, st = run.run()
    A = C.toarray()
    truth = np.array([sla.svdvals(A - z * np.eye(n))[-1] for z in rec.Z])
    assert np.all(np.isfinite(sig))
    assert np.max(np.abs(sig - truth)) <= 1e-4 * normC
    assert st.n_pts >= 1 and st.n_pred_pts >= 1 and st.n_precond_rebuild_pts >= 1
    assert st.n_pts == int(np.sum(st.main_refine_it > 0)) or st.n_pts >= int(np.sum(st.main_refine_it > 0))
