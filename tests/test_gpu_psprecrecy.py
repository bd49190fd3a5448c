"""psPrecRecy and the operator-generic lobpcgSvd on the GPU against the CPU restatement and the
FP64 dense SVD.

* rls_lobpcg_svd on each operator the solvers use (ShiftedMat with the SparseLLTP
  preconditioner, side 'S'; the prediction operator Cz·invF with :shiftchol and
  conv_thresh_type 1, r up to 40; the r = 1 bound estimates γ and λ_n, side 'L'; the
  inverse Schur operator) against oracle/lobpcg.py on the same operators and X0;
* rls_psprecrecy on small af23560-shaped matrices (the synthetic generator at reduced size)
  against oracle/psprecrecy.py and against LAPACK's dense SVD on every grid point, including
  r_pred = 40 (the prediction stage's kernels for wide blocks).

Bars: σ within 1e-4·normC of the dense SVD; LOBPCG σ within 1e-8·normC of
the restatement's converged value for the same operator and X0 (both iterate to the same
tolerance from the same start).
"""
import ctypes as C

import numpy as np
import pytest
import scipy.linalg as sla

import rls_b200 as R
from oracle import recugrid as ogrid
from oracle.lobpcg import LobpcgSvdControl as OCtl, LobpcgSvdKeep, lobpcg_svd
from oracle.precond import lltp_ldiv
from oracle.psprecrecy import (PsPrecRecyControl as OPCtl, PsPrecRecyRun, SparseOp, InvF, Chain, LowerFactor, InvL)
from rls_b200.examples import af23560_shaped

pytestmark = pytest.mark.gpu


def crand(rng, *shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


def small_case(n, per_row=10, half_width=20, seed=3):
    from scipy.sparse.csgraph import reverse_cuthill_mckee
    normC = 645.74 * n / 23560 * 10
    C = af23560_shaped(n, per_row=per_row, half_width=half_width, normC=normC, seed=seed)
    p = np.ascontiguousarray(reverse_cuthill_mckee((abs(C) + abs(C.T)).tocsr(), symmetric_mode=True), dtype=np.int64)
    return C, normC, p


class _K:
    """SparseLLTP ldiv! through the restated substitutions (oracle/precond.py)."""

    def __init__(self, L, p, invp):
        self.L, self.p, self.invp = L, p, invp

    def ldiv(self, B):
        return lltp_ldiv(self.L, self.p, self.invp, B)


@pytest.fixture(scope="module")
def lob_case(cuda_device):
    C, normC, p = small_case(240)
    z0 = -0.2 + 0.3j
    L, invp, _ = R.ic_factor(C, z0, 1e-3, 1e-6, 1e-6, 40, 60, p)
    e = R.Engine(0)
    e.sparse_upload(C)
    R.SparseLLTP(L, p, invp, e)
    yield e, C, normC, p, L, invp
    e.close()


@pytest.mark.parametrize("op,prec,side,r,orth,ctype", [
    ("shifted", "lltp", "S", 6, "lapack", 0),
    ("shifted", None, "S", 3, "shiftchol", 0),
    ("pred", None, "S", 8, "shiftchol", 1),
    ("pred", None, "S", 40, "shiftchol", 1),
    ("pred", None, "L", 1, "lapack", 0),
    ("inv_l", None, "L", 1, "lapack", 0),
])
def test_generic_lobpcg_matches_restatement(lob_case, op, prec, side, r, orth, ctype):
    e, C, normC, p, L, invp = lob_case
    n = C.shape[0]
    z = 0.1 - 0.2j
    rng = np.random.default_rng(r + 7 * len(op))
    X0 = crand(rng, n, r)
    F = LowerFactor(L, p, invp)
    oop = {"shifted": SparseOp(C, -z), "pred": Chain(SparseOp(C, -z), InvF(F)), "inv_l": InvL(F)}[op]
    nC = normC if op == "shifted" else 2.0
    tol = 1e-5 if side == "S" else 1e-6
    kw = dict(m=n, n=n, r=r, tol=tol, side=side, normC=nC, orth_type=orth, conv_range=(1, min(r, 4)),
              conv_thresh_type=ctype)
    s, it, X, sr = e.lobpcg_svd(op, z, R.LobpcgSvdControl(**kw), prec=prec, X0=X0)
    keep = LobpcgSvdKeep(n, n, r)
    keep.S[:, :r] = X0
    s_o, it_o = lobpcg_svd(oop, keep.S[:, :r], _K(L, p, invp) if prec else None, keep, OCtl(**kw))
    assert np.isfinite(s) and it >= 1
    assert abs(it - it_o) <= 2, (it, it_o)
    assert abs(s - s_o) <= 1e-8 * max(nC, abs(s_o)), (s, s_o)
    # the dense truth of the value lobpcgSvd returns
    A = C.toarray()
    if op == "inv_l":
        truth = np.linalg.norm(np.linalg.inv(np.tril(L.toarray())), 2)
    else:
        M = A - z * np.eye(n)
        if op == "pred":
            Li = np.linalg.inv(np.tril(L.toarray()))
            Pm = np.eye(n)[invp, :]                        # P·X = X[invp, :]
            M = M @ Pm @ Li.conj().T
        sv = sla.svdvals(M)
        truth = sv[0] if side == "L" else sv[-1]
    assert abs(s - truth) <= 1e-3 * truth, (s, truth)


def test_generic_lobpcg_inverse_schur_matches_invtri(cuda_device):
    rng = np.random.default_rng(9)
    n = 200
    A = crand(rng, n, n) / np.sqrt(n)
    T = np.triu(sla.schur(A, output="complex")[0])
    e = R.Engine(0)
    e.set_schur(T)
    z = 0.3 + 0.1j
    X0 = crand(rng, n, 6)
    ctl = R.LobpcgSvdControl(m=n, n=n, r=6, conv_range=(1, 1), tol=1e-8, side="L", normC=1.0)
    s1, it1, X1, sr1 = e.lobpcg_svd_invtri(z, ctl, X0=X0)
    s2, it2, X2, sr2 = e.lobpcg_svd("inv_schur", z, ctl, X0=X0)
    e.close()
    truth = sla.svdvals(A - z * np.eye(n))[-1]
    assert abs(sr1[0] - truth) <= 1e-10 and abs(sr2[0] - truth) <= 1e-10
    assert abs(it1 - it2) <= 1


def _pp_control(normC, rp, orth, p_pred):
    kw = dict(tol=1e-4, main_normC=normC, main_tau=1.6, tol_pred=1e-3, pred_tau=1.6, idx_cutoff_pred=0.01,
              pred_orth_type=orth, pred_conv_thresh_type=1, lambda_lower_min=0.01, lambda_upper_max=30.0,
              r_main=6, p_main=30, main_implict_recycle=True, r_pred=rp, p_pred=p_pred, hsl_tol=1e-3,
              hsl_cntl_1=1e-6, hsl_cntl_2=1e-6, hsl_icntl_1=40, hsl_icntl_2=60)
    return R.PsPrecRecyControl(**kw), OPCtl(**kw)


@pytest.mark.parametrize("n,rp,orth,p_pred,grid", [
    (240, 4, "shiftchol", 6, (-1.6, 0.8, -1.55, 1.55, 6, 6, 3)),
    (240, 6, "lapack", 6, (-1.6, 0.8, -1.55, 1.55, 6, 6, 3)),
    (400, 40, "shiftchol", 3, (-1.6, 0.8, -1.55, 1.55, 4, 4, 2)),
])
def test_psprecrecy_matches_restatement_and_dense_svd(cuda_device, n, rp, orth, p_pred, grid):
    C, normC, p = small_case(n)
    rng = np.random.default_rng(n + rp)
    X0m = rng.random((n, 6)) + 1j * rng.random((n, 6))
    X0p = rng.random((n, rp)) + 1j * rng.random((n, rp))
    xb = rng.random((n, 1)) + 1j * rng.random((n, 1))
    ctl, octl = _pp_control(normC, rp, orth, p_pred)
    rec = R.recursion_grid(*grid)
    sig, st = R.psPrecRecy(C, rec, ctl, verbose=0, p=p, X0_main=X0m, X0_pred=X0p, X0_bound=xb)
    run = PsPrecRecyRun(C, ogrid.recursion_grid(*grid), octl, p, X0m, X0p, bound_x0=xb)
    sig_o, st_o = run.run()
    A = C.toarray()
    truth = np.array([sla.svdvals(A - z * np.eye(n))[-1] for z in rec.Z])
    assert np.all(np.isfinite(sig))
    assert np.max(np.abs(sig - truth)) <= 1e-4 * normC, np.max(np.abs(sig - truth))
    assert np.max(np.abs(sig - sig_o)) <= 1e-4 * normC
    # the same trajectory over the leading points: recycle/refine decisions of both stages
    lead = 6
    assert np.array_equal(st.main_refine_it[:lead] > 0, st_o.main_refine_it[:lead] > 0)
    assert np.array_equal(st.pred_refine_it[:lead] > 0, st_o.pred_refine_it[:lead] > 0)
    assert np.array_equal(st.p_count[:lead], st_o.p_count[:lead])
    assert st.n_precond_rebuild_pts >= 1 and st.n_pts >= 1
    assert np.array_equal(st.precond_rebuild_pts[:1], rec.Z[:1])


def test_psprecrecy_range_calls_equal_one_call(cuda_device):
    """rls_psprecrecy_range continues a run: two range calls give the single call's results."""
    C, normC, p = small_case(240)
    n = 240
    rng = np.random.default_rng(17)
    X0m, X0p, xb = crand(rng, n, 6), crand(rng, n, 4), crand(rng, n, 1)
    ctl, _ = _pp_control(normC, 4, "shiftchol", 6)
    rec = R.recursion_grid(-1.6, 0.8, -1.55, 1.55, 6, 6, 3)
    e = R.Engine(0)
    run1 = R.PrecRecyRun(e, C, rec, ctl, p=p, X0_main=X0m, X0_pred=X0p, X0_bound=xb)
    s1, st1 = run1.run()
    run2 = R.PrecRecyRun(e, C, rec, ctl, p=p, X0_main=X0m, X0_pred=X0p, X0_bound=xb)
    run2.run(0, 17)
    s2, st2 = run2.run(17, 36)
    e.close()
    assert np.array_equal(s1, s2)
    assert np.array_equal(st1.main_refine_it, st2.main_refine_it)
    assert st1.n_pred_pts == st2.n_pred_pts


def test_psprecrecy_lanes_equal_runs_on_their_subgrids(cuda_device):
    """PrecRecyLanes: each lane is exactly a psPrecRecy run on its column-aligned part of the
    traversal (same σ bit for bit, same per-point counters), and σ meets the dense SVD."""
    from rls_b200.grid import Recursion
    C, normC, p = small_case(240)
    n = 240
    rng = np.random.default_rng(23)
    X0m, X0p, xb = crand(rng, n, 6), crand(rng, n, 4), crand(rng, n, 1)
    ctl, _ = _pp_control(normC, 4, "shiftchol", 6)
    rec = R.recursion_grid(-1.6, 0.8, -1.55, 1.55, 8, 6, 3)
    sig, st = R.psPrecRecy(C, rec, ctl, verbose=0, p=p, X0_main=X0m, X0_pred=X0p, X0_bound=xb, lanes=3)
    ls = R.PrecRecyLanes(3, C, rec, ctl, p=p, X0_main=X0m, X0_pred=X0p, X0_bound=xb)
    offs = ls.offs
    ls.close()
    assert offs[0] == 0 and offs[-1] == len(rec.Z) and np.all(np.diff(offs) > 0)
    e = R.Engine(0)
    try:
        for l in range(3):
            sub = Recursion(rec.x_st, rec.x_ed, rec.y_st, rec.y_ed, rec.n_x, rec.n_y, rec.k)
            sub.Z = np.ascontiguousarray(rec.Z[offs[l]:offs[l + 1]])
            s1, st1 = R.PrecRecyRun(e, C, sub, ctl, p=p, X0_main=X0m, X0_pred=X0p, X0_bound=xb).run()
            assert np.array_equal(sig[offs[l]:offs[l + 1]], s1)
            assert np.array_equal(st.main_refine_it[offs[l]:offs[l + 1]], st1.main_refine_it)
            assert np.array_equal(st.pred_refine_it[offs[l]:offs[l + 1]], st1.pred_refine_it)
    finally:
        e.close()
    A = C.toarray()
    truth = np.array([sla.svdvals(A - z * np.eye(n))[-1] for z in rec.Z])
    assert np.max(np.abs(sig - truth)) <= 1e-4 * normC
    assert st.n_precond_rebuild_pts >= 3     # one build per lane at least


def test_psprecrecy_rejects_unsupported_settings(cuda_device):
    C, normC, p = small_case(120)
    rec = R.recursion_grid(-1.6, 0.8, -1.55, 1.55, 4, 4, 2)
    e = R.Engine(0)
    for bad in (dict(main_implict_recycle=False), dict(pred_implict_update=False), dict(r_pred=41),
                dict(r_main=9)):
        kw = dict(main_normC=normC, main_implict_recycle=True, r_pred=4, p_pred=4)
        kw.update(bad)
        with pytest.raises(R.ArgumentError):
            R.PrecRecyRun(e, C, rec, R.PsPrecRecyControl(**kw), p=p).run()
    with pytest.raises(R.ArgumentError):
        R.PrecRecyRun(e, C, rec, R.PsPrecRecyControl(main_normC=normC, main_implict_recycle=True, r_pred=4),
                      p=np.zeros(120, dtype=np.int64)).run()
    e.close()
