"""Restatement of src/core/psPrecRecy.jl (the preconditioned two-space grid solver) — test
infrastructure only (see oracle/__init__.py).

Every step follows the reference's loop (psPrecRecy.jl:617-1033): the main recycled space
on M = C, S = I (orth_S = true), the prediction space on M_pred = C·invF, S_pred = invF
(orth_S = false), the two-level preconditioner SparseLLTP_AD, the Ritz-bound estimates γ and
λ_n (:388-422) and the rebuild rule (:201-209, :825-908).  The IC factor comes from
oracle/icfact.py (get_hsl_LLTP restated).  Two inputs the reference draws inside Julia come
from the caller here: the column order p (the reference takes SPQR's qr(C).cpiv, :625, which
needs SuiteSparse) and the random start blocks (rand!, :547, :586, :849).
"""
from __future__ import annotations

import time
from dataclasses import dataclass

import numpy as np
import scipy.linalg as sla
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from .icfact import ic_factor
from .lobpcg import LobpcgSvdControl, LobpcgSvdKeep, check_conv_svd, lobpcg_svd
from .linalg import EPS
from .recycle import fast_svd_rayl_ritz_implicit, resolve_recycle_fail_dist_thresh
from .recyspace import RecycledSpaceGen, fast_rayl_ritz, update_recycled_space


@dataclass
class PsPrecRecyControl:
    """psPrecRecy.jl:220-261 (same fields, same defaults; shift = main_normC²·eps·100)."""
    tol: float = 1e-3
    lobpcg_tol_scale: float = 0.1
    main_normC: float = 10.0
    main_tau: float = 1.666
    shift: float = None
    gap_tau: float = 1e-10
    recycle_fail_dist_thresh: float = float("nan")
    tol_pred: float = 1e-3
    lobpcg_pred_tol_scale: float = 1.0
    pred_conv_range: tuple = None
    pred_tau: float = 1.666
    idx_cutoff_pred: float = 1e-2
    pred_orth_type: str = "lapack"
    pred_conv_thresh_type: int = 0
    lambda_lower_min: float = 0.1
    lambda_upper_max: float = 30.0
    r_main: int = 6
    p_main: int = 60
    p_min_main: int = 1
    main_implict_update: bool = False
    main_implict_recycle: bool = False
    r_pred: int = 20
    p_pred: int = 20
    p_min_pred: int = 1
    pred_implict_update: bool = True
    pred_implict_recycle: bool = True
    hsl_tol: float = 1e-3
    hsl_cntl_1: float = 1e-6
    hsl_cntl_2: float = 1e-5
    hsl_icntl_1: int = 200
    hsl_icntl_2: int = 200
    gamma_tol: float = 1e-3
    lambda_n_tol: float = 1e-3
    inner_verbose_override: int = None
    collect_timing: bool = True

    def __post_init__(self):
        if self.shift is None:
            self.shift = self.main_normC ** 2 * EPS * 100


class PsPrecRecyStats:
    """psPrecRecy.jl:318-350."""

    def __init__(self, nZ):
        i = lambda: np.zeros(nZ, dtype=np.int64)
        c = lambda: np.zeros(nZ, dtype=np.complex128)
        self.p_count, self.pred_p_count, self.r_recy = i(), i(), i()
        self.pts, self.pred_pts, self.precond_rebuild_pts = c(), c(), c()
        self.main_M_vec_apps, self.main_M_vec_apps_no_recycle, self.main_L_vec_apps = i(), i(), i()
        self.pred_M_vec_apps, self.pred_L_vec_apps = i(), i()
        self.main_refine_it, self.pred_refine_it = i(), i()      # per point (an addition)
        self.n_it = self.n_pred_it = self.n_pts = self.n_pred_pts = self.n_precond_rebuild_pts = 0


# ---- operators (RLSMatrices.jl) ------------------------------------------------------------

class SparseOp:
    """C (SparseMatrixCSC) or ShiftedMat(C, s) = C + sI (RLSMatrices.jl:24-64)."""

    def __init__(self, C, s=0.0):
        self.C = sp.csr_matrix(C)
        self.CH = self.C.conj().T.tocsr()
        self.s = complex(s)

    def mul(self, X):
        return self.C @ X + self.s * X

    def mul_adj(self, Y):
        return self.CH @ Y + np.conj(self.s) * Y


class LowerFactor:
    """LowerTriangular(L) of a SparseLLTP, with its permutation (RLSPreconditioner.jl:8-26)."""

    def __init__(self, L, p, invp):
        self.L = sp.tril(sp.csr_matrix(L)).tocsr()
        self.LH = self.L.conj().T.tocsr()
        self.p, self.invp = np.asarray(p), np.asarray(invp)

    def fwd(self, X):     # L \ X
        return spla.spsolve_triangular(self.L, X, lower=True)

    def bwd(self, X):     # Lᴴ \ X
        return spla.spsolve_triangular(self.LH, X, lower=False)


class InvF:
    """invF = P·L⁻ᴴ (MulChainMat(PermMat, InvMat(adjoint(L))), RLSPreconditioner.jl:16-21);
    PermMat·X = X[invp, :], its adjoint X[p, :] (RLSMatrices.jl:330-380)."""

    def __init__(self, F: LowerFactor):
        self.F = F

    def mul(self, X):
        return self.F.bwd(X)[self.F.invp, :]

    def mul_adj(self, Y):
        return self.F.fwd(Y[self.F.p, :])


class Chain:
    """MulChainMat(A, B) = A·B (RLSMatrices.jl:81-195)."""

    def __init__(self, A, B):
        self.A, self.B = A, B

    def mul(self, X):
        return self.A.mul(self.B.mul(X))

    def mul_adj(self, Y):
        return self.B.mul_adj(self.A.mul_adj(Y))


class InvL:
    """InvMat(L) (psPrecRecy.jl:392): L⁻¹, adjoint L⁻ᴴ."""

    def __init__(self, F: LowerFactor):
        self.F = F

    def mul(self, X):
        return self.F.fwd(X)

    def mul_adj(self, Y):
        return self.F.bwd(Y)


class Identity:
    def mul(self, X):
        return X.copy()

    def mul_adj(self, Y):
        return Y.copy()


class LLTP_AD:
    """SparseLLTP_AD ldiv! (RLSPreconditioner.jl:229-262): X = K⁻¹B + E·GramE⁻¹·EᴴB."""

    def __init__(self, F: LowerFactor, E, GramE):
        self.F, self.E = F, E
        self.chol = sla.cho_factor(GramE, lower=False)     # rls_cholesky!(…; uplo = :U)

    def ldiv(self, B):
        coeff = sla.cho_solve(self.chol, self.E.conj().T @ B)
        X = self.F.fwd(B[self.F.p, :])
        X = self.F.bwd(X)[self.F.invp, :]
        return X + self.E @ coeff


# ---- the loop ---------------------------------------------------------------------------

def _pred_idx(lam, r_pred, cutoff):
    """something(findlast(<(cutoff), λ[1:r_pred]), r_pred) (psPrecRecy.jl:752): 1-based."""
    idx = np.flatnonzero(lam[:r_pred] < cutoff)
    return int(idx[-1]) + 1 if idx.size else r_pred


class PsPrecRecyRun:
    """psPrecRecy (psPrecRecy.jl:617-1033) on a sparse square C, resumable over index ranges."""

    def __init__(self, C, rec, ctl: PsPrecRecyControl, p, X0_main, X0_pred, bound_x0=None, log=None, ic=None):
        self.ic = ic or ic_factor        # get_hsl_LLTP's factorisation (the restatement by default)
        self.C = sp.csc_matrix(C, dtype=np.complex128)
        n = self.C.shape[0]
        self.n, self.rec, self.ctl, self.log = n, rec, ctl, log
        self.p = np.asarray(p, dtype=np.int64)
        self.bound_x0 = bound_x0                     # start vectors of the γ / λ_n estimates
        rm, rp = ctl.r_main, ctl.r_pred
        self.rs_main = RecycledSpaceGen(n, ctl.p_main, rm, ctl.p_min_main, orth_S=True,
                                        implict_update=ctl.main_implict_update,
                                        implict_recycle=ctl.main_implict_recycle)
        self.keep_main = LobpcgSvdKeep(n, n, rm)
        self.keep_main.S[:, :rm] = X0_main
        self.sig_recy_main = self.keep_main.sigma[:rm]          # a view, as in :548
        self.ctl_main = LobpcgSvdControl(m=n, n=n, r=rm, conv_range=(1, 1), tol=float(ctl.lobpcg_tol_scale * ctl.tol),
                                         side="S", normC=ctl.main_normC)
        self.rs_pred = RecycledSpaceGen(n, ctl.p_pred, rp, ctl.p_min_pred, orth_S=False,
                                        implict_update=ctl.pred_implict_update,
                                        implict_recycle=ctl.pred_implict_recycle)
        self.keep_pred = LobpcgSvdKeep(n, n, rp)
        self.keep_pred.S[:, :rp] = X0_pred
        self.X0_pred_rebuild = X0_pred
        self.E_pred = np.zeros((n, rp), dtype=np.complex128)
        self.lam_recy_pred = self.keep_pred.lam[:rp]            # a view of keep_pred.λ, as in :591
        self.ctl_pred = LobpcgSvdControl(m=n, n=n, r=rp, tol=float(ctl.tol_pred * ctl.lobpcg_pred_tol_scale),
                                         side="S", orth_type=ctl.pred_orth_type,
                                         conv_range=ctl.pred_conv_range or (1, rp),
                                         conv_thresh_type=ctl.pred_conv_thresh_type)
        self.thresh = resolve_recycle_fail_dist_thresh(ctl.recycle_fail_dist_thresh, rec)
        nZ = len(rec.Z)
        self.sigma = np.full(nZ, np.nan)
        self.st = PsPrecRecyStats(nZ)
        self.M = SparseOp(self.C)
        self.S = Identity()
        self.lam_lower = 0.0
        self.lam_upper = 0.0
        self.last_failed_main = None
        self.last_failed_pred = None
        self.started = False

    # _get_pred_precond! (psPrecRecy.jl:436-462)
    def _precond(self, z):
        ctl, n = self.ctl, self.n
        L, invp, _ = self.ic(self.C, z, ctl.hsl_tol, ctl.hsl_cntl_1, ctl.hsl_cntl_2, ctl.hsl_icntl_1,
                             ctl.hsl_icntl_2, self.p)
        self.F = LowerFactor(L, self.p, invp)
        self.invF = InvF(self.F)
        x0 = self.bound_x0
        # _compute_λ_n (:405-422): lobpcgSvd r = 1, side 'L', on Cz·invF
        kl = LobpcgSvdKeep(n, n, 1)
        cl = LobpcgSvdControl(m=n, n=n, r=1, tol=ctl.lambda_n_tol, side="L", normC=1.0, conv_range=(1, 1))
        sig_n, _ = lobpcg_svd(Chain(SparseOp(self.C, -z), self.invF), None if x0 is None else x0.copy(), None, kl, cl)
        # _compute_γ (:388-402): lobpcgSvd r = 1, side 'L', on L⁻¹
        kg = LobpcgSvdKeep(n, n, 1)
        cg = LobpcgSvdControl(m=n, n=n, r=1, tol=ctl.gamma_tol, side="L", normC=1.0, conv_range=(1, 1))
        gamma, _ = lobpcg_svd(InvL(self.F), None if x0 is None else x0.copy(), None, kg, cg)
        return sig_n ** 2, gamma

    def _record_precond(self, z):
        st = self.st
        if st.n_precond_rebuild_pts > 0 and st.precond_rebuild_pts[st.n_precond_rebuild_pts - 1] == z:
            return
        st.precond_rebuild_pts[st.n_precond_rebuild_pts] = z
        st.n_precond_rebuild_pts += 1

    def _pred_refine(self, z, Cz_pred, M_pred, S_pred, conv_range, normC):
        ctl, rp = self.ctl, self.ctl.r_pred
        self.ctl_pred.normC = normC
        self.ctl_pred.tol = float(ctl.tol_pred * ctl.lobpcg_pred_tol_scale)
        self.ctl_pred.conv_range = conv_range
        X_pred = self.keep_pred.S[:, :rp]
        _, it = lobpcg_svd(Cz_pred, X_pred, None, self.keep_pred, self.ctl_pred)
        return it

    def _pred_update(self, z, M_pred, S_pred, idx_pred):
        ctl, rp = self.ctl, self.ctl.r_pred
        X_pred = self.keep_pred.S[:, :rp]
        force = self.last_failed_pred is not None and abs(z - self.last_failed_pred) <= self.thresh
        update_recycled_space(M_pred, S_pred, z, self.rs_pred, X_pred, tau=ctl.pred_tau, r_sub=idx_pred,
                              force_add=force)
        self.E_pred[:, :] = self.invF.mul(X_pred)

    def run(self, i_begin=0, i_end=None):
        ctl, rec, st = self.ctl, self.rec, self.st
        nZ = len(rec.Z)
        i_end = nZ if i_end is None else i_end
        rm, rp = ctl.r_main, ctl.r_pred
        if not self.started:
            self.z_dagger = complex(rec.Z[0])
            self.lam_dagger_n, self.gamma = self._precond(self.z_dagger)
            self._record_precond(self.z_dagger)
            self.started = True
        X_main = self.keep_main.S[:, :rm]
        W_main = self.keep_main.S[:, rm:2 * rm]
        X_pred = self.keep_pred.S[:, :rp]
        W_pred = self.keep_pred.S[:, rp:2 * rp]
        CX_pred = self.keep_pred.CS[:, :rp]
        for i in range(i_begin, i_end):
            z = complex(rec.Z[i])
            Cz = SparseOp(self.C, -z)
            st.p_count[i] = self.rs_main.p
            st.pred_p_count[i] = self.rs_pred.p
            main_recycled = False
            r_svdrr = 0
            if self.rs_main.p > 0:                                     # :679-714
                if ctl.main_implict_recycle:
                    r_svdrr = fast_svd_rayl_ritz_implicit(self.rs_main, z, X_main, W_main, self.sig_recy_main,
                                                          complex(ctl.shift), ctl.gap_tau)
                else:
                    raise NotImplementedError("main_implict_recycle = false (fastSvdRaylRitz_explicit!)")
                main_recycled = check_conv_svd(W_main, self.sig_recy_main, ctl.tol, "S", normC=ctl.main_normC,
                                               conv_range=(1, 1))
            st.r_recy[i] = r_svdrr
            if main_recycled:
                self.sigma[i] = self.sig_recy_main[0]
                st.main_M_vec_apps[i] = st.main_M_vec_apps_no_recycle[i] = st.main_L_vec_apps[i] = 0
                st.pred_M_vec_apps[i] = st.pred_L_vec_apps[i] = 0
                if self.log:
                    self.log(i, z, "recycled", None)
                continue
            # RecyProjSpace (:727-820)
            dz = abs(z - self.z_dagger)
            pred_normC = np.sqrt(self.lam_dagger_n) + self.gamma * dz
            M_pred = Chain(self.M, self.invF)
            S_pred = self.invF
            Cz_pred = Chain(Cz, self.invF)
            idx_pred = rp
            conv_pred = (1, rp)
            pred_recycled = False
            pred_refined = False
            if self.rs_pred.p > 0:
                fast_rayl_ritz(self.rs_pred, z, X_pred, self.E_pred, W_pred, self.lam_recy_pred)
                idx_pred = _pred_idx(self.lam_recy_pred, rp, ctl.idx_cutoff_pred)
                conv_pred = (1, idx_pred)
                pred_recycled = check_conv_svd(W_pred, None, ctl.tol_pred, "S", normC=pred_normC,
                                               conv_range=conv_pred, conv_thresh_type=1)
            pM = pL = 0
            upd = (3 * rp, 5 * rp) if ctl.pred_implict_recycle else (rp, rp)     # :82-105
            if pred_recycled:
                CX_pred[:, :] = Cz.mul(self.E_pred)                     # :770
                pM += rp
                self.lam_lower = self.lam_recy_pred[rp - 1]
            else:
                pred_refined = True
                it = self._pred_refine(z, Cz_pred, M_pred, S_pred, conv_pred, pred_normC)
                st.n_pred_it += it
                st.pred_refine_it[i] += it
                ops = 2 * (it + 1) * rp if it > 0 else 0                # :67-76
                pM += ops + upd[0]
                pL += ops + upd[1] + rp
                self._pred_update(z, M_pred, S_pred, idx_pred)
                self.lam_lower = self.keep_pred.lam[rp - 1]
            self.lam_upper = pred_normC ** 2
            if self.lam_lower < ctl.lambda_lower_min or self.lam_upper > ctl.lambda_upper_max:   # :825
                self._record_precond(z)
                self.lam_dagger_n, self.gamma = self._precond(z)
                M_pred = Chain(self.M, self.invF)
                S_pred = self.invF
                Cz_pred = Chain(Cz, self.invF)
                self.rs_pred.p = 0
                X_pred[:, :] = self.X0_pred_rebuild                     # rand!(X_pred) (:849)
                self.lam_upper = self.lam_dagger_n
                pred_refined = True
                it = self._pred_refine(z, Cz_pred, M_pred, S_pred, (1, rp), np.sqrt(self.lam_dagger_n))
                st.n_pred_it += it
                st.pred_refine_it[i] += it
                ops = 2 * (it + 1) * rp if it > 0 else 0
                pM += ops + upd[0]
                pL += ops + upd[1] + rp
                idx_pred = _pred_idx(self.lam_recy_pred, rp, ctl.idx_cutoff_pred)
                self._pred_update(z, M_pred, S_pred, idx_pred)
                self.lam_lower = self.keep_pred.lam[rp - 1]
                self.z_dagger = z
            st.pred_p_count[i] = self.rs_pred.p
            if pred_refined:
                st.pred_pts[st.n_pred_pts] = z
                st.n_pred_pts += 1
                self.last_failed_pred = z
            # two-level preconditioner (:910-921)
            GramE = CX_pred.conj().T @ CX_pred
            K_ad = LLTP_AD(self.F, self.E_pred, GramE)
            # main solve (:923-945)
            sig, it = lobpcg_svd(Cz, X_main, K_ad, self.keep_main, self.ctl_main)
            self.sigma[i] = sig
            st.main_refine_it[i] = it
            st.n_it += it
            st.pts[st.n_pts] = z
            st.n_pts += 1
            mM = mL = 0
            if it > 0:
                mM = 2 * (it + 1) * rm
                mL = 2 * it * rm
                force = self.last_failed_main is not None and abs(z - self.last_failed_main) <= self.thresh
                update_recycled_space(self.M, self.S, z, self.rs_main, X_main, tau=ctl.main_tau, force_add=force)
                mM += 3 * rm if ctl.main_implict_recycle else rm          # :58-64
            self.last_failed_main = z
            st.main_M_vec_apps[i] = st.main_M_vec_apps_no_recycle[i] = mM
            st.main_L_vec_apps[i] = mL
            st.pred_M_vec_apps[i] = pM
            st.pred_L_vec_apps[i] = pL
            if self.log:
                self.log(i, z, "refine", it)
        return self.sigma, st
