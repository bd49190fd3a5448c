"""Restatement of src/core/psTriRecy.jl (dense Schur-triangular path).

Test infrastructure only (see oracle/__init__.py).

``pre_process`` (psTriRecy.jl:6-14) reduces a square dense C to its complex
Schur factor T (C = Q T Qᴴ, LAPACK zgees through scipy); M = T and S = I.
Because the similarity is unitary, σ_min(C − zI) = σ_min(T − zI).
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field, fields

import numpy as np
import scipy.linalg as sla

from .linalg import EPS
from .lobpcg import LobpcgSvdControl, LobpcgSvdKeep, lobpcg_svd
from .recycle import (RecycledSpace, fast_svd_rayl_ritz_implicit, update_recycled_space,
                      resolve_recycle_fail_dist_thresh)


@dataclass
class PsTriRecyControl:
    """psTriRecy.jl:350-370.  ``shift`` defaults to normC²·eps·100 (:353)."""
    tol: float = 1e-3
    normC: float = 1.0
    shift: float = None
    gap_tau: float = 1e-10
    gap_tau_scale: float = 0.01
    recy_tau: float = 1.5
    recycle_fail_dist_thresh: float = float("nan")
    r: int = 6
    p: int = 50
    p_min: int = 1
    lobpcg_tol_scale: float = 0.1
    lobpcg_side: str = "L"
    implict_update: bool = False
    implict_recycle: bool = True
    collect_timing: bool = True
    inner_verbose_override: int = None

    def __post_init__(self):
        if self.shift is None:
            self.shift = self.normC ** 2 * EPS * 100


@dataclass
class PsTriRecyStats:
    """psTriRecy.jl:257-292."""
    p_count: np.ndarray
    r_recy: np.ndarray
    pts: np.ndarray
    M_vec_apps: np.ndarray
    M_vec_apps_no_recycle: np.ndarray
    R_vec_apps: np.ndarray
    preprocess_time_ns: int = 0
    recycle_time_ns: int = 0
    qr_time_ns: int = 0
    refine_time_ns: int = 0
    update_time_ns: int = 0
    mv_stats_available: bool = True
    n_it: int = 0
    n_pts: int = 0
    refine_it: np.ndarray = None

    @classmethod
    def alloc(cls, nZ):
        z = lambda: np.zeros(nZ, dtype=np.int64)
        return cls(z(), z(), np.zeros(nZ, dtype=np.complex128), z(), z(), z(), refine_it=z())


class TriOp:
    """Upper-triangular operator M = T (dense Schur factor)."""

    def __init__(self, T):
        self.T = T

    def mul(self, X):
        return self.T @ X

    def mul_adj(self, Y):
        return self.T.conj().T @ Y


class IdentityOp:
    """S = Diagonal(ones) (psTriRecy.jl:13)."""

    def mul(self, X):
        return X.copy()

    def mul_adj(self, Y):
        return Y.copy()


class InvAdjR:
    """InvMat(adjoint(Rz)) (psTriRecy.jl:797; RLSMatrices.jl:390-425).
    mul: R⁻ᴴ X (forward solve with Rᴴ); mul_adj: R⁻¹ Y (back solve with R)."""

    def __init__(self, R):
        self.R = R

    def mul(self, X):
        return sla.solve_triangular(self.R, X, lower=False, trans="C", check_finite=False)

    def mul_adj(self, Y):
        return sla.solve_triangular(self.R, Y, lower=False, trans="N", check_finite=False)


class SparseOp:
    """A sparse M (SciPy) as an operator: mul M·X, mul_adj Mᴴ·Y."""

    def __init__(self, A):
        self.A = A.tocsr()
        self.AH = A.conj().T.tocsr()

    def mul(self, X):
        return np.asarray(self.A @ X)

    def mul_adj(self, Y):
        return np.asarray(self.AH @ Y)


class ColPermOp:
    """S = I[:, p] (psTriRecy.jl:59-60): (S·X)[p[k]] = X[k], Sᴴ·Y = Y[p]."""

    def __init__(self, p):
        self.p = np.asarray(p)

    def mul(self, X):
        Y = np.zeros_like(X)
        Y[self.p] = X
        return Y

    def mul_adj(self, Y):
        return Y[self.p].copy()


class InvAdjLU:
    """(M − zS)⁻ᴴ through SuperLU (scipy splu), for sparse sizes where a dense QR is out of
    reach.  With M − zS = QR, R⁻ᴴ = Qᴴ·(M − zS)⁻ᴴ: the two operators differ by a unitary factor
    on the left, so LOBPCG side 'L' finds the same σ and right singular vectors with either
    (its Gram matrices and residuals see only CᴴC).  mul: (M − zS)⁻ᴴX, mul_adj: (M − zS)⁻¹Y."""

    def __init__(self, A):
        import scipy.sparse.linalg as spla
        self.lu = spla.splu(A.tocsc())

    def mul(self, X):
        return self.lu.solve(np.ascontiguousarray(X), trans="H")

    def mul_adj(self, Y):
        return self.lu.solve(np.ascontiguousarray(Y))


def pre_process_sparse(C, p):
    """psTriRecy.jl:47-61 (sparse branch) with the column order p given (the reference takes
    p = amd(lower(CᴴC))): M = C[:, p], S = I[:, p]."""
    import scipy.sparse as sp
    C = sp.csc_matrix(C, dtype=np.complex128)
    n = C.shape[0]
    M = C[:, p]
    S = sp.identity(n, dtype=np.complex128, format="csc")[:, p]
    return M, S


def pre_process_dense(C):
    """psTriRecy.jl:6-14 (square branch): complex Schur T of C."""
    T, _ = sla.schur(np.asarray(C, dtype=np.complex128), output="complex")
    return np.triu(T)


def _gap_tau(ctl, remaining):
    """psTriRecy.jl:373-378."""
    return ctl.gap_tau * ctl.gap_tau_scale if remaining > 0 else ctl.gap_tau


def residual_norm_ok(W, sigma, tol, normC):
    """_residual_norm_ok (psTriRecy.jl:237-245)."""
    return np.linalg.norm(W[:, 0]) < normC * max(sigma * tol, normC * np.sqrt(2) * EPS)


class PsTriRecyRun:
    """The loop of _psTriRecy_impl (psTriRecy.jl:708-881) on a precomputed Schur factor T,
    resumable over index ranges (state carried between calls as the reference's loop
    carries it between iterations).

    ``X0`` (n×r) replaces the reference's ``rand!(X)`` (psTriRecy.jl:607): the Julia
    RNG stream is not reproducible here, so the caller supplies it.
    """

    def __init__(self, T, rec, ctl: PsTriRecyControl, X0=None, seed=0, log=None, ritz_g1_always=False,
                 sparse=None, factor="qr"):
        n = T.shape[0] if sparse is None else sparse[0].shape[0]
        self.ritz_g1_always = ritz_g1_always
        r = ctl.r
        self.T, self.rec, self.ctl, self.log = T, rec, ctl, log
        if sparse is None:
            self.M, self.S = TriOp(T), IdentityOp()
        else:   # (M, S) of pre_process_sparse
            self.Msp, self.Ssp = sparse
            self.M, self.S = SparseOp(self.Msp), ColPermOp(self.Ssp.tocoo().row[np.argsort(self.Ssp.tocoo().col)])
        self.rs = RecycledSpace(n, n, ctl.p, r, p_min=ctl.p_min)
        self.keep = LobpcgSvdKeep(n, n, r)
        if X0 is None:
            rng = np.random.default_rng(seed)
            X0 = rng.random((n, r)) + 1j * rng.random((n, r))
        self.keep.S[:, :r] = X0
        self.sigma_recy = np.zeros(r)
        self.ctl_main = LobpcgSvdControl(m=n, n=n, r=r, conv_range=(1, 1),
                                         tol=float(ctl.lobpcg_tol_scale * ctl.tol),
                                         side=ctl.lobpcg_side, normC=ctl.normC)
        self.shift = complex(ctl.shift)
        self.thresh = resolve_recycle_fail_dist_thresh(ctl.recycle_fail_dist_thresh, rec)
        self.remaining = 0
        nZ = len(rec.Z)
        self.sigma_min = np.full(nZ, np.nan)
        self.st = PsTriRecyStats.alloc(nZ)
        self.last_failed = None
        self.factor = factor
        if sparse is None:
            self.Rz = T.copy()
            self.diagT = np.diag(T).copy()

    def refine_operator(self, z):
        """InvMat(adjoint(Rz)) (psTriRecy.jl:796-797); on the sparse branch with factor="lu"
        the equivalent (M − zS)⁻ᴴ by sparse LU."""
        if self.T is None and self.factor == "lu":
            return InvAdjLU(self.Msp - z * self.Ssp)
        return InvAdjR(self.shift_factor(z))

    def shift_factor(self, z):
        """get_R_factor!: T − zI on the dense Schur factor (psTriRecy.jl:87-99), or the R of
        qr(M − zS) (ordering = 0) on the sparse branch (psTriRecy.jl:222-234)."""
        if self.T is not None:
            np.fill_diagonal(self.Rz, self.diagT - z)
            return self.Rz
        A = (self.Msp - z * self.Ssp).toarray()
        return np.linalg.qr(A, mode="r")

    def run(self, i_begin=0, i_end=None):
        rec, ctl, rs, keep, st = self.rec, self.ctl, self.rs, self.keep, self.st
        r = ctl.r
        nZ = len(rec.Z)
        i_end = nZ if i_end is None else i_end
        X = keep.S[:, :r]
        W = keep.S[:, r:2 * r]
        for i in range(i_begin, i_end):
            z = complex(rec.Z[i])
            st.p_count[i] = rs.p
            r_svdrr = 0
            m_apps = 0
            r_apps = 0
            if rs.p > 0:
                t0 = time.perf_counter_ns()
                r_svdrr = fast_svd_rayl_ritz_implicit(rs, z, X, W, self.sigma_recy, self.shift,
                                                      _gap_tau(ctl, self.remaining), self.ritz_g1_always)
                self.remaining = self.remaining - 1 if self.remaining > 0 else 0
                st.recycle_time_ns += time.perf_counter_ns() - t0
                st.r_recy[i] = r_svdrr
                if residual_norm_ok(W, self.sigma_recy[0], ctl.tol, ctl.normC):
                    self.sigma_min[i] = self.sigma_recy[0]
                    if self.log is not None:
                        self.log(i, z, "recycled", rs.p, r_svdrr, self.sigma_min[i], 0)
                    continue
            t0 = time.perf_counter_ns()
            _, it = lobpcg_svd(self.refine_operator(z), X, None, keep, self.ctl_main)
            self.sigma_min[i] = keep.sigma[0]
            st.refine_it[i] = it
            if it > 0:
                r_apps += 2 * r + it * r + (it - 1) * r
            st.refine_time_ns += time.perf_counter_ns() - t0
            st.n_it += it
            st.pts[st.n_pts] = z
            st.n_pts += 1
            if i < nZ - 1 and it > 0:
                t0 = time.perf_counter_ns()
                force_add = self.last_failed is not None and abs(z - self.last_failed) <= self.thresh
                update_recycled_space(self.M, self.S, z, rs, keep.S[:, :r], tau=ctl.recy_tau, r_sub=1,
                                      force_add=force_add)
                self.remaining = max(rec.k, 0) if force_add else 0
                m_apps += 3 * r if ctl.implict_recycle else r
                st.update_time_ns += time.perf_counter_ns() - t0
            self.last_failed = z
            st.M_vec_apps[i] = m_apps
            st.M_vec_apps_no_recycle[i] = m_apps
            st.R_vec_apps[i] = r_apps
            if self.log is not None:
                self.log(i, z, "refine", rs.p, r_svdrr, self.sigma_min[i], it)
        return self.sigma_min, st


def ps_tri_recy_schur(T, rec, ctl: PsTriRecyControl, X0=None, seed=0, log=None, ritz_g1_always=False):
    """_psTriRecy_impl (psTriRecy.jl:708-881) on a precomputed Schur factor T.
    Returns (σ_min, stats)."""
    return PsTriRecyRun(T, rec, ctl, X0=X0, seed=seed, log=log, ritz_g1_always=ritz_g1_always).run()


def ps_tri_recy_sparse(C, p, rec, ctl: PsTriRecyControl, X0=None, seed=0, log=None, ritz_g1_always=False,
                       factor="qr"):
    """_psTriRecy_impl on the sparse branch (M = C[:, p], S = I[:, p]).  The shifted factor is
    the dense QR's R (factor="qr", small n) or the equivalent sparse LU operator (factor="lu").
    Returns (σ_min, stats)."""
    return PsTriRecyRun(None, rec, ctl, X0=X0, seed=seed, log=log, ritz_g1_always=ritz_g1_always,
                        sparse=pre_process_sparse(C, p), factor=factor).run()


def dense_sigma_min(C, z):
    """Independent FP64 oracle: smallest singular value of C − zI by dense SVD."""
    A = np.asarray(C, dtype=np.complex128).copy()
    A[np.diag_indices_from(A)] -= z
    return sla.svdvals(A)[-1]
