"""Restatement of src/core/lobpcgSvd.jl (block LOBPCG for extreme singular values).

Test infrastructure only (see oracle/__init__.py).  ``C`` is any object with
``mul(X) -> C X`` and ``mul_adj(Y) -> Cᴴ Y``; ``K`` is ``None`` for the identity
preconditioner (``ldiv!(IdentityMat, ·)`` is a no-op).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .linalg import EPS, qr_inplace, qr_typed, svd_inplace, lq_rows_inplace, orth_inplace, orth_typed


@dataclass
class LobpcgSvdControl:
    """lobpcgSvd.jl:1-55."""
    m: int
    n: int
    r: int
    maxit: int = 2000
    tol: float = 1e-3
    side: str = "S"
    verbose: int = 0
    normC: float = 1.0
    orth_type: str = "lapack"
    conv_range: tuple = None      # 1-based inclusive (first, last); None → (1, r)
    conv_thresh_type: int = 0

    def __post_init__(self):
        if self.conv_range is None:
            self.conv_range = (1, self.r)
        a, b = self.conv_range
        if not (1 <= a <= b <= self.r):
            raise ValueError(f"conv_range={self.conv_range} must satisfy 1 <= first <= last <= r={self.r}")
        if self.orth_type not in ("lapack", "shiftchol"):
            raise ValueError("orth_type must be lapack or shiftchol")
        if self.conv_thresh_type not in (0, 1):
            raise ValueError("conv_thresh_type must be 0 or 1")


class LobpcgSvdKeep:
    """lobpcgSvd.jl:57-80."""

    def __init__(self, m, n, r):
        c = np.complex128
        self.S = np.zeros((n, 3 * r), dtype=c)
        self.CS = np.zeros((m, 3 * r), dtype=c)
        self.G = np.zeros((3 * r, 3 * r), dtype=c)
        self.R = np.zeros((3 * r, 3 * r), dtype=c)
        self.sigma = np.zeros(3 * r)
        self.lam = np.zeros(3 * r)


def svd_rayl_ritz(CS, R_view, G_view, sigma, lam, r, side, orth_type="lapack"):
    """svdRaylRitz! (lobpcgSvd.jl:126-184)."""
    nS = CS.shape[1]
    qr_typed(CS, R_view, orth_type)
    R_work = R_view[:nS, :nS].copy()
    svd_inplace(R_work, sigma, G_view, ascending=(side != "L"))
    if side == "L":
        sigma[:r] = 1.0 / sigma[:r]
        lam[:r] = sigma[:r] ** 2
    else:
        lam[:r] = sigma[:r] ** 2
    if nS > r:
        G_rest = G_view[:, r:nS]
        Q_mat = G_view[:r, r:nS].copy()
        lq_rows_inplace(Q_mat)
        G_view[:, r:2 * r] = G_rest @ Q_mat.conj().T


def basis_update(V, CV, S, CS, R_view, G_view):
    """basisUpdate! (lobpcgSvd.jl:195-220): V ← S G, CV ← CS (R G)."""
    temp_V = S @ G_view
    temp_RG = R_view @ G_view
    temp_CV = CS @ temp_RG
    V[:, :] = temp_V
    CV[:, :] = temp_CV


def residual(C, V, CV, W, lam, side):
    """residual! (lobpcgSvd.jl:227-248)."""
    W[:, :] = C.mul_adj(CV)
    if side == "S":
        W -= V * lam[None, :]
    elif side == "L":
        W[:, :] = W * lam[None, :] - V


def conv_thresh(sigma, normC, tol, typ):
    """lobpcgSvd.jl:295-310."""
    if typ == 0:
        return max(normC * sigma * tol, normC ** 2 * np.sqrt(2) * EPS)
    if typ == 1:
        return max(normC ** 2 * tol, normC ** 2 * np.sqrt(2) * EPS)
    raise ValueError(f"unsupported conv thresh type: {typ}")


def check_conv_svd(W, sigma, tol, side, normC=1.0, conv_range=None, conv_thresh_type=0):
    """check_conv_svd (lobpcgSvd.jl:317-357)."""
    if side != "S":
        return np.linalg.norm(W[:, 0]) < tol
    a, b = conv_range if conv_range is not None else (1, W.shape[1])
    if conv_thresh_type == 0:
        for j in range(a - 1, b):
            if np.linalg.norm(W[:, j]) >= conv_thresh(sigma[j], normC, tol, 0):
                return False
    else:
        th = conv_thresh(0.0, normC, tol, 1)
        for j in range(a - 1, b):
            if np.linalg.norm(W[:, j]) >= th:
                return False
    return True


def lobpcg_svd(C, X0, K, keep: LobpcgSvdKeep, ctl: LobpcgSvdControl, rng=None):
    """lobpcgSvd (lobpcgSvd.jl:365-477).  Returns (σ, it)."""
    r, side = ctl.r, ctl.side
    S, CS, G, R, sigma, lam = keep.S, keep.CS, keep.G, keep.R, keep.sigma, keep.lam
    X, P, W = S[:, :r], S[:, r:2 * r], S[:, 2 * r:3 * r]
    XP = S[:, :2 * r]
    CX, CP, CW = CS[:, :r], CS[:, r:2 * r], CS[:, 2 * r:3 * r]
    CXP = CS[:, :2 * r]
    lam_r = lam[:r]
    R_r, G_r_r = R[:r, :r], G[:r, :r]
    R_2r, G_2r_2r = R[:2 * r, :2 * r], G[:2 * r, :2 * r]
    R_3r, G_3r_2r, G_3r_3r = R[:3 * r, :3 * r], G[:3 * r, :2 * r], G[:3 * r, :3 * r]

    def ldiv(B):
        if K is not None:
            B[:, :] = K.ldiv(B)

    if X0 is not None:
        if X0 is not X:
            X[:, :] = X0
    else:
        rng = rng or np.random.default_rng()
        X[:, :] = rng.random(X.shape) + 1j * rng.random(X.shape)
    ot = ctl.orth_type
    qr_typed(X, None, ot)
    CX[:, :] = C.mul(X)
    svd_rayl_ritz(CX, R_r, G_r_r, sigma, lam, r, side, ot)
    basis_update(X, CX, X, CX, R_r, G_r_r)
    residual(C, X, CX, P, lam_r, side)
    check_conv_svd(P, sigma, ctl.tol, side, ctl.normC, ctl.conv_range, ctl.conv_thresh_type)
    ldiv(P)
    orth_typed(X, P, typ=ot)
    CP[:, :] = C.mul(P)
    for i in range(1, ctl.maxit + 1):
        if i == 1:
            svd_rayl_ritz(CXP, R_2r, G_2r_2r, sigma, lam, r, side, ot)
            basis_update(XP, CXP, XP, CXP, R_2r, G_2r_2r)
        else:
            svd_rayl_ritz(CS, R_3r, G_3r_3r, sigma, lam, r, side, ot)
            basis_update(XP, CXP, S, CS, R_3r, G_3r_2r)
        residual(C, X, CX, W, lam_r, side)
        if check_conv_svd(W, sigma, ctl.tol, side, ctl.normC, ctl.conv_range, ctl.conv_thresh_type):
            return (sigma[0] if side == "S" else 1.0 / sigma[0]), i
        ldiv(W)
        orth_typed(XP, W, typ=ot)
        CW[:, :] = C.mul(W)
    return (sigma[0] if side == "S" else 1.0 / sigma[0]), ctl.maxit
