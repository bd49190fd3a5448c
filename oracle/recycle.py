"""Restatement of src/core/recySpace.jl and src/core/fastRaylRitz.jl.

Test infrastructure only (see oracle/__init__.py).  Indices in comments are
the reference's 1-based ones; the code is 0-based.
"""
from __future__ import annotations

import numpy as np

from .linalg import (EPS, qr_inplace, svd_inplace, eigh_index_range, orth_robust_inplace,
                     block_unitary_rot, block_rot_lmul, block_rot_rmul_adj)


def default_recycle_fail_dist_thresh(rec) -> float:
    """recySpace.jl:22-26."""
    dx = abs(rec.x_ed - rec.x_st) / (rec.n_x - 1) if rec.n_x > 1 else 0.0
    dy = abs(rec.y_ed - rec.y_st) / (rec.n_y - 1) if rec.n_y > 1 else 0.0
    return 1.01 * max(dx, dy)


def resolve_recycle_fail_dist_thresh(thresh: float, rec) -> float:
    """recySpace.jl:29-38."""
    if np.isfinite(thresh):
        if thresh < 0:
            raise ValueError(f"recycle_fail_dist_thresh must be nonnegative, got {thresh}")
        return float(thresh)
    return default_recycle_fail_dist_thresh(rec)


class RecycledSpace:
    """recySpace.jl:40-120, specialised to orth_S=true, implict_update=false,
    implict_recycle=true (the psTriRecy configuration, psTriRecy.jl:591-602).

    With S'S = I the reference aliases J4 to V (recySpace.jl:90-91) and fixes
    H3 = I on the active blocks (recySpace.jl:394-398, :410-412).
    """

    def __init__(self, m, n, p_max, r, p_min=1):
        if p_max <= 0:
            raise ValueError(f"p_max must be positive, got {p_max}")
        if not (0 <= p_min <= p_max):
            raise ValueError("p_min must satisfy 0 <= p_min <= p_max")
        pr = p_max * r
        self.p_max, self.p_min, self.p, self.m, self.n, self.r = p_max, p_min, 0, m, n, r
        self.sn = m
        c = np.complex128
        self.pts = np.zeros(p_max, dtype=c)
        self.V = np.zeros((n, pr), dtype=c)
        self.L = np.zeros((pr, pr), dtype=c)
        self.H1 = np.zeros((pr, pr), dtype=c)
        self.H2 = np.zeros((pr, pr), dtype=c)
        self.H3 = np.zeros((pr, pr), dtype=c)
        self.J1 = np.zeros((n, pr), dtype=c)
        self.J2 = np.zeros((n, pr), dtype=c)
        self.J3 = np.zeros((n, pr), dtype=c)
        self.J5 = np.zeros((m, pr), dtype=c)
        self.J6 = np.zeros((m, pr), dtype=c)

    @property
    def J4(self):
        return self.V  # orth_S: J4 shares storage with V (recySpace.jl:91)


def update_recycled_space(M, S, z, rs: RecycledSpace, X, tau=1.5, r_sub=1, force_add=False):
    """updateRecycledSpace! (recySpace.jl:160-223)."""
    p, r = rs.p, rs.r
    if p > 0:
        V0 = rs.V[:, :p * r]
        X_sub = X[:, :r_sub]
        R = np.zeros((r_sub, r_sub), dtype=np.complex128)
        X_temp = X_sub.copy()
        orth_robust_inplace(V0, X_temp, None, R)
        res0 = np.linalg.norm(R)
        l = 0
        if not force_add:
            l_max = min(p - 1, p + 1 - rs.p_min)
            l = l_max
            for i in range(1, l_max + 2):
                Vl = rs.V[:, i * r:p * r]
                X_temp = X_sub.copy()
                orth_robust_inplace(Vl, X_temp, None, R)
                resl = np.linalg.norm(R)
                if resl / res0 > tau:
                    l = i - 1
                    break
        if l > 0:
            shift_blocks(rs, l)
        if l == 0 and p == rs.p_max:
            shift_blocks(rs, 1)
    add_blocks(rs, X, M, S, z)
    block_unitary_update(rs, S)


def shift_blocks(rs: RecycledSpace, l: int):
    """_shift_blocks! (recySpace.jl:290-340): drop the first l blocks."""
    p, r = rs.p, rs.r
    src = slice(l * r, p * r)
    nk = (p - l) * r
    rs.pts[:p - l] = rs.pts[l:p].copy()
    for A in (rs.V, rs.J1, rs.J2, rs.J3, rs.J5, rs.J6):
        A[:, :nk] = A[:, src].copy()
    for A in (rs.L, rs.H1, rs.H2):
        A[:nk, :nk] = A[src, src].copy()
    rs.p = p - l


def add_blocks(rs: RecycledSpace, X, M, S, z):
    """_add_blocks! (recySpace.jl:344-453), implicit-recycle branch with orth_S."""
    p, r = rs.p, rs.r
    old = slice(0, p * r)
    new = slice(p * r, (p + 1) * r)
    V_new = X.copy()
    Lnn = np.zeros((r, r), dtype=np.complex128)
    if p > 0:
        Lon = np.zeros((p * r, r), dtype=np.complex128)
        orth_robust_inplace(rs.V[:, old], V_new, Lon, Lnn)
        rs.L[old, new] = Lon
    else:
        qr_inplace(V_new, Lnn)
    rs.L[new, new] = Lnn
    rs.V[:, new] = V_new
    J5n = M.mul(V_new)                       # mul_coupled_ms! (RLSPreconditioner.jl:38-48)
    J6n = S.mul(V_new)
    rs.J5[:, new] = J5n
    rs.J6[:, new] = J6n
    J1n = M.mul_adj(J5n)                     # recySpace.jl:377
    J2n = M.mul_adj(J6n)                     # recySpace.jl:380
    J3n = S.mul_adj(J5n)                     # recySpace.jl:385
    rs.J1[:, new] = J1n
    rs.J2[:, new] = J2n
    rs.J3[:, new] = J3n
    rs.H1[new, new] = V_new.conj().T @ J1n   # recySpace.jl:392-398
    rs.H2[new, new] = V_new.conj().T @ J2n
    rs.H3[new, new] = np.eye(r)
    if p > 0:                                # recySpace.jl:404-417
        rs.H1[old, new] = rs.J1[:, old].conj().T @ V_new
        rs.H2[old, new] = rs.J3[:, old].conj().T @ V_new
        rs.H1[new, old] = rs.H1[old, new].conj().T
        rs.H2[new, old] = V_new.conj().T @ rs.J2[:, old]
        rs.H3[old, new] = 0
        rs.H3[new, old] = 0
    rs.pts[p] = z
    rs.p = p + 1


def block_unitary_update(rs: RecycledSpace, S):
    """_block_unitary_update! (recySpace.jl:226-286), implict_update=false, orth_S=true."""
    p, r = rs.p, rs.r
    if p <= 1:
        return
    pr = p * r
    for i in range(1, p):
        ri = rs.L[(i - 1) * r:i * r, (p - 1) * r:p * r]
        rend = rs.L[(p - 1) * r:p * r, (p - 1) * r:p * r]
        U = block_unitary_rot(rend.copy(), ri.copy())
        i1, i2 = p, i
        block_rot_lmul(U, rs.L[:pr, :pr], i1, i2, r)
        for A in (rs.V, rs.J5, rs.J6, rs.J1, rs.J2):
            block_rot_rmul_adj(A[:, :pr], U, i1, i2, r)
        for ib in (i1, i2):                 # recySpace.jl:259-264: J3 = S'J5 on both blocks
            cols = slice((ib - 1) * r, ib * r)
            rs.J3[:, cols] = S.mul_adj(rs.J5[:, cols])
        for H in (rs.H1, rs.H2):            # recySpace.jl:272-275
            block_rot_rmul_adj(H[:pr, :pr], U, i1, i2, r)
            block_rot_lmul(U, H[:pr, :pr], i1, i2, r)


# ----------------------------------------------------------------------------------------
# fastRaylRitz.jl
# ----------------------------------------------------------------------------------------

def affine_combine(z, A1, A2, A3, A4, shift=0.0):
    """affine_conbine! (fastRaylRitz.jl:6-28): A1 − zA2 − z̄A3 + (|z|²+shift)A4."""
    zz = abs(z) ** 2 + shift
    return A1 - z * A2 - np.conj(z) * A3 + zz * A4


def check_rr_dim(lam, gap) -> int:
    """fastRaylRitz.jl:35-47 (returns a 1-based index, 0 if no gap)."""
    for i in range(len(lam) - 1):
        if abs(lam[i] - lam[i + 1]) > gap:
            return i + 1
    return 0


def find_rr_dim(Hz, r, tau, n_init=None, n_max=-1):
    """find_rr_dim! (fastRaylRitz.jl:54-96).  Returns (r_, G) with G holding the
    eigenvectors of the last solve in its leading columns.

    Difference, stated: when no gap is found and the last solve covered fewer
    than n_H columns, the reference reads the trailing columns of G from an
    uninitialised scratch buffer; here those columns come from a full solve.
    """
    n_H = Hz.shape[0]
    if n_init is None:
        n_init = 2 * r
    n_init = min(n_init, n_H)
    n_max = min(n_max, n_H) if n_max > 0 else n_H
    G = np.zeros((n_H, n_H), dtype=np.complex128)
    lam_max, g = eigh_index_range(Hz, n_H, n_H)
    G[:, :1] = g
    gap = lam_max[0] / tau * EPS
    n = n_init
    r_ = 0
    last_n = 0
    while n <= n_max:
        lam, g = eigh_index_range(Hz, 1, n)
        G[:, :n] = g
        last_n = n
        r_ = check_rr_dim(lam[:n], gap)
        if r_ > 0:
            break
        n = n + 2 * r
    if r_ > 0:
        return max(r_, r), G
    if last_n < n_max:
        _, g = eigh_index_range(Hz, 1, n_max)
        G[:, :n_max] = g
    return n_max, G


def fast_svd_rayl_ritz_implicit(rs: RecycledSpace, z, X_recy, W_recy, sigma_recy, shift, tau, ritz_g1_always=False):
    """_fastSvdRaylRitz_impl! implicit branch (fastRaylRitz.jl:99-219).

    ``ritz_g1_always`` (not in the reference) forms G_total = G1·G2 also when
    r_ == pr, where the reference takes G2 alone (fastRaylRitz.jl:199-202).
    """
    p, r = rs.p, rs.r
    pr = p * r
    if pr == 0:
        return 0
    H1, H2, H3 = rs.H1[:pr, :pr], rs.H2[:pr, :pr], rs.H3[:pr, :pr]
    Hz = affine_combine(z, H1, H2, H2.conj().T, H3, shift=shift)
    r_, G = find_rr_dim(Hz, r, tau)
    G1 = G[:, :r_]
    CzX = rs.J5[:, :pr] - z * rs.J6[:, :pr]
    CzX_ = CzX @ G1
    R_ = np.zeros((r_, r_), dtype=np.complex128)
    qr_inplace(CzX_, R_)
    sig = np.zeros(r_)
    G_ = np.zeros((r_, r_), dtype=np.complex128)
    svd_inplace(R_.copy(), sig, G_, ascending=True)
    G2 = G_[:, :r]
    sigma_recy[:r] = sig[:r]
    if r_ < pr or ritz_g1_always:
        G_total = G1 @ G2
    else:
        G_total = G2.copy()   # fastRaylRitz.jl:199-202 uses G2 alone when r_ == pr
    work = affine_combine(z, rs.J1[:, :pr], rs.J2[:, :pr], rs.J3[:, :pr], rs.J4[:, :pr])
    X_recy[:, :] = rs.V[:, :pr] @ G_total
    W_recy[:, :] = work @ G_total - X_recy * (sigma_recy[:r] ** 2)[None, :]
    return r_
