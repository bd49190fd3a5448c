"""Restatement of src/core/recySpace.jl in full generality and of fastRaylRitz! — test
infrastructure only (see oracle/__init__.py).

oracle/recycle.py restates the psTriRecy configuration (orth_S = true, implict_update =
false); this module covers every flag of RecycledSpace (recySpace.jl:40-120), as psPrecRecy
uses it: the main stage with orth_S = true and the prediction stage with orth_S = false and
implict_update = true (psPrecRecy.jl:489-608).  M and S are operators with mul / mul_adj
(square here: m = n, sn = m).  Indices in comments are the reference's 1-based ones.
"""
from __future__ import annotations

import numpy as np

from .linalg import (qr_inplace, orth_robust_inplace, block_unitary_rot, block_rot_lmul, block_rot_rmul_adj,
                     eigh_index_range)
from .recycle import affine_combine


class RecycledSpaceGen:
    """RecycledSpace (recySpace.jl:40-120) for square operators (m = n = sn)."""

    def __init__(self, n, p_max, r, p_min=1, orth_S=False, implict_update=False, implict_recycle=True):
        if p_max <= 0:
            raise ValueError(f"p_max must be positive, got {p_max}")
        if not (0 <= p_min <= p_max):
            raise ValueError("p_min must satisfy 0 <= p_min <= p_max")
        pr = p_max * r
        c = np.complex128
        self.orth_S, self.implict_update, self.implict_recycle = orth_S, implict_update, implict_recycle
        self.p_max, self.p_min, self.p, self.n, self.r = p_max, p_min, 0, n, r
        self.pts = np.zeros(p_max, dtype=c)
        self.V = np.zeros((n, pr), dtype=c)
        self.L = np.zeros((pr, pr), dtype=c)
        self.H1 = np.zeros((pr, pr), dtype=c)
        self.H2 = np.zeros((pr, pr), dtype=c)
        self.H3 = np.zeros((pr, pr), dtype=c)
        shape = (n, pr) if implict_recycle else (0, 0)
        self.J1 = np.zeros(shape, dtype=c)
        self.J2 = np.zeros(shape, dtype=c)
        self.J3 = np.zeros(shape, dtype=c)
        self._J4 = np.zeros(shape if not orth_S else (0, 0), dtype=c)
        self.J5 = np.zeros((n, pr), dtype=c)
        self.J6 = np.zeros((n, pr), dtype=c)

    @property
    def J4(self):
        return self.V if self.orth_S else self._J4   # recySpace.jl:90-91


def update_recycled_space(M, S, z, rs: RecycledSpaceGen, X, tau=1.5, r_sub=1, force_add=False):
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
                if np.linalg.norm(R) / res0 > tau:
                    l = i - 1
                    break
        if l > 0:
            shift_blocks(rs, l)
        if l == 0 and p == rs.p_max:
            shift_blocks(rs, 1)
    add_blocks(rs, X, M, S, z)
    block_unitary_update(rs, S)


def shift_blocks(rs: RecycledSpaceGen, l: int):
    """_shift_blocks! (recySpace.jl:290-340)."""
    p, r = rs.p, rs.r
    src = slice(l * r, p * r)
    nk = (p - l) * r
    rs.pts[:p - l] = rs.pts[l:p].copy()
    tall = [rs.V, rs.J5, rs.J6]
    if rs.implict_recycle:
        tall += [rs.J1, rs.J2, rs.J3] + ([] if rs.orth_S else [rs._J4])
    for A in tall:
        A[:, :nk] = A[:, src].copy()
    sq = [rs.L, rs.H1, rs.H2] + ([] if rs.orth_S else [rs.H3])
    for A in sq:
        A[:nk, :nk] = A[src, src].copy()
    rs.p = p - l


def add_blocks(rs: RecycledSpaceGen, X, M, S, z):
    """_add_blocks! (recySpace.jl:344-453)."""
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
    J5n = M.mul(V_new)                            # mul_coupled_ms! (RLSPreconditioner.jl:38-76)
    J6n = S.mul(V_new)
    rs.J5[:, new] = J5n
    rs.J6[:, new] = J6n
    H3nn = np.eye(r, dtype=np.complex128)
    if rs.implict_recycle:
        J1n = M.mul_adj(J5n)                      # :377
        J2n = M.mul_adj(J6n)                      # :380 (sn == m)
        J3n = S.mul_adj(J5n)                      # :385
        rs.J1[:, new], rs.J2[:, new], rs.J3[:, new] = J1n, J2n, J3n
        if not rs.orth_S:
            J4n = S.mul_adj(J6n)                  # :388
            rs._J4[:, new] = J4n
            H3nn = V_new.conj().T @ J4n           # :399
        rs.H1[new, new] = V_new.conj().T @ J1n    # :392-393
        rs.H2[new, new] = V_new.conj().T @ J2n
        rs.H3[new, new] = H3nn
        if p > 0:                                 # :404-417
            rs.H1[old, new] = rs.J1[:, old].conj().T @ V_new
            rs.H2[old, new] = rs.J3[:, old].conj().T @ V_new
            rs.H1[new, old] = rs.H1[old, new].conj().T
            rs.H2[new, old] = V_new.conj().T @ rs.J2[:, old]
            if rs.orth_S:
                rs.H3[old, new] = 0
                rs.H3[new, old] = 0
            else:
                rs.H3[old, new] = rs.J4[:, old].conj().T @ V_new
                rs.H3[new, old] = rs.H3[old, new].conj().T
    else:                                         # light cache (:420-450)
        rs.H1[new, new] = J5n.conj().T @ J5n
        rs.H2[new, new] = J5n.conj().T @ J6n
        rs.H3[new, new] = H3nn if rs.orth_S else J6n.conj().T @ J6n
        if p > 0:
            rs.H1[old, new] = rs.J5[:, old].conj().T @ J5n
            rs.H1[new, old] = rs.H1[old, new].conj().T
            rs.H2[old, new] = rs.J5[:, old].conj().T @ J6n
            rs.H2[new, old] = J5n.conj().T @ rs.J6[:, old]
            if rs.orth_S:
                rs.H3[old, new] = 0
                rs.H3[new, old] = 0
            else:
                rs.H3[old, new] = rs.J6[:, old].conj().T @ J6n
                rs.H3[new, old] = rs.H3[old, new].conj().T
    rs.pts[p] = z
    rs.p = p + 1


def block_unitary_update(rs: RecycledSpaceGen, S):
    """_block_unitary_update! (recySpace.jl:226-286)."""
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
        for A in (rs.V, rs.J5, rs.J6):
            block_rot_rmul_adj(A[:, :pr], U, i1, i2, r)
        if rs.implict_recycle:
            for A in (rs.J1, rs.J2):
                block_rot_rmul_adj(A[:, :pr], U, i1, i2, r)
            if rs.implict_update:
                block_rot_rmul_adj(rs.J3[:, :pr], U, i1, i2, r)
                if not rs.orth_S:
                    block_rot_rmul_adj(rs._J4[:, :pr], U, i1, i2, r)
            else:
                for ib in (i1, i2):               # :257-266
                    cols = slice((ib - 1) * r, ib * r)
                    rs.J3[:, cols] = S.mul_adj(rs.J5[:, cols])
                    if not rs.orth_S:
                        rs._J4[:, cols] = S.mul_adj(rs.J6[:, cols])
        Hs = (rs.H1, rs.H2) + (() if rs.orth_S else (rs.H3,))
        for H in Hs:
            block_rot_rmul_adj(H[:pr, :pr], U, i1, i2, r)
            block_rot_lmul(U, H[:pr, :pr], i1, i2, r)


def fast_rayl_ritz(rs: RecycledSpaceGen, z, X_recy, E_recy, W_recy, lam_recy):
    """fastRaylRitz! (fastRaylRitz.jl:382-427): Rayleigh–Ritz on the cached normal-equation
    projection; eigenpairs 1..min(2r, pr) of Hz, the first r used."""
    if not rs.implict_recycle:
        raise ValueError("fastRaylRitz! requires recySp.implict_recycle=true")
    p, r = rs.p, rs.r
    pr = p * r
    if pr == 0:
        return
    H1, H2, H3 = rs.H1[:pr, :pr], rs.H2[:pr, :pr], rs.H3[:pr, :pr]
    Hz = affine_combine(z, H1, H2, H2.conj().T, H3)
    iu = min(2 * r, pr)
    lam, G = eigh_index_range(Hz, 1, iu)
    lam_recy[:r] = lam[:r]
    G_ = G[:, :r]
    X_recy[:, :] = rs.V[:, :pr] @ G_
    E_recy[:, :] = rs.J6[:, :pr] @ G_
    work = affine_combine(z, rs.J1[:, :pr], rs.J2[:, :pr], rs.J3[:, :pr], rs.J4[:, :pr])
    W_recy[:, :] = work @ G_ - X_recy * lam_recy[:r][None, :]
