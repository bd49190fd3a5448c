"""Restatement of the small dense kernels of src/types/RLSLinearAlgebra.jl.

Test infrastructure only (see oracle/__init__.py).  Each wrapper reaches the
same LAPACK routine the reference ``ccall``s, through ``scipy.linalg.lapack``.
Arrays are complex128 and column semantics follow Julia (``X[:, j]`` is
column j).
"""
from __future__ import annotations

import numpy as np
import scipy.linalg.lapack as lapack

EPS = np.finfo(np.float64).eps


def qr_inplace(V: np.ndarray, R: np.ndarray | None = None, full_Q: bool = False):
    """rls_qr! (RLSLinearAlgebra.jl:476-606): V ← thin Q (m×n), R ← upper R.

    With ``full_Q`` the m×m unitary Q is returned (rls_qr!(V, Q, nothing),
    used by rls_block_unitary_rot!, RLSLinearAlgebra.jl:164-190).
    """
    m, n = V.shape
    assert m >= n, "QR factorization requires m >= n"
    qr, tau, _, info = lapack.zgeqrf(np.asfortranarray(V))
    assert info == 0
    if R is not None:
        R[:n, :n] = np.triu(qr[:n, :n])
    if full_Q:
        a = np.zeros((m, m), dtype=np.complex128, order="F")
        a[:, :n] = qr
        q, _, info = lapack.zungqr(a, tau)
        assert info == 0
        V[:, :] = q[:, :n]
        return q
    q, _, info = lapack.zungqr(qr, tau)
    assert info == 0
    V[:, :] = q
    return None


def lq_rows_inplace(V: np.ndarray):
    """rls_lq!(V) (RLSLinearAlgebra.jl:1007-1123): V (m×n, m<=n) ← first m rows of Q.

    zgelqf on V is the conjugate transpose of zgeqrf on Vᴴ (LAPACK's zgelq2
    conjugates each row before generating its reflector), so the rows of the
    LQ factor Q are the conjugated columns of the QR factor of Vᴴ.
    """
    m, n = V.shape
    assert m <= n
    Vh = np.ascontiguousarray(V.conj().T)
    qr_inplace(Vh)
    V[:, :] = Vh.conj().T


def svd_inplace(A: np.ndarray, S: np.ndarray, Vout: np.ndarray, ascending: bool):
    """rls_svd!(A, S, Vt; return_V=true, ascending) (RLSLinearAlgebra.jl:255-446).

    zgesdd job 'S'; Vt is converted to V in place; with ``ascending`` the
    singular values and the columns of V are reversed.
    """
    m, n = A.shape
    minmn = min(m, n)
    u, s, vt, info = lapack.zgesdd(np.asfortranarray(A), compute_uv=1, full_matrices=0)
    assert info == 0, f"zgesdd info={info}"
    V = vt[:minmn, :minmn].conj().T
    if ascending:
        s = s[::-1]
        V = V[:, ::-1]
    S[:minmn] = s
    Vout[:minmn, :minmn] = V
    return minmn


def eigh_index_range(A: np.ndarray, il: int, iu: int):
    """rls_eigen!(A, λ, Z; range='I', il, iu) via zheevr, uplo 'U' (RLSLinearAlgebra.jl:903-982).

    ``il``/``iu`` are 1-based like LAPACK.  abstol <= 0 selects LAPACK's default.
    Returns (w[0:iu-il+1], Z[:, 0:iu-il+1]).
    """
    w, z, m, _, info = lapack.zheevr(np.asfortranarray(A), compute_v=1, range="I",
                                     lower=0, il=il, iu=iu, abstol=0.0)
    assert info == 0, f"zheevr info={info}"
    return w[:m].copy(), z[:, :m].copy()


def orth_inplace(V, X, W=None, R=None):
    """rls_orth! two-pass block classical Gram–Schmidt (RLSLinearAlgebra.jl:1127-1160)."""
    nX = X.shape[1]
    W1 = V.conj().T @ X
    X -= V @ W1
    R1 = np.zeros((nX, nX), dtype=np.complex128)
    qr_inplace(X, R1)
    W2 = V.conj().T @ X
    X -= V @ W2
    R2 = np.zeros((nX, nX), dtype=np.complex128)
    qr_inplace(X, R2)
    if W is not None:
        W[:, :] = W2 @ R1 + W1
    if R is not None:
        R[:, :] = R2 @ R1


def orth_robust_inplace(V, X, W=None, R=None, miniter=2, maxiter=4, tol=None):
    """rls_orth_robust! adaptive multi-pass block CGS (RLSLinearAlgebra.jl:1225-1284)."""
    nV, nX = V.shape[1], X.shape[1]
    if tol is None:
        tol = EPS * np.sqrt(float(nV))
    Wtot = None
    Rtot = None
    niter = 0
    for it in range(1, maxiter + 1):
        Wk = V.conj().T @ X
        X -= V @ Wk
        Rk = np.zeros((nX, nX), dtype=np.complex128)
        qr_inplace(X, Rk)
        if it == 1:
            Wtot = Wk.copy()
            Rtot = Rk.copy()
        else:
            Wtot = Wtot + Wk @ Rtot
            Rtot = Rk @ Rtot
        Wk = V.conj().T @ X
        niter = it
        if it >= miniter and np.linalg.norm(Wk) <= tol:
            break
    if W is not None:
        W[:, :] = Wtot
    if R is not None:
        R[:, :] = Rtot
    return niter


def block_unitary_rot(A, B):
    """rls_block_unitary_rot! (RLSLinearAlgebra.jl:164-190): U = Qᴴ of QR([A; B])."""
    r = A.shape[0]
    Y = np.vstack([A, B]).astype(np.complex128)
    Q = qr_inplace(Y, None, full_Q=True)
    return Q.conj().T.copy()


def block_rot_lmul(U, A, i1, i2, r):
    """lmul!(BlockUnitaryRot, A) (RLSLinearAlgebra.jl:59-92); i1, i2 are 1-based block indices."""
    r1 = slice((i1 - 1) * r, i1 * r)
    r2 = slice((i2 - 1) * r, i2 * r)
    A1 = A[r1, :].copy()
    A2 = A[r2, :].copy()
    A[r1, :] = U[:r, :r] @ A1 + U[:r, r:] @ A2
    A[r2, :] = U[r:, :r] @ A1 + U[r:, r:] @ A2


def block_rot_rmul_adj(A, U, i1, i2, r):
    """rmul!(A, adjoint(BlockUnitaryRot)) (RLSLinearAlgebra.jl:106-140) with U' = Uᴴ."""
    Ua = U.conj().T
    c1 = slice((i1 - 1) * r, i1 * r)
    c2 = slice((i2 - 1) * r, i2 * r)
    A1 = A[:, c1].copy()
    A2 = A[:, c2].copy()
    A[:, c1] = A1 @ Ua[:r, :r] + A2 @ Ua[r:, :r]
    A[:, c2] = A1 @ Ua[:r, r:] + A2 @ Ua[r:, r:]


def qr_shiftchol_inplace(X: np.ndarray, R: np.ndarray | None = None, itmax: int = 3):
    """_rls_qr_shiftchol! (RLSLinearAlgebra.jl:725-796): shifted Cholesky-QR.

    X (m×n) ← orthonormal basis; R (when given) ← R_k ⋯ R_1.  On a failed Cholesky of the
    Gram matrix, 11(mn + n(n+1))·eps·max_j‖X_j‖² is added to its diagonal (cumulatively)
    and the factorisation is retried; a sweep stops once ‖XᴴX − I‖_F < 2√n·eps.  Returns
    True when it converged within itmax sweeps (the reference warns otherwise).
    """
    m, n = X.shape
    assert m >= n, "shifted Cholesky-QR requires m >= n"
    if n == 0:
        return True
    conv_tol = 2 * np.sqrt(float(n)) * EPS
    work = X.conj().T @ X
    it = 1
    retries = 0
    while it <= itmax:
        c, info = lapack.zpotrf(work.copy(), lower=0, clean=1)
        if info == 0:
            Rc = np.triu(c)
            if it == 1 and R is not None:
                R[:n, :n] = np.eye(n)
            if R is not None:
                R[:n, :n] = Rc @ R[:n, :n]
            X[:, :] = sla_solve_right_upper(X, Rc)
            work = X.conj().T @ X
            if np.linalg.norm(work - np.eye(n)) < conv_tol:
                return True
            it += 1
        else:
            retries += 1
            if retries > 1000:
                raise RuntimeError("shifted Cholesky-QR: no shift made the Gram matrix factorable")
            gnorm = max(np.linalg.norm(X[:, j]) ** 2 for j in range(n))
            work = work + 11 * (m * n + n * (n + 1)) * EPS * gnorm * np.eye(n)
    return False


def sla_solve_right_upper(X, Rc):
    """X · Rc⁻¹ for upper-triangular Rc (the reference forms trtri(Rc) then trmm; the same
    product to rounding)."""
    import scipy.linalg as sla
    Rinv = sla.solve_triangular(Rc, np.eye(Rc.shape[0], dtype=np.complex128), lower=False)
    return X @ Rinv


def qr_typed(V: np.ndarray, R: np.ndarray | None = None, typ: str = "lapack"):
    """rls_qr!(V, R; type) (RLSLinearAlgebra.jl:584-596)."""
    if typ == "lapack":
        return qr_inplace(V, R)
    if typ == "shiftchol":
        qr_shiftchol_inplace(V, R)
        return None
    raise ValueError(f"unsupported rls_qr! type: {typ}")


def orth_typed(V, X, W=None, R=None, typ="lapack"):
    """rls_orth!(V, X, W, R; type) (RLSLinearAlgebra.jl:1127-1160)."""
    if typ == "lapack":
        return orth_inplace(V, X, W, R)
    nX = X.shape[1]
    W1 = V.conj().T @ X
    X -= V @ W1
    R1 = np.zeros((nX, nX), dtype=np.complex128)
    qr_typed(X, R1, typ)
    W2 = V.conj().T @ X
    X -= V @ W2
    R2 = np.zeros((nX, nX), dtype=np.complex128)
    qr_typed(X, R2, typ)
    if W is not None:
        W[:, :] = W2 @ R1 + W1
    if R is not None:
        R[:, :] = R2 @ R1
