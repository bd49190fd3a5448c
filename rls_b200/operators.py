"""Lazy operator chains of the reference (src/types/RLSMatrices.jl:81-520): MulChainMat,
NormalMat, IdentityMat, PermMat, InvMat and FilledMat.

They compose whatever leaves they are given without forming a product: this package's device
operators (ShiftedMat's ``@``, SparseLLTP's ``ldiv``), NumPy arrays and SciPy sparse matrices.
A leaf needs ``shape`` and ``@`` (or ``ldiv`` under InvMat) and, for ``adjoint()``, either an
``adjoint()`` method or NumPy/SciPy conjugate transposition.  Host buffers flow between the
factors; each factor's own work runs where the leaf runs it.
"""
from __future__ import annotations

import numpy as np

from ._lib import DimensionMismatch


def _adjoint(A):
    if hasattr(A, "adjoint") and callable(A.adjoint):
        return A.adjoint()
    return A.conj().T


def _ldiv(A, X):
    """A \\ X for a leaf: its own ``ldiv``, a sparse solve, or a dense solve."""
    if hasattr(A, "ldiv"):
        return A.ldiv(X)
    import scipy.sparse as sp
    if sp.issparse(A):
        import scipy.sparse.linalg as spla
        return spla.spsolve(sp.csc_matrix(A), X)
    return np.linalg.solve(A, X)


def _check_rows(op, X):
    if X.shape[0] != op.shape[1]:
        raise DimensionMismatch(-2, f"{type(op).__name__} of size {op.shape} applied to {X.shape[0]} rows")


class MulChainMat:
    """A₁·A₂·…·A_L applied right to left (RLSMatrices.jl:81-182); adjoint() reverses the chain
    and takes each factor's adjoint."""

    def __init__(self, *factors):
        if not factors:
            raise DimensionMismatch(-2, "MulChainMat needs at least one factor")
        for a, b in zip(factors, factors[1:]):
            if a.shape[1] != b.shape[0]:
                raise DimensionMismatch(-2, f"MulChainMat link {a.shape} · {b.shape}")
        self.factors = tuple(factors)
        self.shape = (factors[0].shape[0], factors[-1].shape[1])

    def __matmul__(self, X):
        X = np.asarray(X)
        _check_rows(self, X)
        Y = X
        for f in reversed(self.factors):
            Y = f @ Y
        return np.asarray(Y)

    def adjoint(self):
        return MulChainMat(*[_adjoint(f) for f in reversed(self.factors)])


class NormalMat:
    """N = Cᴴ·C, applied as Cᴴ(C X) (RLSMatrices.jl:186-232); Hermitian."""

    def __init__(self, C):
        self.C = C
        self.shape = (C.shape[1], C.shape[1])

    def __matmul__(self, X):
        X = np.asarray(X)
        _check_rows(self, X)
        return MulChainMat(_adjoint(self.C), self.C) @ X

    def adjoint(self):
        return self


class IdentityMat:
    """The n × n identity (RLSMatrices.jl:237-302)."""

    def __init__(self, n: int):
        if n < 0:
            raise DimensionMismatch(-2, f"IdentityMat size must be nonnegative, got n = {n}")
        self.n = n
        self.shape = (n, n)

    def __matmul__(self, X):
        X = np.asarray(X)
        _check_rows(self, X)
        return X.copy()

    def ldiv(self, X):
        return self @ X

    def adjoint(self):
        return self


class PermMat:
    """The permutation P with P·X = X[invp, :] (RLSMatrices.jl:307-357); adjoint() swaps p and
    invp.  0-based index vectors."""

    def __init__(self, p, invp, n: int):
        self.p = np.asarray(p, dtype=np.int64)
        self.invp = np.asarray(invp, dtype=np.int64)
        if self.p.shape != (n,) or self.invp.shape != (n,):
            raise DimensionMismatch(-2, f"PermMat of size {n} with index vectors {self.p.shape}, {self.invp.shape}")
        self.n = n
        self.shape = (n, n)

    def __matmul__(self, X):
        X = np.asarray(X)
        _check_rows(self, X)
        return X[self.invp]

    def adjoint(self):
        return PermMat(self.invp, self.p, self.n)


class InvMat:
    """A⁻¹ applied as A \\ X (RLSMatrices.jl:390-425); adjoint() is InvMat(adjoint(A))."""

    def __init__(self, A):
        self.A = A
        self.shape = tuple(A.shape)

    def __matmul__(self, X):
        X = np.asarray(X)
        _check_rows(self, X)
        return np.asarray(_ldiv(self.A, X))

    def adjoint(self):
        return InvMat(_adjoint(self.A))


class FilledMat:
    """F = [A; 0] with m rows in all (RLSMatrices.jl:441-520): F·X = [A·X; 0], and its adjoint
    [Aᴴ 0]·X = Aᴴ·X[:rows(A), :]."""

    def __init__(self, A, m: int):
        if m < A.shape[0]:
            raise DimensionMismatch(-2, f"FilledMat needs m ≥ {A.shape[0]}, got {m}")
        self.A = A
        self.m = m
        self.shape = (m, A.shape[1])

    def __matmul__(self, X):
        X = np.asarray(X)
        _check_rows(self, X)
        top = np.asarray(self.A @ X)
        out = np.zeros((self.m,) + top.shape[1:], dtype=np.result_type(top, np.complex128))
        out[:top.shape[0]] = top
        return out

    def adjoint(self):
        return _FilledAdjoint(self)


class _FilledAdjoint:
    def __init__(self, F: FilledMat):
        self.F = F
        self.shape = (F.shape[1], F.shape[0])

    def __matmul__(self, X):
        X = np.asarray(X)
        _check_rows(self, X)
        return np.asarray(_adjoint(self.F.A) @ X[:self.F.A.shape[0]])

    def adjoint(self):
        return self.F


def mul_coupled(M, S, V):
    """(M·V, S·V) (mul_coupled_ms!, RLSPreconditioner.jl:38-76): when M = M₀·F and S = S₀·F are
    two-factor chains sharing the same F object, F·V is formed once."""
    V = np.asarray(V)
    if (isinstance(M, MulChainMat) and isinstance(S, MulChainMat) and len(M.factors) == 2
            and len(S.factors) == 2 and M.factors[1] is S.factors[1]):
        FV = np.asarray(M.factors[1] @ V)
        return np.asarray(M.factors[0] @ FV), np.asarray(S.factors[0] @ FV)
    return np.asarray(M @ V), np.asarray(S @ V)
