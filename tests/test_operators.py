"""Lazy operator chains (src/types/RLSMatrices.jl:81-520) against the products they stand for,
with NumPy and SciPy leaves (no device)."""
import numpy as np
import pytest
import scipy.sparse as sp

import rls_b200 as R
from rls_b200.operators import MulChainMat, NormalMat, IdentityMat, PermMat, InvMat, FilledMat


def _c(rng, *shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


def test_mul_chain_and_its_adjoint():
    rng = np.random.default_rng(1)
    A, B, Cm = _c(rng, 7, 5), sp.random(5, 9, density=0.4, random_state=2, format="csr") * (1 - 2j), _c(rng, 9, 4)
    M = MulChainMat(A, B, Cm)
    X = _c(rng, 4, 3)
    D = A @ B.toarray() @ Cm
    assert M.shape == (7, 4)
    assert np.allclose(M @ X, D @ X)
    Y = _c(rng, 7, 2)
    assert M.adjoint().shape == (4, 7)
    assert np.allclose(M.adjoint() @ Y, D.conj().T @ Y)
    x = _c(rng, 5, 1)
    assert np.allclose(MulChainMat(A) @ x, A @ x)                 # one factor
    with pytest.raises(R.DimensionMismatch):
        MulChainMat(A, Cm)
    with pytest.raises(R.DimensionMismatch):
        M @ _c(rng, 5, 1)


def test_normal_identity_and_permutation():
    rng = np.random.default_rng(2)
    Cm = _c(rng, 8, 6)
    X = _c(rng, 6, 2)
    assert np.allclose(NormalMat(Cm) @ X, Cm.conj().T @ (Cm @ X))
    assert NormalMat(Cm).adjoint().shape == (6, 6)
    I = IdentityMat(6)
    assert np.array_equal(I @ X, X) and np.array_equal(I.ldiv(X), X)
    p = rng.permutation(6)
    invp = np.argsort(p)
    P = PermMat(p, invp, 6)
    Pd = np.zeros((6, 6))
    Pd[p, np.arange(6)] = 1.0                      # P e_k = e_{p[k]}
    assert np.array_equal(P @ X, Pd @ X)
    assert np.array_equal(P.adjoint() @ X, Pd.T @ X)
    with pytest.raises(R.DimensionMismatch):
        IdentityMat(-1)


def test_inverse_and_filled():
    rng = np.random.default_rng(3)
    A = _c(rng, 6, 6) + 6 * np.eye(6)
    S = sp.csc_matrix(A)
    X = _c(rng, 6, 2)
    assert np.allclose(A @ (InvMat(A) @ X), X)
    assert np.allclose(A @ (InvMat(S) @ X), X)
    assert np.allclose(A.conj().T @ (InvMat(A).adjoint() @ X), X)
    F = FilledMat(A, 10)
    Z = F @ X
    assert Z.shape == (10, 2) and np.allclose(Z[:6], A @ X) and np.all(Z[6:] == 0)
    W = _c(rng, 10, 3)
    assert np.allclose(F.adjoint() @ W, A.conj().T @ W[:6])
    with pytest.raises(R.DimensionMismatch):
        FilledMat(A, 5)


def test_preconditioned_chain_of_the_pred_stage():
    """Cz·P·L⁻ᴴ (the pred-stage operator of psPrecRecy, RLSPreconditioner.jl:16-25) composed from
    the host IC factor, against the dense product."""
    rng = np.random.default_rng(4)
    n = 50
    Cm = sp.random(n, n, density=0.1, random_state=4, format="csc") + sp.identity(n)
    z = 0.3 + 0.1j
    p = rng.permutation(n)
    L, invp, _ = R.ic_factor(Cm, z, 1e-3, 1e-4, 0.0, 8, 4, p)
    Cz = (Cm - z * sp.identity(n)).tocsc()
    Lt = sp.csc_matrix(L)
    M = MulChainMat(Cz, PermMat(p, invp, n), InvMat(Lt.conj().T.tocsc()))
    X = _c(rng, n, 3)
    Pd = np.zeros((n, n))
    Pd[p, np.arange(n)] = 1.0
    D = Cz.toarray() @ Pd @ np.linalg.inv(L.toarray().conj().T)
    assert np.allclose(M @ X, D @ X)
    assert np.allclose(M.adjoint() @ X, D.conj().T @ X)


class _HostK:
    """A SparseLLTP stand-in whose solve is the CPU restatement (the device solve has its own
    parity tests); only the composition around it is under test here."""

    def __init__(self, L, p, invp):
        self.L, self.p, self.invp = L, p, invp
        self.shape = L.shape

    def ldiv(self, B):
        from oracle.precond import lltp_ldiv
        return lltp_ldiv(self.L, self.p, self.invp, B)


def test_two_level_preconditioner():
    """SparseLLTP_AD: K⁻¹B + E·(GramE⁻¹·(Eᴴ·B)), and update_basis with GramE = (CX)ᴴ(CX)."""
    from rls_b200.examples import ic_factor_banded
    rng = np.random.default_rng(5)
    n, ks = 80, 4
    L = ic_factor_banded(n, 12, 0.5, seed=5)
    p = rng.permutation(n)
    invp = np.argsort(p)
    K = _HostK(L, p, invp)
    E = _c(rng, n, ks)
    CX = _c(rng, n + 3, ks)
    G = CX.conj().T @ CX
    Kad = R.SparseLLTP_AD(K, E, G)
    B = _c(rng, n, 3)
    Ld = L.toarray()
    Pd = np.zeros((n, n))
    Pd[p, np.arange(n)] = 1.0
    Kinv = Pd @ np.linalg.inv(Ld @ Ld.conj().T) @ Pd.T
    ref = Kinv @ B + E @ np.linalg.solve(G, E.conj().T @ B)
    assert np.allclose(Kad.ldiv(B), ref, rtol=1e-10, atol=1e-12)
    X2, CX2 = _c(rng, n, ks), _c(rng, n + 3, ks)
    Kad.update_basis(X2, CX2)
    G2 = CX2.conj().T @ CX2
    ref2 = Kinv @ B + X2 @ np.linalg.solve(G2, X2.conj().T @ B)
    assert np.allclose(Kad.ldiv(B), ref2, rtol=1e-10, atol=1e-12)
    with pytest.raises(R.DimensionMismatch):
        R.SparseLLTP_AD(K, E[:-1], G)
    with pytest.raises(np.linalg.LinAlgError):
        R.SparseLLTP_AD(K, E, -np.eye(ks))


def test_mul_coupled_shares_the_common_factor():
    rng = np.random.default_rng(6)
    calls = []

    class Counted:
        def __init__(self, A):
            self.A, self.shape = A, A.shape

        def __matmul__(self, X):
            calls.append(1)
            return self.A @ X

    F = Counted(_c(rng, 5, 4))
    M0, S0 = _c(rng, 6, 5), _c(rng, 3, 5)
    V = _c(rng, 4, 2)
    MV, SV = R.mul_coupled(MulChainMat(M0, F), MulChainMat(S0, F), V)
    assert len(calls) == 1
    assert np.allclose(MV, M0 @ F.A @ V) and np.allclose(SV, S0 @ F.A @ V)
    MV, SV = R.mul_coupled(MulChainMat(M0, F), MulChainMat(S0, Counted(F.A)), V)
    assert len(calls) == 3 and np.allclose(SV, S0 @ F.A @ V)
