"""The CPU oracle against the independent FP64 dense-SVD oracle and its own committed
golden fixtures (the reference has no tests or golden vectors to pin against)."""
import os

import numpy as np
import pytest

from oracle import recugrid as G
from oracle.linalg import orth_robust_inplace, qr_inplace, block_unitary_rot, lq_rows_inplace, svd_inplace
from oracle.pstrirecy import PsTriRecyControl, ps_tri_recy_schur, pre_process_dense, dense_sigma_min
from oracle.recycle import find_rr_dim, check_rr_dim
from rls_b200.examples import sprand, landau, skewlap3d

HERE = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.parametrize("name,gen", [("sprand200", lambda: sprand(200).toarray()),
                                      ("laser120", lambda: landau(120, 40 * np.pi))])
def test_oracle_reproduces_golden(name, gen):
    g = np.load(os.path.join(HERE, f"pstrirecy_{name}.npz"))
    C = gen()
    T = pre_process_dense(C)
    n, r = T.shape[0], int(g["r"])
    rng = np.random.default_rng(int(g["seed"]))
    X0 = rng.random((n, r)) + 1j * rng.random((n, r))
    grid = tuple(g["grid"][:4]) + tuple(int(x) for x in g["grid"][4:])
    rec = G.recursion_grid(*grid)
    ctl = PsTriRecyControl(normC=float(g["normC"]), tol=1e-4, p_min=1, p=int(g["p"]), r=r, recy_tau=1.6)
    sig, st = ps_tri_recy_schur(T, rec, ctl, X0=X0)
    assert np.max(np.abs(sig - g["sigma"])) <= 1e-8 * float(g["normC"])
    assert np.array_equal(st.refine_it > 0, g["refine_it"] > 0)
    assert np.array_equal(st.p_count, g["p_count"])
    # FP64 dense-SVD truth, independent of the restatement
    assert np.max(np.abs(g["truth"] - np.array([dense_sigma_min(C, z) for z in rec.Z]))) < 1e-12
    assert np.max(np.abs(sig - g["truth"])) <= 1e-4 * float(g["normC"])


def test_oracle_sigma_vs_dense_svd_random():
    rng = np.random.default_rng(0)
    n = 80
    C = (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))) / np.sqrt(n)
    T = pre_process_dense(C)
    rec = G.recursion_grid(-0.5, 0.5, -0.5, 0.5, 5, 4, 2)
    sig, st = ps_tri_recy_schur(T, rec, PsTriRecyControl(normC=2.0, tol=1e-4, p=10, r=3), seed=1)
    truth = np.array([dense_sigma_min(C, z) for z in rec.Z])
    assert np.max(np.abs(sig - truth)) <= 1e-4 * 2.0
    assert st.n_pts >= 1


def test_orth_robust_and_qr():
    rng = np.random.default_rng(1)
    V = np.linalg.qr(rng.standard_normal((50, 12)) + 1j * rng.standard_normal((50, 12)))[0]
    X = rng.standard_normal((50, 3)) + 1j * rng.standard_normal((50, 3))
    X0 = X.copy()
    W = np.zeros((12, 3), dtype=complex)
    R = np.zeros((3, 3), dtype=complex)
    orth_robust_inplace(V, X, W, R)
    assert np.linalg.norm(V.conj().T @ X) < 1e-13
    assert np.linalg.norm(X.conj().T @ X - np.eye(3)) < 1e-13
    assert np.linalg.norm(V @ W + X @ R - X0) < 1e-12


def test_block_unitary_rotation_zeroes_lower_block():
    rng = np.random.default_rng(2)
    A = np.triu(rng.standard_normal((4, 4)) + 1j * rng.standard_normal((4, 4)))
    B = rng.standard_normal((4, 4)) + 1j * rng.standard_normal((4, 4))
    U = block_unitary_rot(A, B)
    Y = U @ np.vstack([A, B])
    assert np.linalg.norm(Y[4:]) < 1e-13
    assert np.linalg.norm(U @ U.conj().T - np.eye(8)) < 1e-13


def test_lq_rows():
    rng = np.random.default_rng(3)
    A = rng.standard_normal((3, 7)) + 1j * rng.standard_normal((3, 7))
    Q = A.copy()
    lq_rows_inplace(Q)
    assert np.linalg.norm(Q @ Q.conj().T - np.eye(3)) < 1e-13
    L = A @ Q.conj().T
    assert np.linalg.norm(np.triu(L, 1)) < 1e-13


def test_check_rr_dim_and_find_rr_dim():
    assert check_rr_dim(np.array([1.0, 1.0, 1.0 + 1e-9, 2.0]), 1e-6) == 3
    assert check_rr_dim(np.array([1.0, 1.0]), 1.0) == 0
    rng = np.random.default_rng(4)
    B = rng.standard_normal((30, 12)) + 1j * rng.standard_normal((30, 12))
    H = B.conj().T @ B
    rr, Gm = find_rr_dim(H, 2, 1e-10)
    assert 2 <= rr <= 12
    w = np.linalg.eigvalsh(H)
    assert np.linalg.norm(H @ Gm[:, :rr] - Gm[:, :rr] * w[:rr]) < 1e-10 * w[-1]


def test_generators_shapes():
    C = sprand(400)
    assert C.shape == (400, 400) and C.dtype == np.complex128
    d = C.diagonal()
    assert np.allclose(d.real[:5] - 3 * np.exp(-np.arange(5) / 10), 0, atol=0.5)
    S = skewlap3d(5)
    assert S.shape == (64, 64) and S.nnz <= 7 * 64
    Ld = landau(64, 40 * np.pi)
    assert Ld.shape == (64, 64)
    # Landau operator is complex symmetric
    assert np.allclose(Ld, Ld.T)


def test_fp64_truth_matches_dense_svd():
    """The parity tests' FP64 truth (block inverse iteration on the Schur factor, tests/truth.py)
    against LAPACK's dense SVD of C − zI, here on the host (torch CPU)."""
    import scipy.linalg as sla
    from rls_b200.examples import sprand
    from truth import sigma_min_schur
    C = sprand(150).toarray()
    T = np.triu(sla.schur(C, output="complex")[0])
    zs = [0.5 + 0.05j, 0.45 + 0.0j, 0.3 - 0.2j, 2.0 + 1.0j]
    sig, bound, its = sigma_min_schur(T, zs, device="cpu")
    ref = np.array([sla.svdvals(C - z * np.eye(150))[-1] for z in zs])
    assert np.all(bound <= 1e-10)
    assert np.max(np.abs(sig - ref)) <= 1e-12 * 3.2
