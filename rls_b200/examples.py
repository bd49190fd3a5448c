"""Synthetic matrices with the shapes and value distributions of the reference's examples.

These generators stand in for example/*/<case>.jl.  The reference draws its
random instances from Julia's RNG (not reproducible outside Julia) and loads
af23560 from a file that is not distributed, so each instance here is built
with NumPy's PCG64 from the same seed and the same construction, and all
engines and checkers read the same bytes.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
from scipy.linalg import eigh_tridiagonal

SEED = 20260318


def sprand(N: int = 4000, seed: int = SEED) -> sp.csc_matrix:
    """example/sprand/sprand.jl:11-23: diag 3·exp(−i/10) + superdiag 0.5 + 0.1·sprandn(N,N,3/N).

    The sprandn pattern is Bernoulli(3/N) per entry with N(0,1) values;
    entries that coincide with the two bands are summed, as Julia's sparse
    addition does.  Returned as complex128 CSC.
    """
    rng = np.random.default_rng(seed)
    d0 = 3.0 * np.exp(-np.arange(N) / 10.0)
    d1 = np.full(N - 1, 0.5)
    A = sp.diags([d0, d1], [0, 1], shape=(N, N), format="csc")
    cnt = rng.binomial(N * N, 3.0 / N)
    lin = rng.choice(N * N, size=cnt, replace=False)
    vals = rng.standard_normal(cnt)
    rows, cols = lin % N, lin // N          # column-major linear index, like Julia
    R = sp.csc_matrix((vals, (rows, cols)), shape=(N, N))
    C = (A + 0.1 * R).astype(np.complex128).tocsc()
    C.sort_indices()
    return C


SPRAND_NORMC = 3.2                                     # sprand.jl:27
SPRAND_GRID = dict(x_st=0.45, x_ed=0.55, y_st=0.0, y_ed=0.1, n_x=200, n_y=200, k=20)


def landau(N: int = 5000, F: float = 40 * np.pi) -> np.ndarray:
    """example/laser/laser.jl:15-55: A_kj = √(iF)·√w_k·√w_j·exp(−iπF(x_k−x_j)²).

    Nodes and weights are Gauss–Legendre by Golub–Welsch (laser.jl:21-34).
    """
    k = np.arange(1, N, dtype=np.float64)
    beta = 0.5 * (1.0 - (2.0 * k) ** (-2)) ** (-0.5)
    nodes, V = eigh_tridiagonal(np.zeros(N), beta)
    w = 2.0 * V[0, :] ** 2
    sw = np.sqrt(w)
    d = nodes[:, None] - nodes[None, :]
    B = np.sqrt(1j * F) * np.exp(-1j * np.pi * F * d * d)
    B *= sw[:, None]
    B *= sw[None, :]
    return B


LASER_NORMC = 1.0                                      # laser_psTriRecy.jl:36
LASER_GRID = dict(x_st=-1.1, x_ed=1.2, y_st=-1.1, y_ed=1.1, n_x=200, n_y=200, k=20)


def skewlap3d(N: int = 25) -> sp.csc_matrix:
    """example/skewlap3d/skewlap3d.jl:11-30: n = (N−1)³, D = N²·tridiag(1.5, −2, 0.5)."""
    m = N - 1
    I = sp.identity(m, format="csc")
    D = (N ** 2) * sp.diags([np.full(m - 1, 1.5), np.full(m, -2.0), np.full(m - 1, 0.5)],
                            [-1, 0, 1], format="csc")
    A = sp.kron(I, sp.kron(I, D)) + sp.kron(I, sp.kron(D, I)) + sp.kron(D, sp.kron(I, I))
    C = A.astype(np.complex128).tocsc()
    C.sort_indices()
    return C


SKEWLAP_NORMC = 7471.59                                # skewlap3d.jl:41
SKEWLAP_GRID = dict(x_st=-550.0, x_ed=100.0, y_st=-200.0, y_ed=200.0, n_x=200, n_y=200, k=20)


def ic_factor_banded(n: int, band: int, fill: float, seed: int, complex_values: bool = True) -> sp.csc_matrix:
    """Synthetic stand-in for the threshold IC factor L that psPrecRecy builds
    (get_hsl_LLTP, src/preconditioner/hsl_preconditioner.jl:159-252): sparse lower triangular,
    each row keeping a random `fill` fraction of the `band` columns to its left (values
    N(0, 1)/band, complex unless complex_values is False) and a diagonal of 1 + the row's
    absolute sum, so that it is well conditioned.  n = 23,560, band = 300, fill = 2/3 gives
    the af23560-shaped factor (≈200 nonzeros per row, 4.7·10⁶ in all).  Returns CSC."""
    rng = np.random.default_rng(seed)
    rows, cols = [], []
    for i in range(n):
        lo = max(0, i - band)
        cand = np.arange(lo, i)
        keep = cand[rng.random(cand.size) < fill]
        rows.append(np.full(keep.size, i))
        cols.append(keep)
    r = np.concatenate(rows) if rows else np.zeros(0, int)
    c = np.concatenate(cols) if cols else np.zeros(0, int)
    v = rng.standard_normal(r.size) / max(band, 1)
    if complex_values:
        v = v + 1j * rng.standard_normal(r.size) / max(band, 1)
    off = sp.csr_matrix((v, (r, c)), shape=(n, n), dtype=np.complex128)
    diag = 1.0 + np.asarray(abs(off).sum(axis=1)).ravel()
    return (off + sp.diags(diag.astype(np.complex128))).tocsc()


AF23560_NORMC = 645.74                                 # af23560_psPrecRecy.jl (normC of af23560.jl)
AF23560_GRID = dict(x_st=-1.6, x_ed=0.8, y_st=-1.55, y_ed=1.55, n_x=200, n_y=200, k=20)


def af23560_shaped(n: int = 23560, per_row: int = 20, half_width: int = 300, normC: float = AF23560_NORMC,
                   seed: int = SEED) -> sp.csc_matrix:
    """Synthetic stand-in for the af23560 matrix of example/af23560/af23560.jl (not distributed):
    real unsymmetric, `per_row` − 1 off-diagonal N(0,1) entries per row at uniform offsets within
    ±`half_width` of the diagonal (coinciding entries summed), and a weakly dominant diagonal
    d_i = Σ_j |c_ij| over the row, so that the spectrum lies in the closed right half-plane and
    reaches towards the origin, where the af23560 grid [-1.6, 0.8] × [-1.55, 1.55] sits.  The
    whole matrix is scaled to ‖C‖₂ = normC (largest singular value by ARPACK).  complex128 CSC
    with sorted indices."""
    import scipy.sparse.linalg as spla
    rng = np.random.default_rng(seed)
    rows = np.repeat(np.arange(n, dtype=np.int64), per_row - 1)
    off = rng.integers(1, half_width + 1, size=rows.size) * np.where(rng.random(rows.size) < 0.5, -1, 1)
    cols = rows + off
    ok = (cols >= 0) & (cols < n)
    rows, cols = rows[ok], cols[ok]
    vals = rng.standard_normal(rows.size)
    B = sp.csr_matrix((vals, (rows, cols)), shape=(n, n))
    B.sum_duplicates()
    d = np.asarray(abs(B).sum(axis=1)).ravel()
    A = (B + sp.diags(d)).tocsc()
    s1 = spla.svds(A, k=1, return_singular_vectors=False, random_state=seed)[0]
    C = (A * (normC / s1)).astype(np.complex128).tocsc()
    C.sort_indices()
    return C
