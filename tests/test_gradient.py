"""Gradient of σ_min(C − zI) with respect to z and to C (rls_sigma_grad).

The reference returns σ only; the gradient is checked against central finite
differences of an FP64 dense SVD (relative agreement 1e-6, the bar for this
quantity) and against the dense singular-vector formula (oracle/gradient.py).
"""
import numpy as np
import pytest

from oracle.gradient import dense_sigma_grad, dense_sigma_min, central_difference
from rls_b200.examples import sprand

FD_RTOL = 1e-6


def _grad_scale(dx, dy):
    return max(abs(dx), abs(dy), 1e-3)


def test_dense_formula_matches_finite_differences():
    rng = np.random.default_rng(4)
    n = 40
    C = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    for z in (0.3 + 0.2j, -1.0 + 0.5j):
        s, dx, dy, u, v, dC = dense_sigma_grad(C, z)
        fx, fy = central_difference(C, z)
        sc = _grad_scale(dx, dy)
        assert abs(dx - fx) <= FD_RTOL * sc and abs(dy - fy) <= FD_RTOL * sc
        for (i, j) in [(0, 0), (3, 17), (n - 1, 5)]:
            h = 1e-6
            Cp, Cm = C.copy(), C.copy()
            Cp[i, j] += h
            Cm[i, j] -= h
            fd = (dense_sigma_min(Cp, z) - dense_sigma_min(Cm, z)) / (2 * h)
            assert abs(dC[i, j] - fd) <= FD_RTOL * max(abs(dC).max(), 1e-3)


@pytest.mark.gpu
@pytest.mark.parametrize("z", [0.5 + 0.05j, 0.47 + 0.01j])
def test_engine_gradient_matches_dense_and_finite_differences(cuda_device, z):
    import rls_b200 as R
    from rls_b200.solvers import Engine, LobpcgSvdControl
    C = sprand(240).toarray().astype(np.complex128)
    T, Q = R.pre_process(C, return_q=True)
    e = Engine(cuda_device)
    e.set_schur(T)
    n = C.shape[0]
    ctl = LobpcgSvdControl(m=n, n=n, r=6, conv_range=(1, 1), tol=1e-6, side="L", normC=3.2)
    rng = np.random.default_rng(5)
    X0 = rng.random((n, 6)) + 1j * rng.random((n, 6))
    _, _, X, _ = e.lobpcg_svd_invtri(z, ctl, X0=X0)
    rows, cols = np.nonzero(C)
    g = e.sigma_grad(z, X[:, 0], refine_steps=3, Q=Q, pattern=(rows, cols))
    s, dx, dy, u, v, dC = dense_sigma_grad(C, z)
    assert abs(g["sigma"] - s) <= 1e-10 * max(s, 1e-12) + 1e-14
    fx, fy = central_difference(C, z)
    sc = _grad_scale(dx, dy)
    assert abs(g["dsdx"] - fx) <= FD_RTOL * sc, (g["dsdx"], fx)
    assert abs(g["dsdy"] - fy) <= FD_RTOL * sc, (g["dsdy"], fy)
    assert abs(g["dsdx"] - dx) <= 1e-9 * sc and abs(g["dsdy"] - dy) <= 1e-9 * sc
    # ∂σ/∂C on the sparsity pattern of C (u, v are unique up to a common phase)
    assert np.max(np.abs(g["dsdC"] - dC[rows, cols])) <= 1e-9 * np.abs(dC).max()
    e.close()


@pytest.mark.gpu
def test_engine_gradient_rejects_bad_input(cuda_device):
    import rls_b200 as R
    from rls_b200._lib import ArgumentError, DimensionMismatch
    from rls_b200.solvers import Engine
    C = sprand(120).toarray()
    e = Engine(cuda_device)
    e.set_schur(R.pre_process(C))
    with pytest.raises(DimensionMismatch):
        e.sigma_grad(0.5, np.ones(7))
    with pytest.raises(ArgumentError):
        e.sigma_grad(0.5, np.zeros(120))
    e.close()


@pytest.mark.gpu
def test_grid_gradient_every_point(cuda_device):
    """∂σ/∂z at every grid point from the loop's own singular pairs (stats dsdx, dsdy): the
    accepted Ritz pair at recycled points (quadratic form on the cached H2), LOBPCG's pair at
    refined ones.  Against the dense-SVD gradient: these come from pairs the solver accepted at
    its tolerance, so they agree to first order in the accepted residual (|uᴴv| ≤ 1, bound
    1e-3), and the same values come out of single-lane and laned runs."""
    import rls_b200 as R
    C = sprand(240).toarray().astype(np.complex128)
    T = R.pre_process(C)
    grid = (0.45, 0.55, 0.0, 0.1, 8, 6, 3)
    rec = R.recursion_grid(*grid)
    n = 240
    rng = np.random.default_rng(8)
    X0 = rng.random((n, 6)) + 1j * rng.random((n, 6))
    ctl = R.PsTriRecyControl(normC=3.2, tol=1e-4, p=20, recy_tau=1.6)
    sig, st = R.psTriRecy(R.SchurFactor(T), rec, ctl, verbose=0, X0=X0, grad=True)
    assert np.all(np.isfinite(st.dsdx)) and np.all(np.isfinite(st.dsdy))
    ref = np.array([dense_sigma_grad(C, z)[1:3] for z in rec.Z])
    err = np.maximum(np.abs(st.dsdx - ref[:, 0]), np.abs(st.dsdy - ref[:, 1]))
    rec_pts = st.refine_it == 0
    print(f"grid gradient: max error recycled {err[rec_pts].max() if rec_pts.any() else 0:.2e}, "
          f"refined {err[~rec_pts].max():.2e}")
    assert rec_pts.any() and (~rec_pts).any()
    assert err.max() <= 1e-3, err.max()
    sig2, st2 = R.psTriRecy(R.SchurFactor(T), rec, ctl, verbose=0, X0=X0, grad=False)
    assert st2.dsdx is None and np.array_equal(sig, sig2)
