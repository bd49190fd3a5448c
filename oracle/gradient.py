"""Dense reference for the gradient of σ_min(C − zI) — test infrastructure only.

No counterpart in the reference project (its solvers return σ only).  With the
smallest singular triplet (σ, u, v) of C − zI from an FP64 dense SVD (LAPACK zgesdd
through NumPy), first-order perturbation of a simple singular value gives
dσ = Re(uᴴ d(C − zI) v), hence
    ∂σ/∂Re z = −Re(uᴴv),  ∂σ/∂Im z = Im(uᴴv),  ∂σ/∂C_ij = Re(conj(u_i) v_j).
"""
from __future__ import annotations

import numpy as np


def dense_sigma_grad(C, z):
    """(σ, ∂σ/∂x, ∂σ/∂y, u, v, ∂σ/∂C) at z = x + iy for dense C."""
    A = np.asarray(C, dtype=np.complex128) - z * np.eye(C.shape[0])
    U, s, Vh = np.linalg.svd(A)
    u, v = U[:, -1], Vh[-1].conj()
    w = np.vdot(u, v)
    return s[-1], -w.real, w.imag, u, v, np.real(np.outer(u.conj(), v))


def dense_sigma_min(C, z):
    A = np.asarray(C, dtype=np.complex128) - z * np.eye(C.shape[0])
    return np.linalg.svd(A, compute_uv=False)[-1]


def central_difference(C, z, h=1e-6):
    """(∂σ/∂x, ∂σ/∂y) by central differences of the dense σ_min."""
    fx = (dense_sigma_min(C, z + h) - dense_sigma_min(C, z - h)) / (2 * h)
    fy = (dense_sigma_min(C, z + 1j * h) - dense_sigma_min(C, z - 1j * h)) / (2 * h)
    return fx, fy
