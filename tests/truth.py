"""FP64 truth for σ_min(T − zI) on an upper-triangular Schur factor, for the parity tests.

Test infrastructure, independent of the engine: block inverse subspace iteration on
(T − zI)ᴴ(T − zI) with cuBLAS triangular solves through torch (the engine's own kernels
are not used), with Rayleigh–Ritz on the block every step.  σ_min(T − zI) = σ_min(C − zI)
because C = Q T Qᴴ with Q unitary.

It returns an error bound from the residual of the Ritz pair beside σ: for the Hermitian
A = RᴴR and a unit vector v, some eigenvalue of A lies within ρ = ‖Av − σ²v‖ of σ², so
|σ_true − σ| ≤ ρ / σ.  Iteration stops once the smallest Ritz value is stationary to
1e-14 and that bound is below `bound_tol`, or after `maxit` steps.
"""
from __future__ import annotations

import numpy as np


def sigma_min_schur(T, zs, block=16, maxit=300, rtol=1e-14, bound_tol=1e-10, seed=0, device="cuda"):
    """σ_min(T − zI) for each z in zs; returns (sigma, err_bound, iterations) as arrays."""
    import torch
    Td = T if isinstance(T, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(T)).to(device)
    n = Td.shape[0]
    b = min(block, n)
    gen = torch.Generator(device=Td.device).manual_seed(seed)
    sig, bound, its = [], [], []
    diag = torch.diagonal(Td).clone()
    R = Td.clone()
    for z in zs:
        torch.diagonal(R).copy_(diag - complex(z))
        Y = torch.randn((n, b), dtype=torch.complex128, device=Td.device, generator=gen)
        Y, _ = torch.linalg.qr(Y)
        prev = np.inf
        s, bnd = np.inf, np.inf
        for it in range(1, maxit + 1):
            W = torch.linalg.solve_triangular(R.mH, Y, upper=False)     # R⁻ᴴ Y
            Y = torch.linalg.solve_triangular(R, W, upper=True)         # R⁻¹ R⁻ᴴ Y
            Y, _ = torch.linalg.qr(Y)
            _, sv, Vh = torch.linalg.svd(R @ Y, full_matrices=False)
            Y = Y @ Vh.mH                                              # Ritz vectors, σ descending
            s = float(sv[-1])
            if abs(prev - s) <= rtol * s:
                v = Y[:, -1:]
                res = R.mH @ (R @ v) - (s * s) * v
                bnd = float(torch.linalg.norm(res)) / max(s, 1e-300)
                if bnd <= bound_tol:
                    break
            prev = s
        sig.append(s)
        bound.append(bnd)
        its.append(it)
    return np.array(sig), np.array(bound), np.array(its)
