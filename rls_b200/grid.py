"""Recursion grid (src/core/recuGrid.jl) through the C ABI.

Same names and semantics as the reference: ``recursion_grid`` builds the block
zigzag order, ``recursion_natural_permutation`` returns a 1-based permutation and
the reorder helpers raise where the reference throws.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import check, lib, ptr, rls_grid, ArgumentError, DimensionMismatch


class Recursion:
    """Grid metadata + traversal order (recuGrid.jl:1-38)."""

    def __init__(self, x_st, x_ed, y_st, y_ed, n_x, n_y, k):
        nx, ny, kk = int(n_x), int(n_y), int(k)
        if nx < 2:
            raise ArgumentError(-1, "n_x must be >= 2")
        if ny < 2:
            raise ArgumentError(-1, "n_y must be >= 2")
        if kk < 1:
            raise ArgumentError(-1, "k must be >= 1")
        self.x_st, self.x_ed = float(x_st), float(x_ed)
        self.y_st, self.y_ed = float(y_st), float(y_ed)
        self.n_x, self.n_y, self.k = nx, ny, kk
        self.dx = (self.x_ed - self.x_st) / (nx - 1)
        self.dy = (self.y_ed - self.y_st) / (ny - 1)
        self.Z = np.zeros(nx * ny, dtype=np.complex128)

    def c_grid(self) -> rls_grid:
        return rls_grid(self.x_st, self.x_ed, self.y_st, self.y_ed, self.n_x, self.n_y, self.k)


def _build(fn, x_st, x_ed, y_st, y_ed, n_x, n_y, k) -> Recursion:
    rec = Recursion(x_st, x_ed, y_st, y_ed, n_x, n_y, k)
    g = rec.c_grid()
    st = fn(C.byref(g), ptr(rec.Z))
    if st == -1 and fn is lib().rls_grid_zigzag and rec.n_y % rec.k != 0:
        raise ArgumentError(st, "n_y must be a multiple of k")
    check(st)
    return rec


def recursion_grid_zigzag(x_st, x_ed, y_st, y_ed, n_x, n_y, k) -> Recursion:
    """recuGrid.jl:157-176."""
    return _build(lib().rls_grid_zigzag, x_st, x_ed, y_st, y_ed, n_x, n_y, k)


def recursion_grid(x_st, x_ed, y_st, y_ed, n_x, n_y, k) -> Recursion:
    """recuGrid.jl:68-73 (default order: block zigzag)."""
    return recursion_grid_zigzag(x_st, x_ed, y_st, y_ed, n_x, n_y, k)


def recursion_grid_linear(x_st, x_ed, y_st, y_ed, n_x, n_y, k) -> Recursion:
    """recuGrid.jl:82-102."""
    return _build(lib().rls_grid_linear, x_st, x_ed, y_st, y_ed, n_x, n_y, k)


def recursion_grid_spiral(x_st, x_ed, y_st, y_ed, n_x, n_y, k) -> Recursion:
    """recuGrid.jl:109-148."""
    return _build(lib().rls_grid_spiral, x_st, x_ed, y_st, y_ed, n_x, n_y, k)


def recursion_natural_permutation(rec: Recursion) -> np.ndarray:
    """recuGrid.jl:196-208 (1-based int64)."""
    n = rec.n_x * rec.n_y
    Z = np.ascontiguousarray(rec.Z, dtype=np.complex128)
    perm = np.zeros(n, dtype=np.int64)
    g = rec.c_grid()
    st = lib().rls_natural_perm(C.byref(g), ptr(Z), len(Z), ptr(perm))
    if st == -2:
        raise DimensionMismatch(st, f"rec.Z length {len(Z)} does not match grid size {n}")
    if st == -1:
        raise ArgumentError(st, "grid point outside the recursion grid, duplicated or missing")
    check(st)
    return perm


def reorder_to_natural(rec: Recursion, v) -> np.ndarray:
    """recuGrid.jl:216-221."""
    v = np.asarray(v)
    n = rec.n_x * rec.n_y
    if v.shape[0] != n:
        raise DimensionMismatch(-2, f"v length {v.shape[0]} does not match grid size {n}")
    return v[recursion_natural_permutation(rec) - 1]


def reorder_to_natural_grid(rec: Recursion, v) -> np.ndarray:
    """recuGrid.jl:229-232: n_y × n_x array, A[iy, ix] at (x[ix], y[iy])."""
    v_nat = reorder_to_natural(rec, v)
    return v_nat.reshape(rec.n_y, rec.n_x).copy()
