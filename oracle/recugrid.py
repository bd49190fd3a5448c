"""Restatement of src/core/recuGrid.jl (grid construction and natural-order remap).

Test infrastructure only (see oracle/__init__.py).  Bit-exact by construction:
every coordinate is ``x_st + (ix-1)*dx`` in IEEE double without contraction,
exactly as recuGrid.jl:41-45 evaluates it, and the natural-index rounding
uses round-half-to-even like Julia's ``round(Int, x)`` (recuGrid.jl:182-183).
Indices returned to callers are 1-based, as in the Julia API.
"""
from __future__ import annotations

import numpy as np


class Recursion:
    """Grid metadata + traversal order (recuGrid.jl:1-38)."""

    def __init__(self, x_st, x_ed, y_st, y_ed, n_x, n_y, k):
        nx, ny, kk = int(n_x), int(n_y), int(k)
        if nx < 2:
            raise ValueError("n_x must be >= 2")            # recuGrid.jl:26
        if ny < 2:
            raise ValueError("n_y must be >= 2")            # recuGrid.jl:27
        if kk < 1:
            raise ValueError("k must be >= 1")              # recuGrid.jl:28
        self.x_st, self.x_ed = float(x_st), float(x_ed)
        self.y_st, self.y_ed = float(y_st), float(y_ed)
        self.n_x, self.n_y, self.k = nx, ny, kk
        self.dx = (self.x_ed - self.x_st) / (nx - 1)        # recuGrid.jl:34
        self.dy = (self.y_ed - self.y_st) / (ny - 1)        # recuGrid.jl:35
        self.Z = np.zeros(nx * ny, dtype=np.complex128)

    def z(self, ix: int, iy: int) -> complex:
        """recuGrid.jl:41-45 (1-based ix, iy)."""
        x = self.x_st + float(ix - 1) * self.dx
        y = self.y_st + float(iy - 1) * self.dy
        return complex(x, y)


def recursion_grid_zigzag(x_st, x_ed, y_st, y_ed, n_x, n_y, k) -> Recursion:
    """recuGrid.jl:157-176 (block zigzag, default order)."""
    rec = Recursion(x_st, x_ed, y_st, y_ed, n_x, n_y, k)
    if rec.n_y % rec.k != 0:
        raise ValueError("n_y must be a multiple of k")     # recuGrid.jl:162
    block_id = 0
    for by in range(1, rec.n_y // rec.k + 1):
        x_range = range(1, rec.n_x + 1) if by % 2 == 1 else range(rec.n_x, 0, -1)
        iy0 = (by - 1) * rec.k + 1
        for j, ix in enumerate(x_range, start=1):
            down = (j % 2 == 1)
            base = block_id * rec.k                          # _set_col_k! recuGrid.jl:48-60
            for l in range(1, rec.k + 1):
                iy = iy0 + l - 1 if down else iy0 + (rec.k - l)
                rec.Z[base + l - 1] = rec.z(ix, iy)
            block_id += 1
    return rec


recursion_grid = recursion_grid_zigzag                         # recuGrid.jl:68-73


def recursion_grid_linear(x_st, x_ed, y_st, y_ed, n_x, n_y, k) -> Recursion:
    """recuGrid.jl:82-102 (row serpentine)."""
    rec = Recursion(x_st, x_ed, y_st, y_ed, n_x, n_y, k)
    idx = 0
    for iy in range(1, rec.n_y + 1):
        xs = range(1, rec.n_x + 1) if iy % 2 == 1 else range(rec.n_x, 0, -1)
        for ix in xs:
            rec.Z[idx] = rec.z(ix, iy)
            idx += 1
    return rec


def recursion_grid_spiral(x_st, x_ed, y_st, y_ed, n_x, n_y, k) -> Recursion:
    """recuGrid.jl:109-148 (clockwise spiral from the upper-left corner)."""
    rec = Recursion(x_st, x_ed, y_st, y_ed, n_x, n_y, k)
    left, right, top, bottom = 1, rec.n_x, 1, rec.n_y
    idx = 0
    while left <= right and top <= bottom:
        for ix in range(left, right + 1):
            rec.Z[idx] = rec.z(ix, top); idx += 1
        top += 1
        if top > bottom:
            break
        for iy in range(top, bottom + 1):
            rec.Z[idx] = rec.z(right, iy); idx += 1
        right -= 1
        if left > right:
            break
        for ix in range(right, left - 1, -1):
            rec.Z[idx] = rec.z(ix, bottom); idx += 1
        bottom -= 1
        if top > bottom:
            break
        for iy in range(bottom, top - 1, -1):
            rec.Z[idx] = rec.z(left, iy); idx += 1
        left += 1
    return rec


def _natural_linear_index(rec: Recursion, z: complex) -> int:
    """recuGrid.jl:179-188; Python's round() is round-half-to-even like Julia's."""
    rx = (z.real - rec.x_st) / rec.dx
    ry = (z.imag - rec.y_st) / rec.dy
    ix = int(round(rx)) + 1
    iy = int(round(ry)) + 1
    if not (1 <= ix <= rec.n_x and 1 <= iy <= rec.n_y):
        raise ValueError(f"point {z} is outside the recursion grid bounds")
    return (iy - 1) * rec.n_x + ix


def recursion_natural_permutation(rec: Recursion) -> np.ndarray:
    """recuGrid.jl:196-208; returns a 1-based int64 permutation."""
    n = rec.n_x * rec.n_y
    perm = np.zeros(n, dtype=np.int64)
    for i in range(1, n + 1):
        j = _natural_linear_index(rec, complex(rec.Z[i - 1]))
        if perm[j - 1] != 0:
            raise ValueError(f"duplicate grid point detected at rec.Z[{i}]")
        perm[j - 1] = i
    for j in range(n):
        if perm[j] <= 0:
            raise ValueError(f"missing grid point for natural index {j + 1}")
    return perm


def reorder_to_natural(rec: Recursion, v) -> np.ndarray:
    """recuGrid.jl:216-221."""
    v = np.asarray(v)
    n = rec.n_x * rec.n_y
    if v.shape[0] != n:
        raise ValueError(f"v length {v.shape[0]} does not match grid size {n}")
    return v[recursion_natural_permutation(rec) - 1]


def reorder_to_natural_grid(rec: Recursion, v) -> np.ndarray:
    """recuGrid.jl:229-232: n_y × n_x array with A[iy, ix]."""
    v_nat = reorder_to_natural(rec, v)
    # Julia reshape(v, n_x, n_y) is column-major: element (ix, iy) = v[(iy-1)*n_x + ix].
    return v_nat.reshape(rec.n_y, rec.n_x).copy()
