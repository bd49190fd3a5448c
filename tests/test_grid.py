"""recuGrid through the C ABI: bit-exact against the restatement and the golden
fixtures (src/core/recuGrid.jl), plus the reference's argument errors."""
import os

import numpy as np
import pytest

import rls_b200 as R
from oracle import recugrid as O

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "recugrid.npz"))
NG = len([k for k in GOLD.files if k.endswith("_params")])


def bits(a):
    return np.ascontiguousarray(a, dtype=np.complex128).view(np.uint64)


@pytest.mark.parametrize("i", range(NG))
@pytest.mark.parametrize("name", ["zigzag", "linear", "spiral"])
def test_grid_matches_golden_bit_exact(built_lib, i, name):
    g = tuple(GOLD[f"g{i}_params"])
    g = g[:4] + tuple(int(x) for x in g[4:])
    fn = {"zigzag": R.recursion_grid_zigzag, "linear": R.recursion_grid_linear,
          "spiral": R.recursion_grid_spiral}[name]
    rec = fn(*g)
    assert np.array_equal(bits(rec.Z), bits(GOLD[f"g{i}_{name}_Z"]))
    perm = R.recursion_natural_permutation(rec)
    assert np.array_equal(perm, GOLD[f"g{i}_{name}_perm"])


def test_oracle_matches_golden(built_lib):
    for i in range(NG):
        g = tuple(GOLD[f"g{i}_params"])
        g = g[:4] + tuple(int(x) for x in g[4:])
        rec = O.recursion_grid(*g)
        assert np.array_equal(bits(rec.Z), bits(GOLD[f"g{i}_zigzag_Z"]))


@pytest.mark.parametrize("g", [(0.45, 0.55, 0.0, 0.1, 200, 200, 20), (-1.1, 1.2, -1.1, 1.1, 200, 200, 20),
                               (-1.6, 0.8, -1.55, 1.55, 200, 200, 20), (-550.0, 100.0, -200.0, 200.0, 200, 200, 20),
                               (0.3, -0.7, 0.9, 0.2, 13, 9, 3)])
def test_full_size_grids_bit_exact(built_lib, g):
    a, b = R.recursion_grid(*g), O.recursion_grid(*g)
    assert np.array_equal(bits(a.Z), bits(b.Z))
    assert np.array_equal(R.recursion_natural_permutation(a), O.recursion_natural_permutation(b))


def test_reorder_helpers(built_lib):
    rec = R.recursion_grid(0.0, 1.0, 0.0, 2.0, 5, 6, 3)
    v = np.arange(30, dtype=np.float64) * 1.5
    nat = R.reorder_to_natural(rec, v)
    orec = O.recursion_grid(0.0, 1.0, 0.0, 2.0, 5, 6, 3)
    assert np.array_equal(nat, O.reorder_to_natural(orec, v))
    grid = R.reorder_to_natural_grid(rec, v)
    assert grid.shape == (6, 5)
    assert np.array_equal(grid, O.reorder_to_natural_grid(orec, v))
    # A[iy, ix] holds the value at grid point (x[ix], y[iy])
    for i, z in enumerate(rec.Z):
        ix = int(round((z.real - rec.x_st) / rec.dx))
        iy = int(round((z.imag - rec.y_st) / rec.dy))
        assert grid[iy, ix] == v[i]


def test_c_abi_reorder_entry_points(built_lib):
    import ctypes as C
    from rls_b200._lib import lib, ptr
    rec = R.recursion_grid(-1.0, 1.0, -1.0, 1.0, 8, 6, 2)
    v = np.linspace(0, 1, 48)
    out = np.zeros(48)
    g = rec.c_grid()
    assert lib().rls_reorder_to_natural(C.byref(g), ptr(rec.Z), 48, ptr(v), ptr(out)) == 0
    assert np.array_equal(out, O.reorder_to_natural(O.recursion_grid(-1.0, 1.0, -1.0, 1.0, 8, 6, 2), v))
    outg = np.zeros(48)
    assert lib().rls_reorder_to_natural_grid(C.byref(g), ptr(rec.Z), 48, ptr(v), ptr(outg)) == 0
    # column-major n_y × n_x
    assert np.array_equal(outg.reshape(8, 6).T, R.reorder_to_natural_grid(rec, v))


def test_round_half_even_ties(built_lib):
    # A point exactly halfway between two grid columns maps by round-half-to-even, as Julia's round(Int, x).
    rec = R.recursion_grid(0.0, 4.0, 0.0, 1.0, 5, 2, 1)
    import ctypes as C
    from rls_b200._lib import lib, ptr
    Z = rec.Z.copy()
    Z[0], Z[1] = complex(0.5, 0.0), complex(1.5, 0.0)     # 0.5 → 0 (even), 1.5 → 2 (even)
    Z[2] = complex(0.0, 0.0)
    perm = np.zeros(10, dtype=np.int64)
    g = rec.c_grid()
    st = lib().rls_natural_perm(C.byref(g), ptr(Z), 10, ptr(perm))
    orec = O.recursion_grid(0.0, 4.0, 0.0, 1.0, 5, 2, 1)
    orec.Z = Z.copy()
    with pytest.raises(ValueError):
        O.recursion_natural_permutation(orec)
    assert st == -1   # the collision at index 0 is reported as a duplicate, like the reference
    assert O._natural_linear_index(orec, complex(0.5, 0.0)) == 1
    assert O._natural_linear_index(orec, complex(1.5, 0.0)) == 3
    assert O._natural_linear_index(orec, complex(2.5, 0.0)) == 3


@pytest.mark.parametrize("args,exc", [((0, 1, 0, 1, 1, 4, 1), ValueError), ((0, 1, 0, 1, 4, 1, 1), ValueError),
                                      ((0, 1, 0, 1, 4, 4, 0), ValueError), ((0, 1, 0, 1, 4, 5, 2), ValueError)])
def test_argument_errors(built_lib, args, exc):
    with pytest.raises(exc):
        R.recursion_grid(*args)
    with pytest.raises(ValueError):
        O.recursion_grid(*args)


def test_reorder_dimension_mismatch(built_lib):
    rec = R.recursion_grid(0, 1, 0, 1, 4, 4, 2)
    with pytest.raises(R.DimensionMismatch):
        R.reorder_to_natural(rec, np.zeros(15))


def test_outside_and_missing_points(built_lib):
    rec = R.recursion_grid(0, 1, 0, 1, 4, 4, 2)
    rec.Z[3] = complex(5.0, 0.0)
    with pytest.raises(R.ArgumentError):
        R.recursion_natural_permutation(rec)


def test_lane_offsets_split_on_column_boundaries():
    """rls_lane_offsets (host only): near-equal lanes starting on k-point columns of the
    zigzag traversal, covering the grid."""
    import ctypes as C
    from rls_b200._lib import lib, ptr, check, DimensionMismatch
    rec = R.recursion_grid(0.45, 0.55, 0.0, 0.1, 200, 200, 20)
    g = rec.c_grid()
    k = 20
    for lanes in (1, 3, 4, 8, 10, 25, 2000):
        off = np.zeros(lanes + 1, dtype=np.int64)
        check(lib().rls_lane_offsets(C.byref(g), len(rec.Z), lanes, ptr(off)), None)
        assert off[0] == 0 and off[-1] == len(rec.Z)
        assert np.all(np.diff(off) > 0)
        assert np.all(off[:-1] % k == 0)
        assert np.diff(off).max() - np.diff(off).min() <= k
    # the first point of every lane starts a column of the traversal: same x as the next k-1 points
    off = np.zeros(9, dtype=np.int64)
    check(lib().rls_lane_offsets(C.byref(g), len(rec.Z), 8, ptr(off)), None)
    for o in off[:-1]:
        assert np.allclose(rec.Z[o:o + k].real, rec.Z[o].real)
    off = np.zeros(2002, dtype=np.int64)
    with pytest.raises(DimensionMismatch):
        check(lib().rls_lane_offsets(C.byref(g), len(rec.Z), 2001, ptr(off)), None)
