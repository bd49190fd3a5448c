"""MatrixMarket input and the example drivers' result layout.

``loaddata(mname)`` mirrors src/utils/loadmtx.jl:1-28: it reads ``<data_dir>/<mname>.mtx`` (the
reference looks in its ``data/`` directory) through the library's MatrixMarket reader
(``rls_mtx_*``, the NIST format that MatrixMarket.jl 0.5's mmread reads) and returns ComplexF64: a
``scipy.sparse.csc_matrix`` for the coordinate format, a dense Fortran-ordered array for the
array format.  A missing file raises ``FileNotFoundError`` where the reference calls
``error("Matrix file not found at ...")``.  loaddata's narrowing to Int32 indices is a Julia
storage choice; the CSC here keeps SciPy's index type.

``save_run`` writes the fields the example drivers serialise after a solve
(example/sprand/sprand_psTriRecy.jl:35-45: σ_min, σ_min_perm, σ_min_grid, stats, elapsed) to a
NumPy ``.npz``; the Julia drivers keep their own ``.jls`` output through the ccall shim.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np
import scipy.sparse as sp

from ._lib import check, lib, ptr


def _path(path) -> bytes:
    return os.fsencode(os.fspath(path))


def mtx_info(path):
    """(m, n, nnz_max, dense) from the banner and size line of a MatrixMarket file."""
    m, n, nz, dense = C.c_int64(0), C.c_int64(0), C.c_int64(0), C.c_int(0)
    check(lib().rls_mtx_info(_path(path), C.byref(m), C.byref(n), C.byref(nz), C.byref(dense)))
    return m.value, n.value, nz.value, bool(dense.value)


def load_mtx(path):
    """A MatrixMarket file as ComplexF64: CSC for the coordinate format, a dense array otherwise."""
    m, n, nz, dense = mtx_info(path)
    if dense:
        A = np.zeros((m, n), dtype=np.complex128, order="F")
        check(lib().rls_mtx_read_dense(_path(path), ptr(A), max(m, 1)))
        return A
    colptr = np.zeros(n + 1, dtype=np.int64)
    nnz = C.c_int64(0)
    # the size line is not trusted for the allocation: a first pass with room for at most 2^24
    # entries, then exactly the count the reader reports (RLS_ERR_DIM carries it)
    cap = max(1, min(nz, 1 << 24))
    while True:
        rowval = np.zeros(cap, dtype=np.int64)
        nzval = np.zeros(cap, dtype=np.complex128)
        st = lib().rls_mtx_read_csc(_path(path), 0, cap, ptr(colptr), ptr(rowval), ptr(nzval), C.byref(nnz))
        if st == -2 and nnz.value > cap:
            cap = nnz.value
            continue
        check(st)
        break
    k = nnz.value
    return sp.csc_matrix((nzval[:k].copy(), rowval[:k].copy(), colptr), shape=(m, n))


def loaddata(mname: str, data_dir=None):
    """loaddata(mname) (loadmtx.jl:1-28): ``<data_dir>/<mname>.mtx`` as ComplexF64.  data_dir
    defaults to ``$RLS_DATA_DIR`` or ``./data``."""
    d = data_dir if data_dir is not None else os.environ.get("RLS_DATA_DIR", "data")
    path = os.path.join(d, mname + ".mtx")
    if not os.path.isfile(path):
        raise FileNotFoundError(f"Matrix file not found at {path}")
    return load_mtx(path)


def save_run(path, rec, sigma_min, stats=None, elapsed: float = 0.0):
    """The drivers' output tuple (σ_min, σ_min_perm, σ_min_grid, stats, elapsed) as ``.npz``:
    stats' array fields become ``stats_<name>`` entries, its scalar fields ``stats_<name>`` 0-d
    arrays."""
    from .grid import reorder_to_natural, reorder_to_natural_grid
    sigma_min = np.asarray(sigma_min, dtype=np.float64)
    out = {
        "sigma_min": sigma_min,
        "sigma_min_perm": reorder_to_natural(rec, sigma_min),
        "sigma_min_grid": reorder_to_natural_grid(rec, sigma_min),
        "elapsed": np.float64(elapsed),
    }
    if stats is not None:
        fields = vars(stats) if hasattr(stats, "__dict__") else {}
        for name, v in fields.items():
            if name.startswith("_") or v is None:
                continue
            a = np.asarray(v)
            if a.dtype == object:
                continue
            out["stats_" + name] = a
    np.savez(path, **out)
