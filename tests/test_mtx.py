"""MatrixMarket input (loaddata, src/utils/loadmtx.jl:1-28) through the C ABI, on the CPU.

The reference reads its matrices with MatrixMarket.jl 0.5's mmread (not vendored); the library's
reader restates the NIST MatrixMarket format.  Each case writes a file, reads it through
``rls_mtx_*`` and compares with SciPy's independent reader (``scipy.io.mmread``) as ComplexF64,
plus the format's edge cases: comments and blank lines, duplicates (summed), explicit zeros,
symmetric / hermitian / skew-symmetric expansion in both formats, and malformed files.
"""
import ctypes as C
import zlib

import numpy as np
import pytest
import scipy.io
import scipy.sparse as sp

from rls_b200 import recursion_grid, reorder_to_natural, reorder_to_natural_grid, PsTriRecyStats
from rls_b200._lib import lib, ptr, ArgumentError
from rls_b200.mtx import load_mtx, loaddata, mtx_info, save_run


def _fmt(field, v):
    v = complex(v)
    if field == "complex":
        return f"{v.real!r} {v.imag!r}"
    if field == "integer":
        return str(int(v.real))
    if field == "pattern":
        return ""
    return repr(float(v.real))


def write_coo(path, m, n, rows, cols, vals, field="real", symm="general", banner="%%MatrixMarket matrix coordinate"):
    with open(path, "w") as f:
        f.write(f"{banner} {field} {symm}\n% written by the test\n")
        f.write(f"{m} {n} {len(rows)}\n")
        for i, j, v in zip(rows, cols, vals):
            f.write(f"{i + 1} {j + 1} {_fmt(field, v)}".rstrip() + "\n")


def write_array(path, A, field="real", symm="general"):
    m, n = A.shape
    with open(path, "w") as f:
        f.write(f"%%MatrixMarket matrix array {field} {symm}\n{m} {n}\n")
        for j in range(n):
            i0 = 0 if symm == "general" else (j + 1 if symm == "skew-symmetric" else j)
            for i in range(i0, m):
                f.write(_fmt(field, A[i, j]) + "\n")


def scipy_dense(path):
    B = scipy.io.mmread(str(path))
    B = B.toarray() if sp.issparse(B) else np.asarray(B)      # toarray() adds up duplicates
    return B.astype(np.complex128)


def as_dense(A):
    return A.toarray() if sp.issparse(A) else np.asarray(A)


def lower_entries(rng, n, field, strict=False):
    rows, cols, vals = [], [], []
    for j in range(n):
        for i in range(j + (1 if strict else 0), n):
            if rng.random() < 0.45 or i == j:
                rows.append(i); cols.append(j)
                v = rng.standard_normal() + 1j * rng.standard_normal()
                if field == "integer":
                    v = complex(int(rng.integers(-9, 10)), 0)
                elif field != "complex":
                    v = complex(v.real, 0)
                vals.append(v)
    return rows, cols, vals


@pytest.mark.parametrize("field", ["real", "complex", "integer", "pattern"])
@pytest.mark.parametrize("symm", ["general", "symmetric", "hermitian", "skew-symmetric"])
def test_coordinate_matches_scipy(tmp_path, field, symm):
    if symm == "hermitian" and field != "complex":
        pytest.skip("hermitian is a complex field")
    if field == "pattern" and symm in ("hermitian", "skew-symmetric"):
        pytest.skip("not a valid pattern storage")
    rng = np.random.default_rng(zlib.crc32(f"{field}/{symm}".encode()))
    n = 23
    if symm == "general":
        m = 17
        rows, cols, vals = [], [], []
        for _ in range(90):
            rows.append(int(rng.integers(m))); cols.append(int(rng.integers(n)))
            v = rng.standard_normal() + 1j * rng.standard_normal()
            vals.append(v if field == "complex" else complex(round(v.real * 5) if field == "integer" else v.real, 0))
        # 90 random positions in 17 × 23: duplicates occur and must add up
    else:
        m = n
        rows, cols, vals = lower_entries(rng, n, field, strict=(symm == "skew-symmetric"))
        if symm == "hermitian":
            vals = [complex(v.real, 0) if i == j else v for i, j, v in zip(rows, cols, vals)]
    path = tmp_path / "a.mtx"
    write_coo(path, m, n, rows, cols, vals, field, symm)
    A = load_mtx(path)
    assert sp.isspmatrix_csc(A) and A.dtype == np.complex128 and A.shape == (m, n)
    np.testing.assert_array_equal(as_dense(A), scipy_dense(path))
    # rows ascend within columns, no duplicate (row, column) pairs
    for j in range(n):
        r = A.indices[A.indptr[j]:A.indptr[j + 1]]
        assert np.all(np.diff(r) > 0)


@pytest.mark.parametrize("field,symm", [("real", "general"), ("complex", "general"), ("integer", "general"),
                                        ("real", "symmetric"), ("complex", "hermitian"),
                                        ("real", "skew-symmetric"), ("complex", "skew-symmetric")])
def test_array_matches_scipy(tmp_path, field, symm):
    rng = np.random.default_rng(5)
    m, n = (7, 5) if symm == "general" else (6, 6)
    A0 = rng.standard_normal((m, n)) + 1j * rng.standard_normal((m, n))
    if field != "complex":
        A0 = A0.real.astype(np.complex128)
    if field == "integer":
        A0 = np.round(A0.real * 5).astype(np.complex128)
    if symm == "hermitian":
        A0[np.diag_indices(n)] = A0.diagonal().real
    path = tmp_path / "d.mtx"
    write_array(path, A0, field, symm)
    A = load_mtx(path)
    assert isinstance(A, np.ndarray) and A.dtype == np.complex128 and A.flags.f_contiguous
    np.testing.assert_array_equal(A, scipy_dense(path))
    assert mtx_info(path) == (m, n, m * n, True)


def test_duplicates_sum_and_explicit_zeros_stay(tmp_path):
    path = tmp_path / "dup.mtx"
    path.write_text("%%MatrixMarket matrix coordinate complex general\n"
                    "%comment\n\n"
                    "3 3 5\n"
                    "1 1 1.5 0.5\n"
                    "3 2 0 0\n"                 # explicit zero, stored
                    "1 1 2.0 -1.0\n"            # duplicate of (1,1): summed
                    "\n"
                    "2 3 -4e-3 1E2\n"
                    "1 1 0.25 0\n")
    A = load_mtx(path)
    assert A.nnz == 3                            # (1,1), (3,2), (2,3)
    assert A[0, 0] == (1.5 + 2.0 + 0.25) + (0.5 - 1.0) * 1j
    assert A[2, 1] == 0 and A.indptr[2] - A.indptr[1] == 1
    assert A[1, 2] == -4e-3 + 100j


def test_banner_case_crlf_and_one_based_output(tmp_path):
    path = tmp_path / "crlf.mtx"
    path.write_bytes(b"%%MatrixMarket MATRIX Coordinate Real Symmetric\r\n% c\r\n2 2 2\r\n1 1 3\r\n2 1 -1\r\n")
    A = load_mtx(path).toarray()
    np.testing.assert_array_equal(A, np.array([[3, -1], [-1, 0]], dtype=np.complex128))
    colptr = np.zeros(3, dtype=np.int64); rowval = np.zeros(4, dtype=np.int64)
    nzval = np.zeros(4, dtype=np.complex128); nnz = C.c_int64(0)
    assert lib().rls_mtx_read_csc(str(path).encode(), 1, 4, ptr(colptr), ptr(rowval), ptr(nzval), C.byref(nnz)) == 0
    assert nnz.value == 3
    np.testing.assert_array_equal(colptr, [1, 3, 4])          # 1-based, as SparseMatrixCSC holds it
    np.testing.assert_array_equal(rowval[:3], [1, 2, 1])


def test_empty_and_capacity(tmp_path):
    path = tmp_path / "empty.mtx"
    path.write_text("%%MatrixMarket matrix coordinate real general\n4 3 0\n")
    A = load_mtx(path)
    assert A.shape == (4, 3) and A.nnz == 0
    path2 = tmp_path / "two.mtx"
    path2.write_text("%%MatrixMarket matrix coordinate real symmetric\n3 3 2\n2 1 1\n3 2 1\n")
    assert mtx_info(path2) == (3, 3, 4, False)
    colptr = np.zeros(4, dtype=np.int64); rowval = np.zeros(3, dtype=np.int64)
    nzval = np.zeros(3, dtype=np.complex128); nnz = C.c_int64(0)
    st = lib().rls_mtx_read_csc(str(path2).encode(), 0, 3, ptr(colptr), ptr(rowval), ptr(nzval), C.byref(nnz))
    assert st == -2 and nnz.value == 4                     # RLS_ERR_DIM, the count it needs


@pytest.mark.parametrize("text,needle", [
    ("%%MatrixMarket tensor coordinate real general\n2 2 0\n", "banner"),
    ("%%MatrixMarket matrix coordinate quaternion general\n2 2 0\n", "field"),
    ("%%MatrixMarket matrix array pattern general\n2 2\n", "pattern"),
    ("%%MatrixMarket matrix coordinate real symmetric\n2 3 0\n", "square"),
    ("%%MatrixMarket matrix coordinate real general\n2 2 2\n1 1 1.0\n", "ends after 1 of 2"),
    ("%%MatrixMarket matrix coordinate real general\n2 2 1\n3 1 1.0\n", "outside"),
    ("%%MatrixMarket matrix coordinate real general\n2 2 1\n1 1 x\n", "bad value"),
    ("%%MatrixMarket matrix coordinate real general\n2 2 1\n1 1 1.0 2.0\n", "trailing"),
    ("%%MatrixMarket matrix coordinate real general\n2 x 1\n", "size line"),
    ("%%MatrixMarket matrix coordinate real general\n2 2 1000000000000\n1 1 1.0\n", "ends after 1 of"),
    ("%%MatrixMarket matrix coordinate real general\n2 2 9000000000000000000\n", "too many entries"),
])
def test_malformed_files_raise(tmp_path, text, needle):
    path = tmp_path / "bad.mtx"
    path.write_text(text)
    with pytest.raises(ArgumentError, match=needle):
        load_mtx(path)


def test_loaddata_missing_file_and_data_dir(tmp_path):
    with pytest.raises(FileNotFoundError, match="Matrix file not found"):
        loaddata("af23560", data_dir=str(tmp_path))
    (tmp_path / "tiny.mtx").write_text("%%MatrixMarket matrix coordinate real general\n2 2 1\n2 1 7\n")
    A = loaddata("tiny", data_dir=str(tmp_path))
    assert A[1, 0] == 7 and A.dtype == np.complex128


def test_save_run_writes_the_driver_fields(tmp_path):
    rec = recursion_grid(0.0, 1.0, 0.0, 1.0, 6, 4, 2)
    sig = np.linspace(1.0, 2.0, len(rec.Z))
    st = PsTriRecyStats.alloc(len(rec.Z))
    st.n_it = 7
    path = tmp_path / "run.npz"
    save_run(path, rec, sig, st, elapsed=1.25)
    z = np.load(path)
    np.testing.assert_array_equal(z["sigma_min"], sig)
    np.testing.assert_array_equal(z["sigma_min_perm"], reorder_to_natural(rec, sig))
    np.testing.assert_array_equal(z["sigma_min_grid"], reorder_to_natural_grid(rec, sig))
    assert float(z["elapsed"]) == 1.25 and int(z["stats_n_it"]) == 7
    assert z["stats_p_count"].shape == (len(rec.Z),)


def test_bench_reads_the_af23560_matrix_from_a_file(tmp_path):
    """bench.py --workload af23560 --mtx PATH: C comes from the file as loaddata reads it, with the
    driver's main_normC and a permutation for the column order."""
    import bench
    rng = np.random.default_rng(11)
    n = 40
    rows, cols, vals = [], [], []
    for i in range(n):
        for j in (i - 2, i, i + 3):
            if 0 <= j < n:
                rows.append(i); cols.append(j); vals.append(complex(rng.standard_normal(), 0))
    path = tmp_path / "af.mtx"
    write_coo(path, n, n, rows, cols, vals)
    C, normC, p = bench.af_inputs(0, mtx=str(path))
    np.testing.assert_array_equal(C.toarray(), scipy_dense(path))
    assert sp.isspmatrix_csc(C) and C.has_sorted_indices
    assert normC == 645.74
    assert sorted(p.tolist()) == list(range(n))
