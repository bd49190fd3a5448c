"""psTriRecy / lobpcgSvd host interface over the C ABI (mirrors src/core/psTriRecy.jl).

``psTriRecy(C, rec; control)`` keeps the reference's call shape: C dense (or
sparse, densified), ``rec`` a Recursion, ``control`` a PsTriRecyControl; it
returns ``(sigma_min, stats)``.  The one-time preprocessing (complex Schur
factor, LAPACK zgees — psTriRecy.jl:6-14) runs on the host as in the reference
and is timed into ``stats.preprocess_time_ns``; everything per grid point runs
on the GPU through librls_b200.so.
"""
from __future__ import annotations

import ctypes as C
import sys
import time
from dataclasses import dataclass, field

import numpy as np

from ._lib import (LOG_FN, check, lib, ptr, c64, rls_lobpcg_control, rls_pstrirecy_control,
                   rls_pstrirecy_stats, ArgumentError, DimensionMismatch)
from .grid import Recursion

EPS = float(np.finfo(np.float64).eps)


def _checked(arr, dtype, min_len: int, name: str, writable: bool = False):
    """arr as a C-contiguous array of dtype holding at least min_len values, for the library to
    read (or, with writable, write in place: then arr must already be such an array)."""
    if writable:
        if not isinstance(arr, np.ndarray) or arr.dtype != dtype or not arr.flags.c_contiguous or \
                not arr.flags.writeable:
            raise ArgumentError(-1, f"{name} must be a writable C-contiguous {np.dtype(dtype).name} array")
        a = arr
    else:
        a = np.ascontiguousarray(arr, dtype=dtype)
    if a.size < min_len:
        raise DimensionMismatch(-2, f"{name} holds {a.size} values, {min_len} needed")
    return a


@dataclass
class PsTriRecyControl:
    """psTriRecy.jl:350-370 (same fields, same defaults; shift = normC²·eps·100)."""
    tol: float = 1e-3
    normC: float = 1.0
    shift: float = None
    gap_tau: float = 1e-10
    gap_tau_scale: float = 0.01
    recy_tau: float = 1.5
    recycle_fail_dist_thresh: float = float("nan")
    r: int = 6
    p: int = 50
    p_min: int = 1
    lobpcg_tol_scale: float = 0.1
    lobpcg_side: str = "L"
    implict_update: bool = False
    implict_recycle: bool = True
    collect_timing: bool = True
    inner_verbose_override: int = None

    def __post_init__(self):
        if self.shift is None:
            self.shift = self.normC ** 2 * EPS * 100

    def c_struct(self) -> rls_pstrirecy_control:
        return rls_pstrirecy_control(
            self.tol, self.normC, self.shift, self.gap_tau, self.gap_tau_scale, self.recy_tau,
            self.recycle_fail_dist_thresh, int(self.r), int(self.p), int(self.p_min), self.lobpcg_tol_scale,
            ord(self.lobpcg_side), int(self.implict_update), int(self.implict_recycle), int(self.collect_timing),
            0, -1 if self.inner_verbose_override is None else int(self.inner_verbose_override))


@dataclass
class PsTriRecyStats:
    """psTriRecy.jl:257-292 (+ refine_it: LOBPCG iterations per point)."""
    p_count: np.ndarray
    r_recy: np.ndarray
    pts: np.ndarray
    M_vec_apps: np.ndarray
    M_vec_apps_no_recycle: np.ndarray
    R_vec_apps: np.ndarray
    refine_it: np.ndarray
    preprocess_time_ns: int = 0
    recycle_time_ns: int = 0
    qr_time_ns: int = 0
    refine_time_ns: int = 0
    update_time_ns: int = 0
    mv_stats_available: bool = True
    n_it: int = 0
    n_pts: int = 0
    dsdx: np.ndarray = None      # ∂σ/∂Re z per point (grad=True)
    dsdy: np.ndarray = None      # ∂σ/∂Im z per point

    @classmethod
    def alloc(cls, nZ, grad: bool = False):
        z = lambda: np.zeros(nZ, dtype=np.int64)
        st = cls(z(), z(), np.zeros(nZ, dtype=np.complex128), z(), z(), z(), z())
        if grad:
            st.dsdx = np.full(nZ, np.nan)
            st.dsdy = np.full(nZ, np.nan)
        return st


@dataclass
class LobpcgSvdControl:
    """lobpcgSvd.jl:1-55."""
    m: int
    n: int
    r: int
    maxit: int = 2000
    tol: float = 1e-3
    side: str = "S"
    verbose: int = 0
    normC: float = 1.0
    orth_type: str = "lapack"
    conv_range: tuple = None
    conv_thresh_type: int = 0

    def __post_init__(self):
        if self.conv_range is None:
            self.conv_range = (1, self.r)
        a, b = self.conv_range
        if not (1 <= a <= b <= self.r):
            raise ArgumentError(-1, f"conv_range={self.conv_range} must satisfy 1 <= first <= last <= r={self.r}")
        if self.orth_type not in ("lapack", "shiftchol"):
            raise ArgumentError(-1, f"orth_type={self.orth_type} must be :lapack or :shiftchol")
        if self.conv_thresh_type not in (0, 1):
            raise ArgumentError(-1, f"conv_thresh_type={self.conv_thresh_type} must be 0 or 1")

    def c_struct(self) -> rls_lobpcg_control:
        return rls_lobpcg_control(self.m, self.n, self.r, self.maxit, self.tol, ord(self.side), self.verbose,
                                  self.normC, 0 if self.orth_type == "lapack" else 1, self.conv_thresh_type,
                                  self.conv_range[0], self.conv_range[1])


def pre_process(C_, return_q: bool = False):
    """psTriRecy.jl:6-14 (square dense branch): upper-triangular complex Schur factor.

    Host LAPACK zgees through SciPy, as the reference's ``schur(C)``.  A sparse C is
    densified first: σ_min(C − zI) is invariant under the unitary similarity, so the
    Schur path computes the same σ as the reference's sparse QR path.  With
    ``return_q`` the Schur vectors Q (C = Q T Qᴴ) are returned too, for the gradient
    with respect to C (Engine.sigma_grad).
    """
    import scipy.linalg as sla
    import scipy.sparse as sp
    if sp.issparse(C_):
        C_ = C_.toarray()
    A = np.asarray(C_, dtype=np.complex128)
    if A.ndim != 2 or A.shape[0] != A.shape[1]:
        raise DimensionMismatch(-2, f"pre_process only supports square matrices here, got size {A.shape}")
    T, Q = sla.schur(A, output="complex", check_finite=True)
    return (np.triu(T), Q) if return_q else np.triu(T)


BAND_QR_MAX_L = 1008   # the device band QR's largest lower bandwidth (rls_set_sparse_tri)


def _csc_arrays(C_):
    import scipy.sparse as sp
    A = sp.csc_matrix(C_, dtype=np.complex128)
    A.sum_duplicates()
    A.sort_indices()
    if A.shape[0] != A.shape[1]:
        raise DimensionMismatch(-2, f"pre_process only supports square matrices, got size {A.shape}")
    return (A.shape[0], np.ascontiguousarray(A.indptr, dtype=np.int64),
            np.ascontiguousarray(A.indices, dtype=np.int64), np.ascontiguousarray(A.data, dtype=np.complex128))


def band_order(C_):
    """The symmetric order sparse psTriRecy takes by default (rls_band_order): the natural or
    the reverse Cuthill–McKee order of |C| + |Cᵀ|, whichever gives the smaller banded-QR work.
    Returns (perm (new → old, 0-based), l, u), l and u the bandwidths of C[perm, perm]."""
    n, colptr, rowval, _ = _csc_arrays(C_)
    perm = np.zeros(n, dtype=np.int64)
    l, u = C.c_int64(0), C.c_int64(0)
    check(lib().rls_band_order(n, ptr(colptr), ptr(rowval), 0, ptr(perm), C.byref(l), C.byref(u)), None)
    return perm, int(l.value), int(u.value)


class SparseTri:
    """A sparse C for psTriRecy's sparse branch (pre_process(C::SparseMatrixCSC),
    psTriRecy.jl:47-61): the CSC arrays and the symmetric order P (perm, new → old; None:
    band_order's).  Each Engine it is installed on holds B = PᵀCP and refactors R of B − zI on
    the device at every refine point."""

    def __init__(self, C_, perm=None):
        self.n, self.colptr, self.rowval, self.nzval = _csc_arrays(C_)
        if perm is None:
            perm, self.l, self.u = band_order(C_)
        else:
            perm = np.ascontiguousarray(perm, dtype=np.int64)
            self.l = self.u = None
        self.perm = perm


class SchurFactor:
    """A precomputed Schur factor T (skip pre_process on repeated runs)."""

    def __init__(self, T, preprocess_time_ns=0):
        self.T = np.asfortranarray(np.asarray(T, dtype=np.complex128))
        self.preprocess_time_ns = preprocess_time_ns


class Engine:
    """One device context (stream, workspaces, uploaded operator) — one per host thread."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        check(lib().rls_ctx_create(C.byref(h), int(device)))
        self._h = h
        self._log_cb = None
        self._T_id = None
        self._Q_id = None
        self.n = 0

    def close(self):
        if self._h:
            lib().rls_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_schur(self, T: np.ndarray):
        T = np.asfortranarray(np.asarray(T, dtype=np.complex128))
        if T.ndim != 2 or T.shape[0] != T.shape[1]:
            raise DimensionMismatch(-2, f"the Schur factor must be square, got shape {T.shape}")
        n = T.shape[0]
        check(lib().rls_set_schur(self._h, n, ptr(T), n), self._h)
        self._T_id = id(T)
        self._Q_id = None
        self.n = n

    def set_sparse_tri(self, S: "SparseTri"):
        """Installs a sparse C for psTriRecy's sparse branch (rls_set_sparse_tri)."""
        check(lib().rls_set_sparse_tri(self._h, S.n, ptr(S.colptr), ptr(S.rowval), ptr(S.nzval), 0, ptr(S.perm)),
              self._h)
        self._T_id = None
        self._Q_id = None
        self.n = S.n

    def band_r(self, z: complex):
        """R of B − zI from the device band QR, dense (test hook rls_test_band_r), with (l, u)."""
        n = self.n
        R = np.zeros((n, n), dtype=np.complex128, order="F")
        l, u = C.c_int64(0), C.c_int64(0)
        z = complex(z)
        check(lib().rls_test_band_r(self._h, c64(z.real, z.imag), ptr(R), n, C.byref(l), C.byref(u)), self._h)
        return R, int(l.value), int(u.value)

    def band_set_panel(self, w: int):
        """Band QR panel width: 8, 16 or 0 (timed choice)."""
        check(lib().rls_band_set_panel(self._h, int(w)), self._h)

    def band_info(self):
        """(l, u, panel width in use, timed ms with 8 and with 16 columns) of the sparse operator."""
        l, u, w = C.c_int64(0), C.c_int64(0), C.c_int(0)
        m8, m16 = C.c_double(0), C.c_double(0)
        check(lib().rls_band_info(self._h, C.byref(l), C.byref(u), C.byref(w), C.byref(m8), C.byref(m16)), self._h)
        return int(l.value), int(u.value), int(w.value), float(m8.value), float(m16.value)

    def band_factor(self, z: complex):
        """One device factorisation R(z) of B − zI (test hook rls_test_band_factor), synchronised."""
        z = complex(z)
        check(lib().rls_test_band_factor(self._h, c64(z.real, z.imag)), self._h)

    def set_log(self, fn, verbose=1):
        if fn is None:
            self._log_cb = None
            check(lib().rls_ctx_set_log(self._h, LOG_FN(), None, 0), self._h)
            return
        cb = LOG_FN(lambda line, user: fn(line.decode()))
        self._log_cb = cb
        check(lib().rls_ctx_set_log(self._h, cb, None, int(verbose)), self._h)

    def pstrirecy(self, rec: Recursion, control: PsTriRecyControl, X0=None, grad: bool = False):
        """psTriRecy on the uploaded Schur factor → (σ, stats); with grad, stats.dsdx and
        stats.dsdy hold ∂σ/∂Re z and ∂σ/∂Im z at every point."""
        nZ = len(rec.Z)
        Z = np.ascontiguousarray(rec.Z, dtype=np.complex128)
        sigma = np.full(nZ, np.nan)
        st = PsTriRecyStats.alloc(nZ, grad)
        cst = self.stats_struct(st)
        x0 = None
        if X0 is not None:
            x0 = np.asfortranarray(np.asarray(X0, dtype=np.complex128))
            if x0.shape != (self.n, control.r):
                raise DimensionMismatch(-2, f"X0 must be {(self.n, control.r)}, got {x0.shape}")
        g = rec.c_grid()
        cc = control.c_struct()
        check(lib().rls_pstrirecy_schur(self._h, ptr(Z), nZ, C.byref(g), C.byref(cc), ptr(x0), ptr(sigma),
                                        C.byref(cst)), self._h)
        for f in ("recycle_time_ns", "qr_time_ns", "refine_time_ns", "update_time_ns", "n_it", "n_pts"):
            setattr(st, f, int(getattr(cst, f)))
        st.mv_stats_available = bool(cst.mv_stats_available)
        return sigma, st

    def stats_struct(self, st: "PsTriRecyStats"):
        cst = rls_pstrirecy_stats()
        i64 = C.POINTER(C.c_int64)
        cst.p_count = st.p_count.ctypes.data_as(i64)
        cst.r_recy = st.r_recy.ctypes.data_as(i64)
        cst.pts = st.pts.ctypes.data_as(C.POINTER(c64))
        cst.M_vec_apps = st.M_vec_apps.ctypes.data_as(i64)
        cst.M_vec_apps_no_recycle = st.M_vec_apps_no_recycle.ctypes.data_as(i64)
        cst.R_vec_apps = st.R_vec_apps.ctypes.data_as(i64)
        cst.refine_it = st.refine_it.ctypes.data_as(i64)
        f64 = C.POINTER(C.c_double)
        if st.dsdx is not None:
            cst.dsdx = st.dsdx.ctypes.data_as(f64)
        if st.dsdy is not None:
            cst.dsdy = st.dsdy.ctypes.data_as(f64)
        return cst

    def pstrirecy_range(self, rec: Recursion, control: PsTriRecyControl, i_begin: int, i_end: int, sigma, st,
                        cst, X0=None):
        """Continues (or, with i_begin == 0, starts) a psTriRecy run over rec.Z[i_begin:i_end];
        sigma/st are the run's full-length outputs, cst the C view of st (stats_struct)."""
        Z = _checked(rec.Z, np.complex128, 0, "rec.Z")
        sigma = _checked(sigma, np.float64, len(Z), "sigma", writable=True)
        x0 = None
        if X0 is not None and i_begin == 0:
            x0 = np.asfortranarray(np.asarray(X0, dtype=np.complex128))
            if x0.shape != (self.n, control.r):
                raise DimensionMismatch(-2, f"X0 must be {(self.n, control.r)}, got {x0.shape}")
        g = rec.c_grid()
        cc = control.c_struct()
        check(lib().rls_pstrirecy_schur_range(self._h, ptr(Z), len(Z), C.byref(g), C.byref(cc), ptr(x0), int(i_begin),
                                              int(i_end), ptr(sigma), C.byref(cst)), self._h)
        for f in ("recycle_time_ns", "qr_time_ns", "refine_time_ns", "update_time_ns", "n_it", "n_pts"):
            setattr(st, f, int(getattr(cst, f)))

    def set_batch(self, max_points: int):
        """Speculative recycle batch size (1 = plain per-point path)."""
        check(lib().rls_ctx_set_batch(self._h, int(max_points)), self._h)

    def set_ritz_basis(self, g1_always: bool):
        """Recycle-step Ritz basis when r_ == p·r: V·G1·G2 (True, default) or the
        reference's V·G2 (False, fastRaylRitz.jl:199-202)."""
        check(lib().rls_ctx_set_ritz_basis(self._h, int(bool(g1_always))), self._h)

    def set_trsm_ctas(self, ctas: int):
        """CTAs per triangular solve (0: one per half block row, the single-traversal
        optimum; fewer leave SMs to concurrent lanes)."""
        check(lib().rls_set_trsm_ctas(self._h, int(ctas)), self._h)

    def set_host_wait(self, spin_us: int):
        """Host waits: spin (spin_us < 0, default) or poll spin_us µs and then sleep."""
        check(lib().rls_ctx_set_host_wait(self._h, int(spin_us)), self._h)

    def set_trsm_backoff(self, max_ns: int):
        """Longest back-off (ns) between the triangular solve's flag polls."""
        check(lib().rls_set_trsm_backoff(self._h, int(max_ns)), self._h)

    def set_graphs(self, on: bool):
        """CUDA-graph replay of the refine's steady LOBPCG iteration (default on)."""
        check(lib().rls_ctx_set_graphs(self._h, int(bool(on))), self._h)

    def stream_ptr(self) -> int:
        return int(lib().rls_ctx_stream(self._h) or 0)

    def launches(self) -> int:
        return int(lib().rls_ctx_launches(self._h))

    def set_profile(self, on: bool):
        check(lib().rls_ctx_set_profile(self._h, int(on)), self._h)

    def profile(self, kernel: int):
        cnt = C.c_int64()
        ms = C.c_double()
        work = C.c_double()
        check(lib().rls_ctx_profile_get(self._h, int(kernel), C.byref(cnt), C.byref(ms), C.byref(work)), self._h)
        return cnt.value, ms.value, work.value

    def lobpcg_svd_invtri(self, z: complex, control: LobpcgSvdControl, X0=None):
        """lobpcgSvd(InvMat(adjoint(T − zI)), X0, I, keep, control) → (σ, it, X, σ_r)."""
        r = control.r
        x0 = None
        if X0 is not None:
            x0 = np.asfortranarray(np.asarray(X0, dtype=np.complex128))
        X = np.zeros((self.n, r), dtype=np.complex128, order="F")
        sr = np.zeros(r)
        s = C.c_double()
        it = C.c_int64()
        cc = control.c_struct()
        check(lib().rls_lobpcg_svd_invtri(self._h, c64(z.real, z.imag), ptr(x0), C.byref(cc), ptr(X), ptr(sr),
                                          C.byref(s), C.byref(it)), self._h)
        return s.value, it.value, X, sr

    OPS = {"inv_schur": 0, "shifted": 1, "pred": 2, "inv_l": 3}

    def lobpcg_svd(self, op: str, z: complex, control: LobpcgSvdControl, prec: str = None, X0=None):
        """lobpcgSvd(C, X0, K, keep, control) (lobpcgSvd.jl:365-477) on one of the context's
        operators: "inv_schur" InvMat(adjoint(T − zI)), "shifted" ShiftedMat(C, −z), "pred"
        ShiftedMat(C, −z)·invF, "inv_l" InvMat(L); K = None or "lltp" (the uploaded SparseLLTP).
        Returns (σ, it, X = keep.S[:, 1:r], keep.σ[1:r])."""
        r = control.r
        n = control.n
        x0 = None
        if X0 is not None:
            x0 = np.asfortranarray(np.asarray(X0, dtype=np.complex128).reshape(n, -1))
        X = np.zeros((n, r), dtype=np.complex128, order="F")
        sr = np.zeros(r)
        s = C.c_double()
        it = C.c_int64()
        cc = control.c_struct()
        check(lib().rls_lobpcg_svd(self._h, self.OPS[op], c64(z.real, z.imag), 0 if prec is None else 1, ptr(x0),
                                   C.byref(cc), ptr(X), ptr(sr), C.byref(s), C.byref(it)), self._h)
        return s.value, it.value, X, sr

    def sparse_upload(self, C):
        """Uploads a sparse C (SciPy sparse, any format) for spmm_shifted / ShiftedMat."""
        import scipy.sparse as sp
        A = sp.csc_matrix(C, dtype=np.complex128)
        A.sort_indices()
        m, n = A.shape
        colptr = np.ascontiguousarray(A.indptr, dtype=np.int64)
        rowval = np.ascontiguousarray(A.indices, dtype=np.int64)
        nzval = np.ascontiguousarray(A.data, dtype=np.complex128)
        check(lib().rls_sparse_upload_csc(self._h, m, n, ptr(colptr), ptr(rowval), ptr(nzval), 0), self._h)
        self.sparse_shape = (m, n)

    def spmm_shifted(self, s: complex, X, adj: bool = False):
        """mul!(Y, ShiftedMat(C, s), X) (RLSMatrices.jl:47-56), or its adjoint: host arrays."""
        m, n = self.sparse_shape
        X = np.asfortranarray(np.asarray(X, dtype=np.complex128))
        vec = X.ndim == 1
        if vec:
            X = X.reshape(-1, 1, order="F")
        rows_in, rows_out = (m, n) if adj else (n, m)
        if X.shape[0] != rows_in:
            raise DimensionMismatch(-2, f"X has {X.shape[0]} rows, expected {rows_in}")
        Y = np.zeros((rows_out, X.shape[1]), dtype=np.complex128, order="F")
        check(lib().rls_spmm_shifted(self._h, c64(s.real, s.imag), int(adj), X.shape[1], ptr(X), X.shape[0], ptr(Y),
                                     rows_out), self._h)
        return Y[:, 0] if vec else Y

    def sigma_grad(self, z: complex, v0, refine_steps: int = 2, Q=None, pattern=None):
        """σ_min(C − zI) and its gradient at z (no reference counterpart).

        v0 (n values) approximates the right singular vector of T − zI (e.g. the first
        Ritz vector of lobpcg_svd_invtri).  Returns a dict with sigma, dsdx = ∂σ/∂Re z,
        dsdy = ∂σ/∂Im z and the Schur-basis singular vectors u, v.  With the Schur vectors
        Q of C (C = Q T Qᴴ, from pre_process; uploaded once per Q) it adds dsdC =
        Re(conj((Qu)_i) (Qv)_j), computed on the device (rls_sigma_grad_pattern): on the
        (rows, cols) index arrays of ``pattern`` when given (the nnz of a sparse C), else the
        dense n × n matrix.
        """
        v0 = np.ascontiguousarray(np.asarray(v0, dtype=np.complex128).reshape(-1))
        if v0.shape[0] != self.n:
            raise DimensionMismatch(-2, f"v0 has {v0.shape[0]} entries, the operator {self.n}")
        u = np.zeros(self.n, dtype=np.complex128)
        v = np.zeros(self.n, dtype=np.complex128)
        sg, dx, dy = C.c_double(), C.c_double(), C.c_double()
        check(lib().rls_sigma_grad(self._h, c64(z.real, z.imag), ptr(v0), int(refine_steps), C.byref(sg),
                                   C.byref(dx), C.byref(dy), ptr(u), ptr(v)), self._h)
        out = {"sigma": sg.value, "dsdx": dx.value, "dsdy": dy.value, "u": u, "v": v}
        if Q is not None:
            if self._Q_id != id(Q):
                Qf = np.asfortranarray(np.asarray(Q, dtype=np.complex128))
                check(lib().rls_set_schur_vectors(self._h, ptr(Qf), Qf.shape[0]), self._h)
                self._Q_id = id(Q)
            if pattern is not None:
                rows = np.ascontiguousarray(pattern[0], dtype=np.int64)
                cols = np.ascontiguousarray(pattern[1], dtype=np.int64)
            else:
                rows = np.ascontiguousarray(np.tile(np.arange(self.n, dtype=np.int64), self.n))
                cols = np.ascontiguousarray(np.repeat(np.arange(self.n, dtype=np.int64), self.n))
            g = np.zeros(rows.size)
            check(lib().rls_sigma_grad_pattern(self._h, ptr(u), ptr(v), rows.size, ptr(rows), ptr(cols), 0, ptr(g)),
                  self._h)
            out["dsdC"] = g if pattern is not None else g.reshape(self.n, self.n, order="F")
        return out


class ShiftedMat:
    """ShiftedMat (src/types/RLSMatrices.jl:24-64) on the device: C − zI with C sparse,
    applied as ``A @ X`` (mul!) and ``A.adjoint() @ X``.  The matrix is uploaded once to
    the given Engine."""

    def __init__(self, C, s: complex, engine: "Engine" = None, adj: bool = False, _uploaded: bool = False):
        self.engine = engine or Engine(0)
        self.s = complex(s)
        self.adj = adj
        if not _uploaded:
            self.engine.sparse_upload(C)
        m, n = self.engine.sparse_shape
        self.shape = (n, m) if adj else (m, n)

    def __matmul__(self, X):
        return self.engine.spmm_shifted(self.s if not self.adj else np.conj(self.s), X, adj=self.adj)

    def adjoint(self) -> "ShiftedMat":
        """adjoint(ShiftedMat) = ShiftedMat(Cᴴ, conj(s)) (RLSMatrices.jl:64-66)."""
        return ShiftedMat(None, np.conj(self.s), self.engine, adj=not self.adj, _uploaded=True)


def ic_factor(Cm, z, tau1, tau2, alpha, lsize, rsize, p):
    """get_hsl_LLTP's factorisation on the host (rls_ic_factor; hsl_preconditioner.jl:159-252):
    returns (L as a SciPy CSC matrix, invp, the diagonal shift used), 0-based p and invp.  No
    device is needed."""
    import scipy.sparse as sp
    A = sp.csc_matrix(Cm, dtype=np.complex128)
    A.sum_duplicates()
    A.sort_indices()
    n = A.shape[0]
    if A.shape != (n, n):
        raise DimensionMismatch(-2, f"get_hsl_LLTP only supports square C, got size {A.shape}")
    p = np.ascontiguousarray(p, dtype=np.int64)
    if p.shape != (n,):
        raise DimensionMismatch(-2, f"permutation length mismatch: length(p)={p.size} n={n}")
    colptr = np.ascontiguousarray(A.indptr, dtype=np.int64)
    rowval = np.ascontiguousarray(A.indices, dtype=np.int64)
    nzval = np.ascontiguousarray(A.data, dtype=np.complex128)
    lsz = min(max(0, int(lsize)), n - 1)
    cap = n + lsz * n
    lcolptr = np.zeros(n + 1, dtype=np.int64)
    lrow = np.zeros(max(cap, 1), dtype=np.int64)
    lval = np.zeros(max(cap, 1), dtype=np.complex128)
    invp = np.zeros(n, dtype=np.int64)
    shift = C.c_double()
    z = complex(z)
    check(lib().rls_ic_factor(n, ptr(colptr), ptr(rowval), ptr(nzval), 0, c64(z.real, z.imag), float(tau1),
                              float(tau2), float(alpha), int(lsize), int(rsize), ptr(p), cap, ptr(lcolptr),
                              ptr(lrow), ptr(lval), ptr(invp), C.byref(shift)), None)
    nl = int(lcolptr[n])
    L = sp.csc_matrix((lval[:nl], lrow[:nl], lcolptr), shape=(n, n))
    return L, invp, shift.value


def get_hsl_LLTP(Cm, z, tau1, tau2, alpha, lsize, rsize, p, engine: "Engine" = None) -> "SparseLLTP":
    """get_hsl_LLTP(C, z, tau1, tau2, α, lsize, rsize, p) (hsl_preconditioner.jl:159-252) with C
    passed as Cm: the IC factor built on the host (ic_factor), uploaded to the device as a
    SparseLLTP."""
    L, invp, _ = ic_factor(Cm, z, tau1, tau2, alpha, lsize, rsize, p)
    return SparseLLTP(L, p, invp, engine)


class SparseLLTP:
    """SparseLLTP (src/preconditioner/RLSPreconditioner.jl:8-26) on the device: the IC factor
    L (sparse; only its lower triangle is used), the permutation p and its stored inverse
    invp (0-based here; the C ABI also takes Julia's 1-based vectors).  ``ldiv(B)`` is
    ldiv!(X, K, B) = P·L⁻ᴴ·L⁻¹·Pᴴ·B (:79-116); ``ldiv(B, out=B)`` is ldiv!(K, B)."""

    def __init__(self, L, p, invp, engine: "Engine" = None):
        import scipy.sparse as sp
        self.engine = engine or Engine(0)
        A = sp.csc_matrix(L, dtype=np.complex128)
        A.sort_indices()
        n = A.shape[0]
        if A.shape != (n, n):
            raise DimensionMismatch(-2, f"SparseLLTP needs a square factor, got {A.shape}")
        p = np.ascontiguousarray(p, dtype=np.int64)
        invp = np.ascontiguousarray(invp, dtype=np.int64)
        if p.shape != (n,) or invp.shape != (n,):
            raise DimensionMismatch(-2, f"permutation lengths {p.shape}, {invp.shape} for n = {n}")
        colptr = np.ascontiguousarray(A.indptr, dtype=np.int64)
        rowval = np.ascontiguousarray(A.indices, dtype=np.int64)
        nzval = np.ascontiguousarray(A.data, dtype=np.complex128)
        check(lib().rls_lltp_upload(self.engine._h, n, ptr(colptr), ptr(rowval), ptr(nzval), ptr(p), ptr(invp), 0),
              self.engine._h)
        self.shape = (n, n)

    def adjoint(self) -> "SparseLLTP":
        """P·L·Lᴴ·Pᴴ is Hermitian, and so is its inverse."""
        return self

    def ldiv(self, B, out=None):
        B = np.asarray(B)
        vec = B.ndim == 1
        Bf = np.asfortranarray(B.reshape(B.shape[0], -1), dtype=np.complex128)
        n, b = Bf.shape
        if n != self.shape[0]:
            raise DimensionMismatch(-2, f"B has {n} rows, the factor {self.shape[0]}")
        X = np.empty((n, b), dtype=np.complex128, order="F")
        check(lib().rls_lltp_ldiv(self.engine._h, b, ptr(Bf), n, ptr(X), n), self.engine._h)
        res = X[:, 0] if vec else X
        if out is not None:
            out[...] = res
            return out
        return res


class SparseLLTP_AD:
    """SparseLLTP_AD (RLSPreconditioner.jl:160-290), the two-level preconditioner of the pred
    stage: ``ldiv(B)`` = K⁻¹B + E·(GramE⁻¹·(Eᴴ·B)), with K a SparseLLTP (its two sparse
    triangular solves on the device) and E (n × ks) with the Cholesky factor of
    GramE = (CE)ᴴ(CE) on the host (ks ≤ 40: two tall-skinny products and a ks × ks solve per
    apply).  The factorisation is plain upper Cholesky, as rls_cholesky! (RLSLinearAlgebra.jl:15-21)
    is; a GramE that is not positive definite raises numpy.linalg.LinAlgError."""

    def __init__(self, K, E, GramE):
        import scipy.linalg as sla
        self.K = K
        self.E = np.array(E, dtype=np.complex128, order="F")
        self.GramE = np.array(GramE, dtype=np.complex128, order="F")
        if self.E.shape[0] != K.shape[0] or self.GramE.shape != (self.E.shape[1], self.E.shape[1]):
            raise DimensionMismatch(-2, f"SparseLLTP_AD: E {self.E.shape}, GramE {self.GramE.shape}, K {K.shape}")
        self.F = sla.cho_factor(self.GramE, lower=False)
        self.shape = K.shape

    def update_basis(self, X, CX):
        """update_sparse_lldiv_ad_basis! (:208-226): E = X, GramE = CXᴴ·CX, refactored."""
        import scipy.linalg as sla
        X = np.asarray(X)
        CX = np.asarray(CX)
        if X.shape != self.E.shape:
            raise DimensionMismatch(-2, f"update_basis: X {X.shape}, E {self.E.shape}")
        self.E[...] = X
        self.GramE = np.asfortranarray(CX.conj().T @ CX)
        self.F = sla.cho_factor(self.GramE, lower=False)

    def ldiv(self, B):
        import scipy.linalg as sla
        B = np.asarray(B, dtype=np.complex128)
        coeff = sla.cho_solve(self.F, self.E.conj().T @ B)
        proj = self.E @ coeff
        X = np.asarray(self.K.ldiv(B))
        return X + proj

    def adjoint(self) -> "SparseLLTP_AD":
        """Both terms are Hermitian."""
        return self


class Lanes:
    """Concurrent grid lanes on one GPU (rls_pstrirecy_schur_lanes_range): one Engine per
    lane, each with the Schur factor uploaded; the traversal is split into near-equal parts
    starting on column boundaries (k points) of the zigzag traversal and every lane runs psTriRecy from an empty recycled space on
    its part, in its own host thread inside the library.  No reference counterpart."""

    def __init__(self, lanes: int, device: int = 0, T=None):
        if lanes < 1:
            raise ArgumentError(-1, f"lanes must be >= 1, got {lanes}")
        self.engines = [Engine(device) for _ in range(lanes)]
        self._arr = (C.c_void_p * lanes)(*[e._h for e in self.engines])
        if T is not None:
            self.set_schur(T)

    @property
    def n(self):
        return self.engines[0].n

    def set_schur(self, T):
        """One host upload to the first lane; the others share its device tiles."""
        self.engines[0].set_schur(T)
        for e in self.engines[1:]:
            check(lib().rls_set_schur_copy(e._h, self.engines[0]._h), e._h)
            e.n = self.engines[0].n

    def set_sparse_tri(self, S: "SparseTri"):
        """Every lane holds its own B = PᵀCP and band factor (R changes with each lane's shift)."""
        for e in self.engines:
            e.set_sparse_tri(S)

    def set_batch(self, max_points: int):
        for e in self.engines:
            e.set_batch(max_points)

    def set_trsm_ctas(self, ctas: int):
        for e in self.engines:
            e.set_trsm_ctas(ctas)

    def set_host_wait(self, spin_us: int):
        for e in self.engines:
            e.set_host_wait(spin_us)

    def set_trsm_backoff(self, max_ns: int):
        for e in self.engines:
            e.set_trsm_backoff(max_ns)

    def set_graphs(self, on: bool):
        for e in self.engines:
            e.set_graphs(on)

    def set_profile(self, on: bool):
        for e in self.engines:
            e.set_profile(on)

    def profile(self, kernel: int):
        cnt, ms, work = 0, 0.0, 0.0
        for e in self.engines:
            c, m, w = e.profile(kernel)
            cnt, ms, work = cnt + c, ms + m, work + w
        return cnt, ms, work

    def launches(self) -> int:
        return sum(e.launches() for e in self.engines)

    def streams(self):
        return [e.stream_ptr() for e in self.engines]

    def offsets(self, rec: Recursion):
        off = np.zeros(len(self.engines) + 1, dtype=np.int64)
        g = rec.c_grid()
        check(lib().rls_lane_offsets(C.byref(g), len(rec.Z), len(self.engines), ptr(off)), None)
        return off

    def pstrirecy_range(self, rec: Recursion, control: PsTriRecyControl, j_begin: int, j_end: int, sigma, st,
                        cst, X0=None):
        """Lane-local points j_begin..j_end-1 of every lane (j_begin == 0 starts the lanes);
        sigma/st are the full-length outputs, cst their C view (Engine.stats_struct)."""
        Z = _checked(rec.Z, np.complex128, 0, "rec.Z")
        sigma = _checked(sigma, np.float64, len(Z), "sigma", writable=True)
        x0 = None
        if X0 is not None and j_begin == 0:
            x0 = np.asfortranarray(np.asarray(X0, dtype=np.complex128))
            if x0.shape != (self.n, control.r):
                raise DimensionMismatch(-2, f"X0 must be {(self.n, control.r)}, got {x0.shape}")
        g = rec.c_grid()
        cc = control.c_struct()
        check(lib().rls_pstrirecy_schur_lanes_range(self._arr, len(self.engines), ptr(Z), len(Z), C.byref(g),
                                                    C.byref(cc), ptr(x0), int(j_begin), int(j_end), ptr(sigma),
                                                    C.byref(cst)), self.engines[0]._h)
        for f in ("recycle_time_ns", "qr_time_ns", "refine_time_ns", "update_time_ns", "n_it", "n_pts"):
            setattr(st, f, int(getattr(cst, f)))

    def pstrirecy(self, rec: Recursion, control: PsTriRecyControl, X0=None, grad: bool = False):
        nZ = len(rec.Z)
        sigma = np.full(nZ, np.nan)
        st = PsTriRecyStats.alloc(nZ, grad)
        cst = self.engines[0].stats_struct(st)
        self.pstrirecy_range(rec, control, 0, nZ, sigma, st, cst, X0=X0)
        st.mv_stats_available = True
        return sigma, st

    def close(self):
        for e in self.engines:
            e.close()


_engines = {}


def _engine(device=0) -> Engine:
    e = _engines.get(device)
    if e is None:
        e = Engine(device)
        _engines[device] = e
    return e


def _print_startup(io, rec, control):
    """psTriRecy.jl:554-577."""
    io.write("[psTriRecy] rec: x_range=[%.6f, %.6f], y_range=[%.6f, %.6f], n_x=%d, n_y=%d, k=%d, n_pts=%d\n"
             % (rec.x_st, rec.x_ed, rec.y_st, rec.y_ed, rec.n_x, rec.n_y, rec.k, rec.n_x * rec.n_y))
    io.write("[psTriRecy] control:\n")
    for f in control.__dataclass_fields__:
        io.write(f"  {f} = {getattr(control, f)!r}\n")


def psTriRecy(C_, rec: Recursion, control: PsTriRecyControl = None, verbose: int = 1, io=None, X0=None,
              device: int = 0, lanes: int = 1, grad: bool = False):
    """psTriRecy (psTriRecy.jl:889-913) → (σ_min in rec.Z order, PsTriRecyStats).

    A SciPy sparse C takes the sparse branch (SparseTri: B = PᵀCP, R of B − zI by the device
    band QR at every refine point) when its ordered lower bandwidth is at most 1008, and the
    dense Schur path otherwise (σ is invariant under the unitary similarity).  A dense C,
    SchurFactor or SparseTri is used as given.

    ``X0`` (n × r) stands in for the reference's ``rand!(X)``; None draws a
    deterministic uniform [0,1) complex block on the device.  ``lanes`` > 1 splits the
    traversal on column boundaries into concurrent lanes on the same GPU (class Lanes);
    1 keeps the reference's single traversal.  ``grad`` fills stats.dsdx / stats.dsdy with
    ∂σ/∂Re z and ∂σ/∂Im z at every point from its own singular pair (no reference
    counterpart).
    """
    import scipy.sparse as sp
    control = control or PsTriRecyControl()
    io = io if io is not None else sys.stdout
    if verbose >= 1:
        _print_startup(io, rec, control)
    t0 = time.perf_counter_ns()
    op = None
    if isinstance(C_, (SchurFactor, SparseTri)):
        op = C_
        pre_ns = getattr(C_, "preprocess_time_ns", 0)
    elif sp.issparse(C_):
        S = SparseTri(C_)
        if S.l <= BAND_QR_MAX_L:           # the sparse branch on the device band QR
            op = S
        else:                              # too wide a band: the unitarily equivalent Schur form
            op = SchurFactor(pre_process(C_))
        pre_ns = time.perf_counter_ns() - t0
    else:
        op = SchurFactor(pre_process(C_))
        pre_ns = time.perf_counter_ns() - t0

    def install(target):
        if isinstance(op, SparseTri):
            target.set_sparse_tri(op)
        else:
            target.set_schur(op.T)

    if lanes > 1:
        ls = Lanes(lanes, device)
        try:
            install(ls)
            sigma, st = ls.pstrirecy(rec, control, X0=X0, grad=grad)
        finally:
            ls.close()
        st.preprocess_time_ns = pre_ns
        return sigma, st
    eng = _engine(device)
    install(eng)
    if verbose >= 1:
        eng.set_log(lambda line: (io.write(line + "\n"), io.write("-" * 100 + "\n")), verbose)
    else:
        eng.set_log(None)
    try:
        sigma, st = eng.pstrirecy(rec, control, X0=X0, grad=grad)
    finally:
        eng.set_log(None)
    st.preprocess_time_ns = pre_ns
    if verbose >= 1:
        io.write(f"Total M vec apps for singular value problem: {int(st.M_vec_apps.sum())}\n")
        if control.collect_timing:
            if st.preprocess_time_ns > 0:
                io.write("Total preprocess time for singular value problem: %.6f seconds\n" % (st.preprocess_time_ns / 1e9))
            io.write("Total recycle time for singular value problem: %.6f seconds\n" % (st.recycle_time_ns / 1e9))
            io.write("Total refine time for singular value problem: %.6f seconds\n" % (st.refine_time_ns / 1e9))
            io.write("Total update time for singular value problem: %.6f seconds\n" % (st.update_time_ns / 1e9))
        io.write(f"Total R vec apps for singular value problem: {int(st.R_vec_apps.sum())}\n")
        io.write(f"Total it for singular value problem: {st.n_it}\n")
        io.write(f"Total pt for singular value problem: {st.n_pts}\n")
    return sigma, st


# ---- psPrecRecy (src/core/psPrecRecy.jl) -------------------------------------------------------

@dataclass
class PsPrecRecyControl:
    """psPrecRecy.jl:220-261 (same fields, same defaults; shift = main_normC²·eps·100).  The Greek
    field names λ_lower_min, λ_upper_max, γ_tol and λ_n_tol are spelt lambda_lower_min,
    lambda_upper_max, gamma_tol and lambda_n_tol; pred_orth_type is "lapack" or "shiftchol" for
    the Symbols :lapack / :shiftchol; pred_conv_range is None or a 1-based (first, last)."""
    tol: float = 1e-3
    lobpcg_tol_scale: float = 0.1
    main_normC: float = 10.0
    main_tau: float = 1.666
    shift: float = None
    gap_tau: float = 1e-10
    recycle_fail_dist_thresh: float = float("nan")
    tol_pred: float = 1e-3
    lobpcg_pred_tol_scale: float = 1.0
    pred_conv_range: tuple = None
    pred_tau: float = 1.666
    idx_cutoff_pred: float = 1e-2
    pred_orth_type: str = "lapack"
    pred_conv_thresh_type: int = 0
    lambda_lower_min: float = 0.1
    lambda_upper_max: float = 30.0
    r_main: int = 6
    p_main: int = 60
    p_min_main: int = 1
    main_implict_update: bool = False
    main_implict_recycle: bool = False
    r_pred: int = 20
    p_pred: int = 20
    p_min_pred: int = 1
    pred_implict_update: bool = True
    pred_implict_recycle: bool = True
    hsl_tol: float = 1e-3
    hsl_cntl_1: float = 1e-6
    hsl_cntl_2: float = 1e-5
    hsl_icntl_1: int = 200
    hsl_icntl_2: int = 200
    gamma_tol: float = 1e-3
    lambda_n_tol: float = 1e-3
    inner_verbose_override: int = None
    collect_timing: bool = True

    def __post_init__(self):
        if self.shift is None:
            self.shift = self.main_normC ** 2 * EPS * 100
        if self.pred_orth_type not in ("lapack", "shiftchol"):
            raise ArgumentError(-1, f"pred_orth_type={self.pred_orth_type} must be :lapack or :shiftchol")

    def c_struct(self) -> "rls_psprecrecy_control":
        from ._lib import rls_psprecrecy_control
        c = rls_psprecrecy_control()
        for f in ("tol", "lobpcg_tol_scale", "main_normC", "main_tau", "shift", "gap_tau", "recycle_fail_dist_thresh",
                  "tol_pred", "lobpcg_pred_tol_scale", "pred_tau", "idx_cutoff_pred", "lambda_lower_min",
                  "lambda_upper_max", "hsl_tol", "hsl_cntl_1", "hsl_cntl_2", "gamma_tol", "lambda_n_tol"):
            setattr(c, f, float(getattr(self, f)))
        for f in ("pred_conv_thresh_type", "r_main", "p_main", "p_min_main", "r_pred", "p_pred", "p_min_pred",
                  "hsl_icntl_1", "hsl_icntl_2"):
            setattr(c, f, int(getattr(self, f)))
        for f in ("main_implict_update", "main_implict_recycle", "pred_implict_update", "pred_implict_recycle",
                  "collect_timing"):
            setattr(c, f, int(bool(getattr(self, f))))
        if self.pred_conv_range is None:
            c.pred_conv_first, c.pred_conv_last = -1, -1
        else:
            c.pred_conv_first, c.pred_conv_last = int(self.pred_conv_range[0]), int(self.pred_conv_range[1])
        c.pred_orth_type = 0 if self.pred_orth_type == "lapack" else 1
        c.inner_verbose_override = -1 if self.inner_verbose_override is None else int(self.inner_verbose_override)
        return c


class PsPrecRecyStats:
    """psPrecRecy.jl:318-350 (+ main_refine_it, pred_refine_it: LOBPCG iterations per point)."""
    _I = ("p_count", "pred_p_count", "r_recy", "main_M_vec_apps", "main_M_vec_apps_no_recycle", "main_L_vec_apps",
          "pred_M_vec_apps", "pred_L_vec_apps", "main_refine_it", "pred_refine_it")
    _Z = ("pts", "pred_pts", "precond_rebuild_pts")
    _S = ("main_recycle_time_ns", "main_refine_time_ns", "main_update_time_ns", "pred_recycle_time_ns",
          "pred_refine_time_ns", "pred_update_time_ns", "precond_time_ns", "n_it", "n_pred_it", "n_pts", "n_pred_pts",
          "n_precond_rebuild_pts")

    def __init__(self, nZ):
        for f in self._I:
            setattr(self, f, np.zeros(nZ, dtype=np.int64))
        for f in self._Z:
            setattr(self, f, np.zeros(nZ, dtype=np.complex128))
        for f in self._S:
            setattr(self, f, 0)

    def c_struct(self):
        from ._lib import rls_psprecrecy_stats
        c = rls_psprecrecy_stats()
        for f in self._I:
            setattr(c, f, getattr(self, f).ctypes.data_as(C.POINTER(C.c_int64)))
        for f in self._Z:
            setattr(c, f, getattr(self, f).ctypes.data_as(C.POINTER(c64)))
        return c

    def read_scalars(self, c):
        for f in self._S:
            setattr(self, f, int(getattr(c, f)))


class PrecRecyRun:
    """One psPrecRecy run on an Engine, resumable over index ranges (rls_psprecrecy_range)."""

    def __init__(self, engine: Engine, C_, rec: Recursion, control: PsPrecRecyControl, p=None, X0_main=None,
                 X0_pred=None, X0_bound=None):
        import scipy.sparse as sp
        A = sp.csc_matrix(C_, dtype=np.complex128)
        A.sum_duplicates()
        A.sort_indices()
        n = A.shape[0]
        if A.shape != (n, n):
            raise DimensionMismatch(-2, f"psPrecRecy needs a square C, got size {A.shape}")
        self.e, self.rec, self.control, self.n = engine, rec, control, n
        self.colptr = np.ascontiguousarray(A.indptr, dtype=np.int64)
        self.rowval = np.ascontiguousarray(A.indices, dtype=np.int64)
        self.nzval = np.ascontiguousarray(A.data, dtype=np.complex128)
        self.p = None if p is None else np.ascontiguousarray(p, dtype=np.int64)
        if self.p is not None and self.p.shape != (n,):
            raise DimensionMismatch(-2, f"p has length {self.p.size}, expected {n}")

        def block(X, k, name):
            if X is None:
                return None
            X = np.asfortranarray(np.asarray(X, dtype=np.complex128).reshape(n, -1))
            if X.shape != (n, k):
                raise DimensionMismatch(-2, f"{name} must be {(n, k)}, got {X.shape}")
            return X
        self.x0 = (block(X0_main, control.r_main, "X0_main"), block(X0_pred, control.r_pred, "X0_pred"),
                   block(X0_bound, 1, "X0_bound"))
        self.Z = _checked(rec.Z, np.complex128, 0, "rec.Z")
        nZ = len(self.Z)
        self.sigma = np.full(nZ, np.nan)
        self.st = PsPrecRecyStats(nZ)
        self._cst = self.st.c_struct()
        self._cc = control.c_struct()
        self._g = rec.c_grid()

    def run(self, i_begin=0, i_end=None):
        i_end = len(self.Z) if i_end is None else i_end
        a, b, c = self.x0
        check(lib().rls_psprecrecy_range(self.e._h, self.n, ptr(self.colptr), ptr(self.rowval), ptr(self.nzval), 0,
                                         ptr(self.p), ptr(self.Z), len(self.Z), C.byref(self._g), C.byref(self._cc),
                                         ptr(a), ptr(b), ptr(c), int(i_begin), int(i_end), ptr(self.sigma),
                                         C.byref(self._cst)), self.e._h)
        self.st.read_scalars(self._cst)
        return self.sigma, self.st


class PrecRecyLanes:
    """psPrecRecy on concurrent lanes of one GPU (no reference counterpart): the traversal is split
    on column boundaries as rls_lane_offsets splits it, and each lane runs the reference's loop on
    its part from its own start (its own Engine, preconditioner built at its first point, both
    recycled spaces), driven from its own host thread (the library calls release the GIL)."""

    def __init__(self, lanes: int, C_, rec: Recursion, control: PsPrecRecyControl, p=None, X0_main=None,
                 X0_pred=None, X0_bound=None, device: int = 0):
        import scipy.sparse as sp
        if lanes < 1:
            raise ArgumentError(-1, f"lanes must be >= 1, got {lanes}")
        A = sp.csc_matrix(C_, dtype=np.complex128)
        nZ = len(rec.Z)
        off = np.zeros(lanes + 1, dtype=np.int64)
        g = rec.c_grid()
        check(lib().rls_lane_offsets(C.byref(g), nZ, lanes, ptr(off)), None)
        self.offs = off
        self.nZ = nZ
        self.engines, self.runs = [], []
        for l in range(lanes):
            sub = Recursion(rec.x_st, rec.x_ed, rec.y_st, rec.y_ed, rec.n_x, rec.n_y, rec.k)
            sub.Z = np.ascontiguousarray(rec.Z[off[l]:off[l + 1]])
            e = Engine(device)
            self.engines.append(e)
            self.runs.append(PrecRecyRun(e, A, sub, control, p=p, X0_main=X0_main, X0_pred=X0_pred,
                                         X0_bound=X0_bound))

    def run(self, j_begin=0, j_end=None):
        """Lane-local points j_begin..j_end−1 of every lane (all lanes at once)."""
        import threading
        errs = [None] * len(self.runs)

        def go(i):
            r = self.runs[i]
            n = len(r.Z)
            b = min(j_begin, n)
            e = n if j_end is None else min(j_end, n)
            if b < e:
                try:
                    r.run(b, e)
                except Exception as exc:  # noqa: BLE001  (re-raised below, first lane first)
                    errs[i] = exc
        th = [threading.Thread(target=go, args=(i,)) for i in range(len(self.runs))]
        for t in th:
            t.start()
        for t in th:
            t.join()
        for e in errs:
            if e is not None:
                raise e
        return self.result()

    def result(self):
        """σ and stats over the whole traversal: per-point arrays in rec.Z order, the point lists
        concatenated lane by lane, times and counts summed."""
        sigma = np.concatenate([r.sigma for r in self.runs])
        st = PsPrecRecyStats(self.nZ)
        for f in PsPrecRecyStats._I:
            setattr(st, f, np.concatenate([getattr(r.st, f) for r in self.runs]))
        for f in PsPrecRecyStats._S:
            setattr(st, f, sum(getattr(r.st, f) for r in self.runs))
        lists = {"pts": "n_pts", "pred_pts": "n_pred_pts", "precond_rebuild_pts": "n_precond_rebuild_pts"}
        for f, cnt in lists.items():
            v = np.zeros(self.nZ, dtype=np.complex128)
            parts = [getattr(r.st, f)[:getattr(r.st, cnt)] for r in self.runs]
            cat = np.concatenate(parts) if parts else v[:0]
            v[:cat.size] = cat
            setattr(st, f, v)
        return sigma, st

    def streams(self):
        return [e.stream_ptr() for e in self.engines]

    def launches(self) -> int:
        return sum(e.launches() for e in self.engines)

    def close(self):
        for e in self.engines:
            e.close()


def psPrecRecy(C_, rec: Recursion, control: PsPrecRecyControl = None, verbose: int = 1, io=None, p=None,
               X0_main=None, X0_pred=None, X0_bound=None, device: int = 0, lanes: int = 1):
    """psPrecRecy (psPrecRecy.jl:617-623; a dense C is made sparse, :1036-1042) →
    (σ_min in rec.Z order, PsPrecRecyStats).

    ``p`` is the column order the reference takes from SPQR (``qr(C).cpiv``, :625), which needs
    SuiteSparse; None here takes reverse Cuthill–McKee of C + Cᵀ as the stand-in fill-reducing
    order.  ``X0_main`` (n × r_main), ``X0_pred`` (n × r_pred) and ``X0_bound`` (n × 1) stand in
    for the reference's rand! draws; None draws fixed uniform [0,1) blocks on the device.
    ``lanes`` > 1 runs column-aligned parts of the traversal concurrently (PrecRecyLanes); 1
    keeps the reference's single traversal.
    """
    import scipy.sparse as sp
    control = control or PsPrecRecyControl()
    io = io if io is not None else sys.stdout
    A = sp.csc_matrix(C_, dtype=np.complex128)
    if p is None:
        from scipy.sparse.csgraph import reverse_cuthill_mckee
        S = abs(A) + abs(A.T)
        p = np.ascontiguousarray(reverse_cuthill_mckee(S.tocsr(), symmetric_mode=True), dtype=np.int64)
    if verbose >= 1:
        io.write("[psPrecRecy] rec: x_range=[%.6f, %.6f], y_range=[%.6f, %.6f], n_x=%d, n_y=%d, k=%d, n_pts=%d\n"
                 % (rec.x_st, rec.x_ed, rec.y_st, rec.y_ed, rec.n_x, rec.n_y, rec.k, rec.n_x * rec.n_y))
        io.write("[psPrecRecy] control:\n")
        for f in control.__dataclass_fields__:
            io.write(f"  {f} = {getattr(control, f)!r}\n")
    if lanes > 1:
        ls = PrecRecyLanes(lanes, A, rec, control, p=p, X0_main=X0_main, X0_pred=X0_pred, X0_bound=X0_bound,
                           device=device)
        try:
            sigma, st = ls.run()
        finally:
            ls.close()
        return sigma, st
    eng = _engine(device)
    if verbose >= 1:
        eng.set_log(lambda line: io.write(line + "\n"), verbose)
    else:
        eng.set_log(None)
    try:
        run = PrecRecyRun(eng, A, rec, control, p=p, X0_main=X0_main, X0_pred=X0_pred, X0_bound=X0_bound)
        sigma, st = run.run()
    finally:
        eng.set_log(None)
    if verbose >= 1:
        io.write(f"Total M vec apps for pred singular value problem: {int(st.pred_M_vec_apps.sum())}\n")
        io.write(f"Total L vec apps for pred singular value problem: {int(st.pred_L_vec_apps.sum())}\n")
        io.write(f"Total it for pred singular value problem: {st.n_pred_it}\n")
        io.write(f"Total pt for pred singular value problem: {st.n_pred_pts}\n")
        io.write(f"Total preconditioner points: {st.n_precond_rebuild_pts}\n")
        io.write(f"Total M vec apps for singular value problem: {int(st.main_M_vec_apps.sum())}\n")
        io.write(f"Total L vec apps for singular value problem: {int(st.main_L_vec_apps.sum())}\n")
        io.write(f"Total it for singular value problem: {st.n_it}\n")
        io.write(f"Total pt for singular value problem: {st.n_pts}\n")
    return sigma, st
