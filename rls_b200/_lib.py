"""ctypes binding of librls_b200.so (the C ABI declared in include/rls_b200.h).

The library is loaded from this package directory; a missing library raises
immediately — there is no fallback implementation.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "librls_b200.so")


class c64(C.Structure):
    _fields_ = [("re", C.c_double), ("im", C.c_double)]


class rls_grid(C.Structure):
    _fields_ = [("x_st", C.c_double), ("x_ed", C.c_double), ("y_st", C.c_double), ("y_ed", C.c_double),
                ("n_x", C.c_int64), ("n_y", C.c_int64), ("k", C.c_int64)]


class rls_pstrirecy_control(C.Structure):
    _fields_ = [("tol", C.c_double), ("normC", C.c_double), ("shift", C.c_double), ("gap_tau", C.c_double),
                ("gap_tau_scale", C.c_double), ("recy_tau", C.c_double),
                ("recycle_fail_dist_thresh", C.c_double), ("r", C.c_int64), ("p", C.c_int64),
                ("p_min", C.c_int64), ("lobpcg_tol_scale", C.c_double), ("lobpcg_side", C.c_uint32),
                ("implict_update", C.c_uint8), ("implict_recycle", C.c_uint8), ("collect_timing", C.c_uint8),
                ("_pad0", C.c_uint8), ("inner_verbose_override", C.c_int64)]


class rls_pstrirecy_stats(C.Structure):
    _fields_ = [("p_count", C.POINTER(C.c_int64)), ("r_recy", C.POINTER(C.c_int64)), ("pts", C.POINTER(c64)),
                ("M_vec_apps", C.POINTER(C.c_int64)), ("M_vec_apps_no_recycle", C.POINTER(C.c_int64)),
                ("R_vec_apps", C.POINTER(C.c_int64)), ("refine_it", C.POINTER(C.c_int64)),
                ("preprocess_time_ns", C.c_uint64), ("recycle_time_ns", C.c_uint64), ("qr_time_ns", C.c_uint64),
                ("refine_time_ns", C.c_uint64), ("update_time_ns", C.c_uint64),
                ("mv_stats_available", C.c_uint8), ("_pad0", C.c_uint8 * 7), ("n_it", C.c_int64),
                ("n_pts", C.c_int64), ("dsdx", C.POINTER(C.c_double)), ("dsdy", C.POINTER(C.c_double))]


class rls_lobpcg_control(C.Structure):
    _fields_ = [("m", C.c_int64), ("n", C.c_int64), ("r", C.c_int64), ("maxit", C.c_int64), ("tol", C.c_double),
                ("side", C.c_uint32), ("verbose", C.c_int32), ("normC", C.c_double), ("orth_type", C.c_int32),
                ("conv_thresh_type", C.c_int32), ("conv_first", C.c_int64), ("conv_last", C.c_int64)]


class rls_psprecrecy_control(C.Structure):
    _fields_ = [("tol", C.c_double), ("lobpcg_tol_scale", C.c_double), ("main_normC", C.c_double),
                ("main_tau", C.c_double), ("shift", C.c_double), ("gap_tau", C.c_double),
                ("recycle_fail_dist_thresh", C.c_double), ("tol_pred", C.c_double),
                ("lobpcg_pred_tol_scale", C.c_double), ("pred_conv_first", C.c_int64), ("pred_conv_last", C.c_int64),
                ("pred_tau", C.c_double), ("idx_cutoff_pred", C.c_double), ("pred_orth_type", C.c_int32),
                ("_pad0", C.c_int32), ("pred_conv_thresh_type", C.c_int64), ("lambda_lower_min", C.c_double),
                ("lambda_upper_max", C.c_double), ("r_main", C.c_int64), ("p_main", C.c_int64),
                ("p_min_main", C.c_int64), ("main_implict_update", C.c_uint8), ("main_implict_recycle", C.c_uint8),
                ("_pad1", C.c_uint8 * 6), ("r_pred", C.c_int64), ("p_pred", C.c_int64), ("p_min_pred", C.c_int64),
                ("pred_implict_update", C.c_uint8), ("pred_implict_recycle", C.c_uint8), ("_pad2", C.c_uint8 * 6),
                ("hsl_tol", C.c_double), ("hsl_cntl_1", C.c_double), ("hsl_cntl_2", C.c_double),
                ("hsl_icntl_1", C.c_int64), ("hsl_icntl_2", C.c_int64), ("gamma_tol", C.c_double),
                ("lambda_n_tol", C.c_double), ("inner_verbose_override", C.c_int64), ("collect_timing", C.c_uint8),
                ("_pad3", C.c_uint8 * 7)]


class rls_psprecrecy_stats(C.Structure):
    _fields_ = [(f, C.POINTER(C.c_int64)) for f in ("p_count", "pred_p_count", "r_recy")] + \
               [(f, C.POINTER(c64)) for f in ("pts", "pred_pts", "precond_rebuild_pts")] + \
               [(f, C.POINTER(C.c_int64)) for f in ("main_M_vec_apps", "main_M_vec_apps_no_recycle", "main_L_vec_apps",
                                                    "pred_M_vec_apps", "pred_L_vec_apps")] + \
               [(f, C.c_uint64) for f in ("main_recycle_time_ns", "main_refine_time_ns", "main_update_time_ns",
                                          "pred_recycle_time_ns", "pred_refine_time_ns", "pred_update_time_ns",
                                          "precond_time_ns")] + \
               [(f, C.c_int64) for f in ("n_it", "n_pred_it", "n_pts", "n_pred_pts", "n_precond_rebuild_pts")] + \
               [(f, C.POINTER(C.c_int64)) for f in ("main_refine_it", "pred_refine_it")]


LOG_FN = C.CFUNCTYPE(None, C.c_char_p, C.c_void_p)
P = C.c_void_p

# name -> (restype, argtypes)
SIGNATURES = {
    "rls_ctx_create": (C.c_int, [C.POINTER(C.c_void_p), C.c_int]),
    "rls_ctx_destroy": (None, [P]),
    "rls_last_error": (C.c_char_p, [P]),
    "rls_status_string": (C.c_char_p, [C.c_int]),
    "rls_ctx_set_log": (C.c_int, [P, LOG_FN, P, C.c_int]),
    "rls_grid_zigzag": (C.c_int, [C.POINTER(rls_grid), P]),
    "rls_grid_linear": (C.c_int, [C.POINTER(rls_grid), P]),
    "rls_grid_spiral": (C.c_int, [C.POINTER(rls_grid), P]),
    "rls_natural_perm": (C.c_int, [C.POINTER(rls_grid), P, C.c_int64, P]),
    "rls_reorder_to_natural": (C.c_int, [C.POINTER(rls_grid), P, C.c_int64, P, P]),
    "rls_reorder_to_natural_grid": (C.c_int, [C.POINTER(rls_grid), P, C.c_int64, P, P]),
    "rls_mtx_info": (C.c_int, [C.c_char_p, P, P, P, P]),
    "rls_mtx_read_csc": (C.c_int, [C.c_char_p, C.c_int, C.c_int64, P, P, P, P]),
    "rls_mtx_read_dense": (C.c_int, [C.c_char_p, P, C.c_int64]),
    "rls_set_schur": (C.c_int, [P, C.c_int64, P, C.c_int64]),
    "rls_set_schur_copy": (C.c_int, [P, P]),
    "rls_set_sparse_tri": (C.c_int, [P, C.c_int64, P, P, P, C.c_int, P]),
    "rls_band_order": (C.c_int, [C.c_int64, P, P, C.c_int, P, P, P]),
    "rls_band_set_panel": (C.c_int, [P, C.c_int]),
    "rls_band_info": (C.c_int, [P, P, P, P, P, P]),
    "rls_pstrirecy_sparse": (C.c_int, [P, C.c_int64, P, P, P, C.c_int, P, P, C.c_int64, C.POINTER(rls_grid),
                                       C.POINTER(rls_pstrirecy_control), P, P, C.POINTER(rls_pstrirecy_stats)]),
    "rls_set_trsm_ctas": (C.c_int, [P, C.c_int]),
    "rls_set_trsm_backoff": (C.c_int, [P, C.c_int]),
    "rls_ctx_set_graphs": (C.c_int, [P, C.c_int]),
    "rls_ctx_set_host_wait": (C.c_int, [P, C.c_int]),
    "rls_pstrirecy_schur": (C.c_int, [P, P, C.c_int64, C.POINTER(rls_grid), C.POINTER(rls_pstrirecy_control), P, P,
                                      C.POINTER(rls_pstrirecy_stats)]),
    "rls_pstrirecy_schur_range": (C.c_int, [P, P, C.c_int64, C.POINTER(rls_grid), C.POINTER(rls_pstrirecy_control), P,
                                            C.c_int64, C.c_int64, P, C.POINTER(rls_pstrirecy_stats)]),
    "rls_lobpcg_svd_invtri": (C.c_int, [P, c64, P, C.POINTER(rls_lobpcg_control), P, P, P, P]),
    "rls_lobpcg_svd": (C.c_int, [P, C.c_int, c64, C.c_int, P, C.POINTER(rls_lobpcg_control), P, P, P, P]),
    "rls_ctx_stream": (C.c_void_p, [P]),
    "rls_tsqr_r_noalloc": (C.c_int, [P, C.c_int64, C.c_int64, C.c_int, P, P]),
    "rls_sigma_grad": (C.c_int, [P, c64, P, C.c_int, P, P, P, P, P]),
    "rls_set_schur_vectors": (C.c_int, [P, P, C.c_int64]),
    "rls_sigma_grad_pattern": (C.c_int, [P, P, P, C.c_int64, P, P, C.c_int, P]),
    "rls_sparse_upload_csc": (C.c_int, [P, C.c_int64, C.c_int64, P, P, P, C.c_int]),
    "rls_spmm_shifted": (C.c_int, [P, c64, C.c_int, C.c_int, P, C.c_int64, P, C.c_int64]),
    "rls_spmm_shifted_dev": (C.c_int, [P, c64, C.c_int, C.c_int, P, C.c_int64, P, C.c_int64]),
    "rls_lltp_upload": (C.c_int, [P, C.c_int64, P, P, P, P, P, C.c_int]),
    "rls_lltp_ldiv": (C.c_int, [P, C.c_int, P, C.c_int64, P, C.c_int64]),
    "rls_lltp_ldiv_dev": (C.c_int, [P, C.c_int, P, C.c_int64, P, C.c_int64]),
    "rls_ic_factor": (C.c_int, [C.c_int64, P, P, P, C.c_int, c64, C.c_double, C.c_double, C.c_double, C.c_int64,
                                C.c_int64, P, C.c_int64, P, P, P, P, P]),
    "rls_lane_offsets": (C.c_int, [C.POINTER(rls_grid), C.c_int64, C.c_int, P]),
    "rls_pstrirecy_schur_lanes": (C.c_int, [P, C.c_int, P, C.c_int64, C.POINTER(rls_grid),
                                            C.POINTER(rls_pstrirecy_control), P, P, C.POINTER(rls_pstrirecy_stats)]),
    "rls_pstrirecy_schur_lanes_range": (C.c_int, [P, C.c_int, P, C.c_int64, C.POINTER(rls_grid),
                                                  C.POINTER(rls_pstrirecy_control), P, C.c_int64, C.c_int64, P,
                                                  C.POINTER(rls_pstrirecy_stats)]),
    "rls_psprecrecy": (C.c_int, [P, C.c_int64, P, P, P, C.c_int, P, P, C.c_int64, C.POINTER(rls_grid),
                                 C.POINTER(rls_psprecrecy_control), P, P, P, P, C.POINTER(rls_psprecrecy_stats)]),
    "rls_psprecrecy_range": (C.c_int, [P, C.c_int64, P, P, P, C.c_int, P, P, C.c_int64, C.POINTER(rls_grid),
                                       C.POINTER(rls_psprecrecy_control), P, P, P, C.c_int64, C.c_int64, P,
                                       C.POINTER(rls_psprecrecy_stats)]),
    "rls_ctx_launches": (C.c_int64, [P]),
    "rls_ctx_set_ritz_basis": (C.c_int, [P, C.c_int]),
    "rls_ctx_set_batch": (C.c_int, [P, C.c_int]),
    "rls_ctx_set_profile": (C.c_int, [P, C.c_int]),
    "rls_ctx_profile_get": (C.c_int, [P, C.c_int, P, P, P]),
    # kernel-level test entry points (include/rls_b200_testing.h)
    "rls_test_setup": (C.c_int, [P, C.c_int, C.c_int]),
    "rls_test_trsm": (C.c_int, [P, c64, C.c_int, C.c_int, P, P]),
    "rls_test_lltp_plan_dense": (C.c_int, [C.c_int64, P, P, P, C.c_int, C.c_int, P, P, P]),
    "rls_test_trmm": (C.c_int, [P, C.c_int, C.c_int, P, P]),
    "rls_test_qr": (C.c_int, [P, C.c_int64, C.c_int, P, P, P]),
    "rls_test_svd_rr": (C.c_int, [P, C.c_int, C.c_int, C.c_int, C.c_int, P, P, P, P]),
    "rls_test_heev_rr": (C.c_int, [P, C.c_int, C.c_int, P, P, c64, C.c_double, C.c_double, P, P, P, P]),
    "rls_test_recip": (C.c_int, [P, C.c_int64, P, P, P]),
    "rls_test_band_r": (C.c_int, [P, c64, P, C.c_int64, P, P]),
    "rls_test_band_factor": (C.c_int, [P, c64]),
    "rls_test_space_update": (C.c_int, [P, c64, P, C.c_double, C.c_int, C.c_int]),
    "rls_test_space_get": (C.c_int, [P, P, P, P, P, P, P, P, P]),
    "rls_test_recycle": (C.c_int, [P, c64, C.c_double, C.c_double, P, P, P, P, P]),
}

_lib = None


def lib():
    """Loads librls_b200.so once; raises if it is missing (no fallback path exists)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"librls_b200.so not built at {LIB_PATH}; run `python -m rls_b200.build`")
        h = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(h, name)
            f.restype = res
            f.argtypes = args
        _lib = h
    return _lib


class RLSError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{msg} (status {status})")
        self.status = status


class DimensionMismatch(RLSError, ValueError):
    """Raised where the reference throws DimensionMismatch."""


class ArgumentError(RLSError, ValueError):
    """Raised where the reference throws ArgumentError."""


class SingularException(RLSError):
    """Raised where the reference throws LinearAlgebra.SingularException."""


def check(status, ctx=None):
    if status == 0:
        return
    L = lib()
    msg = L.rls_last_error(ctx).decode()
    if not msg:
        msg = L.rls_status_string(status).decode()
    if status == -2:
        raise DimensionMismatch(status, msg)
    if status == -1:
        raise ArgumentError(status, msg)
    if status == -8:
        raise SingularException(status, msg)
    raise RLSError(status, msg)


def ptr(a):
    return C.c_void_p(a.ctypes.data) if a is not None else None
