"""B200 σ_min(C − zI) grid engine — the psTriRecy / psPrecRecy hot path of kuandeng/rls on sm_100a.

Public names mirror the reference (src/core/recuGrid.jl, src/core/psTriRecy.jl,
src/core/psPrecRecy.jl, src/core/lobpcgSvd.jl).  All per-grid-point work runs in librls_b200.so; there is
no CPU fallback.
"""
import os as _os

# Concurrent lanes (rls_b200.Lanes) run one CUDA stream each; with the default 8 hardware
# work queues more than 8 streams share queues and serialise.  The CUDA runtime reads this
# when it initialises in this process, so it is set before any CUDA call (a value the
# caller set is kept).
_os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

from .grid import (Recursion, recursion_grid, recursion_grid_zigzag, recursion_grid_linear,
                   recursion_grid_spiral, recursion_natural_permutation, reorder_to_natural,
                   reorder_to_natural_grid)
from .solvers import (PsTriRecyControl, PsTriRecyStats, LobpcgSvdControl, Engine, Lanes, ShiftedMat, SparseLLTP,
                      SparseLLTP_AD, SchurFactor, SparseTri, band_order, pre_process, psTriRecy, ic_factor, get_hsl_LLTP, PsPrecRecyControl,
                      PsPrecRecyStats, PrecRecyRun, PrecRecyLanes, psPrecRecy)
from ._lib import RLSError, ArgumentError, DimensionMismatch, SingularException
from .operators import MulChainMat, NormalMat, IdentityMat, PermMat, InvMat, FilledMat, mul_coupled
from .distributed import psTriRecy_ranks, psPrecRecy_ranks, column_shares
from .mtx import loaddata, load_mtx, save_run

__all__ = [
    "Recursion", "recursion_grid", "recursion_grid_zigzag", "recursion_grid_linear", "recursion_grid_spiral",
    "recursion_natural_permutation", "reorder_to_natural", "reorder_to_natural_grid", "PsTriRecyControl",
    "PsTriRecyStats", "LobpcgSvdControl", "Engine", "Lanes", "ShiftedMat", "SparseLLTP", "SchurFactor", "SparseTri", "band_order",
    "pre_process",
    "psTriRecy", "ic_factor", "get_hsl_LLTP", "SparseLLTP_AD", "mul_coupled", "MulChainMat", "NormalMat", "IdentityMat", "PermMat", "InvMat",
    "FilledMat", "RLSError", "ArgumentError", "DimensionMismatch", "SingularException", "PsPrecRecyControl",
    "PsPrecRecyStats", "PrecRecyRun", "PrecRecyLanes", "psPrecRecy", "psTriRecy_ranks", "psPrecRecy_ranks", "column_shares",
    "loaddata", "load_mtx", "save_run",
]
