"""psTriRecy and psPrecRecy over several GPUs: one rank per GPU, each on a column-aligned share
of the grid.

No reference counterpart (the reference walks the whole traversal in one process).  The
zigzag traversal (recuGrid.jl:157-176) is cut into `world` near-equal contiguous runs of whole
traversal columns (k points each); rank i runs psTriRecy from an empty recycled space on run i,
exactly the reference's loop on that sub-grid, with no collective on the data path.  The one
exchange step is the final gather of σ and the per-point statistics (NCCL all_gather over
NVLink for the nccl backend, gloo on the host otherwise), after which every rank holds the
whole grid's results in rec.Z order.
"""
from __future__ import annotations

import numpy as np

from .grid import Recursion


def column_shares(nZ: int, k: int, world: int) -> np.ndarray:
    """Start offsets (length world + 1) of the ranks' shares: the traversal's columns (k points
    each) split into `world` near-equal contiguous runs."""
    col = max(1, int(k))
    ncols = -(-nZ // col)
    if world < 1 or world > ncols:
        raise ValueError(f"{world} ranks for {ncols} columns of the traversal")
    offs = np.array([min(nZ, (r * ncols // world) * col) for r in range(world)] + [nZ], dtype=np.int64)
    return offs


_STAT_ARRAYS = ("p_count", "r_recy", "M_vec_apps", "M_vec_apps_no_recycle", "R_vec_apps", "refine_it")


def gather_shares(sigma_local, arrays_local: dict, offs, group=None):
    """All-gather of each rank's share (σ and the int64 per-point arrays) into full-length arrays
    on every rank.  Shares are padded to the longest share for the collective."""
    import torch
    import torch.distributed as dist
    world = len(offs) - 1
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    if world == 1:
        return np.asarray(sigma_local), {k: np.asarray(v) for k, v in arrays_local.items()}
    dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    L = int(np.max(np.diff(offs)))
    names = list(arrays_local)
    buf = torch.zeros((1 + len(names), L), dtype=torch.float64, device=dev)
    n_own = int(offs[rank + 1] - offs[rank])
    buf[0, :n_own] = torch.as_tensor(np.asarray(sigma_local, dtype=np.float64)[:n_own], device=dev)
    for q, nm in enumerate(names):
        buf[1 + q, :n_own] = torch.as_tensor(np.asarray(arrays_local[nm], dtype=np.float64)[:n_own], device=dev)
    parts = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf, group=group)
    nZ = int(offs[-1])
    sigma = np.empty(nZ)
    arrays = {nm: np.empty(nZ, dtype=np.int64) for nm in names}
    for r in range(world):
        a, b = int(offs[r]), int(offs[r + 1])
        h = parts[r].cpu().numpy()
        sigma[a:b] = h[0, :b - a]
        for q, nm in enumerate(names):
            arrays[nm][a:b] = np.rint(h[1 + q, :b - a]).astype(np.int64)
    return sigma, arrays


def psTriRecy_ranks(C_, rec: Recursion, control=None, X0=None, group=None, lanes: int = 1, device: int = None,
                    solve=None):
    """psTriRecy on this rank's column-aligned share of rec.Z, then the gather of σ and the
    per-point statistics.  Returns (σ over the whole grid, PsTriRecyStats with the gathered
    per-point arrays and this rank's scalars summed over ranks).  `solve(C_, sub_rec, control,
    X0)` replaces the per-rank solver (default: rls_b200.psTriRecy on `device`, `lanes` lanes)."""
    import torch.distributed as dist
    from .solvers import PsTriRecyControl, PsTriRecyStats, psTriRecy
    control = control or PsTriRecyControl()
    world = dist.get_world_size(group) if dist.is_initialized() else 1
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    offs = column_shares(len(rec.Z), rec.k, world)
    sub = Recursion(rec.x_st, rec.x_ed, rec.y_st, rec.y_ed, rec.n_x, rec.n_y, rec.k)
    sub.Z = np.ascontiguousarray(rec.Z[offs[rank]:offs[rank + 1]])
    if solve is None:
        dev = rank if device is None else device
        sig_l, st_l = psTriRecy(C_, sub, control, verbose=0, X0=X0, device=dev, lanes=lanes)
    else:
        sig_l, st_l = solve(C_, sub, control, X0)
    sigma, arrays = gather_shares(sig_l, {nm: getattr(st_l, nm) for nm in _STAT_ARRAYS}, offs, group)
    st = PsTriRecyStats.alloc(len(rec.Z))
    for nm in _STAT_ARRAYS:
        setattr(st, nm, arrays[nm])
    scal = np.array([st_l.n_it, st_l.n_pts], dtype=np.float64)
    if world > 1:
        import torch
        dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
        t = torch.as_tensor(scal, device=dev)
        dist.all_reduce(t, group=group)
        scal = t.cpu().numpy()
    st.n_it, st.n_pts = int(scal[0]), int(scal[1])
    st.preprocess_time_ns = st_l.preprocess_time_ns
    return sigma, st


_PREC_ARRAYS = ("p_count", "pred_p_count", "r_recy", "main_M_vec_apps", "main_M_vec_apps_no_recycle",
                "main_L_vec_apps", "pred_M_vec_apps", "pred_L_vec_apps", "main_refine_it", "pred_refine_it")
_PREC_SCALARS = ("main_recycle_time_ns", "main_refine_time_ns", "main_update_time_ns", "pred_recycle_time_ns",
                 "pred_refine_time_ns", "pred_update_time_ns", "precond_time_ns", "n_it", "n_pred_it", "n_pts",
                 "n_pred_pts", "n_precond_rebuild_pts")


def psPrecRecy_ranks(C_, rec: Recursion, control=None, group=None, lanes: int = 1, device: int = None, solve=None,
                     **kw):
    """psPrecRecy on this rank's column-aligned share of rec.Z (its own preconditioner, built at
    the share's first point, and its own recycled spaces), then the gather of σ and the per-point
    statistics as psTriRecy_ranks gathers them.  The point lists (pts, pred_pts,
    precond_rebuild_pts) stay per rank; the scalar counters and times are summed over ranks.
    `solve(C_, sub_rec, control)` replaces the per-rank solver (default: rls_b200.psPrecRecy on
    `device` with `lanes` lanes and the keyword arguments kw)."""
    import torch.distributed as dist
    from .solvers import PsPrecRecyControl, PsPrecRecyStats, psPrecRecy
    control = control or PsPrecRecyControl()
    world = dist.get_world_size(group) if dist.is_initialized() else 1
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    offs = column_shares(len(rec.Z), rec.k, world)
    sub = Recursion(rec.x_st, rec.x_ed, rec.y_st, rec.y_ed, rec.n_x, rec.n_y, rec.k)
    sub.Z = np.ascontiguousarray(rec.Z[offs[rank]:offs[rank + 1]])
    if solve is None:
        dev = rank if device is None else device
        sig_l, st_l = psPrecRecy(C_, sub, control, verbose=0, device=dev, lanes=lanes, **kw)
    else:
        sig_l, st_l = solve(C_, sub, control)
    sigma, arrays = gather_shares(sig_l, {nm: getattr(st_l, nm) for nm in _PREC_ARRAYS}, offs, group)
    st = PsPrecRecyStats(len(rec.Z))
    for nm in _PREC_ARRAYS:
        setattr(st, nm, arrays[nm])
    for nm in ("pts", "pred_pts", "precond_rebuild_pts"):
        setattr(st, nm, getattr(st_l, nm))
    scal = np.array([getattr(st_l, nm) for nm in _PREC_SCALARS], dtype=np.float64)
    if world > 1:
        import torch
        dev_t = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
        t = torch.as_tensor(scal, device=dev_t)
        dist.all_reduce(t, group=group)
        scal = t.cpu().numpy()
    for nm, v in zip(_PREC_SCALARS, scal):
        setattr(st, nm, int(v))
    return sigma, st
