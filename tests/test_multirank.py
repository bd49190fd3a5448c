"""Host logic of the multi-rank benchmark, on CPU with two `gloo` ranks.

Each rank runs its own traversal of the grid from the first column of its share, with no
collective on the data path; the only exchange is the max over ranks of the timings.
"""
import json
import os
import socket

import numpy as np
import pytest

import bench


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import torch.distributed as dist
    from datetime import timedelta
    from rls_b200.grid import recursion_grid
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=timedelta(seconds=60))
    try:
        rec = recursion_grid(*bench.GRID)
        off = bench.column_offset(rank, world, len(rec.Z), bench.GRID[6])
        t = bench.max_over_ranks(10.0 * (rank + 1), world, "cpu")
        first = rec.Z[off]
        with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
            json.dump({"off": off, "t": t, "first": [first.real, first.imag]}, f)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2])
def test_column_shares_and_max_over_ranks(tmp_path, world):
    import torch.multiprocessing as mp
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    res = []
    for r in range(world):
        with open(tmp_path / f"rank{r}.json") as f:
            res.append(json.load(f))
    x_st, x_ed, y_st, y_ed, n_x, n_y, k = bench.GRID
    offs = [r["off"] for r in res]
    assert offs[0] == 0
    assert all(o % k == 0 for o in offs)
    assert offs == sorted(set(offs))                      # distinct, increasing shares
    assert all(r["t"] == 10.0 * world for r in res)       # every rank sees the slowest rank's time
    # every rank starts at the first row of y of a grid column in one of the serpentine strips
    dy = (y_ed - y_st) / (n_y - 1)
    for r in res:
        strip = r["off"] // (n_x * k)
        assert np.isclose(r["first"][1], y_st + strip * k * dy)


@pytest.mark.parametrize("world", [1, 2, 4, 8])
def test_column_shares_fit_ten_lanes_per_rank(world):
    """Ranks' shares are near-equal and column-aligned; each holds the benchmark's twenty
    lanes of at least (warm-up + timed steps) × the step it picks."""
    from rls_b200.grid import recursion_grid
    k = bench.GRID[6]
    nZ = len(recursion_grid(*bench.GRID).Z)
    offs = [bench.column_offset(r, world, nZ, k) for r in range(world)] + [nZ]
    sizes = np.diff(offs)
    assert sizes.min() > 0 and sizes.max() - sizes.min() <= k
    nst = 3 + 5
    lanes, s = bench.lane_plan(nZ, world, 20, 200, nst, k)
    assert lanes == 20 and s >= 20
    for size in sizes:
        ncols = size // k
        smallest_lane = (ncols // lanes) * k
        assert smallest_lane >= nst * s


def test_column_offset_rejects_more_ranks_than_columns():
    with pytest.raises(SystemExit):
        bench.column_offset(0, 2001, 200 * 200, 20)


def _fake_solve(C_, sub, control, X0):
    """Stands in for the per-rank GPU solve: σ = |z| + 1 and per-point counters from z."""
    from rls_b200.solvers import PsTriRecyStats
    st = PsTriRecyStats.alloc(len(sub.Z))
    st.refine_it[:] = (np.round(sub.Z.real * 1000).astype(np.int64) % 7)
    st.p_count[:] = np.arange(len(sub.Z))               # local index: shows each share restarts
    st.n_it, st.n_pts = int(st.refine_it.sum()), len(sub.Z)
    return np.abs(sub.Z) + 1.0, st


def _ranks_main(rank, world, port, out_dir):
    import torch.distributed as dist
    from datetime import timedelta
    from rls_b200.grid import recursion_grid
    from rls_b200.distributed import psTriRecy_ranks
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=timedelta(seconds=60))
    try:
        rec = recursion_grid(0.45, 0.55, 0.0, 0.1, 30, 12, 4)
        sig, st = psTriRecy_ranks(None, rec, solve=_fake_solve)
        np.savez(os.path.join(out_dir, f"ranks{rank}.npz"), sig=sig, refine_it=st.refine_it, p_count=st.p_count,
                 n_it=st.n_it, n_pts=st.n_pts)
    finally:
        dist.destroy_process_group()


def test_library_gather_of_rank_shares(tmp_path):
    """rls_b200.distributed.psTriRecy_ranks on two gloo ranks: every rank ends with the whole
    grid's σ and per-point statistics in rec.Z order, each share solved from its own start."""
    import torch.multiprocessing as mp
    from rls_b200.grid import recursion_grid
    from rls_b200.distributed import column_shares
    world = 2
    mp.start_processes(_ranks_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    rec = recursion_grid(0.45, 0.55, 0.0, 0.1, 30, 12, 4)
    offs = column_shares(len(rec.Z), rec.k, world)
    ref_sig = np.abs(rec.Z) + 1.0
    for r in range(world):
        d = np.load(tmp_path / f"ranks{r}.npz")
        assert np.array_equal(d["sig"], ref_sig)
        assert np.array_equal(d["refine_it"], np.round(rec.Z.real * 1000).astype(np.int64) % 7)
        local = np.concatenate([np.arange(offs[q + 1] - offs[q]) for q in range(world)])
        assert np.array_equal(d["p_count"], local)
        assert int(d["n_pts"]) == len(rec.Z)
    assert offs[1] % rec.k == 0 and 0 < offs[1] < len(rec.Z)


def _fake_prec_solve(C_, sub, control):
    """Stands in for the per-rank psPrecRecy: σ = |z| + 2 and per-point counters from z."""
    from rls_b200.solvers import PsPrecRecyStats
    st = PsPrecRecyStats(len(sub.Z))
    st.main_refine_it[:] = (np.round(sub.Z.imag * 1000).astype(np.int64) % 5)
    st.p_count[:] = np.arange(len(sub.Z))
    st.n_pts = int(np.sum(st.main_refine_it > 0))
    st.n_precond_rebuild_pts = 1
    return np.abs(sub.Z) + 2.0, st


def _prec_ranks_main(rank, world, port, out_dir):
    import torch.distributed as dist
    from datetime import timedelta
    from rls_b200.grid import recursion_grid
    from rls_b200.distributed import psPrecRecy_ranks
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=timedelta(seconds=60))
    try:
        rec = recursion_grid(-1.6, 0.8, -1.55, 1.55, 24, 12, 4)
        sig, st = psPrecRecy_ranks(None, rec, solve=_fake_prec_solve)
        np.savez(os.path.join(out_dir, f"prec{rank}.npz"), sig=sig, it=st.main_refine_it, p_count=st.p_count,
                 n_pts=st.n_pts, builds=st.n_precond_rebuild_pts)
    finally:
        dist.destroy_process_group()


def test_library_gather_of_psprecrecy_shares(tmp_path):
    """rls_b200.distributed.psPrecRecy_ranks on two gloo ranks: σ and the per-point counters of
    both shares on every rank in rec.Z order; scalar counters summed (one preconditioner build
    per rank)."""
    import torch.multiprocessing as mp
    from rls_b200.grid import recursion_grid
    from rls_b200.distributed import column_shares
    world = 2
    mp.start_processes(_prec_ranks_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    rec = recursion_grid(-1.6, 0.8, -1.55, 1.55, 24, 12, 4)
    offs = column_shares(len(rec.Z), rec.k, world)
    it_ref = np.round(rec.Z.imag * 1000).astype(np.int64) % 5
    for r in range(world):
        d = np.load(tmp_path / f"prec{r}.npz")
        assert np.array_equal(d["sig"], np.abs(rec.Z) + 2.0)
        assert np.array_equal(d["it"], it_ref)
        local = np.concatenate([np.arange(offs[q + 1] - offs[q]) for q in range(world)])
        assert np.array_equal(d["p_count"], local)
        assert int(d["n_pts"]) == int(np.sum(it_ref > 0))
        assert int(d["builds"]) == world
