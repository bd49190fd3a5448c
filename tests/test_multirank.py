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
