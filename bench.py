#!/usr/bin/env python
"""σ_min grid-point throughput of psTriRecy on the B200 (one JSON line on rank 0).

Workload: the reference's sprand case on its full grid — N = 4000 sparse random C
(example/sprand/sprand.jl:11-27, NumPy PCG64 instance with the script's seed),
densified and reduced once to its complex Schur factor on the host (timed apart,
as the reference's preprocess_time_ns), 200 × 200 grid on [0.45,0.55]×[0,0.1],
k = 20, PsTriRecyControl(normC=3.2, tol=1e-4, p_min=1, p=60, recy_tau=1.6),
complex128 throughout.

A step is `--chunk` consecutive points of each lane's part of the traversal,
processed with the lane's recycled space carried from the previous step exactly as
the reference's loop carries it; W warm-up steps, then K timed steps.  The Schur
factor's tiles (132 MB; 256 MB dense) and every lane's scaled copy of them (132 MB
each) are larger than the 126 MB L2, so every step streams them from HBM.

  value : points / device time of the K timed steps, Schur factor resident in HBM.
          The traversal is split on column boundaries (k points) into --lanes
          near-equal concurrent lanes
          (rls_b200.Lanes: one context, stream and host thread per lane); a step is
          --chunk lane-local points in every lane, and the K timed steps run as one
          lane-parallel call (no wait across lanes between steps); device time is the
          max over the lanes' streams of CUDA-event spans.  single_lane repeats the timed steps
          with one lane (the reference's single recycled space).
  e2e   : fresh lane contexts through the public C ABI with host buffers: upload
          of the Schur factor from host memory (to lane 0, whose device copy the
          other lanes share) plus steps 0..W+K-1 (grid points in, σ out), wall clock.
  --impl reference : the CPU restatement (oracle/, the reference's algorithm with
          LAPACK through SciPy on all host cores) on the same traversal, each step
          a bounded sample of --ref-chunk points.

Multi-GPU (torchrun): every rank takes a contiguous, column-aligned share of the grid
and splits it into --lanes lanes (independent recycled spaces; lanes per GPU fixed, the
step shrinks to fit where a rank's share of the grid is small); the only
collectives are the broadcast of T before timing and the max over ranks of the
timings.
"""
from __future__ import annotations

import argparse
import json
import os

# one hardware work queue per lane stream (read by the CUDA runtime at initialisation)
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "σ_min grid pts/s (psTriRecy, sprand N=4000, 200×200 grid, k=20, tol 1e-4)"
GRID = (0.45, 0.55, 0.0, 0.1, 200, 200, 20)
N_MAT = 4000
NORMC = 3.2
NCU_TRSM_TRAFFIC = 132.54e6 + 3.81e6   # DRAM bytes per k_trsm_half launch (ncu, n = 4000, k = 6)
WORKLOAD = "sprand4000"
# The dense Schur-factor workloads of psTriRecy (the default is the sprand case on its full grid;
# laser5000 is the dense Landau laser operator, example/laser/laser.jl:15-57, normC = 1,
# laser_psTriRecy.jl:28-36).  af23560 (psPrecRecy) has its own leg (run_precrecy).
WORKLOADS = {
    "sprand4000": dict(metric=METRIC, grid=GRID, n=4000, normC=3.2,
                       desc="psTriRecy sprand N=4000 dense-Schur, 200x200 grid [0.45,0.55]x[0,0.1], k=20, "
                            "tol=1e-4, p=60, r=6, recy_tau=1.6"),
    "laser5000": dict(metric="σ_min grid pts/s (psTriRecy, laser N=5000, 200×200 grid, k=20, tol 1e-4)",
                      grid=(-1.1, 1.2, -1.1, 1.1, 200, 200, 20), n=5000, normC=1.0,
                      desc="psTriRecy laser (Landau, F=40π) N=5000 dense-Schur, 200x200 grid [-1.1,1.2]x[-1.1,1.1], "
                           "k=20, tol=1e-4, p=60, r=6, recy_tau=1.6"),
}


def select_workload(name):
    """Rebinds the workload constants (the dense psTriRecy workloads)."""
    global METRIC, GRID, N_MAT, NORMC, WORKLOAD
    w = WORKLOADS[name]
    METRIC, GRID, N_MAT, NORMC, WORKLOAD = w["metric"], w["grid"], w["n"], w["normC"], name


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="sprand4000", choices=["sprand4000", "laser5000", "af23560", "skewlap3d"],
                    help="sprand4000 (default, the headline), laser5000 (dense laser operator), af23560 "
                         "(psPrecRecy on the af23560-shaped synthetic matrix)")
    ap.add_argument("--chunk", type=int, default=200,
                    help="grid points per lane per step (at most; lowered to fit the lane's share of the grid)")
    ap.add_argument("--lanes", type=int, default=20, help="concurrent grid lanes per GPU")
    ap.add_argument("--trsm-backoff", type=int, default=32, help="longest ns between TRSM flag polls")
    ap.add_argument("--no-graphs", action="store_true", help="refine iterations as direct launches")
    ap.add_argument("--batch", type=int, default=0, help="largest speculative recycle batch (0: the library's 16)")
    ap.add_argument("--trsm-ctas", type=int, default=0,
                    help="CTAs per triangular solve in every lane (0: one per half block row)")
    ap.add_argument("--ref-chunk", type=int, default=3, help="grid points per step of the CPU arm")
    ap.add_argument("--pp-chunk", type=int, default=100, help="grid points per step of the af23560 (psPrecRecy) leg")
    ap.add_argument("--pp-lanes", type=int, default=8, help="concurrent lanes of the af23560 (psPrecRecy) leg")
    ap.add_argument("--mtx", default=None,
                    help="af23560 workload: read C from this MatrixMarket file (e.g. the reference's "
                         "data/af23560.mtx) instead of the synthetic af23560-shaped matrix")
    ap.add_argument("--cpu-sample-s", type=float, default=20.0, help="seconds of CPU baseline sampling")
    ap.add_argument("--n", type=int, default=None, help="matrix order (default: the workload's)")
    ap.add_argument("--factor-only", type=int, default=0,
                    help="skewlap3d: time this many band QR factorisations alone (one context) and exit")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-spmm", action="store_true", help="skip the sparse shifted product measurement")
    ap.add_argument("--no-ic", action="store_true", help="skip the IC preconditioner apply measurement")
    ap.add_argument("--plain-steps", type=int, default=5, help="steps timed on the unbatched per-point path")
    ap.add_argument("--accuracy-points", type=int, default=64,
                    help="timed points checked against the FP64 truth after the timed region (0: skip)")
    ap.add_argument("--ncu-window", default=None,
                    help="WARM,COUNT: run WARM points, then COUNT points inside cudaProfilerStart/Stop, and exit "
                         "(for ncu --profile-from-start off); no timing output")
    return ap.parse_args()


def control():
    from oracle.pstrirecy import PsTriRecyControl as OC  # used only by the CPU legs
    return OC


def build_inputs(n):
    from rls_b200.examples import sprand, landau
    from rls_b200.solvers import pre_process
    C = landau(n) if WORKLOAD == "laser5000" else sprand(n).toarray()
    t0 = time.perf_counter()
    T = pre_process(C)
    return C, np.asfortranarray(T), time.perf_counter() - t0


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = str(gpu_index)
        self.rows = []
        self.proc = None
        self.th = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.th = threading.Thread(target=self._read, daemon=True)
        self.th.start()

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9 and parts[0] == self.gpu:
                self.rows.append(parts)

    def stop(self):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if self.th is not None:
            self.th.join(timeout=5)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        def num(x):
            try:
                return float(x)
            except ValueError:
                return None
        sm = [num(r[1]) for r in self.rows if num(r[1]) is not None]
        mx = [num(r[2]) for r in self.rows if num(r[2]) is not None]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if r[5 + i].strip() == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows),
                "power_w_max": max((num(r[3]) or 0.0) for r in self.rows)}


def column_offset(rank, world, nZ, col):
    """First traversal index of this rank's share: the traversal's columns (col = k points
    each, one grid column of a serpentine strip) are split into `world` near-equal contiguous
    runs, and rank i starts its own traversal, with its own recycled space, at run i
    (rls_b200.distributed.column_shares, the library's rank split)."""
    from rls_b200.distributed import column_shares
    try:
        return int(column_shares(nZ, col, world)[rank])
    except ValueError as exc:
        raise SystemExit(str(exc))


def lane_plan(nZ, world, lanes, chunk, nsteps, col):
    """(lanes per rank, points per lane per step) for `world` ranks sharing an nZ-point
    traversal: every rank runs the same number of lanes and the same step, sized so that
    the smallest lane (column-aligned split, shares within two columns of nZ / world / lanes)
    holds `nsteps` steps."""
    share = nZ // world
    lanes = max(1, min(lanes, share // max(col, nsteps)))
    return lanes, max(1, min(chunk, (share // lanes - 2 * col) // nsteps))


def max_over_ranks(x, world, device):
    """The largest of the ranks' values of x (a time), on every rank."""
    if world == 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def banded_sparse(n, per_row, half_width, seed):
    """Synthetic real sparse matrix with the af23560 shape: `per_row` N(0,1) entries per row
    inside a band of half-width `half_width`, plus a dominant diagonal (duplicates summed)."""
    import scipy.sparse as sp
    rng = np.random.default_rng(seed)
    rows = np.repeat(np.arange(n, dtype=np.int64), per_row - 1)
    cols = np.clip(rows + rng.integers(-half_width, half_width + 1, size=rows.size), 0, n - 1)
    vals = rng.standard_normal(rows.size)
    d = np.arange(n, dtype=np.int64)
    A = sp.csc_matrix((np.concatenate([vals, np.full(n, 4.0 * per_row)]),
                       (np.concatenate([rows, d]), np.concatenate([cols, d]))), shape=(n, n))
    A.sum_duplicates()
    return A


def spmm_measure(local, hbm_peak, reps=20, b=6):
    """Shifted sparse product (ShiftedMat mul!) on two synthetic matrices, device-resident
    operands, CUDA-event timing per launch (the engine's profile slot 5)."""
    import torch
    from rls_b200.solvers import Engine
    out = {}
    for name, n, per_row in (("af23560-shaped n=23560, ~20 nnz/row, band ±300", 23560, 20),
                             ("banded n=1,000,000, ~16 nnz/row, band ±300", 1_000_000, 16)):
        A = banded_sparse(n, per_row, 300, 20260318)
        e = Engine(local)
        e.sparse_upload(A)
        X = torch.randn((b, n), dtype=torch.complex128, device="cuda")
        Y = torch.empty((b, n), dtype=torch.complex128, device="cuda")
        from rls_b200._lib import lib, c64
        import ctypes as C
        fn = lib().rls_spmm_shifted_dev
        for _ in range(3):
            fn(e._h, c64(-0.2, 0.1), 0, b, C.c_void_p(X.data_ptr()), n, C.c_void_p(Y.data_ptr()), n)
        torch.cuda.synchronize()
        e.set_profile(True)
        for _ in range(reps):
            for adj in (0, 1):
                fn(e._h, c64(-0.2, 0.1), adj, b, C.c_void_p(X.data_ptr()), n, C.c_void_p(Y.data_ptr()), n)
        cnt, ms, work = e.profile(5)
        e.close()
        achieved = (work / cnt) / (ms / cnt / 1e3) / 1e9
        out[name] = {"nnz": int(A.nnz), "b": b, "launches": cnt, "avg_us": ms / cnt * 1e3,
                     "bytes_per_launch": work / cnt, "achieved_gbs": achieved, "frac": achieved / hbm_peak}
        del X, Y
    return out


def lltp_measure(local, hbm_peak, reps=10, b=6):
    """SparseLLTP ldiv! (psPrecRecy's incomplete-Cholesky preconditioner apply) with b = 6
    device-resident columns, CUDA-event time per call (the engine's profile slot 6), on two
    factors: the one get_hsl_LLTP builds on the host (rls_ic_factor, timed) from the
    af23560-shaped matrix at z = -0.4+0.3i with psPrecRecy's default IC controls (tau1 1e-3,
    tau2 1e-6, alpha 1e-5, lsize = rsize = 200), and a synthetic factor that fills every
    lsize = 200 slot (4.7e6 nonzeros, the bound n(1 + lsize)).  Beside each, as the operator's
    CPU baseline, the same apply by the CPU restatement (SciPy sparse substitution, one thread)."""
    import torch
    import ctypes as C
    from rls_b200._lib import lib
    from rls_b200.examples import ic_factor_banded
    from rls_b200.solvers import Engine, SparseLLTP, ic_factor
    from oracle.precond import lltp_ldiv
    from scipy.sparse.csgraph import reverse_cuthill_mckee
    n = 23560
    A = banded_sparse(n, 20, 300, 20260318)
    # psPrecRecy orders by SPQR's column pivoting (qr(C).cpiv, psPrecRecy.jl:625), which needs
    # SuiteSparse; reverse Cuthill-McKee of C + Cᵀ stands in for that fill-reducing order
    p_ref = np.ascontiguousarray(reverse_cuthill_mckee((A + A.T).tocsr(), symmetric_mode=True), dtype=np.int64)
    t0 = time.perf_counter()
    L_ref, invp_ref, shift = ic_factor(A, -0.4 + 0.3j, 1e-3, 1e-6, 1e-5, 200, 200, p_ref)
    build_s = time.perf_counter() - t0
    L_fill = ic_factor_banded(n, 300, 2.0 / 3.0, seed=20260318, complex_values=False)
    p_fill = np.random.default_rng(7).permutation(n)
    out = {}
    for name, L, p, invp, extra in (
            ("get_hsl_LLTP factor of the af23560-shaped matrix (host build, RCM order)", L_ref, p_ref, invp_ref,
             {"host_build_s": build_s, "shift": shift}),
            ("synthetic af23560-shaped factor filling lsize = 200 (band 300, fill 2/3)", L_fill, p_fill,
             np.argsort(p_fill), {})):
        e = Engine(local)
        SparseLLTP(L, p, invp, e)
        dB = torch.randn((b, n), dtype=torch.complex128, device="cuda")
        dX = torch.empty_like(dB)
        torch.cuda.synchronize()
        fn = lib().rls_lltp_ldiv_dev
        for _ in range(3):
            fn(e._h, b, C.c_void_p(dB.data_ptr()), n, C.c_void_p(dX.data_ptr()), n)
        e.set_profile(True)
        for _ in range(reps):
            fn(e._h, b, C.c_void_p(dB.data_ptr()), n, C.c_void_p(dX.data_ptr()), n)
        cnt, ms, work = e.profile(6)
        e.close()
        achieved = (work / cnt) / (ms / cnt / 1e3) / 1e9
        r = {"n": n, "nnz": int(L.nnz), "b": b, "calls": cnt, "avg_us": ms / cnt * 1e3, "bytes_per_call": work / cnt,
             "achieved_gbs": achieved, "frac": achieved / hbm_peak}
        r.update(extra)
        B = np.random.default_rng(8).standard_normal((n, b)) + 0j
        t0 = time.perf_counter()
        lltp_ldiv(L, p, invp, B)
        r["cpu_baseline"] = {"avg_us": (time.perf_counter() - t0) * 1e6, "cores": 1, "kind": "port",
                             "sample": "one apply, SciPy spsolve_triangular forward and backward"}
        out[name] = r
        del dB, dX
    return out


def cpu_baseline(T, rec, ctl, X0, budget_s, min_pts=2):
    """The oracle (CPU restatement) from the start of the traversal, bounded by time."""
    from oracle.pstrirecy import PsTriRecyRun
    run = PsTriRecyRun(T, rec, ctl, X0=X0)
    t0 = time.perf_counter()
    i = 0
    while i < len(rec.Z) and (i < min_pts or time.perf_counter() - t0 < budget_s):
        run.run(i, i + 1)
        i += 1
    el = time.perf_counter() - t0
    return {"value": i / el, "unit": "pts/s", "cores": os.cpu_count(), "kind": "port",
            "sample": f"first {i} points of the 200x200 traversal (recycled space carried), "
                      f"CPU restatement with SciPy LAPACK on all host threads, {el:.1f} s"}


def base_line(args, n_gpus):
    return {"metric": METRIC, "unit": "pts/s", "n_gpus": n_gpus, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "complex128",
            "data": ("synthetic (sprand generator, NumPy PCG64 seed 20260318)" if WORKLOAD == "sprand4000" else
                     "synthetic (laser.jl's Landau operator, Gauss-Legendre nodes by Golub-Welsch)"),
            "config": {"workload": WORKLOADS[WORKLOAD]["desc"],
                       "n": args.n, "grid": list(GRID), "points_per_step": None,
                       "l2": "inputs larger than L2 (Schur tiles 132 MB and each lane's scaled copy 132 MB, "
                              "streamed every step; L2 126 MB)"}}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import rls_b200.examples  # noqa: F401  (generator only)
    from oracle import recugrid as G
    from oracle.pstrirecy import PsTriRecyControl, PsTriRecyRun
    C, T, pre_s = build_inputs(args.n)
    rec = G.recursion_grid(*GRID)
    ctl = PsTriRecyControl(normC=NORMC, tol=1e-4, p_min=1, p=60, recy_tau=1.6)
    rng = np.random.default_rng(1)
    X0 = rng.random((args.n, 6)) + 1j * rng.random((args.n, 6))
    run = PsTriRecyRun(T, rec, ctl, X0=X0)
    s = args.ref_chunk
    for w in range(args.warmup):
        run.run(w * s, (w + 1) * s)
    t0 = time.perf_counter()
    for k in range(args.steps):
        a = (args.warmup + k) * s
        run.run(a, a + s)
    el = time.perf_counter() - t0
    v = args.steps * s / el
    out = base_line(args, 1)
    out.update({"impl": "reference", "value": v, "ms_per_step": el * 1e3 / args.steps,
                "cpu_baseline": {"value": v, "unit": "pts/s", "cores": os.cpu_count(), "kind": "port",
                                 "sample": f"{s} points per step of the 200x200 traversal after {args.warmup} warm-up "
                                           f"steps; CPU restatement of psTriRecy (SciPy LAPACK, all host threads)"},
                "e2e": {"value": v, "unit": "pts/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
                "preprocess_s": pre_s})
    out["config"]["points_per_step"] = s
    print(json.dumps(out), flush=True)


def run_ours(args):
    import torch
    import torch.distributed as dist
    import rls_b200 as R
    from rls_b200.solvers import Engine, PsTriRecyControl, PsTriRecyStats

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local))

    # inputs: rank 0 reduces C to Schur form, every rank receives T
    if rank == 0:
        C, T, pre_s = build_inputs(args.n)
    else:
        C, T, pre_s = None, None, 0.0
    if world > 1:
        buf = torch.empty((args.n, args.n, 2), dtype=torch.float64, device="cuda")
        if rank == 0:
            buf.copy_(torch.view_as_real(torch.from_numpy(np.ascontiguousarray(T.T))))
        dist.broadcast(buf, 0)
        T = np.asfortranarray(torch.view_as_complex(buf).cpu().numpy().T)
        del buf

    rec = R.recursion_grid(*GRID)
    col = GRID[6]
    off = column_offset(rank, world, len(rec.Z), col)
    end = column_offset(rank + 1, world, len(rec.Z), col) if rank + 1 < world else len(rec.Z)
    sub = R.Recursion(*GRID)
    sub.Z = np.ascontiguousarray(rec.Z[off:end])
    nst = args.warmup + args.steps
    lanes, s = lane_plan(len(rec.Z), world, args.lanes, args.chunk, nst, col)
    ctl = PsTriRecyControl(normC=NORMC, tol=1e-4, p_min=1, p=60, recy_tau=1.6)
    rng = np.random.default_rng(1 + rank)
    X0 = rng.random((args.n, 6)) + 1j * rng.random((args.n, 6))
    need = nst * s

    # plain per-point drop-in (no speculative batching, one lane) on one step, for comparison
    plain = None
    if args.plain_steps > 0:
        engp = Engine(local)
        engp.set_batch(1)
        engp.set_schur(T)
        sigp = np.full(len(sub.Z), np.nan)
        stp = PsTriRecyStats.alloc(len(sub.Z))
        cstp = engp.stats_struct(stp)
        for w in range(args.warmup):
            engp.pstrirecy_range(sub, ctl, w * s, (w + 1) * s, sigp, stp, cstp, X0=X0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for k in range(args.plain_steps):
            a = (args.warmup + k) * s
            engp.pstrirecy_range(sub, ctl, a, a + s, sigp, stp, cstp)
        torch.cuda.synchronize()
        plain = {"value": args.plain_steps * s / (time.perf_counter() - t0), "unit": "pts/s",
                 "steps": args.plain_steps, "mode": "one lane, one recycle step per launch sequence (set_batch(1))"}
        engp.close()

    def timed_lanes(nl, profile, clocks=False):
        """W warm-up and K timed steps of `nl` concurrent lanes; a step is `s` lane-local points
        in every lane.  The K timed steps are one lane-parallel call: each lane walks its K·s
        points without waiting for the other lanes at step boundaries, as one psTriRecy call
        with lanes does over a whole grid.  Device time = max over the lanes' streams of
        CUDA-event spans.  With `profile` every kernel is timed by events (and the refine's
        iterations run as direct launches instead of their captured graph)."""
        ls = R.Lanes(nl, local, T)
        if nl > 1:
            ls.set_trsm_ctas(args.trsm_ctas)
        ls.set_trsm_backoff(args.trsm_backoff)
        if args.no_graphs:
            ls.set_graphs(False)
        if args.batch:
            ls.set_batch(args.batch)
        offs = ls.offsets(sub)
        if need > int(np.min(np.diff(offs))):
            raise SystemExit(f"--chunk × (warmup + steps) = {need} exceeds a lane of {int(np.min(np.diff(offs)))} points")
        sig = np.full(len(sub.Z), np.nan)
        st = PsTriRecyStats.alloc(len(sub.Z))
        cst = ls.engines[0].stats_struct(st)
        for w in range(args.warmup):
            ls.pstrirecy_range(sub, ctl, w * s, (w + 1) * s, sig, st, cst, X0=X0)
        if profile:
            ls.set_profile(True)
        streams = [torch.cuda.ExternalStream(p) for p in ls.streams()]
        ev0 = [torch.cuda.Event(enable_timing=True) for _ in streams]
        ev1 = [torch.cuda.Event(enable_timing=True) for _ in streams]
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        clk = None
        if clocks:
            clk = ClockSampler(local if "CUDA_VISIBLE_DEVICES" not in os.environ else
                               os.environ["CUDA_VISIBLE_DEVICES"].split(",")[local])
            clk.start()
            time.sleep(0.3)
        l0 = ls.launches()
        for e, st_ in zip(ev0, streams):
            e.record(st_)
        ls.pstrirecy_range(sub, ctl, args.warmup * s, need, sig, st, cst)
        for e, st_ in zip(ev1, streams):
            e.record(st_)
        for e in ev1:
            e.synchronize()
        torch.cuda.synchronize()
        l1 = ls.launches()
        if clk is not None:
            clk.stop()
        if world > 1:
            dist.barrier()
        ms = max(e0.elapsed_time(e1) for e0, e1 in zip(ev0, ev1))
        timed = np.concatenate([np.arange(o + args.warmup * s, o + need) for o in offs[:-1]])
        res = {"ms": max_over_ranks(ms, world, "cuda"), "launches": int(l1 - l0), "sig": sig, "timed": timed,
               "refines": int(np.sum(st.refine_it[timed] > 0)), "clk": clk, "offs": offs,
               "refine_it_hist": np.bincount(st.refine_it[timed][st.refine_it[timed] > 0]).tolist()}
        if profile:
            res["prof"] = {k: ls.profile(k) for k in range(4)}
            res["waits"] = ls.profile(4)
        ls.close()
        return res

    single = timed_lanes(1, False) if lanes > 1 else None
    main = timed_lanes(lanes, False, clocks=True)   # the headline: no per-kernel events
    profd = timed_lanes(lanes, True)                # the same steps again, every kernel timed
    ms_max = main["ms"]
    sigma, timed, refines, clk = main["sig"], main["timed"], main["refines"], main["clk"]
    prof, waits = profd["prof"], profd["waits"]

    # accuracy of the timed run itself (after the timed region): σ at sampled timed points of
    # every lane against an FP64 truth (block inverse iteration with cuBLAS triangular solves
    # on the same Schur factor, independent of the engine's kernels; tests/truth.py)
    accuracy = None
    if args.accuracy_points > 0:
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        from truth import sigma_min_schur
        pick = np.unique(np.concatenate([
            timed[np.linspace(0, len(timed) - 1, args.accuracy_points).astype(np.int64)],
            timed[np.argsort(sigma[timed])[:16]]]))                # plus the 16 smallest σ
        t0 = time.perf_counter()
        truth, bound, its = sigma_min_schur(T, sub.Z[pick])
        err = np.abs(sigma[pick] - truth)
        lane_of = np.searchsorted(main["offs"], pick, side="right") - 1
        accuracy = {"points": int(pick.size), "lanes_covered": int(np.unique(lane_of).size),
                    "max_abs_err": float(err.max()), "max_abs_err_over_normC": float(err.max() / NORMC),
                    "bar": "1e-4·normC", "within_bar": bool(err.max() <= 1e-4 * NORMC),
                    "max_rel_err": float(np.max(err / truth)),
                    "truth_max_err_bound": float(bound.max()), "truth_iterations_max": int(its.max()),
                    "truth": "block inverse subspace iteration on (T−zI)ᴴ(T−zI), cuBLAS FP64 triangular solves",
                    "seconds": time.perf_counter() - t0}

    # end to end through the public API on fresh contexts: host buffers, T uploaded to every lane
    e2e = None
    if not args.no_e2e:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ls2 = R.Lanes(lanes, local, T)
        if lanes > 1:
            ls2.set_trsm_ctas(args.trsm_ctas)
        t_setup = time.perf_counter() - t0
        sigma2 = np.full(len(sub.Z), np.nan)
        st2 = PsTriRecyStats.alloc(len(sub.Z))
        cst2 = ls2.engines[0].stats_struct(st2)
        t_steps = []
        for k in range(args.warmup + args.steps):
            t1 = time.perf_counter()
            ls2.pstrirecy_range(sub, ctl, k * s, (k + 1) * s, sigma2, st2, cst2, X0=X0)
            t_steps.append(time.perf_counter() - t1)
        el = max_over_ranks(time.perf_counter() - t0, world, "cuda")
        ls2.close()
        nsteps = args.warmup + args.steps
        T_bytes = args.n * args.n * 16
        e2e = {"value": world * lanes * nsteps * s / el, "unit": "pts/s",
               "h2d_bytes_per_step": int((T_bytes + lanes * nsteps * s * 16) / nsteps),
               "d2h_bytes_per_step": int(lanes * s * 8),
               "span": f"upload of T (host to lane 0, shared by the other {lanes - 1}) + steps 0..{nsteps - 1}",
               "setup_s": t_setup, "step_s": [round(t, 4) for t in t_steps]}
        e2e["matches_device_run"] = bool(np.allclose(sigma2[timed], sigma[timed], rtol=0, atol=1e-12))

    out = base_line(args, world)
    value = world * lanes * args.steps * s / (ms_max / 1e3)
    out.update({"value": value, "ms_per_step": ms_max / args.steps})
    out["config"]["points_per_step"] = lanes * s
    out["config"]["lanes"] = lanes
    out["config"]["chunk"] = s
    out["config"]["trsm_ctas"] = args.trsm_ctas or "one per half block row"
    out["config"]["trsm_backoff_ns"] = args.trsm_backoff
    out["config"]["parallelism"] = (f"grid columns: {world} rank(s) x {lanes} concurrent lane(s) per GPU "
                                    "(independent traversals from column starts)")
    out["config"]["refine_fraction_timed"] = refines / (lanes * args.steps * s)
    out["config"]["refine_iterations_hist"] = main["refine_it_hist"]   # refines by LOBPCG iteration count
    out["preprocess_s"] = pre_s
    out["gpu_launches"] = main["launches"]
    out["profiled_run"] = {"value": world * lanes * args.steps * s / (profd["ms"] / 1e3), "unit": "pts/s",
                           "launches": profd["launches"],
                           "mode": "the same steps with every kernel timed by events and the refine iterations "
                                   "as direct launches (source of kernel_time_ms and roofline)"}
    out["clocks"] = clk.summary()
    if single is not None:
        out["single_lane"] = {"value": world * args.steps * s / (single["ms"] / 1e3), "unit": "pts/s",
                              "mode": "one traversal per GPU (the reference's single recycled space)",
                              "matches_lanes_on_first_lane": bool(np.array_equal(
                                  single["sig"][single["timed"][:args.steps * s]],
                                  sigma[timed[:args.steps * s]]))}
    # roofline of the dominant profiled kernel
    names = {0: "k_trsm_half (R⁻¹/R⁻ᴴ on T−zI, block-row scaled factor)", 1: "k_heev_rr (projected eigensolve)",
             2: "recycle step span (k_batch_czx .. k_batch_xw, or k_gemm_rows per point)", 3: "k_trmm_partial+reduce (T·V, Tᴴ·[J5 V])"}
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except (OSError, ValueError):
        pass
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    shares = {k: v[1] for k, v in prof.items()}
    top = max((k for k in prof if k != 1), key=lambda k: shares[k])
    cnt, tot_ms, work = prof[top]
    achieved = (work / cnt) / (tot_ms / cnt / 1e3) / 1e9 if cnt else 0.0
    # DRAM bytes per launch of the TRSM from one ncu capture of this workload (n = 4000, k = 6):
    # dram__bytes_read.sum + dram__bytes_write.sum of k_trsm_half<6>
    traffic = NCU_TRSM_TRAFFIC if (top == 0 and args.n == N_MAT) else None
    out["roofline"] = {"bound": "hbm", "kernel": names[top], "achieved": achieved, "peak": hbm_peak,
                       "unit": "GB/s", "frac": achieved / hbm_peak, "traffic": traffic,
                       "peak_source": "measured" if "hbm_gbs" in peaks else "fallback",
                       "launches": cnt, "avg_us": tot_ms / max(cnt, 1) * 1e3}
    out["kernel_time_ms"] = {names[k]: {"launches": v[0], "ms": v[1]} for k, v in prof.items()}
    out["host_waits"] = {"count": waits[0], "ms": waits[1], "per_step": waits[0] / args.steps}
    if prof[1][0]:
        c1, t1, f1 = prof[1]
        out["heev_fp64"] = {"gflops": f1 / (t1 / 1e3) / 1e9, "launches": c1, "avg_us": t1 / c1 * 1e3}
    # the sparse operators' legs report a failure in the line instead of losing it
    if rank == 0 and world == 1 and not args.no_spmm:
        try:
            out["spmm_shifted"] = spmm_measure(local, hbm_peak)
        except Exception as exc:  # noqa: BLE001
            out["spmm_shifted"] = {"error": f"{type(exc).__name__}: {exc}"}
    if rank == 0 and world == 1 and not args.no_ic:
        try:
            out["ic_precond_apply"] = lltp_measure(local, hbm_peak)
        except Exception as exc:  # noqa: BLE001
            out["ic_precond_apply"] = {"error": f"{type(exc).__name__}: {exc}"}
    if rank == 0 and world == 1:
        from oracle.pstrirecy import PsTriRecyControl as OC
        from oracle import recugrid as G
        out["cpu_baseline"] = cpu_baseline(T, G.recursion_grid(*GRID),
                                           OC(normC=NORMC, tol=1e-4, p_min=1, p=60, recy_tau=1.6), X0,
                                           args.cpu_sample_s)
    if e2e is not None:
        out["e2e"] = e2e
    if accuracy is not None:
        out["accuracy"] = accuracy
    if plain is not None:
        out["plain_per_point"] = plain
        a0 = args.warmup * s   # lane 0 starts at the rank's first point, as the plain run does
        same = np.allclose(sigp[a0:a0 + args.plain_steps * s], sigma[a0:a0 + args.plain_steps * s], rtol=0,
                           atol=1e-10)
        out["plain_per_point"]["matches_batched"] = bool(same)
    if rank == 0:
        print(json.dumps(out), flush=True)
    if world > 1:
        dist.destroy_process_group()


def run_ncu_window(args):
    import torch
    import rls_b200 as R
    from rls_b200.solvers import Engine, PsTriRecyControl, PsTriRecyStats
    warm, count = (int(x) for x in args.ncu_window.split(","))
    _, T, _ = build_inputs(args.n)
    rec = R.recursion_grid(*GRID)
    ctl = PsTriRecyControl(normC=NORMC, tol=1e-4, p_min=1, p=60, recy_tau=1.6)
    rng = np.random.default_rng(1)
    X0 = rng.random((args.n, 6)) + 1j * rng.random((args.n, 6))
    eng = Engine(0)
    eng.set_schur(T)
    sig = np.full(len(rec.Z), np.nan)
    st = PsTriRecyStats.alloc(len(rec.Z))
    cst = eng.stats_struct(st)
    eng.pstrirecy_range(rec, ctl, 0, warm, sig, st, cst, X0=X0)
    torch.cuda.synchronize()
    torch.cuda.profiler.start()
    eng.pstrirecy_range(rec, ctl, warm, warm + count, sig, st, cst)
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    print(f"profiled points {warm}..{warm + count - 1}: {int(np.sum(st.refine_it[warm:warm + count] > 0))} refines",
          flush=True)


def main():
    args = parse()
    if args.workload == "af23560":
        run_precrecy(args)
        return
    if args.workload == "skewlap3d":
        run_sparse_tri(args)
        return
    select_workload(args.workload)
    if args.n is None:
        args.n = N_MAT
    if args.ncu_window:
        run_ncu_window(args)
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)



# ---- psPrecRecy on the af23560-shaped matrix --------------------------------------------------

AF_GRID = (-1.6, 0.8, -1.55, 1.55, 200, 200, 20)


def af_controls(mod, normC):
    """af23560_psPrecRecy.jl:16-46 as PsPrecRecyControl of `mod` (rls_b200.solvers or the oracle)."""
    return mod.PsPrecRecyControl(
        tol=1e-4, main_normC=normC, main_tau=1.6, gap_tau=1e-10, tol_pred=1e-3, lobpcg_pred_tol_scale=1.0,
        pred_tau=1.6, idx_cutoff_pred=0.01, pred_orth_type="shiftchol", pred_conv_thresh_type=1,
        lambda_lower_min=0.01, lambda_upper_max=30.0, r_main=6, p_main=60, p_min_main=1, main_implict_update=False,
        main_implict_recycle=True, r_pred=40, p_pred=20, p_min_pred=1, pred_implict_update=True,
        pred_implict_recycle=True, hsl_tol=1e-3, hsl_cntl_1=1e-6, hsl_icntl_1=200, hsl_icntl_2=500,
        hsl_cntl_2=1e-6, gamma_tol=1e-3, lambda_n_tol=1e-3)


def af_inputs(n, mtx=None):
    """C (the synthetic af23560-shaped matrix, or the MatrixMarket file `mtx` read as loaddata
    reads it), the driver's main_normC and the column order."""
    from rls_b200.examples import af23560_shaped, AF23560_NORMC
    from scipy.sparse.csgraph import reverse_cuthill_mckee
    if mtx:
        import scipy.sparse as sp
        from rls_b200.mtx import load_mtx
        C = load_mtx(mtx)
        if not sp.issparse(C) or C.shape[0] != C.shape[1]:
            raise SystemExit(f"--mtx {mtx}: psPrecRecy needs a square coordinate-format matrix")
        C = C.tocsc()
        C.sort_indices()
    else:
        C = af23560_shaped(n)
    # psPrecRecy orders by SPQR's column pivoting (qr(C).cpiv, psPrecRecy.jl:625), which needs
    # SuiteSparse; reverse Cuthill-McKee of |C| + |Cᵀ| stands in for that fill-reducing order
    p = np.ascontiguousarray(reverse_cuthill_mckee((abs(C) + abs(C.T)).tocsr(), symmetric_mode=True),
                             dtype=np.int64)
    return C, AF23560_NORMC, p


def sparse_truth(C, zs, block=4, maxit=200, rtol=1e-13):
    """FP64 σ_min(C − zI) by block inverse iteration on (C − zI)ᴴ(C − zI) with SciPy's sparse LU
    (host; independent of the engine), and the residual bound |σ − σ_true| ≤ ‖Aᴴu − σv‖ for the
    pair v, u = Av/σ (the distance to the nearest singular value)."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla
    n = C.shape[0]
    rng = np.random.default_rng(0)
    out, bnd = [], []
    for z in zs:
        A = (C - z * sp.identity(n, format="csc", dtype=np.complex128)).tocsc()
        lu = spla.splu(A)
        Y = np.linalg.qr(rng.standard_normal((n, block)) + 1j * rng.standard_normal((n, block)))[0]
        prev, s = np.inf, np.inf
        for _ in range(maxit):
            Y = lu.solve(lu.solve(Y, trans="H"))
            Y = np.linalg.qr(Y)[0]
            _, sv, Vh = np.linalg.svd(A @ Y, full_matrices=False)
            Y = Y @ Vh.conj().T
            s = sv[-1]
            if abs(prev - s) <= rtol * s:
                break
            prev = s
        v = Y[:, -1] / np.linalg.norm(Y[:, -1])
        Av = A @ v
        s = np.linalg.norm(Av)
        res = A.conj().T @ (Av / s) - s * v
        out.append(s)
        bnd.append(np.linalg.norm(res))
    return np.array(out), np.array(bnd)


def run_precrecy(args):
    """psPrecRecy (af23560-shaped, 200x200 grid, k=20): the prefix of the traversal in steps of
    --pp-chunk points, device time of the timed steps on the engine stream."""
    n = args.n or 23560
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    C, normC, p = af_inputs(n, args.mtx)
    n = C.shape[0]
    s = args.pp_chunk
    nst = args.warmup + args.steps
    if args.mtx:
        data = f"MatrixMarket file {os.path.basename(args.mtx)} (read by rls_mtx_read_csc as loaddata reads it)"
        shape = f"{os.path.basename(args.mtx)} N={n} ({C.nnz} nnz, main_normC=645.74)"
    else:
        data = "synthetic af23560-shaped matrix (rls_b200.examples.af23560_shaped, NumPy PCG64 seed 20260318)"
        shape = f"af23560-shaped N={n} (~20 nnz/row, band ±300, ‖C‖₂=645.74)"
    metric = ("σ_min grid pts/s (psPrecRecy, af23560-shaped N=23560, 200×200 grid, k=20, tol 1e-4)" if not args.mtx
              else f"σ_min grid pts/s (psPrecRecy, {os.path.basename(args.mtx)} N={n}, 200×200 grid, k=20, tol 1e-4)")
    out = {"metric": metric,
           "unit": "pts/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "complex128",
           "data": data,
           "config": {"workload": "psPrecRecy %s, 200x200 "
                                  "grid [-1.6,0.8]x[-1.55,1.55], k=20, tol=1e-4, r_main=6, p_main=60, r_pred=40, "
                                  "p_pred=20, IC lsize=200 rsize=500, RCM column order" % shape,
                      "n": n, "nnz": int(C.nnz), "grid": list(AF_GRID), "points_per_step": s,
                      "span": f"traversal points {args.warmup * s}..{nst * s - 1} after {args.warmup * s} "
                              f"warm-up points (the run's first preconditioner build is in the warm-up)"}}
    if args.impl == "reference":
        from oracle import recugrid as G
        from oracle.psprecrecy import PsPrecRecyRun
        import oracle.psprecrecy as OP
        from rls_b200.solvers import ic_factor as ic_host
        rng = np.random.default_rng(1)
        run = PsPrecRecyRun(C, G.recursion_grid(*AF_GRID), af_controls(OP, normC), p,
                            rng.random((n, 6)) + 1j * rng.random((n, 6)), rng.random((n, 40)) + 1j * rng.random((n, 40)),
                            bound_x0=rng.random((n, 1)) + 1j * rng.random((n, 1)), ic=ic_host)
        rs = args.ref_chunk
        for w in range(args.warmup):
            run.run(w * rs, (w + 1) * rs)
        t0 = time.perf_counter()
        for k in range(args.steps):
            a = (args.warmup + k) * rs
            run.run(a, a + rs)
        el = time.perf_counter() - t0
        v = args.steps * rs / el
        out.update({"impl": "reference", "value": v, "ms_per_step": el * 1e3 / args.steps,
                    "cpu_baseline": {"value": v, "unit": "pts/s", "cores": os.cpu_count(), "kind": "port",
                                     "sample": f"{rs} points per step after {args.warmup} warm-up steps; CPU "
                                               "restatement of psPrecRecy (SciPy sparse solves and LAPACK, all host "
                                               "threads; IC factor by the C++ host build)"},
                    "e2e": {"value": v, "unit": "pts/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}})
        out["config"]["points_per_step"] = rs
        out["config"]["span"] = (f"traversal points {args.warmup * rs}..{(args.warmup + args.steps) * rs - 1} after "
                                 f"{args.warmup * rs} warm-up points")
        print(json.dumps(out), flush=True)
        return
    import torch
    import rls_b200 as R
    from rls_b200.solvers import Engine, PrecRecyRun
    torch.cuda.set_device(0)
    rec = R.recursion_grid(*AF_GRID)
    ctl = af_controls(R, normC)
    rng = np.random.default_rng(1)
    X0m = rng.random((n, 6)) + 1j * rng.random((n, 6))
    X0p = rng.random((n, 40)) + 1j * rng.random((n, 40))
    xb = rng.random((n, 1)) + 1j * rng.random((n, 1))
    e = Engine(0)
    if args.ncu_window:   # warm points, then the profiled window between profiler start/stop
        warm, count = (int(x) for x in args.ncu_window.split(","))
        run = PrecRecyRun(e, C, rec, ctl, p=p, X0_main=X0m, X0_pred=X0p, X0_bound=xb)
        run.run(0, warm)
        torch.cuda.synchronize()
        torch.cuda.profiler.start()
        _, st = run.run(warm, warm + count)
        torch.cuda.synchronize()
        torch.cuda.profiler.stop()
        print(f"profiled points {warm}..{warm + count - 1}", flush=True)
        e.close()
        return
    t0 = time.perf_counter()
    run = PrecRecyRun(e, C, rec, ctl, p=p, X0_main=X0m, X0_pred=X0p, X0_bound=xb)
    run.run(0, args.warmup * s)
    torch.cuda.synchronize()
    t_warm = time.perf_counter() - t0
    e.set_profile(True)
    stream = torch.cuda.ExternalStream(e.stream_ptr())
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clk = ClockSampler(0 if "CUDA_VISIBLE_DEVICES" not in os.environ else os.environ["CUDA_VISIBLE_DEVICES"].split(",")[0])
    clk.start()
    time.sleep(0.3)
    l0 = e.launches()
    ev0.record(stream)
    t1 = time.perf_counter()
    sig, st = run.run(args.warmup * s, nst * s)
    ev1.record(stream)
    ev1.synchronize()
    wall = time.perf_counter() - t1
    l1 = e.launches()
    clk.stop()
    ms = ev0.elapsed_time(ev1)
    prof = {k: e.profile(k) for k in (1, 4, 5, 6)}
    e.close()
    timed = np.arange(args.warmup * s, nst * s)
    v = args.steps * s / (ms / 1e3)
    out.update({"value": v, "ms_per_step": ms / args.steps, "gpu_launches": int(l1 - l0), "clocks": clk.summary(),
                "e2e": {"value": nst * s / (t_warm + wall), "unit": "pts/s",
                        "h2d_bytes_per_step": int((C.nnz * 32 + n * 8 + nst * s * 16) / nst),
                        "d2h_bytes_per_step": int(s * 8),
                        "span": "PrecRecyRun through the public API from host buffers: C uploaded, preconditioner "
                                f"built at z†, steps 0..{nst - 1}, wall clock"},
                "wall_pts_per_s": args.steps * s / wall})
    out["stats"] = {"main_refines_timed": int(np.sum(st.main_refine_it[timed] > 0)),
                    "pred_refines_timed": int(np.sum(st.pred_refine_it[timed] > 0)),
                    "precond_builds": st.n_precond_rebuild_pts, "precond_s": st.precond_time_ns / 1e9,
                    "main_refine_s": st.main_refine_time_ns / 1e9, "pred_refine_s": st.pred_refine_time_ns / 1e9,
                    "pred_update_s": st.pred_update_time_ns / 1e9, "main_recycle_s": st.main_recycle_time_ns / 1e9,
                    "pred_recycle_s": st.pred_recycle_time_ns / 1e9, "main_update_s": st.main_update_time_ns / 1e9}
    names = {1: "pred-stage eigensolve (tridiagonalisation + Sturm + inverse iteration)", 4: "host waits",
             5: "k_spmm_shifted (C − zI and its adjoint)", 6: "IC preconditioner solves (k_sptrsv_wide)"}
    out["kernel_time_ms"] = {names[k]: {"launches": c, "ms": m} for k, (c, m, w) in prof.items() if k != 4}
    out["host_waits"] = {"count": prof[4][0], "ms": prof[4][1]}
    cnt, tot, work = prof[6]
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except (OSError, ValueError):
        pass
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    if cnt:
        ach = (work / cnt) / (tot / cnt / 1e3) / 1e9
        out["roofline"] = {"bound": "hbm", "kernel": names[6], "achieved": ach, "peak": hbm, "unit": "GB/s",
                           "frac": ach / hbm, "traffic": None,
                           "peak_source": "measured" if "hbm_gbs" in peaks else "fallback", "launches": cnt,
                           "avg_us": tot / cnt * 1e3}
    # concurrent lanes (PrecRecyLanes): every lane its own preconditioner and spaces, steps of s
    # lane-local points; the timed steps are one lane-parallel call, device time = the latest lane
    if args.pp_lanes > 1:
        from rls_b200.solvers import PrecRecyLanes
        L = args.pp_lanes
        t0 = time.perf_counter()
        ls = PrecRecyLanes(L, C, rec, ctl, p=p, X0_main=X0m, X0_pred=X0p, X0_bound=xb)
        offs = ls.offs
        if nst * s > int(np.min(np.diff(offs))):
            raise SystemExit(f"--pp-chunk × (warmup + steps) = {nst * s} exceeds a lane of {int(np.min(np.diff(offs)))}")
        ls.run(0, args.warmup * s)
        torch.cuda.synchronize()
        t_warm_l = time.perf_counter() - t0
        streams = [torch.cuda.ExternalStream(q) for q in ls.streams()]
        e0s = [torch.cuda.Event(enable_timing=True) for _ in streams]
        e1s = [torch.cuda.Event(enable_timing=True) for _ in streams]
        l0 = ls.launches()
        for a, q in zip(e0s, streams):
            a.record(q)
        t1 = time.perf_counter()
        sigL, stL = ls.run(args.warmup * s, nst * s)
        for b, q in zip(e1s, streams):
            b.record(q)
        for b in e1s:
            b.synchronize()
        wall_l = time.perf_counter() - t1
        l1 = ls.launches()
        ms_l = max(a.elapsed_time(b) for a, b in zip(e0s, e1s))
        ls.close()
        timedL = np.concatenate([np.arange(o + args.warmup * s, o + nst * s) for o in offs[:-1]])
        out["single_lane"] = {"value": v, "unit": "pts/s", "mode": "one traversal (the reference's single run)"}
        v = L * args.steps * s / (ms_l / 1e3)
        out.update({"value": v, "ms_per_step": ms_l / args.steps, "gpu_launches": int(l1 - l0)})
        out["e2e"] = {"value": L * nst * s / (t_warm_l + wall_l), "unit": "pts/s",
                      "h2d_bytes_per_step": int((L * (C.nnz * 32 + n * 8) + L * nst * s * 16) / nst),
                      "d2h_bytes_per_step": int(L * s * 8),
                      "span": f"PrecRecyLanes through the public API from host buffers: C uploaded to {L} lanes, "
                              f"each lane's preconditioner built at its first point, steps 0..{nst - 1}, wall clock"}
        out["config"]["lanes"] = L
        out["config"]["points_per_step"] = L * s
        out["stats"]["lanes"] = {"main_refines_timed": int(np.sum(stL.main_refine_it[timedL] > 0)),
                                 "pred_refines_timed": int(np.sum(stL.pred_refine_it[timedL] > 0)),
                                 "precond_builds": stL.n_precond_rebuild_pts}
        sig, timed = sigL, timedL
    # accuracy of the timed points against the FP64 sparse-LU truth (after the timed region)
    pick = timed[np.linspace(0, len(timed) - 1, min(args.accuracy_points, len(timed), 8)).astype(np.int64)]
    if args.accuracy_points > 0:
        truth, bound = sparse_truth(C, rec.Z[pick])
        err = np.abs(sig[pick] - truth)
        out["accuracy"] = {"points": int(pick.size), "max_abs_err": float(err.max()),
                           "max_abs_err_over_normC": float(err.max() / normC),
                           "within_bar": bool(err.max() <= 1e-4 * normC), "truth_max_err_bound": float(bound.max()),
                           "truth": "block inverse iteration on (C−zI)ᴴ(C−zI), SciPy sparse LU (host)"}
    if args.cpu_sample_s > 0:
        from oracle import recugrid as G
        from oracle.psprecrecy import PsPrecRecyRun
        import oracle.psprecrecy as OP
        from rls_b200.solvers import ic_factor as ic_host
        runo = PsPrecRecyRun(C, G.recursion_grid(*AF_GRID), af_controls(OP, normC), p, X0m, X0p, bound_x0=xb,
                             ic=ic_host)
        t0 = time.perf_counter()
        i = 0
        while i < nst * s and (i < 2 or time.perf_counter() - t0 < args.cpu_sample_s):
            runo.run(i, i + 1)
            i += 1
        el = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": i / el, "unit": "pts/s", "cores": os.cpu_count(), "kind": "port",
                               "sample": f"first {i} points of the traversal (preconditioner build included), CPU "
                                         f"restatement (SciPy sparse solves, LAPACK; IC by the C++ host build), "
                                         f"{el:.1f} s"}
    print(json.dumps(out), flush=True)



# ---- psTriRecy's sparse branch on the 3-D skew Laplacian ---------------------------------------

SKEW_GRID = (-550.0, 100.0, -200.0, 200.0, 200, 200, 20)


def run_sparse_tri(args):
    """psTriRecy on the sparse skewlap3d matrix (example/skewlap3d/skewlap3d.jl: N = 25,
    n = 24³ = 13,824, normC = 7471.59; skewlap3d_psTriRecy.jl's control), 200 × 200 grid, k = 20,
    with ∂σ/∂z at every point: the sparse branch (B = PᵀCP, band QR of B − zI per refine point)
    on concurrent lanes, steps of --chunk lane-local points as in the dense workloads."""
    import torch
    import torch.distributed as dist
    import rls_b200 as R
    from rls_b200.examples import skewlap3d, SKEWLAP_NORMC
    from rls_b200.solvers import PsTriRecyControl, PsTriRecyStats
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    C = skewlap3d(25)
    n = C.shape[0]
    normC = SKEWLAP_NORMC
    rec = R.recursion_grid(*SKEW_GRID)
    col = SKEW_GRID[6]
    desc = ("psTriRecy sparse branch, skewlap3d N=25 (n=13824, 7-point skew Laplacian, normC=7471.59), 200x200 grid "
            "[-550,100]x[-200,200], k=20, tol=1e-4, p=60, r=6, recy_tau=1.6, dsigma/dz at every point")
    out = {"metric": "σ_min grid pts/s (psTriRecy sparse, skewlap3d n=13824, 200×200 grid, k=20, tol 1e-4)",
           "unit": "pts/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "complex128",
           "data": "synthetic (skewlap3d.jl's matrix: N²·tridiag(1.5, −2, 0.5) in each of three Kronecker directions)",
           "config": {"workload": desc, "n": n, "nnz": int(C.nnz), "grid": list(SKEW_GRID)}}
    ctl = PsTriRecyControl(normC=normC, tol=1e-4, p_min=1, p=60, recy_tau=1.6, implict_recycle=True)
    rng = np.random.default_rng(1 + rank)
    X0 = rng.random((n, 6)) + 1j * rng.random((n, 6))
    nst = args.warmup + args.steps
    if args.impl == "reference":
        if rank != 0:
            return
        from oracle import recugrid as G
        import oracle.pstrirecy as OP
        t0 = time.perf_counter()
        p, l, u = R.band_order(C)
        run = OP.PsTriRecyRun(None, G.recursion_grid(*SKEW_GRID),
                              OP.PsTriRecyControl(normC=normC, tol=1e-4, p_min=1, p=60, recy_tau=1.6), X0=X0,
                              sparse=OP.pre_process_sparse(C, p), factor="lu")
        pre_s = time.perf_counter() - t0
        rs = args.ref_chunk
        for w in range(args.warmup):
            run.run(w * rs, (w + 1) * rs)
        t0 = time.perf_counter()
        for k in range(args.steps):
            a = (args.warmup + k) * rs
            run.run(a, a + rs)
        el = time.perf_counter() - t0
        v = args.steps * rs / el
        out.update({"impl": "reference", "value": v, "ms_per_step": el * 1e3 / args.steps, "preprocess_s": pre_s,
                    "cpu_baseline": {"value": v, "unit": "pts/s", "cores": os.cpu_count(), "kind": "port",
                                     "sample": f"{rs} points per step after {args.warmup} warm-up steps; CPU "
                                               "restatement of the sparse branch with a SuperLU operator in place "
                                               "of SPQR's R (same σ and right singular vectors), all host threads"},
                    "e2e": {"value": v, "unit": "pts/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}})
        out["config"]["points_per_step"] = rs
        print(json.dumps(out), flush=True)
        return
    torch.cuda.set_device(local)
    if args.ncu_window:   # one context: warm points, then the profiled window between profiler start/stop
        warm, count = (int(x) for x in args.ncu_window.split(","))
        S = R.SparseTri(C)
        eng = R.Engine(local)
        eng.set_sparse_tri(S)
        sig = np.full(len(rec.Z), np.nan)
        st = PsTriRecyStats.alloc(len(rec.Z))
        cst = eng.stats_struct(st)
        eng.pstrirecy_range(rec, ctl, 0, warm, sig, st, cst, X0=X0)
        torch.cuda.synchronize()
        torch.cuda.profiler.start()
        eng.pstrirecy_range(rec, ctl, warm, warm + count, sig, st, cst)
        torch.cuda.synchronize()
        torch.cuda.profiler.stop()
        print(f"profiled points {warm}..{warm + count - 1}: {int(np.sum(st.refine_it[warm:warm + count] > 0))} "
              "refines", flush=True)
        eng.close()
        return
    if args.factor_only > 0:   # the refine's factorisation alone: R(z) of B − zI at successive grid points
        if rank != 0:
            return
        S = R.SparseTri(C)
        eng = R.Engine(local)
        eng.set_sparse_tri(S)
        eng.set_profile(True)
        wall = []
        for i in range(args.factor_only):
            t0 = time.perf_counter()
            eng.band_factor(rec.Z[i])
            wall.append(time.perf_counter() - t0)
        cnt, ms_, fl = eng.profile(7)
        _, _, wsel, m8, m16 = eng.band_info()
        eng.close()
        print(json.dumps({"workload": desc, "band": {"l": S.l, "u": S.u},
                          "panel": {"width": wsel, "timed_ms_w8": m8, "timed_ms_w16": m16}, "factorisations": cnt,
                          "device_ms_each": ms_ / max(cnt, 1), "gflops": fl / (ms_ / 1e3) / 1e9 if ms_ else None,
                          "wall_ms": [w * 1e3 for w in wall]}), flush=True)
        return
    if world > 1:
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local))
    t0 = time.perf_counter()
    S = R.SparseTri(C)
    pre_s = time.perf_counter() - t0
    off = column_offset(rank, world, len(rec.Z), col)
    end = column_offset(rank + 1, world, len(rec.Z), col) if rank + 1 < world else len(rec.Z)
    sub = R.Recursion(*SKEW_GRID)
    sub.Z = np.ascontiguousarray(rec.Z[off:end])
    lanes, s = lane_plan(len(rec.Z), world, args.lanes, args.chunk, nst, col)
    need = nst * s

    def timed(nl, profile):
        ls = R.Lanes(nl, local)
        ls.set_sparse_tri(S)
        offs = ls.offsets(sub)
        if need > int(np.min(np.diff(offs))):
            raise SystemExit(f"--chunk × (warmup + steps) = {need} exceeds a lane of {int(np.min(np.diff(offs)))} points")
        sig = np.full(len(sub.Z), np.nan)
        st = PsTriRecyStats.alloc(len(sub.Z), grad=True)
        cst = ls.engines[0].stats_struct(st)
        for w in range(args.warmup):
            ls.pstrirecy_range(sub, ctl, w * s, (w + 1) * s, sig, st, cst, X0=X0)
        if profile:
            ls.set_profile(True)
        streams = [torch.cuda.ExternalStream(q) for q in ls.streams()]
        ev0 = [torch.cuda.Event(enable_timing=True) for _ in streams]
        ev1 = [torch.cuda.Event(enable_timing=True) for _ in streams]
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        clk = None
        if profile:
            clk = ClockSampler(local if "CUDA_VISIBLE_DEVICES" not in os.environ else
                               os.environ["CUDA_VISIBLE_DEVICES"].split(",")[local])
            clk.start()
            time.sleep(0.3)
        l0 = ls.launches()
        for e, q in zip(ev0, streams):
            e.record(q)
        ls.pstrirecy_range(sub, ctl, args.warmup * s, need, sig, st, cst)
        for e, q in zip(ev1, streams):
            e.record(q)
        for e in ev1:
            e.synchronize()
        torch.cuda.synchronize()
        l1 = ls.launches()
        if clk is not None:
            clk.stop()
        if world > 1:
            dist.barrier()
        ms = max(a.elapsed_time(b) for a, b in zip(ev0, ev1))
        tim = np.concatenate([np.arange(o + args.warmup * s, o + need) for o in offs[:-1]])
        res = {"ms": max_over_ranks(ms, world, "cuda"), "launches": int(l1 - l0), "sig": sig, "st": st, "timed": tim,
               "clk": clk, "offs": offs}
        if profile:
            res["prof"] = {k: ls.profile(k) for k in (0, 1, 2, 5, 7)}
            res["waits"] = ls.profile(4)
        res["band_info"] = ls.engines[0].band_info()
        ls.close()
        return res

    single = timed(1, False) if lanes > 1 else None
    main_ = timed(lanes, True)
    ms = main_["ms"]
    sig, st, tim, prof = main_["sig"], main_["st"], main_["timed"], main_["prof"]
    value = world * lanes * args.steps * s / (ms / 1e3)
    out["n_gpus"] = world
    out.update({"value": value, "ms_per_step": ms / args.steps, "gpu_launches": main_["launches"],
                "clocks": main_["clk"].summary(), "preprocess_s": pre_s})
    out["config"].update({"points_per_step": lanes * s, "lanes": lanes, "chunk": s,
                          "band": {"l": S.l, "u": S.u, "order": "reverse Cuthill-McKee of |C|+|Cᵀ| (band_order)",
                                   "panel_width": main_["band_info"][2],
                                   "panel_timed_ms": {"w8": main_["band_info"][3], "w16": main_["band_info"][4]}},
                          "parallelism": f"grid columns: {world} rank(s) x {lanes} concurrent lane(s) per GPU",
                          "refine_fraction_timed": float(np.mean(st.refine_it[tim] > 0)),
                          "l2": "the band array (n·(3l+2u+1)·16 B ≈ 0.3 GB) and R's band tiles exceed L2 (126 MB); "
                                "every refine point rebuilds and streams them"})
    if single is not None:
        out["single_lane"] = {"value": world * args.steps * s / (single["ms"] / 1e3), "unit": "pts/s",
                              "mode": "one traversal per GPU (the reference's single recycled space)"}
    names = {0: "k_trsm_half on R's band tiles", 1: "k_heev_rr (projected eigensolve)",
             2: "recycle step span", 5: "k_spmm_shifted (B and Bᴴ products of the space)",
             7: "band QR of B − zI (k_bqr_panel + k_bqr_update, per refine point)"}
    out["kernel_time_ms"] = {names[k]: {"launches": v[0], "ms": v[1]} for k, v in prof.items()}
    out["host_waits"] = {"count": main_["waits"][0], "ms": main_["waits"][1]}
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except (OSError, ValueError):
        pass
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    cnt, tot, work = prof[0]
    if cnt:
        ach = (work / cnt) / (tot / cnt / 1e3) / 1e9
        out["roofline"] = {"bound": "hbm", "kernel": names[0], "achieved": ach, "peak": hbm, "unit": "GB/s",
                           "frac": ach / hbm, "traffic": None, "launches": cnt, "avg_us": tot / cnt * 1e3,
                           "peak_source": "measured" if "hbm_gbs" in peaks else "fallback"}
    c7, t7, f7 = prof[7]
    if c7:
        out["band_qr_fp64"] = {"gflops": f7 / (t7 / 1e3) / 1e9, "launches": c7, "avg_ms": t7 / c7,
                               "flops_per_factorisation": f7 / c7}
    # gradient and σ at sampled timed points against the FP64 sparse-LU truth (after timing)
    if args.accuracy_points > 0:
        pick = tim[np.linspace(0, len(tim) - 1, min(args.accuracy_points, 24)).astype(np.int64)]
        t0 = time.perf_counter()
        truth, bound = sparse_truth(C, sub.Z[pick])
        err = np.abs(sig[pick] - truth)
        out["accuracy"] = {"points": int(pick.size), "max_abs_err": float(err.max()),
                           "max_abs_err_over_normC": float(err.max() / normC),
                           "max_rel_err": float(np.max(err / truth)), "within_bar": bool(err.max() <= 1e-4 * normC),
                           "truth_max_err_bound": float(bound.max()),
                           "truth": "block inverse iteration on (C−zI)ᴴ(C−zI), SciPy sparse LU (host)",
                           "seconds": time.perf_counter() - t0}
    if not args.no_e2e:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        S2 = R.SparseTri(C)
        ls2 = R.Lanes(lanes, local)
        ls2.set_sparse_tri(S2)
        sig2 = np.full(len(sub.Z), np.nan)
        st2 = PsTriRecyStats.alloc(len(sub.Z), grad=True)
        cst2 = ls2.engines[0].stats_struct(st2)
        for k in range(nst):
            ls2.pstrirecy_range(sub, ctl, k * s, (k + 1) * s, sig2, st2, cst2, X0=X0)
        el = max_over_ranks(time.perf_counter() - t0, world, "cuda")
        ls2.close()
        out["e2e"] = {"value": world * lanes * nst * s / el, "unit": "pts/s",
                      "h2d_bytes_per_step": int((lanes * C.nnz * (16 + 8) + lanes * nst * s * 16) / nst),
                      "d2h_bytes_per_step": int(lanes * s * 24),
                      "span": f"band order + upload of C to each of {lanes} lanes + steps 0..{nst - 1} (σ and ∂σ/∂z "
                              "out), wall clock",
                      "matches_device_run": bool(np.allclose(sig2[tim], sig[tim], rtol=0, atol=1e-12))}
    if rank == 0 and world == 1 and args.cpu_sample_s > 0:
        from oracle import recugrid as G
        import oracle.pstrirecy as OP
        run = OP.PsTriRecyRun(None, G.recursion_grid(*SKEW_GRID),
                              OP.PsTriRecyControl(normC=normC, tol=1e-4, p_min=1, p=60, recy_tau=1.6), X0=X0,
                              sparse=OP.pre_process_sparse(C, S.perm), factor="lu")
        t0 = time.perf_counter()
        i = 0
        while i < 4000 and (i < 2 or time.perf_counter() - t0 < args.cpu_sample_s):
            run.run(i, i + 1)
            i += 1
        el = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": i / el, "unit": "pts/s", "cores": os.cpu_count(), "kind": "port",
                               "sample": f"first {i} points of the traversal, CPU restatement of the sparse branch "
                                         f"with a SuperLU operator in place of SPQR's R, {el:.1f} s"}
    if rank == 0:
        print(json.dumps(out), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
