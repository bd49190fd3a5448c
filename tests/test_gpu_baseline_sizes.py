"""σ_min at the sizes of the benchmark configurations, against the oracle and an FP64 truth.

* sprand N = 4000 on the 20 × 20 grid of [0.45, 0.55] × [0, 0.1] with k = 4, p = 60, r = 6,
  recy_tau = 1.6, tol = 1e-4 (the plain psTriRecy configuration): every one of the 400
  points against the FP64 truth, and the leading 60 points (where the restatement spends several
  seconds per point on the host) against the CPU restatement of the reference's loop.
* laser N = 5000 (Landau operator, F = 40π): the leading 400 points of the 200 × 200
  traversal of [-1.1, 1.2] × [-1.1, 1.1] with k = 20, against the FP64 truth on all of them.

Bar: |σ − σ_ref| ≤ 1e-4·normC on every point; the FP64 truth is
block inverse iteration with cuBLAS triangular solves (tests/truth.py), whose own error
bound is checked to be far below the bar.  Trajectory: with the reference's Ritz-basis
choice the engine takes the oracle's recycle/refine decisions on the leading 40 points.
"""
import numpy as np
import pytest

import rls_b200 as R
from oracle import recugrid as ogrid
from oracle.pstrirecy import PsTriRecyControl as OControl, PsTriRecyRun
from rls_b200.examples import landau, sprand
from truth import sigma_min_schur

pytestmark = pytest.mark.gpu


def _x0(n, r, seed):
    rng = np.random.default_rng(seed)
    return rng.random((n, r)) + 1j * rng.random((n, r))


@pytest.fixture(scope="module")
def sprand4000(cuda_device):
    return R.pre_process(sprand(4000).toarray())


def test_sprand4000_config1_every_point(sprand4000):
    T = sprand4000
    n, r, normC = 4000, 6, 3.2
    grid = (0.45, 0.55, 0.0, 0.1, 20, 20, 4)
    rec = R.recursion_grid(*grid)
    X0 = _x0(n, r, 41)
    ctl = R.PsTriRecyControl(normC=normC, tol=1e-4, p_min=1, p=60, r=r, recy_tau=1.6)
    runs = {}
    for g1 in (True, False):
        e = R.Engine(0)
        e.set_ritz_basis(g1)
        e.set_schur(T)
        runs[g1] = e.pstrirecy(rec, ctl, X0=X0)
        e.close()
    sig, st = runs[True]
    sig_r, st_r = runs[False]
    # the reference's algorithm, restated (its Ritz-basis choice)
    octl = OControl(normC=normC, tol=1e-4, p_min=1, p=60, r=r, recy_tau=1.6)
    lo = 60
    run = PsTriRecyRun(T, ogrid.recursion_grid(*grid), octl, X0=X0)
    sig_full, st_o = run.run(0, lo)
    sig_o = sig_full[:lo]
    truth, bound, _ = sigma_min_schur(T, rec.Z)
    assert np.max(bound) <= 1e-6 * normC, np.max(bound)
    for s in (sig, sig_r):
        assert np.all(np.isfinite(s))
        assert np.max(np.abs(s[:lo] - sig_o)) <= 1e-4 * normC
        assert np.max(np.abs(s - truth)) <= 1e-4 * normC, np.max(np.abs(s - truth))
    assert np.max(np.abs(sig_o - truth[:lo])) <= 1e-4 * normC
    lead = 40
    assert np.array_equal(st_r.refine_it[:lead] > 0, st_o.refine_it[:lead] > 0)
    assert np.array_equal(st_r.p_count[:lead], st_o.p_count[:lead])
    assert np.array_equal(st_r.r_recy[:lead], st_o.r_recy[:lead])
    agree = np.mean((st_r.refine_it[:lo] > 0) == (st_o.refine_it[:lo] > 0))
    assert agree >= 0.9, agree
    # refined points carry LOBPCG's tighter tolerance (0.1·tol): far inside the bar
    ref = st.refine_it > 0
    assert np.max(np.abs(sig[ref] - truth[ref])) <= 1e-5 * normC


def test_laser5000_leading_points(cuda_device):
    C = landau(5000)
    T = R.pre_process(C)
    n, r, normC = 5000, 6, 1.0
    rec = R.recursion_grid(-1.1, 1.2, -1.1, 1.1, 200, 200, 20)
    lead = 400
    ctl = R.PsTriRecyControl(normC=normC, tol=1e-4, p=60, recy_tau=1.6)
    e = R.Engine(0)
    e.set_schur(T)
    sigma = np.full(len(rec.Z), np.nan)
    st = R.PsTriRecyStats.alloc(len(rec.Z))
    cst = e.stats_struct(st)
    e.pstrirecy_range(rec, ctl, 0, lead, sigma, st, cst, X0=_x0(n, r, 43))
    e.close()
    truth, bound, _ = sigma_min_schur(T, rec.Z[:lead])
    assert np.max(bound) <= 1e-6 * normC, np.max(bound)
    assert np.all(np.isfinite(sigma[:lead]))
    assert np.max(np.abs(sigma[:lead] - truth)) <= 1e-4 * normC, np.max(np.abs(sigma[:lead] - truth))
    assert np.all(np.isnan(sigma[lead:]))
    assert 0 < np.sum(st.refine_it[:lead] > 0) < lead     # both paths (recycle and refine) ran
