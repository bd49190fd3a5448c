"""psTriRecy on the GPU against the CPU oracle and the FP64 dense-SVD oracle.

Bar: |σ_gpu − σ_oracle| <= 1e-4·normC on every grid point
and the relative residual of every accepted point <= tol; the dense SVD gives
the FP64 truth on sampled points.
"""
import numpy as np
import pytest

from oracle.pstrirecy import PsTriRecyControl as OControl, ps_tri_recy_schur, dense_sigma_min
from oracle.lobpcg import LobpcgSvdControl as OLobCtl, LobpcgSvdKeep, lobpcg_svd
from oracle.pstrirecy import InvAdjR
from oracle import recugrid as ogrid
import rls_b200 as R
from rls_b200._lib import lib, check
from rls_b200.examples import sprand, landau

pytestmark = pytest.mark.gpu


def _case_sprand(N=240, grid=(0.45, 0.55, 0.0, 0.1, 12, 10, 5)):
    C = sprand(N).toarray()
    return C, 3.2, grid


def _x0(n, r, seed=3):
    rng = np.random.default_rng(seed)
    return rng.random((n, r)) + 1j * rng.random((n, r))


@pytest.fixture(scope="module")
def sprand_case(cuda_device):
    C, normC, grid = _case_sprand()
    T = R.pre_process(C)
    return C, T, normC, grid


def test_lobpcg_single_point_matches_oracle(sprand_case):
    C, T, normC, grid = sprand_case
    n, r = T.shape[0], 6
    X0 = _x0(n, r)
    z = 0.5 + 0.05j
    eng = R.Engine(0)
    eng.set_schur(T)
    ctl = R.LobpcgSvdControl(m=n, n=n, r=r, conv_range=(1, 1), tol=1e-5, side="L", normC=normC)
    s, it, X, sr = eng.lobpcg_svd_invtri(z, ctl, X0=X0)
    keep = LobpcgSvdKeep(n, n, r)
    keep.S[:, :r] = X0
    octl = OLobCtl(m=n, n=n, r=r, conv_range=(1, 1), tol=1e-5, side="L", normC=normC)
    Rz = T - z * np.eye(n)
    s_o, it_o = lobpcg_svd(InvAdjR(Rz), keep.S[:, :r], None, keep, octl)
    assert abs(it - it_o) <= 1
    truth = dense_sigma_min(C, z)
    assert abs(sr[0] - truth) <= 1e-6 * normC
    assert abs(sr[0] - keep.sigma[0]) <= 1e-6 * normC
    # Ritz vector of σ_min agrees with the oracle's up to phase
    ov = abs(np.vdot(X[:, 0], keep.S[:, 0])) / (np.linalg.norm(X[:, 0]) * np.linalg.norm(keep.S[:, 0]))
    assert ov > 1 - 1e-6


def test_sleeping_host_waits_give_identical_sigma(sprand_case):
    """rls_ctx_set_host_wait only changes how the host thread waits: σ and the per-point
    statistics are bit-identical to the spinning default."""
    C, T, normC, grid = sprand_case
    rec = R.recursion_grid(*grid)
    n, r = T.shape[0], 6
    ctl = R.PsTriRecyControl(normC=normC, tol=1e-4, p_min=1, p=20, r=r, recy_tau=1.6)
    out = []
    for spin in (-1, 0, 50):
        e = R.Engine(0)
        e.set_schur(T)
        e.set_host_wait(spin)
        out.append(e.pstrirecy(rec, ctl, X0=_x0(n, r)))
        e.close()
    for sig, st in out[1:]:
        assert np.array_equal(sig, out[0][0])
        assert np.array_equal(st.refine_it, out[0][1].refine_it)


def test_shared_schur_tiles_survive_reupload_and_source_close(sprand_case):
    """rls_set_schur_copy shares the source's device tiles: a later rls_set_schur on the source
    leaves the sharer's operator unchanged, and the sharer keeps working after the source closes."""
    C, T, normC, grid = sprand_case
    n, r = T.shape[0], 6
    X0 = _x0(n, r)
    z = 0.5 + 0.05j
    ctl = R.LobpcgSvdControl(m=n, n=n, r=r, conv_range=(1, 1), tol=1e-6, side="L", normC=normC)
    T2 = 2.0 * T                                         # σ_min(2T − zI) = 2·σ_min(T − z/2·I)
    src, dst = R.Engine(0), R.Engine(0)
    src.set_schur(T)
    check(lib().rls_set_schur_copy(dst._h, src._h), dst._h)
    dst.n = src.n
    truth = dense_sigma_min(C, z)
    s_dst0 = dst.lobpcg_svd_invtri(z, ctl, X0=X0)[3][0]
    src.set_schur(T2)
    s_src = src.lobpcg_svd_invtri(z, ctl, X0=X0)[3][0]
    s_dst1 = dst.lobpcg_svd_invtri(z, ctl, X0=X0)[3][0]
    src.close()
    s_dst2 = dst.lobpcg_svd_invtri(z, ctl, X0=X0)[3][0]
    dst.close()
    assert abs(s_dst0 - truth) <= 1e-6 * normC
    assert s_dst1 == s_dst0 and s_dst2 == s_dst0
    assert abs(s_src - 2.0 * dense_sigma_min(C, z / 2)) <= 1e-4 * normC


@pytest.mark.parametrize("p,r", [(60, 6), (6, 2)])
def test_pstrirecy_matches_oracle(sprand_case, p, r):
    C, T, normC, grid = sprand_case
    n = T.shape[0]
    X0 = _x0(n, r)
    rec = R.recursion_grid(*grid)
    ctl = R.PsTriRecyControl(normC=normC, tol=1e-4, p_min=1, p=p, r=r, recy_tau=1.6)
    sig, st = R.psTriRecy(R.SchurFactor(T), rec, ctl, verbose=0, X0=X0)
    orec = ogrid.recursion_grid(*grid)
    octl = OControl(normC=normC, tol=1e-4, p_min=1, p=p, r=r, recy_tau=1.6)
    # the reference's algorithm (σ bar) and the same with the full Ritz basis (trajectory)
    sig_ref, _ = ps_tri_recy_schur(T, orec, octl, X0=X0)
    sig_o, st_o = ps_tri_recy_schur(T, orec, octl, X0=X0, ritz_g1_always=True)
    assert np.all(np.isfinite(sig))
    assert np.max(np.abs(sig - sig_ref)) <= 1e-4 * normC
    assert np.max(np.abs(sig - sig_o)) <= 1e-4 * normC
    # dense-SVD truth on every grid point (n is small)
    truth = np.array([dense_sigma_min(C, z) for z in rec.Z])
    assert np.max(np.abs(sig - truth)) <= 1e-4 * normC
    # Identical trajectory over the leading points: same space size, same recycle
    # decision, same Ritz dimension.  (Later points may diverge: the unconverged
    # Ritz vectors that enter the space differ at rounding level, and the
    # recycle-acceptance test is a threshold on them.)
    lead = 40
    assert np.array_equal(st.p_count[:lead], st_o.p_count[:lead]), (st.p_count[:lead], st_o.p_count[:lead])
    assert np.array_equal(st.refine_it[:lead] > 0, st_o.refine_it[:lead] > 0)
    assert np.array_equal(st.r_recy[:lead], st_o.r_recy[:lead])
    assert st.n_pts == int(np.sum(st.refine_it > 0))
    # and most recycle/refine decisions over the whole grid
    agree = np.mean((st.refine_it > 0) == (st_o.refine_it > 0))
    assert agree >= 0.9, agree


def test_pstrirecy_laser_small(cuda_device):
    C = landau(180, 40 * np.pi)
    T = R.pre_process(C)
    n, r = T.shape[0], 6
    X0 = _x0(n, r, seed=11)
    grid = (-1.1, 1.2, -1.1, 1.1, 8, 8, 4)
    rec = R.recursion_grid(*grid)
    ctl = R.PsTriRecyControl(normC=1.0, tol=1e-4, recy_tau=1.6, p=60)
    sig, st = R.psTriRecy(R.SchurFactor(T), rec, ctl, verbose=0, X0=X0)
    truth = np.array([dense_sigma_min(C, z) for z in rec.Z])
    assert np.max(np.abs(sig - truth)) <= 1e-4


def test_batched_recycle_matches_per_point(sprand_case):
    """Speculative batches give the sequential loop's results: same σ, same decisions."""
    C, T, normC, grid = sprand_case
    n, r = T.shape[0], 6
    X0 = _x0(n, r, seed=21)
    grid2 = (0.45, 0.55, 0.0, 0.1, 16, 12, 6)
    rec = R.recursion_grid(*grid2)
    ctl = R.PsTriRecyControl(normC=normC, tol=1e-4, p_min=1, p=20, r=r, recy_tau=1.6)
    out = {}
    for B in (1, 4, 16):
        eng = R.Engine(0)
        eng.set_batch(B)
        eng.set_schur(T)
        out[B] = eng.pstrirecy(rec, ctl, X0=X0)
        eng.close()
    s1, st1 = out[1]
    assert np.sum(st1.refine_it == 0) > 0.5 * len(s1)   # the grid exercises recycling
    for B in (4, 16):
        sB, stB = out[B]
        assert np.max(np.abs(sB - s1)) <= 1e-8 * normC
        assert np.array_equal(stB.refine_it > 0, st1.refine_it > 0)
        assert np.array_equal(stB.p_count, st1.p_count)
        assert np.array_equal(stB.r_recy, st1.r_recy)


def test_lanes_cover_grid_and_match_truth(sprand_case):
    """Concurrent lanes: every point computed, σ within the bar of the dense SVD, the first
    lane identical to the single traversal over its points, stats merged per point."""
    C, T, normC, _ = sprand_case
    grid = (0.45, 0.55, 0.0, 0.1, 12, 20, 2)          # strips of 24 points, 10 strips
    rec = R.recursion_grid(*grid)
    n, r = T.shape[0], 6
    X0 = _x0(n, r)
    ctl = R.PsTriRecyControl(normC=normC, tol=1e-4, p_min=1, p=20, r=r, recy_tau=1.6)
    e = R.Engine(0)
    e.set_schur(T)
    sig1, st1 = e.pstrirecy(rec, ctl, X0=X0)
    e.close()
    ls = R.Lanes(3, 0, T)
    off = ls.offsets(rec)
    sigL, stL = ls.pstrirecy(rec, ctl, X0=X0)
    ls.close()
    assert np.all(np.isfinite(sigL))
    assert np.max(np.abs(sigL - sig1)) <= 1e-4 * normC
    sel = np.arange(0, len(rec.Z), 7)
    truth = np.array([dense_sigma_min(T, z) for z in rec.Z[sel]])
    assert np.max(np.abs(sigL[sel] - truth)) <= 1e-4 * normC
    assert np.array_equal(sigL[:off[1]], sig1[:off[1]])
    assert np.array_equal(stL.refine_it[:off[1]], st1.refine_it[:off[1]])
    assert stL.n_pts == int(np.sum(stL.refine_it > 0))
    for b in off[:-1]:
        assert stL.refine_it[b] > 0 and stL.p_count[b] == 0   # each lane starts from an empty space


def test_graph_replay_equals_direct_launches(sprand_case):
    """The refine's steady LOBPCG iteration replayed from its captured graph gives the direct
    launches' results bit for bit (σ, iteration counts, space sizes), and a TRSM setting change
    recaptures it."""
    C, T, normC, grid = sprand_case
    n = T.shape[0]
    X0 = _x0(n, 6)
    rec = R.recursion_grid(*grid)
    ctl = R.PsTriRecyControl(normC=normC, tol=1e-4, p_min=1, p=20, recy_tau=1.6)
    out = []
    for graphs, ctas in ((False, 0), (True, 0), (True, 5)):
        e = R.Engine(0)
        try:
            e.set_schur(T)
            e.set_graphs(graphs)
            e.set_trsm_ctas(ctas)
            out.append(e.pstrirecy(rec, ctl, X0=X0))
        finally:
            e.close()
    (s0, st0), (s1, st1), (s2, st2) = out
    assert np.array_equal(s0, s1) and np.array_equal(s0, s2)
    assert np.array_equal(st0.refine_it, st1.refine_it) and np.array_equal(st0.p_count, st1.p_count)
    assert int(np.max(st0.refine_it)) >= 2      # some refine reached the replayed iterations
