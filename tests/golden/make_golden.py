"""Generates the committed golden fixtures under tests/golden/ from the CPU oracle.

    python tests/golden/make_golden.py

The reference (Julia) ships no tests or golden vectors and cannot run here, so
these fixtures pin the oracle's own outputs; every σ in them is also checked
against an FP64 dense SVD at generation time (independent of the oracle).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import recugrid as G                      # noqa: E402
from oracle.pstrirecy import PsTriRecyControl, ps_tri_recy_schur, pre_process_dense, dense_sigma_min  # noqa: E402
from rls_b200.examples import sprand, landau          # noqa: E402

GRIDS = [
    (0.45, 0.55, 0.0, 0.1, 20, 20, 4),
    (-1.1, 1.2, -1.1, 1.1, 10, 12, 3),
    (-550.0, 100.0, -200.0, 200.0, 7, 6, 6),
    (0.1, 0.2, 0.3, 0.4, 3, 5, 1),
    (0.0, 1.0, 0.0, 1.0, 4, 4, 4),
    (-1.0, 1.0, -0.5, 0.5, 11, 10, 5),
]


def grids():
    out = {}
    for i, g in enumerate(GRIDS):
        for name, fn in (("zigzag", G.recursion_grid_zigzag), ("linear", G.recursion_grid_linear),
                         ("spiral", G.recursion_grid_spiral)):
            rec = fn(*g)
            out[f"g{i}_{name}_Z"] = rec.Z
            out[f"g{i}_{name}_perm"] = G.recursion_natural_permutation(rec)
        out[f"g{i}_params"] = np.array(g, dtype=np.float64)
    np.savez_compressed(os.path.join(HERE, "recugrid.npz"), **out)


def solver_case(name, C, normC, grid, p, r, seed):
    T = pre_process_dense(C)
    n = T.shape[0]
    rng = np.random.default_rng(seed)
    X0 = rng.random((n, r)) + 1j * rng.random((n, r))
    rec = G.recursion_grid(*grid)
    ctl = PsTriRecyControl(normC=normC, tol=1e-4, p_min=1, p=p, r=r, recy_tau=1.6)
    sig, st = ps_tri_recy_schur(T, rec, ctl, X0=X0)
    truth = np.array([dense_sigma_min(C, z) for z in rec.Z])
    assert np.max(np.abs(sig - truth)) <= 1e-4 * normC
    np.savez_compressed(os.path.join(HERE, f"pstrirecy_{name}.npz"), sigma=sig, truth=truth, Z=rec.Z,
                        grid=np.array(grid), p_count=st.p_count, r_recy=st.r_recy, refine_it=st.refine_it,
                        n_it=st.n_it, n_pts=st.n_pts, p=p, r=r, seed=seed, normC=normC)


if __name__ == "__main__":
    grids()
    solver_case("sprand200", sprand(200).toarray(), 3.2, (0.45, 0.55, 0.0, 0.1, 6, 6, 3), 60, 6, 5)
    solver_case("laser120", landau(120, 40 * np.pi), 1.0, (-1.1, 1.2, -1.1, 1.1, 6, 6, 2), 20, 4, 9)
    print("golden fixtures written to", HERE)
