"""CPU oracle for the σ_min(C − zI) grid engine — TEST INFRASTRUCTURE ONLY.

This package restates, in NumPy/SciPy, the algorithm of kuandeng/rls's
``psTriRecy`` hot path (grid ordering, recycled-subspace Rayleigh–Ritz,
block LOBPCG for singular values, recycled-space update).  Every function
cites the reference file:line it follows.  LAPACK is reached through
``scipy.linalg.lapack`` exactly where the reference ``ccall``s it
(zgeqrf/zungqr, zgesdd, zheevr, zgees).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg may import this package, and only as the checker.  The product path
(``rls_b200``) never imports it.

Parity status: UNPINNED against the reference itself.  The reference is pure
Julia, ships no tests, fixtures or golden vectors, and Julia is not installed
(so the reference cannot be run to produce any).  The restatement is checked
instead against an independent FP64 dense-SVD oracle (``dense_sigma_min``)
and against the committed fixtures under ``tests/golden/`` that this package
generated.
"""
