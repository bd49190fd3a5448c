"""CPU restatement of the incomplete-Cholesky preconditioner apply — test infrastructure only.

SparseLLTP ldiv! (src/preconditioner/RLSPreconditioner.jl:79-116): for the factor L (sparse,
only its lower triangle used, as LowerTriangular(L) does), the permutation p and the stored
inverse invp,
    temp = B[p, :]          (:96-101)
    X    = L  \\ temp        (:103-104)
    temp = Lᴴ \\ X           (:105-106)
    X    = temp[invp, :]    (:108-113)
The triangular solves are SciPy's sparse forward / backward substitutions (FP64); a zero
diagonal raises SingularException(j) with the first such 1-based j, as Julia's sparse
triangular ldiv! does.  Parity is pinned to this definition (the reference ships no test
vectors for this operator).
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla


class SingularException(Exception):
    def __init__(self, j):
        super().__init__(f"SingularException({j})")
        self.j = j


def lltp_ldiv(L, p, invp, B):
    """X = P·L⁻ᴴ·L⁻¹·Pᴴ·B with 0-based p and invp (RLSPreconditioner.jl:79-116)."""
    Lt = sp.tril(sp.csr_matrix(L, dtype=np.complex128)).tocsr()
    Lt.sum_duplicates()
    d = Lt.diagonal()
    zero = np.flatnonzero(d == 0)
    if zero.size:
        raise SingularException(int(zero[0]) + 1)
    B = np.asarray(B, dtype=np.complex128)
    vec = B.ndim == 1
    B2 = B.reshape(B.shape[0], -1)
    temp = B2[np.asarray(p), :]
    X = spla.spsolve_triangular(Lt, temp, lower=True)
    temp = spla.spsolve_triangular(Lt.conj().T.tocsr(), X, lower=False)
    out = temp[np.asarray(invp), :]
    return out[:, 0] if vec else out

