"""The allocation-free R factor, rls_tsqr_r_noalloc, against the engine's own QR entry point.

rls_tsqr_r_noalloc serves callers that must not have this library allocate device memory
(an application whose pool allocator already holds the free memory, or a hot loop where
cudaMalloc would synchronise the device).  Its reduction tree lives in one fixed device
array shared by every call, so the checks below make two calls in a row on one stream:
the second runs on scratch that still holds the first call's contents.  Both R factors
must match what rls_test_qr (the context-based path over the same TSQR kernel) returns
for the same blocks.

The file is named to be collected last, and passes alone in a fresh process as well as
after the other GPU tests.  Test-side device buffers come from torch; the entry point
itself allocates nothing.
"""
import ctypes as C

import numpy as np
import pytest
import scipy.linalg as sla

from rls_b200._lib import lib, check, ptr, DimensionMismatch
from rls_b200.solvers import Engine

pytestmark = pytest.mark.gpu

# Same bound as the QR kernel tests: FP64 results within 1e-12 of the operand's norm.
RTOL = 1e-12
MAX_ROWS, MAX_COLS = 131072, 8


def crand(rng, *shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


@pytest.fixture(scope="module")
def qr_engine(cuda_device):
    rng = np.random.default_rng(11)
    n = 3000
    T = np.triu(crand(rng, n, n)) / np.sqrt(n) + 2.0 * np.eye(n)
    e = Engine(cuda_device)
    e.set_schur(T)
    check(lib().rls_test_setup(e._h, 6, 20), e._h)
    return e


def reference_r(e, A):
    m, k = A.shape
    R = np.zeros((k, k), dtype=np.complex128, order="F")
    Af = np.asfortranarray(A)          # named, so that it outlives the call that reads it
    check(lib().rls_test_qr(e._h, m, k, ptr(Af), ptr(R), None), e._h)
    return R


def to_device(torch, A, lda):
    """A (m × k) as a column-major device block with leading dimension lda."""
    m, k = A.shape
    buf = torch.zeros((k, lda), dtype=torch.complex128, device="cuda")
    buf[:, :m] = torch.from_numpy(np.ascontiguousarray(A.T)).to("cuda")
    return buf


def noalloc(torch, dA, lda, m, k, dR):
    stream = torch.cuda.current_stream().cuda_stream
    return lib().rls_tsqr_r_noalloc(C.c_void_p(dA.data_ptr()), lda, m, k, C.c_void_p(dR.data_ptr()),
                                    C.c_void_p(stream))


def test_two_calls_in_a_row_match_engine_qr(qr_engine):
    import torch
    rng = np.random.default_rng(5)
    cases = [(2900, 8, 3000), (1000, 3, 1000)]   # (m, k, lda); the second reuses stale scratch
    blocks, dRs = [], []
    for m, k, lda in cases:
        A = crand(rng, m, k) * np.logspace(0, -6, k)[None, :]
        blocks.append((A, to_device(torch, A, lda)))
        dRs.append(torch.full((k, k), complex(np.nan, np.nan), dtype=torch.complex128, device="cuda"))
    torch.cuda.synchronize()
    for (m, k, lda), (_, dA), dR in zip(cases, blocks, dRs):
        check(noalloc(torch, dA, lda, m, k, dR), None)
    torch.cuda.synchronize()
    for (m, k, lda), (A, _), dR in zip(cases, blocks, dRs):
        R = dR.cpu().numpy().T            # device buffer is column-major, ld = k
        Rref = reference_r(qr_engine, A)
        nA = np.linalg.norm(A)
        assert np.all(np.isfinite(R))
        assert np.allclose(np.tril(R, -1), 0)
        assert np.linalg.norm(R - Rref) <= RTOL * nA, (m, k, np.linalg.norm(R - Rref) / nA)
        # independent of the shared TSQR kernel: RᴴR reproduces AᴴA, and |diag R| matches
        # LAPACK's Householder QR
        assert np.linalg.norm(R.conj().T @ R - A.conj().T @ A) <= RTOL * nA ** 2
        assert np.allclose(np.abs(np.diag(R)), np.abs(np.diag(sla.qr(A, mode="r")[0])), rtol=1e-9, atol=0)


def test_largest_block_gives_gram_factor(cuda_device):
    """At the stated maximum size (131072 × 8) RᴴR reproduces AᴴA."""
    import torch
    rng = np.random.default_rng(9)
    m, k = MAX_ROWS, MAX_COLS
    A = crand(rng, m, k)
    dA = to_device(torch, A, m)
    dR = torch.zeros((k, k), dtype=torch.complex128, device="cuda")
    torch.cuda.synchronize()
    check(noalloc(torch, dA, m, m, k, dR), None)
    torch.cuda.synchronize()
    R = dR.cpu().numpy().T
    G = A.conj().T @ A
    assert np.linalg.norm(R.conj().T @ R - G) <= RTOL * np.linalg.norm(A) ** 2
    assert np.allclose(np.abs(np.diag(R)), np.abs(np.diag(sla.qr(A, mode="r")[0])), rtol=1e-10, atol=0)


@pytest.mark.parametrize("m,k,lda", [(MAX_ROWS + 1, 4, MAX_ROWS + 1), (100, MAX_COLS + 1, 100), (100, 4, 99),
                                     (0, 4, 1)])
def test_sizes_beyond_the_limits_are_rejected(cuda_device, m, k, lda):
    """Checked on the host before any launch; the message names the limit."""
    import torch
    dA = torch.zeros(8, dtype=torch.complex128, device="cuda")
    dR = torch.zeros(8, dtype=torch.complex128, device="cuda")
    st = noalloc(torch, dA, lda, m, k, dR)
    assert st == -2
    with pytest.raises(DimensionMismatch) as ei:
        check(st, None)
    assert "rls_tsqr_r_noalloc" in str(ei.value)
