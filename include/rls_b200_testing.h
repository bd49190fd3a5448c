/*
 * rls_b200_testing.h — kernel-level entry points of librls_b200.so used by the
 * parity tests.  They have no counterpart in the reference: each runs one device
 * routine of the engine on host inputs so that it can be compared with the
 * LAPACK routine the reference calls at that point.  Host pointers, column-major.
 * All but rls_test_lltp_plan_dense and rls_test_recip need rls_set_schur() and
 * rls_test_setup() first.
 */
#ifndef RLS_B200_TESTING_H
#define RLS_B200_TESTING_H

#include "rls_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Host only (no context, no device): the block-row form that rls_lltp_upload builds for
 * L (op = 0) or Lᴴ (op = 1), checked for what the device solve relies on (every off-block
 * term reads a block row solved before its own, indices in range, in-block terms strictly
 * on the solved side of the diagonal) and written out as the dense n × n operator it
 * stands for (n ≤ 4096, column-major; dense = NULL checks only, any n).  singular_at receives the first 1-based index with
 * a zero diagonal (0 if none), levels the longest chain of dependent block rows.  Compare
 * tril(L) or its adjoint. */
int rls_test_lltp_plan_dense(int64_t n, const int64_t* colptr, const int64_t* rowval, const rls_c64* nzval,
                             int base, int op, rls_c64* dense, int64_t* singular_at, int* levels);

/* Allocates the recycled-space and LOBPCG workspaces for block size r and p_max blocks. */
int rls_test_setup(rls_ctx* ctx, int r, int p_max);
/* X = (T − zI)⁻¹ B (adj = 0) or (T − zI)⁻ᴴ B (adj = 1); n × k.  Compare ZTRSM. */
int rls_test_trsm(rls_ctx* ctx, rls_c64 z, int adj, int k, const rls_c64* B, rls_c64* X);
/* Y = T X (adj = 0) or Tᴴ X (adj = 1); n × k.  Compare ZTRMM. */
int rls_test_trmm(rls_ctx* ctx, int adj, int k, const rls_c64* X, rls_c64* Y);
/* R of the QR factorisation of A (m × k); with Q != NULL also the orthonormal Q.
 * Compare ZGEQRF/ZUNGQR (rls_qr!). */
int rls_test_qr(rls_ctx* ctx, int64_t m, int k, const rls_c64* A, rls_c64* R, rls_c64* Q);
/* SVD Rayleigh–Ritz on R (nS × nS): σ (nS), λ (r), G (nS × nS).  Compare
 * svdRaylRitz! after its QR (ZGESDD + ZGELQF). */
int rls_test_svd_rr(rls_ctx* ctx, int nS, int r, int sideL, int lq, const rls_c64* R, double* sigma,
                    double* lam, rls_c64* G);
/* find_rr_dim! on Hz = H1 − zH2 − z̄H2ᴴ + (|z|²+shift)I: Ritz dimension, eigenvalues
 * (entries not computed are 0) and G (pr × rr).  Compare ZHEEVR.  clk (6 values,
 * may be NULL) receives the SM clock at the kernel's phase boundaries. */
int rls_test_heev_rr(rls_ctx* ctx, int pr, int r, const rls_c64* H1, const rls_c64* H2, rls_c64 z,
                     double shift, double tau, int* rr, double* lam, rls_c64* G, long long* clk);

/* The eigensolver's reciprocal (hardware estimate refined by two Newton steps) and CUDA's
 * 1.0/q on the same n inputs (host arrays).  Needs a context only. */
int rls_test_recip(rls_ctx* ctx, int64_t n, const double* q, double* r_nr, double* r_div);

/* updateRecycledSpace! (recySpace.jl:160-223) with X (n × r) on the device space
 * (r_sub = 1).  Compare the CPU restatement. */
int rls_test_space_update(rls_ctx* ctx, rls_c64 z, const rls_c64* X, double tau, int force_add, int p_min);
/* Copies out p and the device space: V, J1 = TᴴTV, J2 = TᴴV, J5 = TV (n × p r) and
 * L, H1, H2 (p r × p r).  NULL outputs are skipped. */
int rls_test_space_get(rls_ctx* ctx, int* p, rls_c64* V, rls_c64* J1, rls_c64* J2, rls_c64* J5, rls_c64* L,
                       rls_c64* H1, rls_c64* H2);
/* fastSvdRaylRitz_implicit! (fastRaylRitz.jl:99-219) on the device space: Ritz
 * dimension, σ (r), X, W (n × r) and |W[:,1]|. */
int rls_test_recycle(rls_ctx* ctx, rls_c64 z, double shift, double gap_tau, int* rr, double* sigma, rls_c64* X,
                     rls_c64* W, double* w0norm);

/* The band QR of a context given rls_set_sparse_tri: R of B − zI (B = PᵀCP) read back from the
 * band tiles the triangular solve uses, as a dense upper-triangular n × n matrix (column-major,
 * leading dimension ldr; zero outside the band), with the bandwidths l and u of B. */
int rls_test_band_r(rls_ctx* ctx, rls_c64 z, rls_c64* R, int64_t ldr, int64_t* l, int64_t* u);
/* The same factorisation (and the solve's scaled band tiles) without the read-back. */
int rls_test_band_factor(rls_ctx* ctx, rls_c64 z);

#ifdef __cplusplus
}
#endif

#endif /* RLS_B200_TESTING_H */
