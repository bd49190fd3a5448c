// Device kernels for psPrecRecy's prediction stage (src/core/psPrecRecy.jl:727-908), where the
// recycled space has r_pred = 40 columns per block and up to p_pred = 20 blocks (pr ≤ 800),
// beyond the shared-memory kernels of the main stage (r ≤ 8, pr ≤ 360):
//   * shifted Cholesky-QR sweeps on Gram matrices of up to 3r = 120 columns in global memory
//     (_rls_qr_shiftchol!, src/types/RLSLinearAlgebra.jl:725-796);
//   * the Hermitian eigensolve of fastRaylRitz! (fastRaylRitz.jl:382-427) at pr ≤ 800: Hz built
//     with a general H3 (orth_S = false), Householder tridiagonalisation one column per pair of
//     multi-CTA launches (symmetric matrix-vector product, then the rank-2 update, whose CTA 0
//     also forms the next reflector), Sturm multisection and inverse iteration for the r
//     smallest eigenpairs, and a multi-CTA back-transformation;
//   * block-unitary rotations for any r (_block_unitary_update!, recySpace.jl:226-286), with
//     each 2r × 2r rotation staged in shared memory;
//   * column norms for the convergence tests of check_conv_svd (lobpcgSvd.jl:317-357).
// All FP64 complex.  Published methods only: Householder tridiagonalisation (Golub & Van Loan
// §8.3.1) with reflectors in the convention of LAPACK's zlarfg, bisection by Sturm counts
// (Barth, Martin & Wilkinson 1967), inverse iteration (Wilkinson), Cholesky-QR with a diagonal
// shift (Fukaya et al. 2020), as the reference's own LAPACK calls compute them.
#pragma once
#include "common.cuh"
#include "heev.cuh"
#include "small.cuh"

// ------------------------------------------------------------------------------------
// One sweep of the shifted Cholesky-QR on the Gram matrix W = XᴴX (k×k, ld k, global; only
// the upper triangle is read).  Factors W = RcᴴRc; while the factorisation breaks down, adds
// 11(mk + k(k+1))·eps·max_j W_jj to W's diagonal (in place, cumulatively, as the reference
// does) and retries.  Writes Rinv = Rc⁻¹ and Rtot ← Rc·Rtot (Rtot ← Rc on the first sweep).
// ws: 2k² cplx of global scratch.  One CTA.
// ------------------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_shiftchol_sweep(int k, int64_t m, cplx* W, cplx* Rinv, cplx* Rtot,
                                                         int first, cplx* ws, int* err) {
  cplx* F = ws;
  cplx* T = ws + (size_t)k * k;
  __shared__ double s_gmax;
  bool ok = false;
  for (int attempt = 0; attempt < 64 && !ok; ++attempt) {
    for (int q = threadIdx.x; q < k * k; q += blockDim.x) {
      const int i = q % k, c = q / k;
      cplx g = W[q];
      if (i == c) g = cmk(g.x, 0.0);
      F[q] = (i <= c) ? g : czero();
    }
    __syncthreads();
    ok = chol_upper(F, k, k);
    if (!ok) {
      if (threadIdx.x == 0) {
        double gm = 0.0;
        for (int i = 0; i < k; ++i) gm = fmax(gm, W[(size_t)i * k + i].x);
        s_gmax = gm;
      }
      __syncthreads();
      const double shift = 11.0 * ((double)m * k + (double)k * (k + 1)) * 2.220446049250313e-16 * s_gmax;
      for (int i = threadIdx.x; i < k; i += blockDim.x) W[(size_t)i * k + i].x += shift;
      __syncthreads();
    }
  }
  if (!ok) {
    if (threadIdx.x == 0) atomicOr(err, DEVERR_BREAKDOWN);
    for (int q = threadIdx.x; q < k * k; q += blockDim.x) F[q] = ((q % k) == (q / k)) ? cmk(1.0, 0.0) : czero();
    __syncthreads();
  }
  trtri_upper(F, k, Rinv, k, k);
  if (first) {
    for (int q = threadIdx.x; q < k * k; q += blockDim.x) Rtot[q] = F[q];
  } else {
    for (int q = threadIdx.x; q < k * k; q += blockDim.x) {
      const int i = q % k, c = q / k;
      cplx s = czero();
      for (int l = i; l <= c; ++l) s = cfma(F[(size_t)l * k + i], Rtot[(size_t)c * k + l], s);
      T[q] = s;
    }
    __syncthreads();
    for (int q = threadIdx.x; q < k * k; q += blockDim.x) Rtot[q] = T[q];
  }
}

// ‖W − I‖_F² of the k×k W (ld k) into out[0], one CTA, deterministic.
__global__ void k_dist_identity2(int k, const cplx* __restrict__ W, double* out) {
  __shared__ double red[32];
  double s = 0.0;
  for (int q = threadIdx.x; q < k * k; q += blockDim.x) {
    const cplx w = W[q];
    const double re = ((q % k) == (q / k)) ? w.x - 1.0 : w.x;
    s += re * re + w.y * w.y;
  }
  s = block_sum(s, red);
  if (threadIdx.x == 0) out[0] = s;
}

// Cholesky factor R (upper, GramE = RᴴR) and its inverse of the k×k GramE, as rls_cholesky!
// (RLSLinearAlgebra.jl:15-21, uplo :U) computes it; a non-positive pivot sets DEVERR_POSDEF
// (the reference throws PosDefException).  Global scratch ws (k²).  One CTA.
__global__ void __launch_bounds__(256) k_chol_plain(int k, const cplx* __restrict__ G, cplx* R, cplx* Rinv,
                                                    cplx* ws, int* err) {
  for (int q = threadIdx.x; q < k * k; q += blockDim.x) {
    const int i = q % k, c = q / k;
    cplx g = G[q];
    if (i == c) g = cmk(g.x, 0.0);
    ws[q] = (i <= c) ? g : czero();
  }
  __syncthreads();
  if (!chol_upper(ws, k, k)) {
    if (threadIdx.x == 0) atomicOr(err, DEVERR_POSDEF);
    for (int q = threadIdx.x; q < k * k; q += blockDim.x) ws[q] = ((q % k) == (q / k)) ? cmk(1.0, 0.0) : czero();
    __syncthreads();
  }
  if (R)
    for (int q = threadIdx.x; q < k * k; q += blockDim.x) R[q] = ws[q];
  trtri_upper(ws, k, Rinv, k, k);
}

// ------------------------------------------------------------------------------------
// Column norms: out[j] = ‖A[:, j]‖² for j < k (grid.x = k, one CTA per column).
// ------------------------------------------------------------------------------------
__global__ void k_colnorm2(int64_t nrows, const cplx* __restrict__ A, int64_t lda, double* out) {
  __shared__ double red[32];
  const cplx* a = A + (int64_t)blockIdx.x * lda;
  double s = 0.0;
  for (int64_t i = threadIdx.x; i < nrows; i += blockDim.x) s += cabs2(a[i]);
  s = block_sum(s, red);
  if (threadIdx.x == 0) out[blockIdx.x] = s;
}

// ------------------------------------------------------------------------------------
// Hz = H1 − z·H2 − z̄·H2ᴴ + (|z|² + shift)·H3 (affine_conbine!, fastRaylRitz.jl:6-28) from the
// upper triangles, written to both triangles of A (n×n, ld lda).  H3 == nullptr stands for I.
// z is read from device memory, so that a captured launch sequence serves every shift.
// ------------------------------------------------------------------------------------
__global__ void k_hz_build(int n, const cplx* __restrict__ H1, const cplx* __restrict__ H2,
                           const cplx* __restrict__ H3, int ldh, const cplx* __restrict__ zp, double shift, cplx* A,
                           int lda) {
  const cplx z = *zp;
  const double zz = z.x * z.x + z.y * z.y + shift;
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < (int64_t)n * n;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(q % n), j = (int)(q / n);
    const int ii = min(i, j), jj = max(i, j);
    cplx h = H1[(int64_t)jj * ldh + ii];
    h = cfms(z, H2[(int64_t)jj * ldh + ii], h);
    h = cfms(cconj(z), cconj(H2[(int64_t)ii * ldh + jj]), h);
    if (H3) h = cfma(cmk(zz, 0.0), H3[(int64_t)jj * ldh + ii], h);
    else if (ii == jj) h.x += zz;
    if (ii == jj) h.y = 0.0;
    A[(int64_t)j * lda + i] = (i <= j) ? h : cconj(h);
  }
}

// Reflector of column k of the Hermitian A (rows k+1..n-1; the column is final): v (rows
// k+1..n-1, v[k+1] = 1) into vbuf, τ into tau[k], e[k] = β, d[k] = A(k,k); the tail of the
// reflector is kept in A below row k+1 for the back-transformation.  One warp.
__device__ void trd_reflector(int k, int n, cplx* A, int lda, cplx* vbuf, cplx* tau, double* d, double* e) {
  const int lane = threadIdx.x & 31;
  const int m0 = k + 1;
  double x2 = 0.0;
  for (int i = m0 + 1 + lane; i < n; i += 32) x2 += cabs2(A[(int64_t)k * lda + i]);
  x2 = warp_sum(x2);
  const cplx alpha = A[(int64_t)k * lda + m0];
  double beta;
  cplx t, sc;
  householder_coeffs(alpha, x2, &beta, &t, &sc);
  for (int i = m0 + lane; i < n; i += 32) {
    const cplx vi = (i == m0) ? cmk(1.0, 0.0) : cmul(A[(int64_t)k * lda + i], sc);
    vbuf[i] = vi;
    if (i > m0) A[(int64_t)k * lda + i] = vi;
  }
  if (lane == 0) {
    tau[k] = t;
    e[k] = beta;
    d[k] = A[(int64_t)k * lda + k].x;
  }
}

__global__ void k_trd_first(int n, cplx* A, int lda, cplx* vbuf, cplx* tau, double* d, double* e) {
  if (n == 1) {                       // nothing to reduce: the 1 × 1 matrix is its own eigenvalue
    if (threadIdx.x == 0) d[0] = A[0].x;
    return;
  }
  if (threadIdx.x < 32) trd_reflector(0, n, A, lda, vbuf, tau, d, e);
}

// Step k, part 1: y_i = τ_k · Σ_j A(i, j) v_j for i ≥ k+1 (row i of A is column i conjugated:
// one warp per row, a contiguous sweep), and per-CTA partial sums of yᴴv into part[].
__global__ void __launch_bounds__(256) k_trd_symv(int k, int n, const cplx* __restrict__ A, int lda,
                                                  const cplx* __restrict__ v, const cplx* __restrict__ tau,
                                                  cplx* y, cplx* part) {
  __shared__ cplx red[8];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int m0 = k + 1;
  const cplx t = tau[k];
  cplx yv = czero();
  for (int i = m0 + blockIdx.x * 8 + w; i < n; i += gridDim.x * 8) {
    cplx s = czero();
    const cplx* col = A + (int64_t)i * lda;
    for (int j = m0 + lane; j < n; j += 32) s = cfmac(col[j], v[j], s);
    s = warp_sum(s);
    const cplx yi = cmul(t, s);
    if (lane == 0) y[i] = yi;
    yv = cfmac(yi, v[i], yv);
  }
  if (lane == 0) red[w] = yv;
  __syncthreads();
  if (threadIdx.x == 0) {
    cplx s = czero();
    for (int q = 0; q < 8; ++q) s = cadd(s, red[q]);
    part[blockIdx.x] = s;
  }
}

// Step k, part 2: α₂ = −½ τ yᴴv (partials summed in a fixed order by every CTA), w = y + α₂v,
// A −= v wᴴ + w vᴴ on the trailing block (columns spread over the CTAs).  The CTA that owns
// column k+1 then forms reflector k+1 from it (next launch reads it from vnext).
__global__ void __launch_bounds__(256) k_trd_update(int k, int n, cplx* A, int lda, const cplx* __restrict__ v,
                                                    cplx* tau, const cplx* __restrict__ y,
                                                    const cplx* __restrict__ part, int nparts, cplx* vnext,
                                                    double* d, double* e) {
  __shared__ cplx s_a2;
  const int m0 = k + 1;
  const cplx t = tau[k];
  if (threadIdx.x == 0) {
    cplx s = czero();
    for (int q = 0; q < nparts; ++q) s = cadd(s, part[q]);
    s_a2 = cscale(cmul(t, s), -0.5);
  }
  __syncthreads();
  const cplx a2 = s_a2;
  const bool active = (t.x != 0.0 || t.y != 0.0);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  // column j = m0 + blockIdx.x + gridDim.x·s: CTA 0 owns column m0 = k+1
  for (int j = m0 + blockIdx.x; j < n && active; j += gridDim.x) {
    const cplx vj = v[j], wj = cfma(a2, vj, y[j]);
    cplx* col = A + (int64_t)j * lda;
    for (int i = m0 + threadIdx.x; i < n; i += blockDim.x) {
      const cplx vi = v[i], wi = cfma(a2, vi, y[i]);
      cplx aij = col[i];
      aij = csub(aij, cmulc(wj, vi));
      aij = csub(aij, cmulc(vj, wi));
      col[i] = aij;
    }
  }
  (void)lane; (void)w;
  if (blockIdx.x == 0 && k + 1 < n - 1) {
    __syncthreads();
    if (threadIdx.x < 32) trd_reflector(k + 1, n, A, lda, vnext, tau, d, e);
  }
  if (blockIdx.x == 0 && k + 1 == n - 1 && threadIdx.x == 0) d[n - 1] = A[(int64_t)(n - 1) * lda + (n - 1)].x;
}

// Eigenvalues 0..nvec-1 (ascending) of the real symmetric tridiagonal (d, e) by Sturm
// multisection (one warp per eigenvalue), eigenvectors by inverse iteration with a partially
// pivoted tridiagonal LU (one warp per vector, lu: 16 warps × 6n doubles of global scratch),
// then CGS2 over the vectors in index order.  S (n × nvec, ld lds) gets the real vectors.
// One CTA of 512 threads.
__global__ void __launch_bounds__(512) k_trd_eigvecs(int n, const double* __restrict__ d,
                                                     const double* __restrict__ e, int nvec, double* lam_out,
                                                     cplx* S, int lds, double* lu, double* e2g, int* err) {
  __shared__ double red[32];
  __shared__ double s_gl, s_gu, s_piv, s_nrm;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  double* e2 = e2g;
  for (int i = threadIdx.x; i < n - 1; i += blockDim.x) e2[i] = e[i] * e[i];
  __syncthreads();
  if (threadIdx.x == 0) {
    double gl = 1e300, gu = -1e300, emax = 0.0;
    for (int i = 0; i < n; ++i) {
      const double off = ((i > 0) ? fabs(e[i - 1]) : 0.0) + ((i < n - 1) ? fabs(e[i]) : 0.0);
      gl = fmin(gl, d[i] - off);
      gu = fmax(gu, d[i] + off);
      if (i < n - 1) emax = fmax(emax, e2[i]);
    }
    const double tnorm = fmax(fabs(gl), fabs(gu));
    gl -= 2.0 * tnorm * 2.220446049250313e-16 * n + 1e-300;
    gu += 2.0 * tnorm * 2.220446049250313e-16 * n + 1e-300;
    s_gl = gl; s_gu = gu;
    s_piv = fmax(2.2250738585072014e-308, 2.2250738585072014e-308 * emax) * 4.0;
  }
  __syncthreads();
  const double gl = s_gl, gu = s_gu, pivmin = s_piv;
  const double atol = 1e-14 * fmax(fabs(gl), fabs(gu));
  for (int j = warp; j < nvec; j += nw) {
    const double lj = (n == 1) ? d[0] : warp_eig_index(d, e2, n, j, gl, gu, pivmin, atol);
    if (lane == 0) lam_out[j] = lj;
  }
  __syncthreads();
  {
    const double tnorm = fmax(fabs(gl), fabs(gu));
    const double tiny = 2.220446049250313e-16 * tnorm + 1e-300;
    for (int j = warp; j < nvec; j += nw) {
      double* l6 = lu + (int64_t)warp * 6 * n;
      double *u0 = l6, *u1 = l6 + n, *u2 = l6 + 2 * n, *l = l6 + 3 * n, *pv = l6 + 4 * n, *x = l6 + 5 * n;
      const double lamj = lam_out[j] + tiny * ((j & 1) ? 1.0 : -1.0);
      if (lane == 0) tri_lu(d, e, n, lamj, u0, u1, u2, l, pv, tiny);
      for (int i = lane; i < n; i += 32) {
        uint32_t h = (uint32_t)(i * 2654435761u) ^ (uint32_t)((j + 1) * 2246822519u);
        h ^= h >> 15; h *= 2654435761u; h ^= h >> 13;
        x[i] = 0.5 + (double)(h & 0xffff) / 65536.0;
      }
      __syncwarp();
      for (int it = 0; it < 2; ++it) {
        if (lane == 0) tri_solve(n, u0, u1, u2, l, pv, x);
        __syncwarp();
        double ss = 0.0;
        for (int i = lane; i < n; i += 32) ss += x[i] * x[i];
        ss = warp_sum(ss);
        const double inv = (ss > 0.0 && isfinite(ss)) ? 1.0 / sqrt(ss) : 0.0;
        for (int i = lane; i < n; i += 32) x[i] *= inv;
        __syncwarp();
      }
      for (int i = lane; i < n; i += 32) S[(int64_t)j * lds + i] = cmk(x[i], 0.0);
      __syncwarp();
    }
  }
  __syncthreads();
  // CGS2 in index order (keeps a cluster's invariant subspace); coefficients in lu's first row
  double* coef = lu;
  for (int j = 0; j < nvec; ++j) {
    double* gj = reinterpret_cast<double*>(S + (int64_t)j * lds);
    for (int pass = 0; pass < 2 && j > 0; ++pass) {
      for (int q = warp; q < j; q += nw) {
        const double* gq = reinterpret_cast<const double*>(S + (int64_t)q * lds);
        double sq = 0.0;
        for (int i = lane; i < n; i += 32) sq += gq[2 * i] * gj[2 * i];
        sq = warp_sum(sq);
        if (lane == 0) coef[q] = sq;
      }
      __syncthreads();
      for (int i = threadIdx.x; i < n; i += blockDim.x) {
        double acc = 0.0;
        for (int q = 0; q < j; ++q) acc += coef[q] * reinterpret_cast<const double*>(S + (int64_t)q * lds)[2 * i];
        gj[2 * i] -= acc;
      }
      __syncthreads();
    }
    double sq = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) sq += gj[2 * i] * gj[2 * i];
    sq = block_sum(sq, red);
    if (threadIdx.x == 0) s_nrm = (sq > 0.0) ? 1.0 / sqrt(sq) : 0.0;
    __syncthreads();
    const double inv = s_nrm;
    for (int i = threadIdx.x; i < n; i += blockDim.x) gj[2 * i] *= inv;
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    bool bad = false;
    for (int j = 0; j < nvec; ++j) bad |= !isfinite(lam_out[j]);
    if (bad) atomicOr(err, DEVERR_NONFINITE);
  }
}

// Back-transformation G = H_0 H_1 ⋯ H_{n-2} S (H_{n-2} applied first), 16 lanes per vector,
// vectors spread over the CTAs (blockDim 256: 16 vectors per CTA).  G is S, in place.
__global__ void __launch_bounds__(256) k_trd_backtransform(int n, const cplx* __restrict__ A, int lda,
                                                           const cplx* __restrict__ tau, cplx* G, int ldg,
                                                           int nvec) {
  const int half = threadIdx.x >> 4, hl = threadIdx.x & 15;
  const int j = blockIdx.x * (blockDim.x >> 4) + half;
  const bool act = j < nvec;
  cplx* sj = G + (int64_t)(act ? j : 0) * ldg;
  for (int k = n - 2; k >= 0; --k) {
    const int m0 = k + 1;
    const cplx t = tau[k];
    if (t.x == 0.0 && t.y == 0.0) continue;
    cplx sum = czero();
    if (act)
      for (int i = m0 + hl; i < n; i += 16) {
        const cplx vi = (i == m0) ? cmk(1.0, 0.0) : A[(int64_t)k * lda + i];
        sum = cfmac(vi, sj[i], sum);
      }
#pragma unroll
    for (int o = 8; o > 0; o >>= 1) {
      sum.x += __shfl_xor_sync(0xffffffffu, sum.x, o);
      sum.y += __shfl_xor_sync(0xffffffffu, sum.y, o);
    }
    const cplx f = cmul(t, sum);
    if (act)
      for (int i = m0 + hl; i < n; i += 16) {
        const cplx vi = (i == m0) ? cmk(1.0, 0.0) : A[(int64_t)k * lda + i];
        sj[i] = cfms(vi, f, sj[i]);
      }
    __syncwarp();
  }
}

// ------------------------------------------------------------------------------------
// Block-unitary rotations for any block width r (the main stage's kernels in rotate.cuh
// hold a 2r × r block per warp and serve r ≤ 8).  Conventions as there: rotation i is
// U_i = Qᴴ, Q the full unitary of the Householder QR of [L(p,p); L(i,p)] (2r × r);
// U_i is stored column-major (2r × 2r).
// k_blockrot_coeffs_g: one CTA; the last block column of L is copied to ws (pr × r), the
// 2r × r block and the 2r × 2r Q are formed in ws too.
// ------------------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_blockrot_coeffs_g(int p, int r, const cplx* __restrict__ L, int ld,
                                                           cplx* Uout, cplx* ws) {
  __shared__ double red[32];
  const int r2 = 2 * r, pr = p * r, bp = p - 1;
  cplx* Lc = ws;                          // pr × r
  cplx* Y = Lc + (size_t)pr * r;          // 2r × r
  cplx* Q = Y + (size_t)r2 * r;           // 2r × 2r
  cplx* tau = Q + (size_t)r2 * r2;        // r
  cplx* wb = tau + r;                     // 2r
  for (int q = threadIdx.x; q < pr * r; q += blockDim.x) Lc[q] = L[(int64_t)(bp * r + q / pr) * ld + (q % pr)];
  __syncthreads();
  for (int i = 0; i < p - 1; ++i) {
    for (int q = threadIdx.x; q < r2 * r; q += blockDim.x) {
      const int a = q % r2, c = q / r2;
      const int row = (a < r) ? bp * r + a : i * r + (a - r);
      Y[(size_t)c * r2 + a] = Lc[(size_t)c * pr + row];
    }
    __syncthreads();
    house_qr_block(Y, r2, r2, r, tau, wb, red);
    // Q = H_0 ⋯ H_{r-1} applied to I (last reflector first), then U = Qᴴ
    for (int q = threadIdx.x; q < r2 * r2; q += blockDim.x) Q[q] = ((q % r2) == (q / r2)) ? cmk(1.0, 0.0) : czero();
    __syncthreads();
    for (int j = r - 1; j >= 0; --j) {
      const cplx tj = tau[j];
      for (int c = threadIdx.x; c < r2; c += blockDim.x) {
        cplx s = czero();
        for (int a = j; a < r2; ++a) {
          const cplx va = (a == j) ? cmk(1.0, 0.0) : Y[(size_t)j * r2 + a];
          s = cfmac(va, Q[(size_t)c * r2 + a], s);
        }
        const cplx f = cmul(tj, s);
        for (int a = j; a < r2; ++a) {
          const cplx va = (a == j) ? cmk(1.0, 0.0) : Y[(size_t)j * r2 + a];
          Q[(size_t)c * r2 + a] = cfms(va, f, Q[(size_t)c * r2 + a]);
        }
      }
      __syncthreads();
    }
    cplx* U = Uout + (size_t)i * r2 * r2;
    for (int q = threadIdx.x; q < r2 * r2; q += blockDim.x) {
      const int a = q % r2, c = q / r2;             // U(a, c) = conj(Q(c, a))
      U[q] = cconj(Q[(size_t)a * r2 + c]);
    }
    // the rotated last block column: block p ← R, block i ← 0
    for (int q = threadIdx.x; q < r2 * r; q += blockDim.x) {
      const int a = q % r2, c = q / r2;
      const int row = (a < r) ? bp * r + a : i * r + (a - r);
      Lc[(size_t)c * pr + row] = (a < r && a <= c) ? Y[(size_t)c * r2 + a] : czero();
    }
    __syncthreads();
  }
}

// Right products [X_p, X_i] ← [X_p, X_i] U_iᴴ, i = 0..p-2 in order, on up to 10 arrays
// (blockIdx.y selects one): BR_ROWS rows per CTA; U_i and the row tile in shared memory.
// Dynamic shared memory: (BR_ROWS · 2r + (2r)²) cplx.
constexpr int BR_ROWS = 32;
struct RotArraysG {
  cplx* a[10];
  int64_t nrows[10];
  int64_t ld[10];
};

__global__ void __launch_bounds__(256) k_blockrot_apply_g(int p, int r, RotArraysG arr,
                                                          const cplx* __restrict__ Ulist) {
  extern __shared__ cplx sm[];
  const int r2 = 2 * r;
  cplx* old = sm;                       // BR_ROWS × r2, old[row * r2 + a]
  cplx* U = old + BR_ROWS * r2;         // r2 × r2
  cplx* A = arr.a[blockIdx.y];
  const int64_t nrows = arr.nrows[blockIdx.y], ld = arr.ld[blockIdx.y];
  const int64_t r0 = (int64_t)blockIdx.x * BR_ROWS;
  if (r0 >= nrows || !A) return;
  const int bp = p - 1;
  for (int q = threadIdx.x; q < BR_ROWS * r; q += blockDim.x) {
    const int tr = q % BR_ROWS, a = q / BR_ROWS;
    const int64_t row = r0 + tr;
    old[tr * r2 + a] = (row < nrows) ? A[(int64_t)(bp * r + a) * ld + row] : czero();
  }
  for (int i = 0; i < p - 1; ++i) {
    for (int q = threadIdx.x; q < BR_ROWS * r; q += blockDim.x) {
      const int tr = q % BR_ROWS, a = q / BR_ROWS;
      const int64_t row = r0 + tr;
      old[tr * r2 + r + a] = (row < nrows) ? A[(int64_t)(i * r + a) * ld + row] : czero();
    }
    for (int q = threadIdx.x; q < r2 * r2; q += blockDim.x) U[q] = Ulist[(size_t)i * r2 * r2 + q];
    __syncthreads();
    // out(tr, a) = Σ_l old(tr, l) · conj(U(a, l)); a thread owns (tr, a) pairs
    constexpr int MAXO = 16;
    cplx outv[MAXO];
    int nout = 0;
    for (int q = threadIdx.x; q < BR_ROWS * r2 && nout < MAXO; q += blockDim.x, ++nout) {
      const int tr = q % BR_ROWS, a = q / BR_ROWS;
      cplx s = czero();
      for (int l = 0; l < r2; ++l) s = cfma(old[tr * r2 + l], cconj(U[(size_t)l * r2 + a]), s);
      outv[nout] = s;
    }
    __syncthreads();
    nout = 0;
    for (int q = threadIdx.x; q < BR_ROWS * r2 && nout < MAXO; q += blockDim.x, ++nout) {
      const int tr = q % BR_ROWS, a = q / BR_ROWS;
      const int64_t row = r0 + tr;
      if (a < r) old[tr * r2 + a] = outv[nout];
      else if (row < nrows) A[(int64_t)(i * r + (a - r)) * ld + row] = outv[nout];
    }
    __syncthreads();
  }
  for (int q = threadIdx.x; q < BR_ROWS * r; q += blockDim.x) {
    const int tr = q % BR_ROWS, a = q / BR_ROWS;
    const int64_t row = r0 + tr;
    if (row < nrows) A[(int64_t)(bp * r + a) * ld + row] = old[tr * r2 + a];
  }
}

// Left products [X_p; X_i] ← U_i [X_p; X_i] on the block rows of up to 4 pr×pr matrices
// (blockIdx.y), BR_ROWS columns per CTA.  Same shared-memory layout as k_blockrot_apply_g.
struct RotMatsG {
  cplx* m[4];
};

__global__ void __launch_bounds__(256) k_blockrot_left_g(int p, int r, RotMatsG mats, int ld,
                                                         const cplx* __restrict__ Ulist) {
  extern __shared__ cplx sm[];
  const int r2 = 2 * r, pr = p * r;
  cplx* old = sm;                       // BR_ROWS (columns) × r2
  cplx* U = old + BR_ROWS * r2;
  cplx* M = mats.m[blockIdx.y];
  if (!M) return;
  const int c0 = blockIdx.x * BR_ROWS;
  const int bp = p - 1;
  for (int q = threadIdx.x; q < BR_ROWS * r; q += blockDim.x) {
    const int tc = q % BR_ROWS, a = q / BR_ROWS;
    const int col = c0 + tc;
    old[tc * r2 + a] = (col < pr) ? M[(int64_t)col * ld + bp * r + a] : czero();
  }
  for (int i = 0; i < p - 1; ++i) {
    for (int q = threadIdx.x; q < BR_ROWS * r; q += blockDim.x) {
      const int tc = q % BR_ROWS, a = q / BR_ROWS;
      const int col = c0 + tc;
      old[tc * r2 + r + a] = (col < pr) ? M[(int64_t)col * ld + i * r + a] : czero();
    }
    for (int q = threadIdx.x; q < r2 * r2; q += blockDim.x) U[q] = Ulist[(size_t)i * r2 * r2 + q];
    __syncthreads();
    constexpr int MAXO = 16;
    cplx outv[MAXO];
    int nout = 0;
    for (int q = threadIdx.x; q < BR_ROWS * r2 && nout < MAXO; q += blockDim.x, ++nout) {
      const int tc = q % BR_ROWS, a = q / BR_ROWS;
      cplx s = czero();
      for (int l = 0; l < r2; ++l) s = cfma(U[(size_t)l * r2 + a], old[tc * r2 + l], s);
      outv[nout] = s;
    }
    __syncthreads();
    nout = 0;
    for (int q = threadIdx.x; q < BR_ROWS * r2 && nout < MAXO; q += blockDim.x, ++nout) {
      const int tc = q % BR_ROWS, a = q / BR_ROWS;
      const int col = c0 + tc;
      if (a < r) old[tc * r2 + a] = outv[nout];
      else if (col < pr) M[(int64_t)col * ld + i * r + (a - r)] = outv[nout];
    }
    __syncthreads();
  }
  for (int q = threadIdx.x; q < BR_ROWS * r; q += blockDim.x) {
    const int tc = q % BR_ROWS, a = q / BR_ROWS;
    const int col = c0 + tc;
    if (col < pr) M[(int64_t)col * ld + bp * r + a] = old[tc * r2 + a];
  }
}

inline size_t blockrot_g_smem(int r) { return ((size_t)BR_ROWS * 2 * r + (size_t)4 * r * r) * sizeof(cplx); }
