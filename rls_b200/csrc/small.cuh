// Small dense FP64 kernels run by a single CTA: Householder QR factors (TSQR leaves),
// one-sided Jacobi SVD, Cholesky/triangular inverse, the LQ step of LOBPCG's
// Rayleigh–Ritz, block-unitary rotations of the recycled space, small GEMM.
#pragma once
#include "common.cuh"

// ------------------------------------------------------------------------------------
// Householder reflector in the convention of LAPACK's zlarfg: given alpha and
// |x|^2, returns beta (real), tau and the scale 1/(alpha − beta) for x, so that
// (I − tau v vᴴ)ᴴ [alpha; x] = [beta; 0] with v = [1; x/(alpha − beta)].
// The magnitude of beta is |[alpha; x]|; its sign is −sign(Re alpha).
// ------------------------------------------------------------------------------------
__device__ __forceinline__ void householder_coeffs(cplx alpha, double xnorm2, double* beta, cplx* tau,
                                                   cplx* scal) {
  if (xnorm2 == 0.0 && alpha.y == 0.0) {
    *beta = alpha.x;
    *tau = czero();
    *scal = czero();
    return;
  }
  const double nrm = sqrt(alpha.x * alpha.x + alpha.y * alpha.y + xnorm2);
  const double b = (alpha.x >= 0.0) ? -nrm : nrm;
  *beta = b;
  *tau = cmk((b - alpha.x) / b, -alpha.y / b);
  *scal = cinv(cmk(alpha.x - b, alpha.y));
}

// ------------------------------------------------------------------------------------
// In-place Householder QR of the m×k block A (column-major, lda) held by one CTA.
// On exit the upper triangle holds R (diagonal real, LAPACK signs) and the strict
// lower part holds the reflector tails; tau[j] holds the reflector scalars.
// Requires blockDim.x a multiple of 32, `red` >= 32 doubles, `wbuf` >= k cplx.
// ------------------------------------------------------------------------------------
__device__ void house_qr_block(cplx* A, int lda, int m, int k, cplx* tau, cplx* wbuf, double* red) {
  __shared__ double s_beta;
  __shared__ cplx s_tau, s_scal;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int kk = min(m, k);
  for (int j = 0; j < kk; ++j) {
    double x2 = 0.0;
    for (int i = j + 1 + threadIdx.x; i < m; i += blockDim.x) x2 += cabs2(A[j * lda + i]);
    x2 = block_sum(x2, red);
    if (threadIdx.x == 0) {
      double beta; cplx t, sc;
      householder_coeffs(A[j * lda + j], x2, &beta, &t, &sc);
      s_beta = beta; s_tau = t; s_scal = sc;
      tau[j] = t;
    }
    __syncthreads();
    const cplx sc = s_scal, t = s_tau;
    for (int i = j + 1 + threadIdx.x; i < m; i += blockDim.x) A[j * lda + i] = cmul(A[j * lda + i], sc);
    __syncthreads();
    if (threadIdx.x == 0) A[j * lda + j] = cmk(s_beta, 0.0);
    // w_c = vᴴ A[j:, c]   (v_j = 1)
    for (int c = j + 1 + warp; c < k; c += nw) {
      cplx s = czero();
      for (int i = j + lane; i < m; i += 32) {
        const cplx v = (i == j) ? cmk(1.0, 0.0) : A[j * lda + i];
        s = cfmac(v, A[c * lda + i], s);
      }
      s = warp_sum(s);
      if (lane == 0) wbuf[c] = s;
    }
    __syncthreads();
    // A[j:, c] -= conj(tau) v w_c
    const cplx tc = cconj(t);
    const int rows = m - j, cols = k - j - 1;
    for (int q = threadIdx.x; q < rows * cols; q += blockDim.x) {
      const int i = j + q % rows, c = j + 1 + q / rows;
      const cplx v = (i == j) ? cmk(1.0, 0.0) : A[j * lda + i];
      A[c * lda + i] = cfms(cmul(tc, v), wbuf[c], A[c * lda + i]);
    }
    __syncthreads();
  }
}

// ------------------------------------------------------------------------------------
// TSQR leaf: CTA b factors rows [b*mb, min(m, (b+1)*mb)) of A (m×k) and writes its
// R (k×k, zeros below the diagonal) into rows [b*k, b*k+k) of `stack` (ld = lds).
// Shared memory: mb*k + 2k cplx.
// ------------------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_tsqr_leaf(int64_t m, int k, int mb, const cplx* __restrict__ A,
                                                   int64_t lda, cplx* __restrict__ stack, int64_t lds) {
  extern __shared__ cplx sm[];
  __shared__ double red[32];
  cplx* sA = sm;
  cplx* tau = sA + (size_t)mb * k;
  cplx* wbuf = tau + k;
  const int64_t r0 = (int64_t)blockIdx.x * mb;
  const int rows = (int)min((int64_t)mb, m - r0);
  for (int q = threadIdx.x; q < mb * k; q += blockDim.x) {
    const int i = q % mb, c = q / mb;
    sA[c * mb + i] = (i < rows) ? A[(int64_t)c * lda + r0 + i] : czero();
  }
  __syncthreads();
  house_qr_block(sA, mb, max(rows, k), k, tau, wbuf, red);
  for (int q = threadIdx.x; q < k * k; q += blockDim.x) {
    const int i = q % k, c = q / k;
    stack[(int64_t)c * lds + (int64_t)blockIdx.x * k + i] = (i <= c) ? sA[c * mb + i] : czero();
  }
}

// ------------------------------------------------------------------------------------
// One-warp TSQR leaf for narrow blocks (k <= 8): warp w of the CTA factors rows
// [leaf*64, leaf*64 + 64) of A (m × k), leaf = blockIdx.x*8 + w, each lane holding two
// rows in registers; reductions are warp shuffles only.  R (k × k, zeros below the
// diagonal) goes to rows [leaf*k, leaf*k + k) of `stack` (ld = lds).
// ------------------------------------------------------------------------------------
template <int KW>
__global__ void __launch_bounds__(256) k_tsqr_warp(int64_t m, int k, const cplx* __restrict__ A, int64_t lda,
                                                   cplx* __restrict__ stack, int64_t lds, int64_t nleaf) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t leaf = (int64_t)blockIdx.x * 8 + w;
  if (leaf >= nleaf) return;
  const int64_t r0 = leaf * 64;
  cplx a0[KW], a1[KW];   // rows r0 + lane and r0 + 32 + lane
#pragma unroll
  for (int c = 0; c < KW; ++c) {
    const int64_t i0 = r0 + lane, i1 = r0 + 32 + lane;
    a0[c] = (c < k && i0 < m) ? A[(int64_t)c * lda + i0] : czero();
    a1[c] = (c < k && i1 < m) ? A[(int64_t)c * lda + i1] : czero();
  }
  // R row j lives in lane j's register rj[] after step j (k <= 8 < 32)
  cplx rrow[KW];
#pragma unroll
  for (int c = 0; c < KW; ++c) rrow[c] = czero();
#pragma unroll
  for (int j = 0; j < KW; ++j) {
    if (j < k) {
      // pivot row j: held by lane j (row j < 32 of the leaf) in a0
      const cplx alpha = cmk(__shfl_sync(0xffffffffu, a0[j].x, j), __shfl_sync(0xffffffffu, a0[j].y, j));
      double x2 = (lane > j ? cabs2(a0[j]) : 0.0) + cabs2(a1[j]);
      x2 = warp_sum(x2);
      double beta; cplx t, sc;
      householder_coeffs(alpha, x2, &beta, &t, &sc);
      // v: v_j = 1 (lane j, a0), v_i = x_i * sc below; rows above j are 0
      const cplx v0 = (lane == j) ? cmk(1.0, 0.0) : ((lane > j) ? cmul(a0[j], sc) : czero());
      const cplx v1 = cmul(a1[j], sc);
      const cplx tc = cconj(t);
      // columns c > j: s_c = vᴴ a_c, a_c −= conj(τ) v s_c
#pragma unroll
      for (int c = 0; c < KW; ++c) {
        if (c > j && c < k) {
          cplx sdot = cfmac(v1, a1[c], cfmac(v0, a0[c], czero()));
          sdot = warp_sum(sdot);
          const cplx f = cmul(tc, sdot);
          a0[c] = cfms(v0, f, a0[c]);
          a1[c] = cfms(v1, f, a1[c]);
        }
      }
      // column j becomes [.., beta at row j, 0 below]
      if (lane == j) a0[j] = cmk(beta, 0.0);
      else if (lane > j) a0[j] = czero();
      a1[j] = czero();
    }
  }
  // R = upper k×k of the leaf (rows 0..k-1 are lanes 0..k-1 of a0)
#pragma unroll
  for (int c = 0; c < KW; ++c)
    if (c < k && lane < k) stack[(int64_t)c * lds + leaf * k + lane] = (lane <= c) ? a0[c] : czero();
}

// Generic in-global Householder QR factor R of an m×k matrix by one CTA (slow path for
// wide k).  A is overwritten.  R (k×k, ldr) gets the upper triangle, zeros below.
__global__ void __launch_bounds__(512) k_house_r_global(int m, int k, cplx* A, int lda, cplx* tau,
                                                        cplx* wbuf, cplx* R, int ldr) {
  __shared__ double red[32];
  house_qr_block(A, lda, m, k, tau, wbuf, red);
  for (int q = threadIdx.x; q < k * k; q += blockDim.x) {
    const int i = q % k, c = q / k;
    R[c * ldr + i] = (i <= c && i < m) ? A[c * lda + i] : czero();
  }
}

// ------------------------------------------------------------------------------------
// One-sided (Hestenes) Jacobi SVD of the n×n matrix A by one CTA, columns updated in
// place; V accumulates the right rotations.  Pairs follow the round-robin schedule,
// one warp per pair.  On exit sigma[i] = |A(:,i)| sorted descending (or ascending)
// with V's columns permuted alike.  `A`, `V` may live in shared or global memory.
// ------------------------------------------------------------------------------------
__device__ void jacobi_svd(cplx* A, int lda, cplx* V, int ldv, int n, double* sigma, bool ascending,
                           int* perm_buf, double* nrm_buf) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const double eps = 2.220446049250313e-16;
  __shared__ int s_rot;
  for (int q = threadIdx.x; q < n * n; q += blockDim.x) {
    const int i = q % n, c = q / n;
    V[c * ldv + i] = (i == c) ? cmk(1.0, 0.0) : czero();
  }
  __syncthreads();
  const int np = (n + 1) & ~1;  // even number of slots (slot n is a dummy when n is odd)
  for (int sweep = 0; sweep < 40; ++sweep) {
    if (threadIdx.x == 0) s_rot = 0;
    __syncthreads();
    for (int step = 0; step < np - 1; ++step) {
      for (int pi = warp; pi < np / 2; pi += nw) {
        // round-robin: slot 0 fixed, others rotate
        int a = (pi == 0) ? 0 : ((pi + step - 1) % (np - 1)) + 1;
        int b = ((np - 1 - pi + step - 1) % (np - 1)) + 1;
        if (pi == 0) b = ((step + np - 2) % (np - 1)) + 1;
        int p = min(a, b), qq = max(a, b);
        if (qq >= n || p == qq) continue;
        double al = 0.0, be = 0.0;
        cplx ga = czero();
        for (int i = lane; i < n; i += 32) {
          const cplx x = A[p * lda + i], y = A[qq * lda + i];
          al += cabs2(x); be += cabs2(y); ga = cfmac(x, y, ga);
        }
        al = warp_sum(al); be = warp_sum(be); ga = warp_sum(ga);
        const double gabs = sqrt(cabs2(ga));
        if (gabs > eps * sqrt(al * be) && gabs > 1e-300) {
          const double zeta = (be - al) / (2.0 * gabs);
          const double t = (zeta >= 0.0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
          const double cs = 1.0 / sqrt(1.0 + t * t), sn = cs * t;
          const cplx ph = cmk(ga.x / gabs, -ga.y / gabs);  // e^{-i phi}
          for (int i = lane; i < n; i += 32) {
            const cplx x = A[p * lda + i], y = cmul(ph, A[qq * lda + i]);
            A[p * lda + i] = csub(cscale(x, cs), cscale(y, sn));
            A[qq * lda + i] = cadd(cscale(x, sn), cscale(y, cs));
            const cplx vx = V[p * ldv + i], vy = cmul(ph, V[qq * ldv + i]);
            V[p * ldv + i] = csub(cscale(vx, cs), cscale(vy, sn));
            V[qq * ldv + i] = cadd(cscale(vx, sn), cscale(vy, cs));
          }
          if (lane == 0) s_rot = 1;
        }
      }
      __syncthreads();
    }
    const int rot = s_rot;
    __syncthreads();
    if (!rot) break;
  }
  // norms and sort (selection by rank; n is small)
  for (int c = warp; c < n; c += nw) {
    double s = 0.0;
    for (int i = lane; i < n; i += 32) s += cabs2(A[c * lda + i]);
    s = warp_sum(s);
    if (lane == 0) nrm_buf[c] = sqrt(s);
  }
  __syncthreads();
  for (int c = threadIdx.x; c < n; c += blockDim.x) {
    int rank = 0;
    const double v = nrm_buf[c];
    for (int o = 0; o < n; ++o) {
      const double w = nrm_buf[o];
      const bool before = ascending ? (w < v || (w == v && o < c)) : (w > v || (w == v && o < c));
      rank += before ? 1 : 0;
    }
    perm_buf[rank] = c;
  }
  __syncthreads();
  for (int c = threadIdx.x; c < n; c += blockDim.x) sigma[c] = nrm_buf[perm_buf[c]];
  // permute V's columns through A's storage (A is no longer needed)
  for (int q = threadIdx.x; q < n * n; q += blockDim.x) {
    const int i = q % n, c = q / n;
    A[c * lda + i] = V[perm_buf[c] * ldv + i];
  }
  __syncthreads();
  for (int q = threadIdx.x; q < n * n; q += blockDim.x) {
    const int i = q % n, c = q / n;
    V[c * ldv + i] = A[c * lda + i];
  }
  __syncthreads();
}

// ------------------------------------------------------------------------------------
// Explicit thin Q (m×k, m >= k) of the Householder QR of B (m×k) by one warp, in
// place (B is overwritten with Q).  Q = H_0 H_1 ... H_{k-1} [I; 0] is accumulated
// backwards as LAPACK's zung2r does.
// ------------------------------------------------------------------------------------
__device__ void warp_house_q(cplx* B, int ldb, int m, int k, cplx* tau) {
  const int lane = threadIdx.x & 31;
  for (int j = 0; j < k; ++j) {
    double x2 = 0.0;
    for (int i = j + 1 + lane; i < m; i += 32) x2 += cabs2(B[j * ldb + i]);
    x2 = warp_sum(x2);
    double beta; cplx t, sc;
    householder_coeffs(B[j * ldb + j], x2, &beta, &t, &sc);
    __syncwarp();
    for (int i = j + 1 + lane; i < m; i += 32) B[j * ldb + i] = cmul(B[j * ldb + i], sc);
    __syncwarp();
    if (lane == 0) { B[j * ldb + j] = cmk(beta, 0.0); tau[j] = t; }
    __syncwarp();
    for (int c = j + 1; c < k; ++c) {   // apply H_jᴴ to column c
      cplx s = czero();
      for (int i = j + lane; i < m; i += 32) {
        const cplx v = (i == j) ? cmk(1.0, 0.0) : B[j * ldb + i];
        s = cfmac(v, B[c * ldb + i], s);
      }
      s = warp_sum(s);
      const cplx f = cmul(cconj(t), s);
      __syncwarp();
      for (int i = j + lane; i < m; i += 32) {
        const cplx v = (i == j) ? cmk(1.0, 0.0) : B[j * ldb + i];
        B[c * ldb + i] = cfms(v, f, B[c * ldb + i]);
      }
      __syncwarp();
    }
  }
  for (int j = k - 1; j >= 0; --j) {
    const cplx tj = tau[j];
    for (int c = j + 1; c < k; ++c) {   // apply H_j to Q[j:, c]
      cplx s = czero();
      for (int i = j + lane; i < m; i += 32) {
        const cplx v = (i == j) ? cmk(1.0, 0.0) : B[j * ldb + i];
        s = cfmac(v, B[c * ldb + i], s);
      }
      s = warp_sum(s);
      const cplx f = cmul(tj, s);
      __syncwarp();
      for (int i = j + lane; i < m; i += 32) {
        const cplx v = (i == j) ? cmk(1.0, 0.0) : B[j * ldb + i];
        B[c * ldb + i] = cfms(v, f, B[c * ldb + i]);
      }
      __syncwarp();
    }
    for (int i = lane; i < m; i += 32) {
      cplx q;
      if (i < j) q = czero();
      else if (i == j) q = csub(cmk(1.0, 0.0), tj);
      else q = cneg(cmul(tj, B[j * ldb + i]));
      B[j * ldb + i] = q;
    }
    __syncwarp();
  }
}

// ------------------------------------------------------------------------------------
// SVD Rayleigh–Ritz on a triangular factor (svdRaylRitz!, lobpcgSvd.jl:126-184, after
// its QR step): R (nS×nS) = U Σ Gᴴ by one-sided Jacobi; side 'L' keeps the largest
// singular values and inverts the first r; otherwise ascending order.  With lq != 0
// and nS > r, columns r..2r-1 of G become G[:, r:nS] · Q_matᴴ, Q_mat the LQ factor of
// G[0:r, r:nS] (lobpcgSvd.jl:166-180).  One CTA.  A and V live in shared memory when
// gA == nullptr (nS <= 80), otherwise in the global scratch gA, gV (nS*nS each).
// Dynamic shared memory: [2 nS² (shared path)] + 2 nS r + r cplx + 3 nS doubles/ints.
// ------------------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_svd_rr(int nS, int r, int sideL, int lq, const cplx* __restrict__ R,
                                                int ldr, double* sigma, double* lam, cplx* G, int ldg, cplx* gA,
                                                cplx* gV) {
  extern __shared__ cplx sm[];
  const bool glob = (gA != nullptr);
  cplx* A = glob ? gA : sm;                       // nS*nS
  cplx* V = glob ? gV : sm + nS * nS;             // nS*nS
  cplx* Bq = glob ? sm : sm + 2 * nS * nS;        // (nS-r)*r
  cplx* tmp = Bq + nS * r;                        // nS*r
  cplx* tau = tmp + nS * r;                       // r
  double* nrm = reinterpret_cast<double*>(tau + r);
  double* ssig = nrm + nS;
  int* perm = reinterpret_cast<int*>(ssig + nS);
  for (int q = threadIdx.x; q < nS * nS; q += blockDim.x) {
    const int i = q % nS, c = q / nS;
    A[q] = R[c * ldr + i];
  }
  __syncthreads();
  jacobi_svd(A, nS, V, nS, nS, ssig, /*ascending=*/!sideL, perm, nrm);
  for (int i = threadIdx.x; i < nS; i += blockDim.x) {
    double s = ssig[i];
    if (i < r) {
      if (sideL) s = 1.0 / s;
      lam[i] = s * s;
    }
    sigma[i] = s;
  }
  if (lq && nS > r) {
    const int m = nS - r;
    // Bq = (G[0:r, r:nS])ᴴ  (m × r)
    for (int q = threadIdx.x; q < m * r; q += blockDim.x) {
      const int i = q % m, c = q / m;
      Bq[c * m + i] = cconj(V[(r + i) * nS + c]);
    }
    __syncthreads();
    if (threadIdx.x < 32) warp_house_q(Bq, m, m, r, tau);
    __syncthreads();
    // tmp = G[:, r:nS] · Bq   (nS × r)
    for (int q = threadIdx.x; q < nS * r; q += blockDim.x) {
      const int i = q % nS, c = q / nS;
      cplx s = czero();
      for (int l = 0; l < m; ++l) s = cfma(V[(r + l) * nS + i], Bq[c * m + l], s);
      tmp[c * nS + i] = s;
    }
    __syncthreads();
    for (int q = threadIdx.x; q < nS * r; q += blockDim.x) {
      const int i = q % nS, c = q / nS;
      V[(r + c) * nS + i] = tmp[c * nS + i];
    }
    __syncthreads();
  }
  for (int q = threadIdx.x; q < nS * nS; q += blockDim.x) {
    const int i = q % nS, c = q / nS;
    G[c * ldg + i] = V[q];
  }
}

// Dynamic shared memory the shared-memory path of k_svd_rr may take (below the 227 KB opt-in).
constexpr size_t kSvdSmemShared = 200 * 1024;

inline size_t svd_rr_smem_bytes(int nS, int r, bool glob) {
  size_t s = ((size_t)2 * nS * r + r) * sizeof(cplx) + (size_t)nS * (2 * sizeof(double) + sizeof(int)) + 16;
  if (!glob) s += (size_t)2 * nS * nS * sizeof(cplx);
  return s;
}

// ------------------------------------------------------------------------------------
// Cholesky of the k×k Hermitian G (upper factor, G = RᴴR) in shared memory by one
// CTA; returns false on a non-positive pivot.  Only the upper triangle is read.
// ------------------------------------------------------------------------------------
__device__ bool chol_upper(cplx* G, int ldg, int k) {
  __shared__ int s_ok;
  if (threadIdx.x == 0) s_ok = 1;
  __syncthreads();
  for (int j = 0; j < k; ++j) {
    if (threadIdx.x == 0) {
      const double d = G[j * ldg + j].x;
      if (!(d > 0.0) || !isfinite(d)) s_ok = 0;
      G[j * ldg + j] = cmk(sqrt(fmax(d, 0.0)), 0.0);
    }
    __syncthreads();
    if (!s_ok) return false;
    const double rjj = G[j * ldg + j].x;
    for (int c = j + 1 + threadIdx.x; c < k; c += blockDim.x) G[c * ldg + j] = cscale(G[c * ldg + j], 1.0 / rjj);
    __syncthreads();
    // trailing update: G[i, c] -= conj(R[j, i]) R[j, c]  for j < i <= c
    const int nt = k - j - 1;
    for (int q = threadIdx.x; q < nt * nt; q += blockDim.x) {
      const int i = j + 1 + q % nt, c = j + 1 + q / nt;
      if (i <= c) G[c * ldg + i] = csub(G[c * ldg + i], cmulc(G[i * ldg + j], G[c * ldg + j]));
    }
    __syncthreads();
  }
  for (int q = threadIdx.x; q < k * k; q += blockDim.x) {
    const int i = q % k, c = q / k;
    if (i > c) G[c * ldg + i] = czero();
  }
  __syncthreads();
  return true;
}

// Inverse of the upper-triangular k×k R (in place in Y; R preserved), shared memory.
__device__ void trtri_upper(const cplx* R, int ldr, cplx* Y, int ldy, int k) {
  for (int q = threadIdx.x; q < k * k; q += blockDim.x) {
    const int i = q % k, c = q / k;
    Y[c * ldy + i] = (i == c) ? cmk(1.0, 0.0) : czero();
  }
  __syncthreads();
  for (int i = k - 1; i >= 0; --i) {
    const cplx dinv = cinv(R[i * ldr + i]);
    for (int c = i + threadIdx.x; c < k; c += blockDim.x) Y[c * ldy + i] = cmul(Y[c * ldy + i], dinv);
    __syncthreads();
    const int nl = i, nc = k - i;
    for (int q = threadIdx.x; q < nl * nc; q += blockDim.x) {
      const int l = q % nl, c = i + q / nl;
      Y[c * ldy + l] = cfms(R[i * ldr + l], Y[c * ldy + i], Y[c * ldy + l]);
    }
    __syncthreads();
  }
}

// ------------------------------------------------------------------------------------
// CholQR step on a Gram matrix: given G = XᴴX (k×k), computes R = chol(G) and
// Rinv = R⁻¹ (both k×k, ld k).  On breakdown adds the shift of the reference's
// shifted Cholesky-QR (11(mk + k(k+1))·eps·max_j G_jj) and retries up to 3 times;
// err gets DEVERR_BREAKDOWN if it still fails.  Optionally Rtot ← R·Rtot.
// ------------------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_chol_inv(int k, int64_t m, const cplx* __restrict__ Gin, int ldgin,
                                                  cplx* R, cplx* Rinv, cplx* Rtot, int* err) {
  extern __shared__ cplx sm[];
  cplx* G = sm;               // k*k
  cplx* Y = sm + k * k;       // k*k
  cplx* T = Y + k * k;        // k*k (for Rtot product)
  __shared__ double s_gmax;
  double shift = 0.0;
  bool ok = false;
  for (int attempt = 0; attempt < 4 && !ok; ++attempt) {
    for (int q = threadIdx.x; q < k * k; q += blockDim.x) {
      const int i = q % k, c = q / k;
      cplx g = Gin[c * ldgin + i];
      if (i == c) g = cmk(g.x + shift, 0.0);
      G[c * k + i] = g;
    }
    if (threadIdx.x == 0) {
      double gm = 0.0;
      for (int i = 0; i < k; ++i) gm = fmax(gm, Gin[i * ldgin + i].x);
      s_gmax = gm;
    }
    __syncthreads();
    ok = chol_upper(G, k, k);
    if (!ok) {
      const double eps = 2.220446049250313e-16;
      shift = 11.0 * ((double)m * k + (double)k * (k + 1)) * eps * s_gmax * (double)(1 << attempt);
    }
    __syncthreads();
  }
  if (!ok) {
    if (threadIdx.x == 0) atomicOr(err, DEVERR_BREAKDOWN);
    for (int q = threadIdx.x; q < k * k; q += blockDim.x) {
      const int i = q % k, c = q / k;
      G[c * k + i] = (i == c) ? cmk(1.0, 0.0) : czero();
    }
    __syncthreads();
  }
  trtri_upper(G, k, Y, k, k);
  for (int q = threadIdx.x; q < k * k; q += blockDim.x) {
    if (R) R[q] = G[q];
    Rinv[q] = Y[q];
  }
  if (Rtot) {
    __syncthreads();
    for (int q = threadIdx.x; q < k * k; q += blockDim.x) {
      const int i = q % k, c = q / k;
      cplx s = czero();
      for (int l = i; l < k; ++l) s = cfma(G[l * k + i], Rtot[c * k + l], s);
      T[q] = s;
    }
    __syncthreads();
    for (int q = threadIdx.x; q < k * k; q += blockDim.x) Rtot[q] = T[q];
  }
}

// Inverse of an upper-triangular k×k R (global, ld k) into Rinv, one CTA.  Tiny
// diagonal entries (|r_ii| <= 1e-300) are replaced by 1e-300 and flagged.
__global__ void __launch_bounds__(256) k_trtri(int k, const cplx* __restrict__ Rin, cplx* Rinv, int* err) {
  extern __shared__ cplx sm[];
  cplx* R = sm;
  cplx* Y = sm + k * k;
  for (int q = threadIdx.x; q < k * k; q += blockDim.x) {
    const int i = q % k, c = q / k;
    cplx v = (i <= c) ? Rin[q] : czero();
    if (i == c && cabs2(v) < 1e-600) { v = cmk(1e-300, 0.0); atomicOr(err, DEVERR_BREAKDOWN); }
    R[q] = v;
  }
  __syncthreads();
  trtri_upper(R, k, Y, k, k);
  for (int q = threadIdx.x; q < k * k; q += blockDim.x) Rinv[q] = Y[q];
}

// C (m×n, ldc) = alpha * op(A) * op(B) + beta * C for small matrices, one CTA;
// opA/opB: 0 = N, 1 = conjugate transpose.  A is m×kk after op, B kk×n after op.
__global__ void k_small_gemm(int m, int n, int kk, cplx alpha, const cplx* A, int lda, int opA,
                             const cplx* B, int ldb, int opB, cplx beta, cplx* C, int ldc) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < m * n; q += gridDim.x * blockDim.x) {
    const int i = q % m, c = q / m;
    cplx s = czero();
    for (int l = 0; l < kk; ++l) {
      const cplx a = opA ? cconj(A[i * lda + l]) : A[l * lda + i];
      const cplx b = opB ? cconj(B[l * ldb + c]) : B[c * ldb + l];
      s = cfma(a, b, s);
    }
    cplx out = cmul(alpha, s);
    if (beta.x != 0.0 || beta.y != 0.0) out = cfma(beta, C[c * ldc + i], out);
    C[c * ldc + i] = out;
  }
}
