// Projected Hermitian eigenproblem of the recycle step (find_rr_dim!,
// src/core/fastRaylRitz.jl:54-96) on the device, FP64, one CTA per grid point.
//
//   Hz = H1 − z·H2 − z̄·H2ᴴ + (|z|² + shift)·I          (affine_conbine!, :6-28; H3 = I)
//   λ_max, then the smallest eigenvalues in steps of 2r until a gap > λ_max/τ·eps,
//   r_ = max(first gap index, r) or pr when none; eigenvectors of the r_ smallest.
//
// Method (published algorithms, written for this kernel):
//   1. Householder tridiagonalisation Hz = Q T Qᴴ (Golub & Van Loan §8.3.1), reflectors
//      in the convention of LAPACK's zlarfg, T real symmetric tridiagonal;
//   2. eigenvalues of T by Sturm-count multisection: a warp evaluates 32 Sturm
//      counts per round (Barth, Martin & Wilkinson 1967 bisection, 32-way);
//   3. eigenvectors of T by inverse iteration with a partially pivoted tridiagonal
//      LU (Wilkinson), one warp per vector, then classical Gram–Schmidt with
//      re-orthogonalisation over the vectors (which keeps a cluster's invariant subspace);
//   4. back-transformation by the stored reflectors: G = Q S.
// Like zheevr with uplo 'U', only the upper triangle of Hz is used.
#pragma once
#include "common.cuh"
#include "small.cuh"

#include <algorithm>

#define HEEV_THREADS 512

struct HeevWork {
  cplx* A;        // per problem pr_max*pr_max (global path)
  double* lu;     // per problem 16 warps × 6 × pr_max doubles
};

// Numbers of eigenvalues of the tridiagonal (d, e²) below x1 and below x2 (two
// interleaved Sturm sequences).
__device__ __forceinline__ void sturm_count2(const double* d, const double* e2, int n, double x1, double x2,
                                             double pivmin, int* c1, int* c2) {
  double q1 = d[0] - x1, q2 = d[0] - x2;
  if (fabs(q1) < pivmin) q1 = -pivmin;
  if (fabs(q2) < pivmin) q2 = -pivmin;
  int n1 = (q1 < 0.0), n2 = (q2 < 0.0);
  for (int i = 1; i < n; ++i) {
    const double di = d[i], ei = e2[i - 1];
    q1 = di - x1 - ei * recip_nr(q1);
    q2 = di - x2 - ei * recip_nr(q2);
    if (fabs(q1) < pivmin) q1 = -pivmin;
    if (fabs(q2) < pivmin) q2 = -pivmin;
    n1 += (q1 < 0.0);
    n2 += (q2 < 0.0);
  }
  *c1 = n1;
  *c2 = n2;
}

// Eigenvalue with 0-based index `idx` (ascending) by 65-way multisection, one warp:
// lane l evaluates the counts at the interior points 2l+1 and 2l+2 of 65 intervals.
__device__ double warp_eig_index(const double* d, const double* e2, int n, int idx, double gl, double gu,
                                 double pivmin, double atol) {
  const int lane = threadIdx.x & 31;
  double lo = gl, hi = gu;
  for (int round = 0; round < 12 && (hi - lo) > atol; ++round) {
    const double h = (hi - lo) / 65.0;
    int c1, c2;
    sturm_count2(d, e2, n, lo + h * (2 * lane + 1), lo + h * (2 * lane + 2), pivmin, &c1, &c2);
    // counts are monotone in the point index: number of points with count <= idx
    const int nle = __popc(__ballot_sync(0xffffffffu, c1 <= idx)) + __popc(__ballot_sync(0xffffffffu, c2 <= idx));
    const double nlo = lo + h * nle;
    const double nhi = (nle < 64) ? lo + h * (nle + 1) : hi;
    lo = nlo; hi = nhi;
  }
  return 0.5 * (lo + hi);
}

// Partially pivoted LU of (T − λI) and solves, on lane 0 of a warp.
// Storage (6 arrays of n): u0 (reciprocal pivots), u1, u2 (superdiagonals), l
// (multipliers), piv.
__device__ void tri_lu(const double* d, const double* e, int n, double lam, double* u0, double* u1, double* u2,
                       double* l, double* piv, double tiny) {
  double a = d[0] - lam;
  double b = (n > 1) ? e[0] : 0.0;
  for (int i = 0; i < n - 1; ++i) {
    const double c = e[i];                      // subdiagonal entry (i+1, i)
    const double an = d[i + 1] - lam;           // next diagonal
    const double bn = (i + 1 < n - 1) ? e[i + 1] : 0.0;
    if (fabs(a) >= fabs(c)) {
      const double aa = (a == 0.0) ? tiny : a;
      const double ia = 1.0 / aa;
      const double m = c * ia;
      piv[i] = 0.0; l[i] = m;
      u0[i] = ia; u1[i] = b; u2[i] = 0.0;
      a = an - m * b;
      b = bn;
    } else {
      const double ic = 1.0 / c;
      const double m = a * ic;
      piv[i] = 1.0; l[i] = m;
      u0[i] = ic; u1[i] = an; u2[i] = bn;
      a = b - m * an;
      b = -m * bn;
    }
  }
  u0[n - 1] = 1.0 / ((a == 0.0) ? tiny : a);
}

__device__ void tri_solve(int n, const double* u0, const double* u1, const double* u2, const double* l,
                          const double* piv, double* x) {
  for (int i = 0; i < n - 1; ++i) {             // apply P and L⁻¹
    if (piv[i] != 0.0) { const double t = x[i]; x[i] = x[i + 1]; x[i + 1] = t; }
    x[i + 1] -= l[i] * x[i];
  }
  x[n - 1] *= u0[n - 1];                         // U⁻¹ (three bands, reciprocal pivots)
  if (n > 1) x[n - 2] = (x[n - 2] - u1[n - 2] * x[n - 1]) * u0[n - 2];
  for (int i = n - 3; i >= 0; --i) x[i] = (x[i] - u1[i] * x[i + 1] - u2[i] * x[i + 2]) * u0[i];
}

// Shared-memory plan of one launch, computed on the host (heev_plan).
struct HeevPlan {
  int lda;      // leading dimension of Hz in shared memory (≡ 4 mod 8), 0: Hz in global scratch
  int nlu;      // warps whose tridiagonal LU factors live in shared memory (0: global scratch)
  int gs_cap;   // eigenvectors kept in shared memory (0: worked on in Gout directly)
  size_t bytes; // dynamic shared memory
};

__global__ void __launch_bounds__(HEEV_THREADS) k_heev_rr(int pr, int r, const cplx* __restrict__ H1,
                                                          const cplx* __restrict__ H2, int ldh,
                                                          const cplx* __restrict__ zs,
                                                          const double* __restrict__ taus, double shift,
                                                          HeevWork work, int prmax, cplx* Gout, int ldg,
                                                          int64_t gstride, int* rr_out, double* lam_out,
                                                          int* err, HeevPlan plan, long long* clk) {
  extern __shared__ double dsm[];
  const int b = blockIdx.x;
  const int n = pr;
  const int nlu = plan.nlu;
  // shared layout: [A (n × lda cplx)] v v1 tau (n cplx) yp (4n cplx) d e e2 lam (n doubles)
  // LU (nlu·6n doubles) S (gs_cap·n cplx)
  cplx* base = reinterpret_cast<cplx*>(dsm);
  const int lda = plan.lda > 0 ? plan.lda : n;
  cplx* A = plan.lda > 0 ? base : work.A + (int64_t)b * prmax * prmax;
  cplx* v = base + (plan.lda > 0 ? (size_t)n * lda : 0);
  cplx* v1 = v + n;
  cplx* tau = v1 + n;
  double* d = reinterpret_cast<double*>(tau + 5 * n);   // yp: tau + n .. tau + 5n
  double* e = d + n;
  double* e2 = e + n;
  double* lam = e2 + n;
  double* lusm = lam + n;
  cplx* Ssm = reinterpret_cast<cplx*>(lusm + (size_t)nlu * 6 * n);
  __shared__ double red[32];
  __shared__ int s_rr;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const cplx z = zs[b];
  const double zz = z.x * z.x + z.y * z.y + shift;
  cplx* G = Gout + (int64_t)b * gstride;

  if (clk && threadIdx.x == 0) clk[(int64_t)b * 8 + 0] = clock64();
  // 1. Hz from the upper triangle, mirrored (affine_conbine!, element (ii, jj), ii <= jj).
  for (int q = threadIdx.x; q < n * n; q += blockDim.x) {
    const int i = q % n, j = q / n;
    const int ii = min(i, j), jj = max(i, j);
    cplx h = H1[(int64_t)jj * ldh + ii];
    h = cfms(z, H2[(int64_t)jj * ldh + ii], h);
    h = cfms(cconj(z), cconj(H2[(int64_t)ii * ldh + jj]), h);
    if (ii == jj) h = cmk(h.x + zz, 0.0);
    A[j * lda + i] = (i <= j) ? h : cconj(h);
  }
  __syncthreads();

  // 2. Householder tridiagonalisation: for column k reduce A[k+1:, k].  Both triangles of
  //    the trailing block are kept, so every access to A reads a column with a lane per row
  //    (conflict-free).  Two barriers per column (B and D below); reflectors alternate
  //    between two buffers.
  auto make_reflector = [&](int k) {   // warp 0; column k (rows ≥ k+1) is final
    const int m0 = k + 1;
    cplx* vk = (k & 1) ? v1 : v;
    double x2 = 0.0;
    for (int i = m0 + 1 + lane; i < n; i += 32) x2 += cabs2(A[k * lda + i]);
    x2 = warp_sum(x2);
    // Householder coefficients in the convention of LAPACK's zlarfg (β real, τ complex);
    // the divisions are reciprocals refined by Newton–Raphson (recip_nr).
    const cplx alpha = A[k * lda + m0];
    double beta;
    cplx t, sc;
    if (x2 == 0.0 && alpha.y == 0.0) {
      beta = alpha.x; t = czero(); sc = czero();
    } else {
      const double nrm = sqrt(alpha.x * alpha.x + alpha.y * alpha.y + x2);
      beta = (alpha.x >= 0.0) ? -nrm : nrm;
      const double ib = recip_nr(beta);
      t = cmk((beta - alpha.x) * ib, -alpha.y * ib);
      const double ar = alpha.x - beta, ai = alpha.y;             // sc = 1 / (α − β)
      const double id = recip_nr(ar * ar + ai * ai);
      sc = cmk(ar * id, -ai * id);
    }
    for (int i = m0 + lane; i < n; i += 32) {
      const cplx vi = (i == m0) ? cmk(1.0, 0.0) : cmul(A[k * lda + i], sc);
      vk[i] = vi;
      if (i > m0) A[k * lda + i] = vi;      // reflector tail kept for the back-transformation
    }
    if (lane == 0) {
      tau[k] = t;
      e[k] = beta;
      d[k] = A[k * lda + k].x;
    }
  };
  // B and D of column k (m0 = k + 1, trailing block rows and columns m0..n−1):
  //   B  partial products P_c(i) = Σ_{j ≡ m0+c (mod 4)} A(i,j) v_j: warp w takes the row
  //      groups g ≡ w (mod 4) (32 rows each, a lane per row) and column residue c = w/4, four
  //      independent sums per thread, into yp[c·n + i]; each warp also forms its share of
  //      Σ conj(P_c(i)) v_i (one warp sum per warp), so yᴴv = conj(τ)·Σ_w yvp[w] with y = τ Σ_c P_c.
  //   D  α₂ = −½ τ yᴴv = −½|τ|² Σ_w yvp[w]; w_i = τ Σ_c P_c(i) + α₂ v_i is rebuilt from the
  //      partials wherever it is needed; A −= v wᴴ + w vᴴ: columns m0+1.. by warps 1..15,
  //      column m0 by warp 0, which then forms the next reflector.
  constexpr int NWH = HEEV_THREADS / 32, RGS = 4, CCH = NWH / RGS;
  static_assert(CCH == 4, "four column residues");
  cplx* yp = tau + n;                 // CCH × n partial products
  __shared__ cplx yvp[NWH];
  if (n > 1 && warp == 0) make_reflector(0);
  __syncthreads();
  for (int k = 0; k < n - 1; ++k) {
    const int m0 = k + 1;
    const cplx t = tau[k];
    const cplx* vk = (k & 1) ? v1 : v;
    const bool active = (t.x != 0.0 || t.y != 0.0);
    if (active) {   // B
      const int c = warp / RGS;
      cplx yv = czero();
      for (int g = warp % RGS; m0 + g * 32 < n; g += RGS) {
        const int i = m0 + g * 32 + lane;
        if (i < n) {
          cplx s0 = czero(), s1 = czero(), s2 = czero(), s3 = czero();
          int j = m0 + c;
          for (; j + 3 * CCH < n; j += 4 * CCH) {
            s0 = cfma(A[j * lda + i], vk[j], s0);                       // A(i,j) v_j
            s1 = cfma(A[(j + CCH) * lda + i], vk[j + CCH], s1);
            s2 = cfma(A[(j + 2 * CCH) * lda + i], vk[j + 2 * CCH], s2);
            s3 = cfma(A[(j + 3 * CCH) * lda + i], vk[j + 3 * CCH], s3);
          }
          for (; j < n; j += CCH) s0 = cfma(A[j * lda + i], vk[j], s0);
          const cplx s = cadd(cadd(s0, s1), cadd(s2, s3));
          yp[c * n + i] = s;
          yv = cfmac(s, vk[i], yv);                                     // conj(P_c(i)) v_i
        }
      }
      yv = warp_sum(yv);
      if (lane == 0) yvp[warp] = yv;
    }
    __syncthreads();
    if (active) {   // D
      cplx ys = yvp[0];
#pragma unroll
      for (int q = 1; q < NWH; ++q) ys = cadd(ys, yvp[q]);
      const cplx a2 = cscale(ys, -0.5 * (t.x * t.x + t.y * t.y));
      auto wrow = [&](int i) {
        const cplx s = cadd(cadd(cadd(yp[i], yp[n + i]), yp[2 * n + i]), yp[3 * n + i]);
        return cfma(a2, vk[i], cmul(t, s));
      };
      if (warp == 0) {   // column m0, all trailing rows
        const cplx vj = vk[m0], wj = wrow(m0);
        for (int i = m0 + lane; i < n; i += 32) {
          const cplx vi = vk[i], wi = wrow(i);
          cplx aij = A[m0 * lda + i];
          aij = csub(aij, cmulc(wj, vi));    // v_i conj(w_j)
          aij = csub(aij, cmulc(vj, wi));    // w_i conj(v_j)
          A[m0 * lda + i] = aij;
        }
        __syncwarp();
      } else {           // columns m0+warp, m0+warp+15, ..., rows in blocks of four groups
        for (int g0 = 0; m0 + g0 * 32 < n; g0 += 4) {
          cplx vi[4], wi[4];
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const int i = m0 + (g0 + q) * 32 + lane;
            vi[q] = (i < n) ? vk[i] : czero();
            wi[q] = (i < n) ? wrow(i) : czero();
          }
          for (int j = m0 + warp; j < n; j += NWH - 1) {
            const cplx vj = vk[j], wj = wrow(j);
            cplx a[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
              const int i = m0 + (g0 + q) * 32 + lane;
              a[q] = (i < n) ? A[j * lda + i] : czero();
            }
#pragma unroll
            for (int q = 0; q < 4; ++q) {
              const int i = m0 + (g0 + q) * 32 + lane;
              if (i < n) A[j * lda + i] = csub(csub(a[q], cmulc(wj, vi[q])), cmulc(vj, wi[q]));
            }
          }
        }
      }
    }
    if (warp == 0 && k + 1 < n - 1) make_reflector(k + 1);
    __syncthreads();
  }
  if (threadIdx.x == 0) d[n - 1] = A[(n - 1) * lda + (n - 1)].x;
  for (int i = threadIdx.x; i < n - 1; i += blockDim.x) e2[i] = e[i] * e[i];
  __syncthreads();

  // Gershgorin interval and pivot floor.
  __shared__ double s_gl, s_gu, s_piv;
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

  // 3. λ_max and the smallest eigenvalues with the gap rule of find_rr_dim!.  The last
  //    warp computes λ_max while the others compute λ_0, λ_1, ... in the same pass.
  if (clk && threadIdx.x == 0) clk[(int64_t)b * 8 + 1] = clock64();
  {
    const int idx = (warp == nw - 1) ? n - 1 : warp;
    if (warp == nw - 1 || idx < n - 1) {
      const double li = warp_eig_index(d, e2, n, idx, gl, gu, pivmin, atol);
      if (lane == 0) lam[idx] = li;
    }
  }
  __syncthreads();
  const double gap = lam[n - 1] / taus[b] * 2.220446049250313e-16;
  const int n_init = min(2 * r, n);
  int n_last = n_init;                      // largest n of the sequence 2r, 4r, ... <= n
  while (n_last + 2 * r <= n) n_last += 2 * r;
  int computed = min(n - 1, nw - 1);        // eigenvalues 0..computed-1 known
  int rr = 0;
  int ncheck = n_init;
  while (true) {
    while (computed < ncheck) {
      const int idx = computed + warp;
      if (idx < ncheck && idx < n - 1) {
        const double li = warp_eig_index(d, e2, n, idx, gl, gu, pivmin, atol);
        if (lane == 0) lam[idx] = li;
      }
      computed = min(ncheck, computed + nw);
      __syncthreads();
    }
    if (threadIdx.x == 0) {
      int g = 0;
      for (int i = 0; i + 1 < ncheck; ++i)
        if (fabs(lam[i] - lam[i + 1]) > gap) { g = i + 1; break; }
      s_rr = g;
    }
    __syncthreads();
    rr = s_rr;
    if (rr > 0 || ncheck >= n_last) break;
    ncheck += 2 * r;
  }
  rr = (rr > 0) ? max(rr, r) : n;
  while (computed < rr) {
    const int idx = computed + warp;
    if (idx < rr && idx < n - 1) {
      const double li = warp_eig_index(d, e2, n, idx, gl, gu, pivmin, atol);
      if (lane == 0) lam[idx] = li;
    }
    computed = min(rr, computed + nw);
    __syncthreads();
  }

  // 4. Inverse iteration, one warp per eigenvector, into S (shared when rr fits).
  if (clk && threadIdx.x == 0) clk[(int64_t)b * 8 + 2] = clock64();
  const bool s_shared = rr <= plan.gs_cap;
  cplx* S = s_shared ? Ssm : G;
  const int lds = s_shared ? n : ldg;
  {
    const double tnorm = fmax(fabs(gl), fabs(gu));
    const double tiny = 2.220446049250313e-16 * tnorm + 1e-300;
    const int nwk = (nlu > 0) ? min(nlu, nw) : nw;
    for (int j = warp; j < rr && warp < nwk; j += nwk) {
      const int ldl = (nlu > 0) ? n : prmax;
      double* lu = (nlu > 0) ? lusm + (int64_t)warp * 6 * n : work.lu + ((int64_t)b * 16 + warp) * 6 * prmax;
      double *u0 = lu, *u1 = lu + ldl, *u2 = lu + 2 * ldl, *l = lu + 3 * ldl, *pv = lu + 4 * ldl,
             *x = lu + 5 * ldl;
      const double lamj = lam[j] + tiny * ((j & 1) ? 1.0 : -1.0);
      if (lane == 0) tri_lu(d, e, n, lamj, u0, u1, u2, l, pv, tiny);
      for (int i = lane; i < n; i += 32) {       // deterministic start vector
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
    }
  }
  __syncthreads();
  if (clk && threadIdx.x == 0) clk[(int64_t)b * 8 + 3] = clock64();
  // Block-wide classical Gram–Schmidt with one re-orthogonalisation (CGS2) over the rr
  // real vectors, in index order.  v (no longer needed) holds the coefficients.
  {
    double* coef = reinterpret_cast<double*>(v);
    __shared__ double s_nrm;
    for (int j = 0; j < rr; ++j) {
      double* gj = reinterpret_cast<double*>(S + (int64_t)j * lds);   // stride-2 real parts
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
  }
  if (clk && threadIdx.x == 0) clk[(int64_t)b * 8 + 4] = clock64();
  // 5. Back-transformation G = H_0 H_1 ... H_{n-2} S (apply H_{n-2} first).  A group of
  //    16 lanes owns one vector: dot product, 4-level reduction, update, no barrier.
  {
    const int half = threadIdx.x >> 4, hl = threadIdx.x & 15, nh = blockDim.x >> 4;
    for (int j0 = 0; j0 < rr; j0 += nh) {
      const int j = j0 + half;
      const bool act = j < rr;
      cplx* sj = S + (int64_t)(act ? j : 0) * lds;
      for (int k = n - 2; k >= 0; --k) {
        const int m0 = k + 1;
        const cplx t = tau[k];
        if (t.x == 0.0 && t.y == 0.0) continue;
        cplx sum = czero();
        if (act)
          for (int i = m0 + hl; i < n; i += 16) {
            const cplx vi = (i == m0) ? cmk(1.0, 0.0) : A[k * lda + i];
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
            const cplx vi = (i == m0) ? cmk(1.0, 0.0) : A[k * lda + i];
            sj[i] = cfms(vi, f, sj[i]);
          }
        __syncwarp();
      }
    }
  }
  __syncthreads();
  if (s_shared)
    for (int q = threadIdx.x; q < rr * n; q += blockDim.x) G[(int64_t)(q / n) * ldg + (q % n)] = S[q];
  if (clk && threadIdx.x == 0) clk[(int64_t)b * 8 + 5] = clock64();
  if (threadIdx.x == 0) {
    rr_out[b] = rr;
    bool bad = !isfinite(lam[n - 1]);
    for (int i = 0; i < rr && i < n - 1; ++i) bad |= !isfinite(lam[i]);
    if (bad) atomicOr(err, DEVERR_NONFINITE);
  }
  if (lam_out) {
    for (int i = threadIdx.x; i < n; i += blockDim.x)
      lam_out[(int64_t)b * prmax + i] = (i < computed || i == n - 1) ? lam[i] : 0.0;
  }
}

// Shared-memory plan for order pr within `avail` bytes: Hz in shared memory when it
// fits next to the vectors, then up to 8 LU warps, then as many eigenvectors (<= 32)
// as fit.
inline HeevPlan heev_plan(int pr, size_t avail) {
  HeevPlan p{};
  const size_t vec = (size_t)7 * pr * sizeof(cplx) + (size_t)4 * pr * sizeof(double);
  int lda = pr + ((4 - pr % 8) + 8) % 8;                    // ≡ 4 (mod 8)
  size_t need = vec + (size_t)pr * lda * sizeof(cplx);
  const size_t lu1 = (size_t)6 * pr * sizeof(double);
  const size_t s1 = (size_t)pr * sizeof(cplx);
  if (need + 2 * lu1 + 6 * s1 <= avail) {
    p.lda = lda;
  } else {
    p.lda = 0;
    need = vec;
  }
  p.nlu = (int)std::min<size_t>(8, (avail - need) / lu1);
  need += (size_t)p.nlu * lu1;
  p.gs_cap = (int)std::min<size_t>(32, (avail - need) / s1);
  need += (size_t)p.gs_cap * s1;
  p.bytes = need;
  return p;
}
