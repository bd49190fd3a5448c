// Batched recycle step: the recycle step (fastSvdRaylRitz_implicit!,
// src/core/fastRaylRitz.jl:99-219) of B consecutive grid points against the same
// recycled space, one launch per stage, grid.y (or grid.x) = point.  Ritz dimensions
// are read from device memory (written by the batched eigensolve), so the stages
// follow each other without a host round trip.  Points whose Ritz dimension exceeds
// BATCH_KMAX are skipped here and flagged for the per-point path.
#pragma once
#include "common.cuh"
#include "small.cuh"

#define BATCH_KMAX 16
#define BATCH_MAX 32

struct BatchDesc {
  int B, pr, r, ldh;
  int64_t np;                 // rows (n_pad), leading dimension of the tall arrays
  const cplx *J1, *J2, *J5, *V;
  const cplx* zs;             // B shifts
  const int* rr;              // B Ritz dimensions (from the eigensolve)
  const cplx* G1;             // eigenvectors, point b at G1 + b*g1_stride, leading dimension ldg1
  int64_t g1_stride;
  int ldg1;
  cplx* czx;                  // point b: np × BATCH_KMAX at czx + b*np*BATCH_KMAX
  cplx* stack[2];             // TSQR stacks, point b at stack + b*stack_stride
  int64_t stack_stride;
  cplx* Rb;                   // point b: BATCH_KMAX² (ld = rr_b) at Rb + b*BATCH_KMAX²
  double* sig;                // point b: BATCH_KMAX singular values at sig + b*BATCH_KMAX
  cplx* G2;                   // point b: BATCH_KMAX² (ld = rr_b)
  cplx* Gtot;                 // point b: pr × r (ld pr) at Gtot + b*pr_max*r
  int64_t gtot_stride;
  cplx* XW;                   // point b: X (np × r) then W (np × r) at XW + b*2*np*r
  double* colpart;            // point b: ntiles partial |W[:,1]|² at colpart + b*ntiles
  int ntiles;
  double* w0sq;               // B
  int g1_always;              // r_ == pr: G1·G2 (1) or G2 (0)
};

__device__ __forceinline__ bool batch_ok(const BatchDesc& d, int b) {
  const int k = d.rr[b];
  return k >= 1 && k <= BATCH_KMAX;
}

// CzX_b = (J5 − z_b V) G1_b  (np × rr_b).  CTA (tile, b): 64 rows, 256 threads, thread
// (row = t % 64, column group g = t / 64) owning columns 4g..4g+3.  G1_b (pr × 16, zero
// beyond rr_b) sits in shared memory for broadcast reads; y = J5 − z V is staged in
// chunks of CZX_KC inner indices, so each value of J5 and V is read once per CTA.
// Column groups beyond rr_b (a warp-uniform test) skip the arithmetic.
// Dynamic shared memory: czx_smem_bytes(pr).
#define CZX_KC 32
__global__ void __launch_bounds__(256) k_batch_czx(BatchDesc d) {
  extern __shared__ cplx smc[];
  const int b = blockIdx.y;
  if (!batch_ok(d, b)) return;
  const int k2 = d.rr[b], pr = d.pr;
  cplx* sG = smc;                          // G1_b[kk][j] at sG[kk*BATCH_KMAX + j]
  cplx* sY = sG + pr * BATCH_KMAX;         // y[kk][row] at sY[kk*64 + row]
  const cplx mz = cneg(d.zs[b]);
  const cplx* G = d.G1 + (int64_t)b * d.g1_stride;
  for (int q = threadIdx.x; q < pr * BATCH_KMAX; q += blockDim.x) {
    const int kk = q / BATCH_KMAX, j = q % BATCH_KMAX;
    sG[q] = (j < k2) ? G[(int64_t)j * d.ldg1 + kk] : czero();
  }
  const int row = threadIdx.x & 63, g = threadIdx.x >> 6;
  const int64_t r0 = (int64_t)blockIdx.x * 64;
  const bool active = g * 4 < k2;
  cplx acc[4];
#pragma unroll
  for (int c = 0; c < 4; ++c) acc[c] = czero();
  for (int k0 = 0; k0 < pr; k0 += CZX_KC) {
    __syncthreads();
    for (int q = threadIdx.x; q < 64 * CZX_KC; q += blockDim.x) {
      const int rr = q % 64, kk = q / 64;
      const int64_t gr = r0 + rr;
      cplx y = czero();
      if (k0 + kk < pr && gr < d.np) {
        const int64_t off = (int64_t)(k0 + kk) * d.np + gr;
        y = cfma(mz, d.V[off], d.J5[off]);
      }
      sY[kk * 64 + rr] = y;
    }
    __syncthreads();
    if (active) {
      const int kmax = min(CZX_KC, pr - k0);
#pragma unroll 4
      for (int kk = 0; kk < kmax; ++kk) {
        const cplx y = sY[kk * 64 + row];
        const cplx* gk = sG + (k0 + kk) * BATCH_KMAX + g * 4;
#pragma unroll
        for (int c = 0; c < 4; ++c) acc[c] = cfma(y, gk[c], acc[c]);
      }
    }
  }
  cplx* out = d.czx + (int64_t)b * d.np * BATCH_KMAX;
  if (r0 + row < d.np) {
#pragma unroll
    for (int c = 0; c < 4; ++c)
      if (g * 4 + c < k2) out[(int64_t)(g * 4 + c) * d.np + r0 + row] = acc[c];
  }
}

inline size_t czx_smem_bytes(int pr) { return ((size_t)pr * BATCH_KMAX + 64 * CZX_KC) * sizeof(cplx); }

// One TSQR level for every point: leaf CTA (blockIdx.x, b) factors rows
// [leaf*mb, leaf*mb + mb) of the m_b × k_b input (level 0: CzX_b with m_b = np;
// level L: the previous stack, m_b = ceil(m_{L-1}/mb)·k_b) and writes its R into
// rows [leaf*k_b, leaf*k_b + k_b) of the output stack (ld = ld_out).  The last
// level (final != 0) writes R_b (k_b × k_b, ld k_b) to d.Rb.
__global__ void __launch_bounds__(256) k_batch_tsqr(BatchDesc d, int level, int mb, int64_t ld_in,
                                                    int64_t ld_out, int final_level) {
  extern __shared__ cplx sm[];
  __shared__ double red[32];
  const int b = blockIdx.y;
  if (!batch_ok(d, b)) return;
  const int k = d.rr[b];
  int64_t m = d.np;                        // this point's rows at `level`
  for (int l = 0; l < level; ++l) m = ((m + mb - 1) / mb) * k;
  const int64_t r0 = (int64_t)blockIdx.x * mb;
  if (r0 >= m) return;
  const cplx* src = (level == 0) ? d.czx + (int64_t)b * d.np * BATCH_KMAX
                                 : d.stack[(level - 1) & 1] + (int64_t)b * d.stack_stride;
  cplx* sA = sm;
  cplx* tau = sA + (size_t)mb * BATCH_KMAX;
  cplx* wbuf = tau + BATCH_KMAX;
  const int rows = (int)min((int64_t)mb, m - r0);
  for (int q = threadIdx.x; q < mb * k; q += blockDim.x) {
    const int i = q % mb, c = q / mb;
    sA[c * mb + i] = (i < rows) ? src[(int64_t)c * ld_in + r0 + i] : czero();
  }
  __syncthreads();
  house_qr_block(sA, mb, max(rows, k), k, tau, wbuf, red);
  if (final_level) {
    cplx* R = d.Rb + (int64_t)b * BATCH_KMAX * BATCH_KMAX;
    for (int q = threadIdx.x; q < k * k; q += blockDim.x) {
      const int i = q % k, c = q / k;
      R[c * k + i] = (i <= c) ? sA[c * mb + i] : czero();
    }
  } else {
    cplx* dst = d.stack[level & 1] + (int64_t)b * d.stack_stride;
    for (int q = threadIdx.x; q < k * k; q += blockDim.x) {
      const int i = q % k, c = q / k;
      dst[(int64_t)c * ld_out + (int64_t)blockIdx.x * k + i] = (i <= c) ? sA[c * mb + i] : czero();
    }
  }
}

// SVD of R_b (ascending) and G_total_b = G1_b G2_b[:, 0:r] (or G2 when r_ == pr and the
// reference's basis is requested).  One CTA per point.
__global__ void __launch_bounds__(256) k_batch_svd_gtot(BatchDesc d) {
  __shared__ cplx A[BATCH_KMAX * BATCH_KMAX], Vm[BATCH_KMAX * BATCH_KMAX];
  __shared__ double nrm[BATCH_KMAX], ssig[BATCH_KMAX];
  __shared__ int perm[BATCH_KMAX];
  const int b = blockIdx.x;
  if (!batch_ok(d, b)) return;
  const int k = d.rr[b];
  const cplx* R = d.Rb + (int64_t)b * BATCH_KMAX * BATCH_KMAX;
  for (int q = threadIdx.x; q < k * k; q += blockDim.x) A[q] = R[q];
  __syncthreads();
  jacobi_svd(A, k, Vm, k, k, ssig, /*ascending=*/true, perm, nrm);
  for (int i = threadIdx.x; i < k; i += blockDim.x) d.sig[(int64_t)b * BATCH_KMAX + i] = ssig[i];
  const int r = d.r, pr = d.pr;
  const cplx* G1 = d.G1 + (int64_t)b * d.g1_stride;
  cplx* Gt = d.Gtot + (int64_t)b * d.gtot_stride;
  const bool full = (k == pr) && !d.g1_always;
  for (int q = threadIdx.x; q < pr * r; q += blockDim.x) {
    const int i = q % pr, c = q / pr;
    cplx s = czero();
    if (full) {
      s = (i < k) ? Vm[c * k + i] : czero();
    } else {
      for (int l = 0; l < k; ++l) s = cfma(G1[(int64_t)l * d.ldg1 + i], Vm[c * k + l], s);
    }
    Gt[(int64_t)c * pr + i] = s;
  }
}

// X_b = V G_b, W_b = (J1 − z J2 − z̄ J5 + |z|² V) G_b − X_b Σ_b², partial |W_b[:,1]|².
// CTA (tile, b): XW_ROWS rows, one thread per row with R columns of X and of W in
// registers; G_b (pr × R) sits in shared memory for broadcast reads.  R = r exactly.
// Dynamic shared memory: pr·R cplx.
#define XW_ROWS 256
template <int R>
__global__ void __launch_bounds__(XW_ROWS) k_batch_xw(BatchDesc d) {
  extern __shared__ cplx smx[];
  const int b = blockIdx.y;
  if (!batch_ok(d, b)) return;
  const int pr = d.pr;
  const cplx z = d.zs[b];
  const cplx mz = cneg(z), mzc = cneg(cconj(z));
  const double zz = z.x * z.x + z.y * z.y;
  const cplx* G = d.Gtot + (int64_t)b * d.gtot_stride;   // column j at G + j*pr
  for (int q = threadIdx.x; q < pr * R; q += blockDim.x) {
    const int kk = q / R, j = q % R;
    smx[q] = G[(int64_t)j * pr + kk];
  }
  __syncthreads();
  const int64_t row = (int64_t)blockIdx.x * XW_ROWS + threadIdx.x;
  cplx ax[R], aw[R];
#pragma unroll
  for (int j = 0; j < R; ++j) { ax[j] = czero(); aw[j] = czero(); }
  if (row < d.np) {
#pragma unroll 2
    for (int kk = 0; kk < pr; ++kk) {
      const int64_t off = (int64_t)kk * d.np + row;
      const cplx vv = d.V[off];
      cplx y = d.J1[off];
      y = cfma(mz, d.J2[off], y);
      y = cfma(mzc, d.J5[off], y);
      y = cadd(y, cscale(vv, zz));
      const cplx* gk = smx + kk * R;
#pragma unroll
      for (int j = 0; j < R; ++j) {
        const cplx gv = gk[j];
        ax[j] = cfma(vv, gv, ax[j]);
        aw[j] = cfma(y, gv, aw[j]);
      }
    }
  }
  cplx* X = d.XW + (int64_t)b * 2 * d.np * d.r;
  cplx* W = X + d.np * d.r;
  const double* sg = d.sig + (int64_t)b * BATCH_KMAX;
  double c0 = 0.0;
  if (row < d.np) {
#pragma unroll
    for (int j = 0; j < R; ++j) {
      const cplx o = csub(aw[j], cscale(ax[j], sg[j] * sg[j]));
      X[(int64_t)j * d.np + row] = ax[j];
      W[(int64_t)j * d.np + row] = o;
      if (j == 0) c0 = cabs2(o);
    }
  }
  __shared__ double sred[32];
  const double s = block_sum(c0, sred);
  if (threadIdx.x == 0) d.colpart[(int64_t)b * d.ntiles + blockIdx.x] = s;
}

__global__ void k_batch_w0(BatchDesc d) {
  __shared__ double red[32];
  const int b = blockIdx.x;
  double s = 0.0;
  if (batch_ok(d, b))
    for (int i = threadIdx.x; i < d.ntiles; i += blockDim.x) s += d.colpart[(int64_t)b * d.ntiles + i];
  s = block_sum(s, red);
  if (threadIdx.x == 0) d.w0sq[b] = batch_ok(d, b) ? s : -1.0;
}

// Quadratic form q_b = g_bᴴ·H2·g_b of each point's leading Ritz coefficient vector g_b =
// G_total_b[:, 0] (pr values, ld pr, point b at G + b·gstride) with the space's
// H2 = J5ᴴV (pr × pr, ld ldh).  vᴴ(M − zS)v of the recycled singular vector v = V·g_b is
// conj(q_b) − z (Vᴴ J5 = H2ᴴ, ‖v‖ = 1): the gradient of σ with respect to z at recycled
// points.  One CTA per point, deterministic.
__global__ void k_batch_quad(int pr, const cplx* __restrict__ G, int64_t gstride, const cplx* __restrict__ H2,
                             int ldh, const int* __restrict__ rr, cplx* out) {
  __shared__ cplx red[32];
  const int b = blockIdx.x;
  const cplx* g = G + (int64_t)b * gstride;
  cplx s = czero();
  if (!rr || (rr[b] >= 1 && rr[b] <= BATCH_KMAX)) {
    for (int i = threadIdx.x; i < pr; i += blockDim.x) {
      cplx hg = czero();
      for (int j = 0; j < pr; ++j) hg = cfma(H2[(int64_t)j * ldh + i], g[j], hg);
      s = cfmac(g[i], hg, s);
    }
  }
  s = block_sum(s, red);
  if (threadIdx.x == 0) out[b] = s;
}
