// Block-unitary rotations of the recycled space (_block_unitary_update!,
// src/core/recySpace.jl:226-286; rls_block_unitary_rot!, lmul!/rmul!,
// src/types/RLSLinearAlgebra.jl:59-190).
//
// Rotation i (i = 1..p-1) is U_i = Qᴴ with Q the full unitary of the Householder
// QR of [L(p,p); L(i,p)] (2r × r).  It mixes block p with block i:
//   rows of L, H1, H2:     [X_p; X_i] ← U_i [X_p; X_i]
//   columns of V, J*, H*:  [X_p, X_i] ← [X_p, X_i] U_iᴴ
// The rotations depend only on the last block column of L (k_blockrot_coeffs, one
// warp); k_blockrot_apply then streams the rows of each array once applying all p-1
// right products, and k_blockrot_left the columns of L, H1, H2 for the left products.
// The QR of each 2r × r block follows LAPACK's zgeqrf/zlarfg conventions.
#pragma once
#include "common.cuh"
#include "small.cuh"

// Rotation coefficients from the last block column of L alone: rotation i (i < p-1,
// 0-based) is determined by [L(p-1, p-1); L(i, p-1)] after rotations 0..i-1, and those
// only change block row p-1 of that column.  One warp; Lc (pr × r) in shared memory.
// Lane a holds row a of the 2r × r block Y (r <= 8, so 2r <= 16 lanes): each Householder
// step of the QR of Y is a handful of warp sums, and Q = H_0 ... H_{r-1} (applied to the
// identity, last reflector first) is kept one row per lane.  U_i = Qᴴ goes to Uout.
// The reflectors follow LAPACK's zlarfg convention (β real), with Newton-refined
// reciprocals in place of divisions.
__global__ void __launch_bounds__(32) k_blockrot_coeffs(int p, int r, const cplx* __restrict__ L, int ld,
                                                        cplx* Uout) {
  extern __shared__ cplx sm[];
  const int r2 = 2 * r, pr = p * r, bp = p - 1, lane = threadIdx.x;
  cplx* Lc = sm;                 // pr × r: the last block column of L
  for (int q = lane; q < pr * r; q += 32) Lc[q] = L[(int64_t)(bp * r + q / pr) * ld + (q % pr)];
  __syncwarp();
  const bool act = lane < r2;
  const int lrow = (lane < r) ? bp * r + lane : 0;   // row of Lc this lane reads / writes
  for (int i = 0; i < p - 1; ++i) {
    const int row = (lane < r) ? lrow : i * r + (lane - r);
    cplx y[8], v[8];
    cplx tau[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) y[c] = (act && c < r) ? Lc[c * pr + row] : czero();
    // Householder QR of Y, column by column
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      if (j >= r) break;
      const cplx alpha = cmk(__shfl_sync(0xffffffffu, y[j].x, j), __shfl_sync(0xffffffffu, y[j].y, j));
      const double x2 = warp_sum((act && lane > j) ? cabs2(y[j]) : 0.0);
      double beta;
      cplx t, sc;
      if (x2 == 0.0 && alpha.y == 0.0) {
        beta = alpha.x; t = czero(); sc = czero();
      } else {
        const double nrm = sqrt(alpha.x * alpha.x + alpha.y * alpha.y + x2);
        beta = (alpha.x >= 0.0) ? -nrm : nrm;
        const double ib = recip_nr(beta);
        t = cmk((beta - alpha.x) * ib, -alpha.y * ib);
        const double ar = alpha.x - beta, ai = alpha.y;
        const double id = recip_nr(ar * ar + ai * ai);
        sc = cmk(ar * id, -ai * id);
      }
      const cplx vj = (lane == j) ? cmk(1.0, 0.0) : ((act && lane > j) ? cmul(y[j], sc) : czero());
      v[j] = vj;
      tau[j] = t;
      const cplx tc = cconj(t);
#pragma unroll
      for (int c = 0; c < 8; ++c) {   // apply H_jᴴ to the columns c > j
        if (c > j && c < r) {
          const cplx s = warp_sum(cmulc(vj, y[c]));
          y[c] = cfms(vj, cmul(tc, s), y[c]);
        }
      }
      if (lane == j) y[j] = cmk(beta, 0.0);
      else if (lane > j) y[j] = czero();
    }
    // Q = H_0 ... H_{r-1} I, row `lane` of Q in q[]
    cplx q[16];
#pragma unroll
    for (int c = 0; c < 16; ++c) q[c] = (c == lane) ? cmk(1.0, 0.0) : czero();
#pragma unroll
    for (int j = 7; j >= 0; --j) {
      if (j >= r) continue;
      const cplx vj = v[j], tj = tau[j];
#pragma unroll
      for (int c = 0; c < 16; ++c) {
        if (c < r2) {
          const cplx s = warp_sum(cmulc(vj, q[c]));
          q[c] = cfms(vj, cmul(tj, s), q[c]);
        }
      }
    }
    cplx* U = Uout + (int64_t)i * r2 * r2;
    if (act) {
#pragma unroll
      for (int c = 0; c < 16; ++c)
        if (c < r2) U[lane * r2 + c] = cconj(q[c]);   // U(c, lane) = conj(Q(lane, c))
    }
    // new column blocks: [R; 0]
    __syncwarp();
    if (act) {
#pragma unroll
      for (int c = 0; c < 8; ++c)
        if (c < r) Lc[c * pr + row] = (lane < r && lane <= c) ? y[c] : czero();
    }
    __syncwarp();
  }
}

// Row-parallel right multiplications [X_p, X_i] ← [X_p, X_i] U_iᴴ, i = 0..p-2 in order,
// on up to 6 arrays (blockIdx.y selects one): 32 rows per CTA, one thread per (row,
// output column); blockDim = 32 · 2r.
struct RotArrays {
  cplx* a[6];
  int64_t nrows[6];
  int64_t ld[6];
};

__global__ void k_blockrot_apply(int p, int r, RotArrays arr, const cplx* __restrict__ Ulist) {
  extern __shared__ cplx sm[];
  const int r2 = 2 * r;
  cplx* old = sm;               // 32 × r2 (per row: [blk p | blk i])
  cplx* U = old + 32 * r2;      // r2 × r2
  cplx* A = arr.a[blockIdx.y];
  const int64_t nrows = arr.nrows[blockIdx.y], ld = arr.ld[blockIdx.y];
  const int64_t r0 = (int64_t)blockIdx.x * 32;
  if (r0 >= nrows) return;
  const int tr = threadIdx.x % 32, a = threadIdx.x / 32;   // row in tile, output column
  const int64_t row = r0 + tr;
  const int bp = p - 1;
  const bool valid = row < nrows;
  if (a < r) old[tr * r2 + a] = valid ? A[(int64_t)(bp * r + a) * ld + row] : czero();
  for (int i = 0; i < p - 1; ++i) {
    if (a >= r) old[tr * r2 + a] = valid ? A[(int64_t)(i * r + (a - r)) * ld + row] : czero();
    for (int q = threadIdx.x; q < r2 * r2; q += blockDim.x) U[q] = Ulist[(int64_t)i * r2 * r2 + q];
    __syncthreads();
    cplx s = czero();
    for (int l = 0; l < r2; ++l) s = cfma(old[tr * r2 + l], cconj(U[l * r2 + a]), s);
    __syncthreads();
    if (a < r) old[tr * r2 + a] = s;
    else if (valid) A[(int64_t)(i * r + (a - r)) * ld + row] = s;
    __syncthreads();
  }
  if (a < r && valid) A[(int64_t)(bp * r + a) * ld + row] = old[tr * r2 + a];
}

// Column-parallel left multiplications [X_p; X_i] ← U_i [X_p; X_i] on the block rows of
// up to 3 pr×pr matrices (blockIdx.y): 32 columns per CTA, one thread per (column,
// output row); blockDim = 32 · 2r.
struct RotMats {
  cplx* m[3];
};

__global__ void k_blockrot_left(int p, int r, RotMats mats, int ld, const cplx* __restrict__ Ulist) {
  extern __shared__ cplx sm[];
  const int r2 = 2 * r, pr = p * r;
  cplx* old = sm;               // 32 × r2 (per column: [blk p | blk i])
  cplx* U = old + 32 * r2;
  cplx* M = mats.m[blockIdx.y];
  const int c0 = blockIdx.x * 32;
  const int tc = threadIdx.x % 32, a = threadIdx.x / 32;
  const int col = c0 + tc;
  const bool valid = col < pr;
  const int bp = p - 1;
  if (a < r) old[tc * r2 + a] = valid ? M[(int64_t)col * ld + bp * r + a] : czero();
  for (int i = 0; i < p - 1; ++i) {
    if (a >= r) old[tc * r2 + a] = valid ? M[(int64_t)col * ld + i * r + (a - r)] : czero();
    for (int q = threadIdx.x; q < r2 * r2; q += blockDim.x) U[q] = Ulist[(int64_t)i * r2 * r2 + q];
    __syncthreads();
    cplx s = czero();
    for (int l = 0; l < r2; ++l) s = cfma(U[l * r2 + a], old[tc * r2 + l], s);
    __syncthreads();
    if (a < r) old[tc * r2 + a] = s;
    else if (valid) M[(int64_t)col * ld + i * r + (a - r)] = s;
    __syncthreads();
  }
  if (a < r && valid) M[(int64_t)col * ld + bp * r + a] = old[tc * r2 + a];
}
