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
#pragma once
#include "common.cuh"
#include "small.cuh"

// Full m×m Q of the Householder QR of Y (m×k, m <= 32, in place: Y ← R and reflector
// tails), one warp.  Lane c owns column c, so every dot product is a serial loop in one
// lane: no shuffles on the dependency chain.
__device__ void warp_house_fullq(cplx* Y, int ldy, int m, int k, cplx* Q, int ldq, cplx* tau) {
  const int lane = threadIdx.x & 31;
  __shared__ cplx s_t[32];
  for (int j = 0; j < k; ++j) {
    if (lane == 0) {
      double x2 = 0.0;
      for (int i = j + 1; i < m; ++i) x2 += cabs2(Y[j * ldy + i]);
      double beta; cplx t, sc;
      householder_coeffs(Y[j * ldy + j], x2, &beta, &t, &sc);
      for (int i = j + 1; i < m; ++i) Y[j * ldy + i] = cmul(Y[j * ldy + i], sc);
      Y[j * ldy + j] = cmk(beta, 0.0);
      tau[j] = t;
      s_t[0] = t;
    }
    __syncwarp();
    const cplx tc = cconj(s_t[0]);
    const int c = j + 1 + lane;
    if (c < k) {   // apply H_jᴴ to column c
      cplx s = Y[c * ldy + j];
      for (int i = j + 1; i < m; ++i) s = cfmac(Y[j * ldy + i], Y[c * ldy + i], s);
      const cplx f = cmul(tc, s);
      Y[c * ldy + j] = csub(Y[c * ldy + j], f);
      for (int i = j + 1; i < m; ++i) Y[c * ldy + i] = cfms(Y[j * ldy + i], f, Y[c * ldy + i]);
    }
    __syncwarp();
  }
  // Q = H_0 ... H_{k-1} I_m, last reflector first; lane c owns column c of Q.
  if (lane < m) {
    for (int i = 0; i < m; ++i) Q[lane * ldq + i] = (i == lane) ? cmk(1.0, 0.0) : czero();
    for (int j = k - 1; j >= 0; --j) {
      const cplx tj = tau[j];
      cplx s = Q[lane * ldq + j];
      for (int i = j + 1; i < m; ++i) s = cfmac(Y[j * ldy + i], Q[lane * ldq + i], s);
      const cplx f = cmul(tj, s);
      Q[lane * ldq + j] = csub(Q[lane * ldq + j], f);
      for (int i = j + 1; i < m; ++i) Q[lane * ldq + i] = cfms(Y[j * ldy + i], f, Q[lane * ldq + i]);
    }
  }
  __syncwarp();
}

// Rotation coefficients from the last block column of L alone: rotation i (i < p-1,
// 0-based) is determined by [L(p-1, p-1); L(i, p-1)] after rotations 0..i-1, and those
// only change block row p-1 of that column.  One warp; Lc (pr × r) in shared memory.
__global__ void k_blockrot_coeffs(int p, int r, const cplx* __restrict__ L, int ld, cplx* Uout) {
  extern __shared__ cplx sm[];
  const int r2 = 2 * r, pr = p * r, bp = p - 1, lane = threadIdx.x;
  cplx* Lc = sm;                 // pr × r
  cplx* Y = Lc + pr * r;         // r2 × r
  cplx* Q = Y + r2 * r;          // r2 × r2
  cplx* tau = Q + r2 * r2;       // r
  for (int q = lane; q < pr * r; q += 32) Lc[q] = L[(int64_t)(bp * r + q / pr) * ld + (q % pr)];
  __syncwarp();
  for (int i = 0; i < p - 1; ++i) {
    for (int q = lane; q < r2 * r; q += 32) {
      const int a = q % r2, c = q / r2;
      Y[c * r2 + a] = Lc[c * pr + ((a < r) ? bp * r + a : i * r + (a - r))];
    }
    __syncwarp();
    warp_house_fullq(Y, r2, r2, r, Q, r2, tau);   // Y ← R (upper part), Q full
    __syncwarp();
    cplx* U = Uout + (int64_t)i * r2 * r2;
    for (int q = lane; q < r2 * r2; q += 32) {
      const int a = q % r2, c = q / r2;
      U[c * r2 + a] = cconj(Q[a * r2 + c]);        // U = Qᴴ
    }
    // new column blocks: [R; 0] (U·Y)
    for (int q = lane; q < r2 * r; q += 32) {
      const int a = q % r2, c = q / r2;
      const int row = (a < r) ? bp * r + a : i * r + (a - r);
      Lc[c * pr + row] = (a < r && a <= c) ? Y[c * r2 + a] : czero();
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
