// Block-unitary rotations of the recycled space (_block_unitary_update!,
// src/core/recySpace.jl:226-286; rls_block_unitary_rot!, lmul!/rmul!,
// src/types/RLSLinearAlgebra.jl:59-190).
//
// Rotation i (i = 1..p-1) is U_i = Qᴴ with Q the full unitary of the Householder
// QR of [L(p,p); L(i,p)] (2r × r).  It mixes block p with block i:
//   rows of L, H1, H2:     [X_p; X_i] ← U_i [X_p; X_i]
//   columns of V, J*, H*:  [X_p, X_i] ← [X_p, X_i] U_iᴴ
// The rotations depend only on L, so k_blockrot_prep computes all of them (and
// rotates the small pr×pr matrices) in one CTA; k_blockrot_apply then streams each
// tall array once, applying the p-1 rotations row by row from shared memory.
#pragma once
#include "common.cuh"
#include "small.cuh"

// Full m×m Q of the Householder QR of Y (m×k, in place destroyed), one warp.
__device__ void warp_house_fullq(cplx* Y, int ldy, int m, int k, cplx* Q, int ldq, cplx* tau) {
  const int lane = threadIdx.x & 31;
  for (int j = 0; j < k; ++j) {
    double x2 = 0.0;
    for (int i = j + 1 + lane; i < m; i += 32) x2 += cabs2(Y[j * ldy + i]);
    x2 = warp_sum(x2);
    double beta; cplx t, sc;
    householder_coeffs(Y[j * ldy + j], x2, &beta, &t, &sc);
    __syncwarp();
    for (int i = j + 1 + lane; i < m; i += 32) Y[j * ldy + i] = cmul(Y[j * ldy + i], sc);
    __syncwarp();
    if (lane == 0) { Y[j * ldy + j] = cmk(beta, 0.0); tau[j] = t; }
    __syncwarp();
    for (int c = j + 1; c < k; ++c) {
      cplx s = czero();
      for (int i = j + lane; i < m; i += 32) {
        const cplx v = (i == j) ? cmk(1.0, 0.0) : Y[j * ldy + i];
        s = cfmac(v, Y[c * ldy + i], s);
      }
      s = warp_sum(s);
      const cplx f = cmul(cconj(t), s);
      __syncwarp();
      for (int i = j + lane; i < m; i += 32) {
        const cplx v = (i == j) ? cmk(1.0, 0.0) : Y[j * ldy + i];
        Y[c * ldy + i] = cfms(v, f, Y[c * ldy + i]);
      }
      __syncwarp();
    }
  }
  // Q = H_0 ... H_{k-1} I_m: apply reflectors to the identity, last one first.
  for (int q = lane; q < m * m; q += 32) Q[(q / m) * ldq + (q % m)] = ((q % m) == (q / m)) ? cmk(1.0, 0.0) : czero();
  __syncwarp();
  for (int j = k - 1; j >= 0; --j) {
    const cplx tj = tau[j];
    for (int c = 0; c < m; ++c) {
      cplx s = czero();
      for (int i = j + lane; i < m; i += 32) {
        const cplx v = (i == j) ? cmk(1.0, 0.0) : Y[j * ldy + i];
        s = cfmac(v, Q[c * ldq + i], s);
      }
      s = warp_sum(s);
      const cplx f = cmul(tj, s);
      __syncwarp();
      for (int i = j + lane; i < m; i += 32) {
        const cplx v = (i == j) ? cmk(1.0, 0.0) : Y[j * ldy + i];
        Q[c * ldq + i] = cfms(v, f, Q[c * ldq + i]);
      }
      __syncwarp();
    }
  }
}

// Rows (bp, bi) of the pr-column matrix M (ld) ← U [rows bp; rows bi]; U is 2r×2r.
__device__ void rot_rows(cplx* M, int ld, int pr, int r, int bp, int bi, const cplx* U, cplx* tmp) {
  const int r2 = 2 * r;
  for (int q = threadIdx.x; q < r2 * pr; q += blockDim.x) {
    const int a = q % r2, c = q / r2;
    const int row = (a < r) ? bp * r + a : bi * r + (a - r);
    tmp[q] = M[(int64_t)c * ld + row];
  }
  __syncthreads();
  for (int q = threadIdx.x; q < r2 * pr; q += blockDim.x) {
    const int a = q % r2, c = q / r2;
    cplx s = czero();
    for (int l = 0; l < r2; ++l) s = cfma(U[l * r2 + a], tmp[c * r2 + l], s);
    const int row = (a < r) ? bp * r + a : bi * r + (a - r);
    M[(int64_t)c * ld + row] = s;
  }
  __syncthreads();
}

// Columns (bp, bi) of the pr-row matrix M ← [cols bp, cols bi] Uᴴ.
__device__ void rot_cols(cplx* M, int ld, int pr, int r, int bp, int bi, const cplx* U, cplx* tmp) {
  const int r2 = 2 * r;
  for (int q = threadIdx.x; q < r2 * pr; q += blockDim.x) {
    const int row = q % pr, a = q / pr;
    const int col = (a < r) ? bp * r + a : bi * r + (a - r);
    tmp[q] = M[(int64_t)col * ld + row];
  }
  __syncthreads();
  for (int q = threadIdx.x; q < r2 * pr; q += blockDim.x) {
    const int row = q % pr, a = q / pr;
    cplx s = czero();
    // new[:, a] = sum_l old[:, l] * conj(U[a, l])
    for (int l = 0; l < r2; ++l) s = cfma(tmp[l * pr + row], cconj(U[l * r2 + a]), s);
    const int col = (a < r) ? bp * r + a : bi * r + (a - r);
    M[(int64_t)col * ld + row] = s;
  }
  __syncthreads();
}

// One CTA.  p >= 2 blocks (1-based block p is the newest).  Writes U_1..U_{p-1}
// (each 2r×2r, column-major) to Uout and rotates L (rows), H1 and H2 (both sides).
// Shared memory: (2r*r + 4r*r + 2r) + 2r*pr cplx.
__global__ void __launch_bounds__(256) k_blockrot_prep(int p, int r, cplx* L, cplx* H1, cplx* H2, int ld,
                                                       cplx* Uout) {
  extern __shared__ cplx sm[];
  const int r2 = 2 * r, pr = p * r;
  cplx* Y = sm;                 // r2 × r
  cplx* Q = Y + r2 * r;         // r2 × r2
  cplx* U = Q + r2 * r2;        // r2 × r2
  cplx* tau = U + r2 * r2;      // r
  cplx* tmp = tau + r;          // r2 × pr
  const int bp = p - 1;
  for (int i = 0; i < p - 1; ++i) {
    // Y = [L(bp, bp); L(i, bp)]
    for (int q = threadIdx.x; q < r2 * r; q += blockDim.x) {
      const int a = q % r2, c = q / r2;
      const int row = (a < r) ? bp * r + a : i * r + (a - r);
      Y[c * r2 + a] = L[(int64_t)(bp * r + c) * ld + row];
    }
    __syncthreads();
    if (threadIdx.x < 32) warp_house_fullq(Y, r2, r2, r, Q, r2, tau);
    __syncthreads();
    for (int q = threadIdx.x; q < r2 * r2; q += blockDim.x) {
      const int a = q % r2, c = q / r2;
      U[c * r2 + a] = cconj(Q[a * r2 + c]);          // U = Qᴴ
    }
    __syncthreads();
    for (int q = threadIdx.x; q < r2 * r2; q += blockDim.x) Uout[(int64_t)i * r2 * r2 + q] = U[q];
    rot_rows(L, ld, pr, r, bp, i, U, tmp);            // lmul!(bu, L)
    rot_cols(H1, ld, pr, r, bp, i, U, tmp);           // rmul!(H1, bu')
    rot_rows(H1, ld, pr, r, bp, i, U, tmp);           // lmul!(bu, H1)
    rot_cols(H2, ld, pr, r, bp, i, U, tmp);
    rot_rows(H2, ld, pr, r, bp, i, U, tmp);
  }
}

// Streams the rows of up to 4 tall arrays (blockIdx.y selects the array) and applies
// [X_p, X_i] ← [X_p, X_i] U_iᴴ for i = 0..p-2 in order.  32 rows per CTA, one thread
// per (row, output column); blockDim = 32 * 2r.
struct RotArrays {
  cplx* a[4];
};

__global__ void k_blockrot_apply(int64_t nrows, int p, int r, RotArrays arr, int64_t ld,
                                 const cplx* __restrict__ Ulist) {
  extern __shared__ cplx sm[];
  const int r2 = 2 * r;
  cplx* old = sm;               // 32 × r2 (row-major per row: [blk p | blk i])
  cplx* U = old + 32 * r2;      // r2 × r2
  cplx* A = arr.a[blockIdx.y];
  const int64_t r0 = (int64_t)blockIdx.x * 32;
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
