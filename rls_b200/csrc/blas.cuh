// Streaming kernels over tall n-row blocks and the tiled Schur factor.
//
// Layout (shared by every kernel here):
//   * tall blocks (V, J1, J2, J5, LOBPCG S/CS, ...) are column-major with
//     leading dimension ld = n_pad (a multiple of TILE); rows n..n_pad-1 are
//     kept at zero so every kernel may run over n_pad rows;
//   * the upper-triangular Schur factor T is stored by TILE×TILE tiles, tile
//     (I, J) (J >= I) at tile index J*(J+1)/2 + I, each tile column-major with
//     leading dimension TILE.  Rows/columns beyond n are zero.
#pragma once
#include "common.cuh"

#define TILE 64

__host__ __device__ __forceinline__ int64_t tile_index(int I, int J) {
  return (int64_t)J * (J + 1) / 2 + I;
}

// Tile slots of an upper-triangular factor whose tiles vanish beyond tile bandwidth bw
// (J − I ≤ bw): the packed layout above when bw ≥ nb − 1, else tile (I, J) at slot
// J·(bw + 1) + (J − I) (slots with J − I > J unused).  The banded R of a sparse shifted
// factor uses the second form.
__host__ __device__ __forceinline__ int64_t tile_index_bw(int I, int J, int nb, int bw) {
  return (bw >= nb - 1) ? tile_index(I, J) : (int64_t)J * (bw + 1) + (J - I);
}
__host__ __device__ __forceinline__ int64_t tile_slots(int nb, int bw) {
  return (bw >= nb - 1) ? (int64_t)nb * (nb + 1) / 2 : (int64_t)nb * (bw + 1);
}

// ------------------------------------------------------------------------------------
// Gram: C (k1×k2) = alpha·AᴴB + beta·C in one launch.  Grid (row chunks, ceil(k1/8)):
// warp w of CTA (c, g) owns column g·8+w of A and sums conj(A)·B over chunk c's rows,
// writing its partial to part[c][col][:].  The last CTA of column group g to finish
// (atomic counter, after a fence) sums the partials of that group over the chunks in a
// fixed order — four threads per output over chunks ≡ q (mod 4), then a fixed shuffle
// tree — so the result does not depend on which CTA finishes last; it then resets the
// counter.  K2 is the exact column count of B when EXACT, else an upper bound.
// ------------------------------------------------------------------------------------
template <int K2, bool EXACT>
__global__ void __launch_bounds__(256) k_gram(int64_t nrows, int64_t chunk, const cplx* __restrict__ A,
                                              int64_t lda, int k1, const cplx* __restrict__ B, int64_t ldb,
                                              int k2, cplx* part, int* counters, cplx alpha, cplx beta, cplx* C,
                                              int64_t ldc) {
  const int kk2 = EXACT ? K2 : k2;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int col = blockIdx.y * 8 + w;
  const int64_t r0 = (int64_t)blockIdx.x * chunk;
  const int64_t r1 = min(nrows, r0 + chunk);
  cplx acc[K2];
#pragma unroll
  for (int j = 0; j < K2; ++j) acc[j] = czero();
  if (col < k1) {
    const cplx* a = A + (int64_t)col * lda;
    for (int64_t row = r0 + lane; row < r1; row += 32) {
      const cplx av = a[row];
#pragma unroll
      for (int j = 0; j < K2; ++j)
        if (EXACT || j < k2) acc[j] = cfmac(av, __ldg(&B[(int64_t)j * ldb + row]), acc[j]);
    }
  }
#pragma unroll
  for (int j = 0; j < K2; ++j) {
    if (EXACT || j < k2) {
      const cplx s = warp_sum(acc[j]);
      if (lane == 0 && col < k1) part[((int64_t)blockIdx.x * k1 + col) * kk2 + j] = s;
    }
  }
  __shared__ int s_last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    s_last = (atomicAdd(&counters[blockIdx.y], 1) == (int)gridDim.x - 1);
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  const int i0 = blockIdx.y * 8, ni = min(8, k1 - i0), nout = ni * kk2, nc = (int)gridDim.x;
  const int q = threadIdx.x & 3;
  for (int base = 0; base < nout; base += (int)blockDim.x / 4) {
    const int o = base + (int)threadIdx.x / 4;
    const bool valid = o < nout;
    const int i = i0 + (valid ? o / kk2 : 0), j = valid ? o % kk2 : 0;
    cplx s0 = czero(), s1 = czero();
    if (valid) {
      int c = q;
      for (; c + 4 < nc; c += 8) {
        s0 = cadd(s0, __ldcg(&part[((int64_t)c * k1 + i) * kk2 + j]));
        s1 = cadd(s1, __ldcg(&part[((int64_t)(c + 4) * k1 + i) * kk2 + j]));
      }
      if (c < nc) s0 = cadd(s0, __ldcg(&part[((int64_t)c * k1 + i) * kk2 + j]));
    }
    cplx s = cadd(s0, s1);
    s.x += __shfl_xor_sync(0xffffffffu, s.x, 1);
    s.y += __shfl_xor_sync(0xffffffffu, s.y, 1);
    s.x += __shfl_xor_sync(0xffffffffu, s.x, 2);
    s.y += __shfl_xor_sync(0xffffffffu, s.y, 2);
    if (valid && q == 0) {
      cplx out = cmul(alpha, s);
      if (beta.x != 0.0 || beta.y != 0.0) out = cfma(beta, C[(int64_t)j * ldc + i], out);
      C[(int64_t)j * ldc + i] = out;
    }
  }
  if (threadIdx.x == 0) counters[blockIdx.y] = 0;
}

// ------------------------------------------------------------------------------------
// Row-streaming GEMM with an affine combination of up to 4 sources:
//   Y = sum_q coef_q * A_q           (row by row, never materialised)
//   C = alpha * Y * B + beta * C     (B: k1 × k2 small, k2 <= 32)
// Optional second product X = A_xsrc * B (same B) and epilogue C -= X * diag(sig²),
// plus per-CTA partial |C[:,0]|^2 sums.  One thread per row; a row of C is written
// only after all reads of that row, so C may alias A_q when k1 == k2.
// ------------------------------------------------------------------------------------
struct CombSrc {
  const cplx* a[4];
  cplx coef[4];
  int nsrc;
};

// Tile of 32 rows per CTA; warp w of the 8 sums the inner index range
// [w·kc, (w+1)·kc) for its lane's row, then the warps' partial sums are combined
// through shared memory (8 × 32 × K2MAX cplx).  Rows are owned by one CTA and all
// reads of a row precede the barrier before its writes, so C may alias a source.
template <int K2MAX>
__global__ void __launch_bounds__(256) k_gemm_rows(int64_t nrows, CombSrc src, int64_t lda, int k1,
                                                   const cplx* __restrict__ B, int64_t ldb, int k2,
                                                   cplx alpha, cplx beta, cplx* C, int64_t ldc,
                                                   int xsrc, cplx* X, int64_t ldx,
                                                   const double* __restrict__ sig,
                                                   double* __restrict__ col0_part) {
  extern __shared__ cplx red[];   // [2][8][K2MAX][32]
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t row = (int64_t)blockIdx.x * 32 + lane;
  const int kc = (k1 + 7) / 8;
  const int kb = w * kc, ke = min(k1, kb + kc);
  cplx acc[K2MAX], accx[K2MAX];
#pragma unroll
  for (int j = 0; j < K2MAX; ++j) { acc[j] = czero(); accx[j] = czero(); }
  if (row < nrows) {
    for (int kk = kb; kk < ke; ++kk) {
      const int64_t off = (int64_t)kk * lda + row;
      cplx y = czero(), xv = czero();
      for (int q = 0; q < src.nsrc; ++q) {
        const cplx v = src.a[q][off];
        y = cfma(src.coef[q], v, y);
        if (q == xsrc) xv = v;
      }
#pragma unroll
      for (int j = 0; j < K2MAX; ++j) {
        if (j < k2) {
          const cplx bb = __ldg(&B[(int64_t)j * ldb + kk]);
          acc[j] = cfma(y, bb, acc[j]);
          if (xsrc >= 0) accx[j] = cfma(xv, bb, accx[j]);
        }
      }
    }
  }
#pragma unroll
  for (int j = 0; j < K2MAX; ++j) {
    if (j < k2) {
      red[((0 * 8 + w) * K2MAX + j) * 32 + lane] = acc[j];
      if (xsrc >= 0) red[((1 * 8 + w) * K2MAX + j) * 32 + lane] = accx[j];
    }
  }
  __syncthreads();
  // thread (lane, w) finalises outputs j = w, w+8, ... of its lane's row
  double c0 = 0.0;
  for (int j = w; j < k2; j += 8) {
    cplx sacc = czero(), sx = czero();
    for (int q = 0; q < 8; ++q) {
      sacc = cadd(sacc, red[((0 * 8 + q) * K2MAX + j) * 32 + lane]);
      if (xsrc >= 0) sx = cadd(sx, red[((1 * 8 + q) * K2MAX + j) * 32 + lane]);
    }
    if (row < nrows) {
      cplx out = cmul(alpha, sacc);
      if (beta.x != 0.0 || beta.y != 0.0) out = cfma(beta, C[(int64_t)j * ldc + row], out);
      if (xsrc >= 0) {
        if (sig) out = csub(out, cscale(sx, sig[j] * sig[j]));
        X[(int64_t)j * ldx + row] = sx;
      }
      C[(int64_t)j * ldc + row] = out;
      if (j == 0) c0 = cabs2(out);
    }
  }
  if (col0_part) {
    __shared__ double sred[32];
    const double s = block_sum(c0, sred);
    if (threadIdx.x == 0) col0_part[blockIdx.x] = s;
  }
}

// ------------------------------------------------------------------------------------
// Tiled TRMM: Y = T X (adj=0) or Y = Tᴴ X (adj=1), X/Y n_pad × k (k <= 16).
// Work unit u = (output tile row/col O, chunk of up to UT source tiles); partials
// land in part[u] and k_trmm_reduce sums the units of each O in a fixed order.
// ------------------------------------------------------------------------------------
#define TRMM_UT 8

// Loads tile `tp` (TILE×TILE, column-major) into shared memory with row stride
// TILE_LDS.  For adj the tile is stored transposed so that both T·x and Tᴴ·x read
// consecutive addresses across threads (the odd stride keeps the 16-byte slots of
// eight consecutive threads in distinct banks).
#define TILE_LDS (TILE + 1)
__device__ __forceinline__ void load_tile(cplx* sT, const cplx* __restrict__ tp, int adj) {
  for (int t = threadIdx.x; t < TILE * TILE; t += blockDim.x) {
    const int rr = t % TILE, cc = t / TILE;
    cp_async16(adj ? &sT[rr * TILE_LDS + cc]     // element (rr, cc) at "column" rr
                   : &sT[cc * TILE_LDS + rr],    // element (rr, cc) at column cc
               &tp[t]);
  }
  cp_async_wait_all();
}

// acc[c] += (adj ? Tᴴ : T)[row, inner-range] · sX[inner-range, c]; the inner dimension is
// split into NG ranges of TILE/NG, range `grp` here.
template <int KMAX, int NG = 4>
__device__ __forceinline__ void tile_apply(const cplx* sT, const cplx* sX, int k, int adj, int row, int grp,
                                           cplx* acc) {
  constexpr int W = TILE / NG;
  if (!adj) {
    for (int jj = grp * W; jj < grp * W + W; ++jj) {
      const cplx tv = sT[jj * TILE_LDS + row];
#pragma unroll
      for (int c = 0; c < KMAX; ++c)
        if (c < k) acc[c] = cfma(tv, sX[c * TILE + jj], acc[c]);
    }
  } else {
    for (int ii = grp * W; ii < grp * W + W; ++ii) {
      const cplx tv = sT[ii * TILE_LDS + row];   // T[ii, row]
#pragma unroll
      for (int c = 0; c < KMAX; ++c)
        if (c < k) acc[c] = cfmac(tv, sX[c * TILE + ii], acc[c]);
    }
  }
}

template <int KMAX>
__global__ void __launch_bounds__(256) k_trmm_partial(int nb, const cplx* __restrict__ T,
                                                      const cplx* __restrict__ X, int64_t ldx, int k,
                                                      int adj, const int* __restrict__ unit_O,
                                                      const int* __restrict__ unit_s,
                                                      cplx* __restrict__ part) {
  extern __shared__ cplx sm[];
  cplx* sT = sm;                       // TILE*TILE_LDS
  cplx* sX = sm + TILE * TILE_LDS;     // TILE*k
  cplx* sAcc = sm;                     // 4 × TILE*k partial sums, reuses sT after the loop (k <= 16)
  const int u = blockIdx.x;
  const int O = unit_O[u], s0 = unit_s[u];
  const int row = threadIdx.x & (TILE - 1), grp = threadIdx.x >> 6;  // 4 groups split the inner dim
  cplx acc[KMAX];
#pragma unroll
  for (int c = 0; c < KMAX; ++c) acc[c] = czero();
  // Source tiles: adj=0: T(O, J), J = O + s0 .. ; adj=1: T(I, O), I = s0 ..
  const int nsrc = adj ? (O + 1) : (nb - O);
  const int s1 = min(nsrc, s0 + TRMM_UT);
  for (int s = s0; s < s1; ++s) {
    const int I = adj ? s : O;
    const int J = adj ? O : O + s;
    const int xb = adj ? I : J;  // tile of X that multiplies
    __syncthreads();
    load_tile(sT, T + tile_index(I, J) * (TILE * TILE), adj);
    for (int t = threadIdx.x; t < TILE * k; t += blockDim.x) {
      const int rr = t % TILE, c = t / TILE;
      sX[c * TILE + rr] = X[(int64_t)c * ldx + (int64_t)xb * TILE + rr];
    }
    __syncthreads();
    tile_apply<KMAX>(sT, sX, k, adj, row, grp, acc);
  }
  __syncthreads();
#pragma unroll
  for (int c = 0; c < KMAX; ++c)
    if (c < k) sAcc[(grp * k + c) * TILE + row] = acc[c];
  __syncthreads();
  for (int t = threadIdx.x; t < TILE * k; t += blockDim.x) {
    const int rr = t % TILE, c = t / TILE;
    cplx v = sAcc[(0 * k + c) * TILE + rr];
    v = cadd(v, sAcc[(1 * k + c) * TILE + rr]);
    v = cadd(v, sAcc[(2 * k + c) * TILE + rr]);
    v = cadd(v, sAcc[(3 * k + c) * TILE + rr]);
    part[((int64_t)u * 16 + c) * TILE + rr] = v;
  }
}

__global__ void k_trmm_reduce(int nb, int k, const int* __restrict__ O_first, const int* __restrict__ O_count,
                              const cplx* __restrict__ part, cplx* Y, int64_t ldy) {
  const int O = blockIdx.x;
  for (int t = threadIdx.x; t < TILE * k; t += blockDim.x) {
    const int rr = t % TILE, c = t / TILE;
    cplx s = czero();
    for (int u = O_first[O]; u < O_first[O] + O_count[O]; ++u) s = cadd(s, part[((int64_t)u * 16 + c) * TILE + rr]);
    Y[(int64_t)c * ldy + (int64_t)O * TILE + rr] = s;
  }
}

// Inverses D_b⁻¹ of the diagonal tiles of R = T − zI, one CTA per tile (512 threads).
// Warp w solves U y = e_j for the columns j ∈ {w, 31−w, 32+w, 63−w} (equal work per
// warp) by column-oriented back substitution: lane i holds rows i and i+32 of the
// right-hand side, y_l is broadcast by shuffle and every lane updates its rows < l.
// Pad rows (global row ≥ n) get 1 on the diagonal, so the pad stays inert.
// Dynamic shared memory: TILE·TILE_LDS cplx.
__global__ void __launch_bounds__(512) k_diag_inv(int nb, int bw, int64_t n, const cplx* __restrict__ T, cplx z,
                                                  cplx* __restrict__ Dinv, int* err) {
  extern __shared__ cplx sm[];
  cplx* sU = sm;                    // U[r][c] at sU[c*TILE_LDS + r], zero below the diagonal
  __shared__ cplx sdi[TILE];        // 1 / U[i][i]
  const int I = blockIdx.x;
  const cplx* tp = T + tile_index_bw(I, I, nb, bw) * (TILE * TILE);
  for (int t = threadIdx.x; t < TILE * TILE; t += blockDim.x) {
    const int rr = t % TILE, cc = t / TILE;
    const int64_t g = (int64_t)I * TILE + rr;
    cplx u = tp[t];
    if (rr == cc) u = (g < n) ? csub(u, z) : cmk(1.0, 0.0);
    sU[cc * TILE_LDS + rr] = (rr <= cc) ? u : czero();
  }
  __syncthreads();
  if (threadIdx.x < TILE) sdi[threadIdx.x] = cinv(sU[threadIdx.x * TILE_LDS + threadIdx.x]);
  __syncthreads();
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  bool bad = false;
  const int cols[4] = {w, 31 - w, 32 + w, 63 - w};
  cplx* out = Dinv + (int64_t)I * TILE * TILE;
  for (int q = 0; q < 4; ++q) {
    const int j = cols[q];
    cplx y0 = (lane == j) ? cmk(1.0, 0.0) : czero();        // row lane
    cplx y1 = (lane + 32 == j) ? cmk(1.0, 0.0) : czero();   // row lane + 32
    for (int l = j; l >= 0; --l) {
      const int src = l & 31;
      const cplx mine = (l >= 32) ? y1 : y0;
      const cplx rl = cmk(__shfl_sync(0xffffffffu, mine.x, src), __shfl_sync(0xffffffffu, mine.y, src));
      const cplx yl = cmul(rl, sdi[l]);
      if (lane == src) {
        if (l >= 32) y1 = yl;
        else y0 = yl;
      }
      if (lane < l) y0 = cfms(sU[l * TILE_LDS + lane], yl, y0);
      if (lane + 32 < l) y1 = cfms(sU[l * TILE_LDS + lane + 32], yl, y1);
    }
    if (!isfinite(y0.x) || !isfinite(y0.y) || !isfinite(y1.x) || !isfinite(y1.y)) bad = true;
    out[j * TILE + lane] = y0;
    out[j * TILE + lane + 32] = y1;
  }
  if (bad) atomicOr(err, DEVERR_NONFINITE);
}

// Block-row scaled factor of the shifted solve: G(I, J) = D_I⁻¹ · T(I, J) for every tile
// J > I, stored in the packed tile layout of T (diagonal slots unused).  With
// R = D·(I + G) the solves need no D⁻¹ product on their dependency chain:
//   R x = b   ⇔  x_b = D_b⁻¹ b_b − Σ_{J>b} G(b,J) x_J
//   Rᴴ x = b  ⇔  u_b = b_b − Σ_{J<b} G(J,b)ᴴ u_J,  x_b = D_b⁻ᴴ u_b.
// Grid: two CTAs per tile slot (tile_slots(nb, bw) slots), CTA h computing output rows
// [32h, 32h+32); 256 threads.  Warp w owns the four rows 4w..4w+3 (A values broadcast),
// lane the columns lane and lane+32.  D_I⁻¹ is upper triangular, so warp w sums only
// l ≥ 32h + 4w (a warp-uniform start).  The result is staged in shared memory and
// written out coalesced.
// Dynamic shared memory (scale_smem_bytes): 64×33 + 64×65 cplx, two CTAs per SM.
#define SC_ALD 33
__global__ void __launch_bounds__(256) k_trsm_scale(int nb, int bw, const cplx* __restrict__ T,
                                                    const cplx* __restrict__ Dinv, cplx* __restrict__ G) {
  extern __shared__ cplx sm[];
  cplx* sA = sm;                      // D⁻¹[32h + i][l] at sA[l*SC_ALD + i]
  cplx* sB = sm + TILE * SC_ALD;      // T[l][c] at sB[c*TILE_LDS + l]; output staging afterwards
  const int64_t idx = blockIdx.x >> 1;
  const int h = blockIdx.x & 1;
  int I, J;
  if (bw >= nb - 1) {
    J = (int)((sqrt(8.0 * (double)idx + 1.0) - 1.0) * 0.5);
    while ((int64_t)J * (J + 1) / 2 > idx) --J;
    while ((int64_t)(J + 1) * (J + 2) / 2 <= idx) ++J;
    I = (int)(idx - (int64_t)J * (J + 1) / 2);
  } else {
    J = (int)(idx / (bw + 1));
    I = J - (int)(idx % (bw + 1));
    if (I < 0) return;
  }
  if (I >= J) return;
  const cplx* dp = Dinv + (int64_t)I * TILE * TILE;
  const cplx* tp = T + idx * (TILE * TILE);
  for (int q = threadIdx.x; q < 32 * TILE; q += blockDim.x) {
    const int r = q % 32, l = q / 32;
    cp_async16(&sA[l * SC_ALD + r], &dp[l * TILE + h * 32 + r]);
  }
  for (int q = threadIdx.x; q < TILE * TILE; q += blockDim.x) {
    const int r = q % TILE, c = q / TILE;
    cp_async16(&sB[c * TILE_LDS + r], &tp[q]);
  }
  cp_async_wait_all();
  __syncthreads();
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  cplx acc[4][2];
#pragma unroll
  for (int a = 0; a < 4; ++a) { acc[a][0] = czero(); acc[a][1] = czero(); }
  for (int l = 32 * h + 4 * w; l < TILE; ++l) {
    cplx av[4], bv[2];
#pragma unroll
    for (int a = 0; a < 4; ++a) av[a] = sA[l * SC_ALD + 4 * w + a];
#pragma unroll
    for (int c = 0; c < 2; ++c) bv[c] = sB[(lane + 32 * c) * TILE_LDS + l];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int c = 0; c < 2; ++c) acc[a][c] = cfma(av[a], bv[c], acc[a][c]);
  }
  __syncthreads();   // sB is reused for the output block (32 rows × 64 columns, ld 33)
  cplx* sO = sB;
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int c = 0; c < 2; ++c) sO[(lane + 32 * c) * SC_ALD + 4 * w + a] = acc[a][c];
  __syncthreads();
  cplx* out = G + idx * (TILE * TILE);
  for (int q = threadIdx.x; q < 32 * TILE; q += blockDim.x) {
    const int r = q % 32, c = q / 32;
    out[c * TILE + h * 32 + r] = sO[c * SC_ALD + r];
  }
}

inline size_t scale_smem_bytes() { return ((size_t)TILE * SC_ALD + (size_t)TILE * TILE_LDS) * sizeof(cplx); }

// ------------------------------------------------------------------------------------
// Dataflow triangular solve on the scaled factor (k_trsm_scale), half block rows.
//   adj = 0: R x = b   → x_b = D_b⁻¹ b_b − Σ_{J>b} G(b,J) x_J, written to X;
//   adj = 1: Rᴴ x = b  → u_b = b_b − Σ_{J<b} G(J,b)ᴴ u_J, written to U; k_trsm_finish
//            then forms X = D⁻ᴴ U block by block.
// Work unit: a half block row (32 rows of a 64-row block), 2·nb units, 256 threads per
// CTA.  Units are taken by ticket in dependency order, and a CTA takes tickets until they
// run out, so any grid of 1..2·nb CTAs solves the system: a unit only waits on units with
// smaller tickets, each held by a CTA that is already running, so every wait ends even
// when not all CTAs are resident.  A smaller grid leaves SMs to concurrent work.
// Waits are bounded by RLS_SPIN_LIMIT polls; on expiry the CTA records
// DEVERR_SPIN_TIMEOUT and carries on, so the launch always terminates.  Each
// dependency costs one 32×64×k product; the next tile is prefetched into registers
// while the current dependency is awaited and applied.  Published halves carry an
// epoch in flags[2·block + half] (st.release / ld.acquire at gpu scope).  X must not
// alias B.  K (the number of columns, 1..8) is a template parameter.
// ------------------------------------------------------------------------------------
__device__ __forceinline__ int ld_acquire(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(int* p, int v) {
  asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

#define HT_LDS 33   // shared-memory leading dimension of a 32-row half tile

// Prefetch of a 32×64 half tile into registers (8 values per thread of 256):
//   trans = 0: A[r][jj] = M[h*32 + r][jj]          (M column-major 64×64)
//   trans = 1: A[r][jj] = conj(M[jj][h*32 + r])
struct HalfTile {
  cplx v[8];
  __device__ __forceinline__ void load(const cplx* __restrict__ M, int h, int trans) {
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int idx = i * 256 + threadIdx.x;
      v[i] = trans ? M[(h * 32 + idx / 64) * TILE + (idx % 64)] : M[(idx / 32) * TILE + h * 32 + (idx % 32)];
    }
  }
  __device__ __forceinline__ void store(cplx* sA, int trans) const {
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int idx = i * 256 + threadIdx.x;
      if (trans) sA[(idx % 64) * HT_LDS + idx / 64] = cconj(v[i]);
      else sA[(idx / 32) * HT_LDS + (idx % 32)] = v[i];
    }
  }
};

// sAcc[c][r] (op)= Σ_jj A[r][jj]·sX[c][jj] for the 32×64 half tile in sA and exactly K
// columns: warp w sums jj ∈ [8w, 8w+8) for row = lane, and the eight partial sums are
// combined through sPart.  op: 0 set, 1 subtract.  Starts and ends with the block
// synchronised.
template <int K>
__device__ __forceinline__ void half_product(const cplx* sA, const cplx* sX, cplx* sPart, cplx* sAcc, int op) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  cplx acc[K];
#pragma unroll
  for (int c = 0; c < K; ++c) acc[c] = czero();
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    const int jj = w * 8 + q;
    const cplx a = sA[jj * HT_LDS + lane];
#pragma unroll
    for (int c = 0; c < K; ++c) acc[c] = cfma(a, sX[c * TILE + jj], acc[c]);
  }
#pragma unroll
  for (int c = 0; c < K; ++c) sPart[(w * K + c) * 32 + lane] = acc[c];
  __syncthreads();
  if (threadIdx.x < 32 * K) {
    const int r = threadIdx.x & 31, c = threadIdx.x >> 5;
    cplx v = sPart[c * 32 + r];
#pragma unroll
    for (int q = 1; q < 8; ++q) v = cadd(v, sPart[(q * K + c) * 32 + r]);
    sAcc[c * 32 + r] = op ? csub(sAcc[c * 32 + r], v) : v;
  }
  __syncthreads();
}

template <int K>
__global__ void __launch_bounds__(256, 2) k_trsm_half(int nb, int bw, const cplx* __restrict__ G,
                                                   const cplx* __restrict__ Dinv,
                                                   const cplx* __restrict__ B, cplx* __restrict__ X, cplx* U,
                                                   int64_t ldx, int adj, int* __restrict__ ticket, int* flags,
                                                   int* err, int sleep_cap) {
  extern __shared__ cplx sm[];
  cplx* sA = sm;                       // TILE·HT_LDS
  cplx* sX = sA + TILE * HT_LDS;       // TILE·K
  cplx* sAcc = sX + TILE * K;          // 32·K
  cplx* sPart = sAcc + 32 * K;         // 8·K·32
  __shared__ int sblk;
  // ticket[0]: the work counter; ticket[1]: the epoch of the previous solve.  This solve's flags
  // carry epoch = ticket[1] + 1; the CTA that takes the last exit ticket (every other CTA has
  // taken its own by then, after reading ticket[1]) stores the epoch and rearms the counter, so
  // a solve needs no host-side reset and replays unchanged from a captured graph.
  const int epoch = __ldcg(&ticket[1]) + 1;
  for (;;) {
    // every thread has read the previous ticket: the unit below passes at least one barrier
    if (threadIdx.x == 0) sblk = atomicAdd(ticket, 1);
    __syncthreads();
    const int unit = sblk;
    if (unit >= 2 * nb) {                              // uniform over the block
      if (threadIdx.x == 0 && unit == 2 * nb + (int)gridDim.x - 1) {
        if (epoch >= (1 << 30)) {   // wrap: flags back to 0, the next solve uses epoch 1
          for (int q = 0; q < 2 * nb; ++q) flags[q] = 0;
          ticket[1] = 0;
        } else {
          ticket[1] = epoch;
        }
        ticket[0] = 0;
      }
      break;
    }
    const int pos = unit >> 1, h = unit & 1;
    const int b = adj ? pos : (nb - 1 - pos);
    const int64_t r0 = (int64_t)b * TILE + h * 32;   // first row of this half
    cplx* out = adj ? U : X;                          // where the chain's values live
    // dependencies in the order they complete: J = b+1..min(nb−1, b+bw) from the far end
    // (forward), J = max(0, b−bw)..b−1 (adjoint)
    const int dlo = adj ? max(0, b - bw) : b + 1;
    const int dhi = adj ? b - 1 : min(nb - 1, b + bw);
    const int ndep = dhi - dlo + 1;
    HalfTile pf;
    auto dep_of = [&](int d) { return adj ? dlo + d : dhi - d; };
    auto tile_of = [&](int dep) {
      return adj ? G + tile_index_bw(dep, b, nb, bw) * (TILE * TILE) : G + tile_index_bw(b, dep, nb, bw) * (TILE * TILE);
    };
    if (ndep > 0) pf.load(tile_of(dep_of(0)), h, adj);
    // start value: D_b⁻¹ b_b (forward) or b_b (adjoint) on this half's rows
    if (!adj) {
      HalfTile dt;
      dt.load(Dinv + (int64_t)b * TILE * TILE, h, 0);
      for (int q = threadIdx.x; q < TILE * K; q += blockDim.x) {
        const int rr = q % TILE, c = q / TILE;
        sX[c * TILE + rr] = B[(int64_t)c * ldx + (int64_t)b * TILE + rr];
      }
      dt.store(sA, 0);
      __syncthreads();
      half_product<K>(sA, sX, sPart, sAcc, 0);
    } else {
      for (int q = threadIdx.x; q < 32 * K; q += blockDim.x) {
        const int rr = q % 32, c = q / 32;
        sAcc[c * 32 + rr] = B[(int64_t)c * ldx + r0 + rr];
      }
      __syncthreads();
    }
    for (int d = 0; d < ndep; ++d) {
      const int dep = dep_of(d);
      pf.store(sA, adj);
      if (d + 1 < ndep) pf.load(tile_of(dep_of(d + 1)), h, adj);   // in flight during the wait
      if ((threadIdx.x & 31) == 0 && threadIdx.x < 64) {             // threads 0 and 32: one half each
        const int* f = &flags[2 * dep + (threadIdx.x >> 5)];
        int spins = 0;
        unsigned ns = 32;   // back-off between polls after 64 spins: 32 ns doubling up to sleep_cap
        while (ld_acquire(f) != epoch) {
          if (++spins > RLS_SPIN_LIMIT) { atomicOr(err, DEVERR_SPIN_TIMEOUT); break; }
          if (spins > 64) {
            __nanosleep(ns);
            if (ns < (unsigned)sleep_cap) ns <<= 1;
          }
        }
      }
      __syncthreads();
      for (int q = threadIdx.x; q < TILE * K; q += blockDim.x) {
        const int rr = q % TILE, c = q / TILE;
        sX[c * TILE + rr] = __ldcg(&out[(int64_t)c * ldx + (int64_t)dep * TILE + rr]);
      }
      __syncthreads();
      half_product<K>(sA, sX, sPart, sAcc, 1);
    }
    for (int q = threadIdx.x; q < 32 * K; q += blockDim.x) {
      const int rr = q % 32, c = q / 32;
      out[(int64_t)c * ldx + r0 + rr] = sAcc[c * 32 + rr];
    }
    // bar.sync orders every thread's stores before thread 0's release (cumulative).
    __syncthreads();
    if (threadIdx.x == 0) st_release(&flags[2 * b + h], epoch);
  }
}

// X_b = D_b⁻ᴴ U_b on each half block row (grid 2·nb, 256 threads): the last step of the
// adjoint solve.
template <int K>
__global__ void __launch_bounds__(256) k_trsm_finish(const cplx* __restrict__ Dinv, const cplx* __restrict__ U,
                                                     cplx* __restrict__ X, int64_t ldx) {
  extern __shared__ cplx sm[];
  cplx* sA = sm;                       // TILE·HT_LDS
  cplx* sX = sA + TILE * HT_LDS;       // TILE·K
  cplx* sAcc = sX + TILE * K;          // 32·K
  cplx* sPart = sAcc + 32 * K;         // 8·K·32
  const int b = blockIdx.x >> 1, h = blockIdx.x & 1;
  HalfTile dt;
  dt.load(Dinv + (int64_t)b * TILE * TILE, h, 1);
  for (int q = threadIdx.x; q < TILE * K; q += blockDim.x) {
    const int rr = q % TILE, c = q / TILE;
    sX[c * TILE + rr] = U[(int64_t)c * ldx + (int64_t)b * TILE + rr];
  }
  dt.store(sA, 1);
  __syncthreads();
  half_product<K>(sA, sX, sPart, sAcc, 0);
  for (int q = threadIdx.x; q < 32 * K; q += blockDim.x) {
    const int rr = q % 32, c = q / 32;
    X[(int64_t)c * ldx + (int64_t)b * TILE + h * 32 + rr] = sAcc[c * 32 + rr];
  }
}

// Dynamic shared memory of k_trsm_half / k_trsm_finish for K columns.
inline size_t trsm_half_smem_bytes(int K) {
  return ((size_t)TILE * HT_LDS + (size_t)TILE * K + 32 * K + 8 * K * 32) * sizeof(cplx);
}

// Y[:, 0:k] = lam[j] * Y[:, j] - X[:, j]  (side 'L') or Y - X*lam (side 'S');
// also per-CTA partial |Y[:,0]|^2.
__global__ void k_residual_fix(int64_t nrows, cplx* Y, int64_t ldy, const cplx* X, int64_t ldx, int k,
                               const double* lam, int sideL, double* col0_part) {
  const int64_t row = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  double c0 = 0.0;
  if (row < nrows) {
    for (int j = 0; j < k; ++j) {
      const cplx y = Y[(int64_t)j * ldy + row], x = X[(int64_t)j * ldx + row];
      const cplx o = sideL ? csub(cscale(y, lam[j]), x) : csub(y, cscale(x, lam[j]));
      Y[(int64_t)j * ldy + row] = o;
      if (j == 0) c0 = cabs2(o);
    }
  }
  __shared__ double red[32];
  const double s = block_sum(c0, red);
  if (threadIdx.x == 0 && col0_part) col0_part[blockIdx.x] = s;
}

// Column-range copy for block shifts: dst[:, j] = src[:, j] for j < ncols.
__global__ void k_copy_cols(int64_t nrows, int ncols, const cplx* __restrict__ src, int64_t lds,
                            cplx* __restrict__ dst, int64_t ldd) {
  const int64_t row = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int c = blockIdx.y;
  if (row < nrows && c < ncols) dst[(int64_t)c * ldd + row] = src[(int64_t)c * lds + row];
}

// Sum of n doubles into out[0] (deterministic, one CTA).
__global__ void k_sum(const double* __restrict__ v, int n, double* out) {
  __shared__ double red[32];
  double s = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) s += v[i];
  s = block_sum(s, red);
  if (threadIdx.x == 0) out[0] = s;
}
