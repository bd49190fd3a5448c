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

// ------------------------------------------------------------------------------------
// Gram: C (k1×k2) = alpha·AᴴB + beta·C.  Phase 1: grid (row chunks, ceil(k1/8)); warp w
// owns column (blockIdx.y*8+w) of A and sums over the chunk's rows; k2 <= K2MAX.
// ------------------------------------------------------------------------------------
template <int K2MAX>
__global__ void __launch_bounds__(256) k_gram_partial(int64_t nrows, int64_t chunk,
                                                      const cplx* __restrict__ A, int64_t lda, int k1,
                                                      const cplx* __restrict__ B, int64_t ldb, int k2,
                                                      cplx* __restrict__ part) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int col = blockIdx.y * 8 + w;
  const int64_t r0 = (int64_t)blockIdx.x * chunk;
  const int64_t r1 = min(nrows, r0 + chunk);
  cplx acc[K2MAX];
#pragma unroll
  for (int j = 0; j < K2MAX; ++j) acc[j] = czero();
  if (col < k1) {
    const cplx* a = A + (int64_t)col * lda;
    for (int64_t row = r0 + lane; row < r1; row += 32) {
      const cplx av = a[row];
#pragma unroll
      for (int j = 0; j < K2MAX; ++j)
        if (j < k2) acc[j] = cfmac(av, __ldg(&B[(int64_t)j * ldb + row]), acc[j]);
    }
  }
#pragma unroll
  for (int j = 0; j < K2MAX; ++j) {
    if (j < k2) {
      cplx s = warp_sum(acc[j]);
      if (lane == 0 && col < k1) part[((int64_t)blockIdx.x * k1 + col) * k2 + j] = s;
    }
  }
}

__global__ void k_gram_reduce(int nchunks, int k1, int k2, const cplx* __restrict__ part, cplx alpha,
                              cplx beta, cplx* C, int64_t ldc) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= k1 * k2) return;
  const int i = t / k2, j = t % k2;
  cplx s = czero();
  for (int c = 0; c < nchunks; ++c) s = cadd(s, part[((int64_t)c * k1 + i) * k2 + j]);
  cplx out = cmul(alpha, s);
  if (beta.x != 0.0 || beta.y != 0.0) out = cfma(beta, C[(int64_t)j * ldc + i], out);
  C[(int64_t)j * ldc + i] = out;
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
    const cplx v = tp[t];
    if (!adj) sT[cc * TILE_LDS + rr] = v;   // element (rr, cc) at column cc
    else sT[rr * TILE_LDS + cc] = v;        // element (rr, cc) at "column" rr
  }
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

// ------------------------------------------------------------------------------------
// Inverse of each shifted diagonal tile D_I = T_II − z·I (upper triangular), rows
// beyond n set to the identity.  One CTA (256 threads) per tile; right-looking
// back substitution on all 64 right-hand sides at once.
// ------------------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_diag_inv(int nb, int64_t n, const cplx* __restrict__ T, cplx z,
                                                  cplx* __restrict__ Dinv, int* err) {
  extern __shared__ cplx sm[];
  cplx* sU = sm;                    // TILE*TILE
  cplx* sY = sm + TILE * TILE;      // TILE*TILE
  const int I = blockIdx.x;
  const cplx* tp = T + tile_index(I, I) * (TILE * TILE);
  for (int t = threadIdx.x; t < TILE * TILE; t += blockDim.x) {
    const int rr = t % TILE, cc = t / TILE;
    const int64_t g = (int64_t)I * TILE + rr;
    cplx u = tp[t];
    if (rr == cc) u = (g < n) ? csub(u, z) : cmk(1.0, 0.0);
    sU[t] = (rr <= cc) ? u : czero();
    sY[t] = (rr == cc) ? cmk(1.0, 0.0) : czero();
  }
  __syncthreads();
  for (int i = TILE - 1; i >= 0; --i) {
    const cplx dinv = cinv(sU[i * TILE + i]);
    // row i of Y: columns c >= i
    for (int c = i + threadIdx.x; c < TILE; c += blockDim.x) sY[c * TILE + i] = cmul(sY[c * TILE + i], dinv);
    __syncthreads();
    // rows l < i: Y[l, c] -= U[l, i] * Y[i, c]  (c >= i)
    const int nl = i, ncol = TILE - i;
    for (int t = threadIdx.x; t < nl * ncol; t += blockDim.x) {
      const int l = t % nl, c = i + t / nl;
      sY[c * TILE + l] = cfms(sU[i * TILE + l], sY[c * TILE + i], sY[c * TILE + l]);
    }
    __syncthreads();
  }
  bool bad = false;
  for (int t = threadIdx.x; t < TILE * TILE; t += blockDim.x) {
    const cplx y = sY[t];
    if (!isfinite(y.x) || !isfinite(y.y)) bad = true;
    Dinv[(int64_t)I * TILE * TILE + t] = y;
  }
  if (bad) atomicOr(err, DEVERR_NONFINITE);
}

// E tiles for the last step of the dataflow solve, per shift:
//   adj = 0: E_b = D_b⁻¹ T(b, b+1)        (b < nb-1)
//   adj = 1: E_b = D_b⁻ᴴ T(b-1, b)ᴴ       (b > 0)
// so that X_b = D_b⁻¹ acc − E_b X_{b±1} needs one tile product after the last wait.
// grid (nb, 2); one CTA computes one 64×64×64 complex product from shared memory.
__global__ void __launch_bounds__(256) k_trsm_etiles(int nb, const cplx* __restrict__ T,
                                                     const cplx* __restrict__ Dinv, cplx* __restrict__ E) {
  extern __shared__ cplx sm[];
  cplx* sD = sm;                  // TILE*TILE (column-major)
  cplx* sT = sm + TILE * TILE;    // TILE*TILE
  const int b = blockIdx.x, adj = blockIdx.y;
  cplx* out = E + ((int64_t)adj * nb + b) * TILE * TILE;
  if ((!adj && b == nb - 1) || (adj && b == 0)) return;
  const cplx* dp = Dinv + (int64_t)b * TILE * TILE;
  const cplx* tp = adj ? T + tile_index(b - 1, b) * (TILE * TILE) : T + tile_index(b, b + 1) * (TILE * TILE);
  for (int q = threadIdx.x; q < TILE * TILE; q += blockDim.x) { sD[q] = dp[q]; sT[q] = tp[q]; }
  __syncthreads();
  // thread: row i = tid % 64, columns c = tid/64 + 4·m
  const int i = threadIdx.x & 63, c0 = threadIdx.x >> 6;
  for (int c = c0; c < TILE; c += 4) {
    cplx s = czero();
    if (!adj) {
      for (int l = 0; l < TILE; ++l) s = cfma(sD[l * TILE + i], sT[c * TILE + l], s);          // D⁻¹[i,l]·T[l,c]
    } else {
      for (int l = 0; l < TILE; ++l) s = cfma(cconj(sD[i * TILE + l]), cconj(sT[l * TILE + c]), s);  // D⁻ᴴ[i,l]·Tᴴ[l,c]
    }
    out[c * TILE + i] = s;
  }
}

// ------------------------------------------------------------------------------------
// Dataflow triangular solve with the shifted Schur factor R = T − zI.
//   adj = 0: R X = B   (back substitution, tiles of block row I, J > I)
//   adj = 1: Rᴴ X = B  (forward substitution, tiles of block column J, I < J)
// One CTA per tile row; CTAs take row blocks by ticket in dependency order, so a
// CTA only ever waits on blocks owned by CTAs that started before it.  Each wait
// is bounded by RLS_SPIN_LIMIT polls; on expiry the CTA records DEVERR_SPIN_TIMEOUT
// and finishes with whatever it has, so the launch always terminates.
// X may alias B.  k <= 24.
// ------------------------------------------------------------------------------------
__device__ __forceinline__ int ld_acquire(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(int* p, int v) {
  asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Shared memory: 2·TILE·TILE_LDS (tile, diagonal inverse) + (2 + NG)·TILE·k cplx.
// All dependencies but the last are subtracted from the right-hand side as they
// arrive; y = D_b⁻¹·acc is then formed before waiting for the last one, which enters
// through the precomputed E_b (k_trsm_etiles): X_b = y − E_b·X_last.  E_b is stored
// like a tile of T with adj = 0 semantics, so it is loaded untransposed.
template <int KMAX, int NG>
__global__ void __launch_bounds__(64 * NG) k_trsm_dataflow(int nb, const cplx* __restrict__ T,
                                                          const cplx* __restrict__ Dinv,
                                                          const cplx* __restrict__ E, const cplx* B,
                                                          cplx* X, int64_t ldx, int k, int adj,
                                                          int* __restrict__ ticket, int* flags, int epoch,
                                                          int* err) {
  extern __shared__ cplx sm[];
  cplx* sT = sm;                         // TILE*TILE_LDS
  cplx* sD = sT + TILE * TILE_LDS;       // TILE*TILE_LDS: this block's diagonal inverse
  cplx* sX = sD + TILE * TILE_LDS;       // TILE*k (dependency block)
  cplx* sAcc = sX + TILE * k;            // TILE*k (running right-hand side)
  cplx* sPart = sAcc + TILE * k;         // NG × TILE*k partial products
  __shared__ int sblk;
  if (threadIdx.x == 0) sblk = atomicAdd(ticket, 1);
  __syncthreads();
  const int t = sblk;
  const int b = adj ? t : (nb - 1 - t);
  const int row = threadIdx.x & (TILE - 1), grp = threadIdx.x >> 6;
  load_tile(sD, Dinv + (int64_t)b * TILE * TILE, adj);
  for (int q = threadIdx.x; q < TILE * k; q += blockDim.x) {
    const int rr = q % TILE, c = q / TILE;
    sAcc[c * TILE + rr] = B[(int64_t)c * ldx + (int64_t)b * TILE + rr];
  }
  auto wait_flag = [&](int dep) {
    if (threadIdx.x == 0) {
      int spins = 0;
      while (ld_acquire(&flags[dep]) != epoch) {
        if (++spins > RLS_SPIN_LIMIT) { atomicOr(err, DEVERR_SPIN_TIMEOUT); break; }
        if (spins > 64) __nanosleep(32);
      }
    }
    __syncthreads();
  };
  auto load_x = [&](int dep) {
    for (int q = threadIdx.x; q < TILE * k; q += blockDim.x) {
      const int rr = q % TILE, c = q / TILE;
      sX[c * TILE + rr] = __ldcg(&X[(int64_t)c * ldx + (int64_t)dep * TILE + rr]);
    }
    __syncthreads();
  };
  // sPart ← products of the tile in `tile` (op per `op_adj`) with `vec`
  auto product = [&](const cplx* tile, const cplx* vec, int op_adj) {
    cplx acc[KMAX];
#pragma unroll
    for (int c = 0; c < KMAX; ++c) acc[c] = czero();
    tile_apply<KMAX, NG>(tile, vec, k, op_adj, row, grp, acc);
#pragma unroll
    for (int c = 0; c < KMAX; ++c)
      if (c < k) sPart[(grp * k + c) * TILE + row] = acc[c];
    __syncthreads();
  };
  const int ndep = adj ? b : (nb - 1 - b);
  for (int d = 0; d + 1 < ndep; ++d) {
    const int dep = adj ? d : (nb - 1 - d);
    const cplx* tp = adj ? T + tile_index(dep, b) * (TILE * TILE) : T + tile_index(b, dep) * (TILE * TILE);
    __syncthreads();
    load_tile(sT, tp, adj);   // independent of X: issued before the wait
    wait_flag(dep);
    load_x(dep);
    product(sT, sX, adj);
    for (int q = threadIdx.x; q < TILE * k; q += blockDim.x) {
      const int rr = q % TILE, c = q / TILE;
      cplx v = sAcc[c * TILE + rr];
#pragma unroll
      for (int gq = 0; gq < NG; ++gq) v = csub(v, sPart[(gq * k + c) * TILE + rr]);
      sAcc[c * TILE + rr] = v;
    }
  }
  // y = D_b⁻¹ acc (adj: D_b⁻ᴴ acc), kept in sAcc
  __syncthreads();
  product(sD, sAcc, adj);
  for (int q = threadIdx.x; q < TILE * k; q += blockDim.x) {
    const int rr = q % TILE, c = q / TILE;
    cplx v = sPart[(0 * k + c) * TILE + rr];
#pragma unroll
    for (int gq = 1; gq < NG; ++gq) v = cadd(v, sPart[(gq * k + c) * TILE + rr]);
    sAcc[c * TILE + rr] = v;
  }
  if (ndep > 0) {
    const int dep = adj ? b - 1 : b + 1;
    load_tile(sT, E + ((int64_t)adj * nb + b) * TILE * TILE, 0);
    wait_flag(dep);
    load_x(dep);
    product(sT, sX, 0);
    for (int q = threadIdx.x; q < TILE * k; q += blockDim.x) {
      const int rr = q % TILE, c = q / TILE;
      cplx v = sAcc[c * TILE + rr];
#pragma unroll
      for (int gq = 0; gq < NG; ++gq) v = csub(v, sPart[(gq * k + c) * TILE + rr]);
      sAcc[c * TILE + rr] = v;
    }
  }
  __syncthreads();
  for (int q = threadIdx.x; q < TILE * k; q += blockDim.x) {
    const int rr = q % TILE, c = q / TILE;
    X[(int64_t)c * ldx + (int64_t)b * TILE + rr] = sAcc[c * TILE + rr];
  }
  // bar.sync orders every thread's stores before thread 0's release (cumulative).
  __syncthreads();
  if (threadIdx.x == 0) st_release(&flags[b], epoch);
}

inline size_t trsm_smem_bytes(int k, int ng) {
  return ((size_t)2 * TILE * TILE_LDS + (size_t)(2 + ng) * TILE * k) * sizeof(cplx);
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
