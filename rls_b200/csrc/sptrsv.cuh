// Sparse triangular solves for the incomplete-Cholesky preconditioner of psPrecRecy:
// SparseLLTP ldiv! (src/preconditioner/RLSPreconditioner.jl:79-116),
//   X = P · L⁻ᴴ · L⁻¹ · Pᴴ · B,  i.e. temp = B[p, :]; X = L \ temp; temp = Lᴴ \ X; X = temp[invp, :],
// with L sparse lower triangular (the IC factor, CSC, as LowerTriangular(L) sees it).
//
// Schedule: block rows of 32 consecutive rows, one warp per block row and one lane per row,
// taken by ticket in dependency order (ascending for L, descending for Lᴴ), so a block row
// only waits on block rows whose warps started before it: every wait ends even when not
// all warps are resident, and a block row starts as soon as the block rows it reads are
// published (dataflow; the level-set parallelism of a level schedule without a barrier
// per level).  A lane first sums its row's off-block terms, waiting on each producing
// block row's flag (entries ordered so the nearest block rows come last), then the warp
// solves the 32 × 32 diagonal block in 32 shuffle steps with the multipliers in registers.
// For the banded IC factors of psPrecRecy, whose row i almost always reads row i − 1, the
// critical path is n/32 block hand-offs instead of n row hand-offs.
//
// Flags carry an epoch (st.release / ld.acquire at gpu scope); every wait is bounded by
// RLS_SPIN_LIMIT polls, after which the lane records DEVERR_SPIN_TIMEOUT and carries on,
// so a launch always terminates.
#pragma once
#include "common.cuh"

constexpr int SPT_ROWS = 32;   // rows per block row (one warp)

// One triangular operator in block-row form (rows of L, or rows of Lᴴ).
struct TriBlocks {
  int64_t n = 0;
  int64_t nblk = 0;             // ceil(n / 32)
  int64_t nnz_off = 0;
  int64_t* rowptr = nullptr;    // n + 1: off-block entries of row i
  int32_t* col = nullptr;       // nnz_off: the solution row each entry reads
  cplx* val = nullptr;          // nnz_off: its coefficient
  cplx* blk = nullptr;          // nblk·32·32: blk[(b·32 + s)·32 + r] = coefficient of x[32b+s] in row 32b+r
  cplx* dinv = nullptr;         // n: 1 / diagonal
};

__device__ __forceinline__ int spt_ld_acquire(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void spt_st_release(int* p, int v) {
  asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// out[:, 0:K] = A⁻¹ · rhs[gather, 0:K]  (gather = nullptr: identity).  BACK: block rows and the
// in-block sweep run from the last row to the first (the operator is upper triangular).
// 128 threads per CTA (4 warps), any grid.  out must not alias rhs.
template <int K, bool BACK>
__global__ void __launch_bounds__(128) k_sptrsv_blocks(TriBlocks A, const cplx* __restrict__ rhs, int64_t ldr,
                                                       const int64_t* __restrict__ gather, cplx* out, int64_t ldo,
                                                       int* ticket, int* flags, int epoch, int* err) {
  const int lane = threadIdx.x & 31;
  for (;;) {
    int t = 0;
    if (lane == 0) t = atomicAdd(ticket, 1);
    t = __shfl_sync(0xffffffffu, t, 0);
    if (t >= A.nblk) break;                           // uniform over the warp
    const int64_t b = BACK ? (A.nblk - 1 - t) : t;
    const int64_t i = b * SPT_ROWS + lane;
    const bool live = i < A.n;
    // this row's in-block multipliers, in flight while the off-block terms are gathered
    cplx m[SPT_ROWS];
    const cplx* mb = A.blk + b * (SPT_ROWS * SPT_ROWS);
#pragma unroll
    for (int s = 0; s < SPT_ROWS; ++s) m[s] = mb[s * SPT_ROWS + lane];
    cplx acc[K], r[K];
    cplx d = czero();
#pragma unroll
    for (int c = 0; c < K; ++c) { acc[c] = czero(); r[c] = czero(); }
    if (live) {
      d = A.dinv[i];
      const int64_t src = gather ? gather[i] : i;
#pragma unroll
      for (int c = 0; c < K; ++c) r[c] = rhs[(int64_t)c * ldr + src];
      const int64_t e1 = A.rowptr[i + 1];
      int64_t waited = -1;
      for (int64_t e = A.rowptr[i]; e < e1; ++e) {
        const int64_t j = A.col[e];
        const cplx v = A.val[e];
        const int64_t jb = j / SPT_ROWS;
        if (jb != waited) {
          int spins = 0;
          while (spt_ld_acquire(&flags[jb]) != epoch) {
            if (++spins > RLS_SPIN_LIMIT) { atomicOr(err, DEVERR_SPIN_TIMEOUT); break; }
            if (spins > 64) __nanosleep(64);
          }
          waited = jb;
        }
#pragma unroll
        for (int c = 0; c < K; ++c) acc[c] = cfma(v, __ldcg(&out[(int64_t)c * ldo + j]), acc[c]);
      }
    }
    // in-block sweep: at step s, lane s's row is final; every row subtracts its multiple of it
    cplx x[K];
#pragma unroll
    for (int c = 0; c < K; ++c) x[c] = czero();
#pragma unroll
    for (int q = 0; q < SPT_ROWS; ++q) {
      const int s = BACK ? (SPT_ROWS - 1 - q) : q;
#pragma unroll
      for (int c = 0; c < K; ++c) {
        const cplx mine = cmul(csub(r[c], acc[c]), d);
        cplx xs;
        xs.x = __shfl_sync(0xffffffffu, mine.x, s);
        xs.y = __shfl_sync(0xffffffffu, mine.y, s);
        if (lane == s) x[c] = xs;
        acc[c] = cfma(m[s], xs, acc[c]);
      }
    }
    if (live) {
#pragma unroll
      for (int c = 0; c < K; ++c) out[(int64_t)c * ldo + i] = x[c];
    }
    __threadfence();
    __syncwarp();
    if (lane == 0) spt_st_release(&flags[b], epoch);
  }
}

// X[i, 0:K] = W[src[i], 0:K] (W column-major with ld n): the final X = temp[invp, :].
template <int K>
__global__ void __launch_bounds__(256) k_gather_rows(int64_t n, const int64_t* __restrict__ src,
                                                     const cplx* __restrict__ W, int64_t ldw, cplx* X,
                                                     int64_t ldx) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t s = src[i];
#pragma unroll
  for (int c = 0; c < K; ++c) X[(int64_t)c * ldx + i] = W[(int64_t)c * ldw + s];
}
