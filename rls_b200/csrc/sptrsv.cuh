// Sparse triangular solves for the incomplete-Cholesky preconditioner of psPrecRecy:
// SparseLLTP ldiv! (src/preconditioner/RLSPreconditioner.jl:79-116),
//   X = P · L⁻ᴴ · L⁻¹ · Pᴴ · B,  i.e. temp = B[p, :]; X = L \ temp; temp = Lᴴ \ X; X = temp[invp, :],
// with L sparse lower triangular (the IC factor, CSC, as LowerTriangular(L) sees it).
//
// Schedule: block rows of 32 consecutive rows, one CTA of eight warps per block row (lane =
// row), taken by ticket in dependency order (ascending for L, descending for Lᴴ), so a block
// row only waits on block rows whose CTAs started before it: every wait ends even when not all
// CTAs are resident, and a block row starts as soon as the block rows it reads are published
// (dataflow; the level-set parallelism of a level schedule without a barrier per level).  The
// plan lists, per block row, the block rows it reads in the order they finish, and per row
// where its terms from each of them end: the warps wait on each in turn (lane 0 of each warp
// polls the block row's flag, alone on its 128-byte line, with a capped exponential back-off),
// then stream strided shares of every row's terms from that block row four at a time with
// independent loads.  Warp 0 then solves the 32 × 32 diagonal block in 32 shuffle steps,
// multipliers in shared memory.  For the banded IC factors of psPrecRecy, whose row i almost
// always reads row i − 1, the critical path is n/32 block hand-offs, each carrying only the
// terms of the block row just finished.
//
// Flags carry an epoch (st.release / ld.acquire at gpu scope; the polling lane's acquire
// reaches the other lanes through __syncwarp); every wait is bounded by RLS_SPIN_LIMIT
// polls, after which the warp records DEVERR_SPIN_TIMEOUT and carries on, so a launch
// always terminates.
#pragma once
#include "common.cuh"

constexpr int SPT_ROWS = 32;          // rows per block row (one warp)
constexpr int SPT_FLAG_STRIDE = 32;   // ints between two block rows' flags (128 bytes)

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
  int64_t ndeps = 0;
  int64_t* depptr = nullptr;    // nblk + 1: block row b reads deps[depptr[b] .. depptr[b+1])
  int32_t* deps = nullptr;      // ndeps: those block rows, in the order they finish
  int64_t* segend = nullptr;    // ndeps·32: segend[k·32 + r] = end of row 32b+r's terms from deps[k]
};

__device__ __forceinline__ int spt_ld_acquire(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void spt_st_release(int* p, int v) {
  asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
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

// out[:, 0:K] = A⁻¹ · rhs[gather, 0:K]  (gather = nullptr: identity).  BACK: block rows and the
// in-block sweep run from the last row to the first (the operator is upper triangular).  out
// must not alias rhs; flags: one per block row, SPT_FLAG_STRIDE ints apart; any grid.
// A CTA of SPW_WARPS warps per block row: every warp takes a strided share
// (offset w, stride SPW_WARPS) of each row's terms from each dependency, waiting for that
// dependency's flag first, so a block row's terms from block rows finished long ago stream
// while the block row finished last is still being solved; after its flag only about
// (terms from it) / SPW_WARPS loads per lane remain on the critical path.  The warps' partial
// sums meet in shared memory in a fixed order (deterministic), and warp 0 does the in-block
// sweep and publishes the block row.
constexpr int SPW_WARPS = 8;

template <int K, bool BACK>
__global__ void __launch_bounds__(32 * SPW_WARPS) k_sptrsv_wide(TriBlocks A, const cplx* __restrict__ rhs, int64_t ldr,
                                                                const int64_t* __restrict__ gather, cplx* out,
                                                                int64_t ldo, int* ticket, int* flags, int epoch,
                                                                int* err) {
  __shared__ cplx sm_m[SPT_ROWS * SPT_ROWS];
  __shared__ cplx sm_acc[SPW_WARPS - 1][K][SPT_ROWS];   // warps 1.. (warp 0 keeps its own)
  __shared__ int s_t;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (;;) {
    if (threadIdx.x == 0) s_t = atomicAdd(ticket, 1);
    __syncthreads();
    const int t = s_t;
    if (t >= A.nblk) break;                               // uniform over the CTA
    const int64_t b = BACK ? (A.nblk - 1 - t) : t;
    const int64_t i = b * SPT_ROWS + lane;
    const bool live = i < A.n;
    const cplx* mb = A.blk + b * (SPT_ROWS * SPT_ROWS);
    for (int q = threadIdx.x; q < SPT_ROWS * SPT_ROWS; q += blockDim.x) sm_m[q] = mb[q];
    cplx acc[K];
#pragma unroll
    for (int c = 0; c < K; ++c) acc[c] = czero();
    int64_t e = live ? A.rowptr[i] : 0;
    const int64_t k1 = A.depptr[b + 1];
    for (int64_t k = A.depptr[b]; k < k1; ++k) {
      if (lane == 0) {
        const int* f = &flags[(int64_t)A.deps[k] * SPT_FLAG_STRIDE];
        int spins = 0;
        unsigned ns = 32;
        while (spt_ld_acquire(f) != epoch) {
          if (++spins > RLS_SPIN_LIMIT) { atomicOr(err, DEVERR_SPIN_TIMEOUT); break; }
          if (spins > 16) {
            __nanosleep(ns);
            if (ns < 256) ns <<= 1;
          }
        }
      }
      __syncwarp();
      const int64_t eend = live ? A.segend[k * SPT_ROWS + lane] : 0;
      int64_t q = e + w;
      for (; q + 3 * SPW_WARPS < eend; q += 4 * SPW_WARPS) {
        int64_t j[4];
        cplx v[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          j[u] = A.col[q + u * SPW_WARPS];
          v[u] = A.val[q + u * SPW_WARPS];
        }
        cplx xv[4][K];
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
          for (int c = 0; c < K; ++c) xv[u][c] = __ldcg(&out[(int64_t)c * ldo + j[u]]);
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
          for (int c = 0; c < K; ++c) acc[c] = cfma(v[u], xv[u][c], acc[c]);
      }
      for (; q < eend; q += SPW_WARPS) {
        const int64_t jj = A.col[q];
        const cplx vv = A.val[q];
#pragma unroll
        for (int c = 0; c < K; ++c) acc[c] = cfma(vv, __ldcg(&out[(int64_t)c * ldo + jj]), acc[c]);
      }
      e = eend;
    }
    if (w > 0) {
#pragma unroll
      for (int c = 0; c < K; ++c) sm_acc[w - 1][c][lane] = acc[c];
    }
    __syncthreads();
    if (w == 0) {
      cplx r[K], x[K];
      cplx d = czero();
#pragma unroll
      for (int c = 0; c < K; ++c) {
        cplx s = acc[c];
        for (int q = 0; q < SPW_WARPS - 1; ++q) s = cadd(s, sm_acc[q][c][lane]);
        acc[c] = s;
        r[c] = czero();
        x[c] = czero();
      }
      if (live) {
        d = A.dinv[i];
        const int64_t src = gather ? gather[i] : i;
#pragma unroll
        for (int c = 0; c < K; ++c) r[c] = rhs[(int64_t)c * ldr + src];
      }
#pragma unroll 4
      for (int qq = 0; qq < SPT_ROWS; ++qq) {
        const int s = BACK ? (SPT_ROWS - 1 - qq) : qq;
        const cplx ms = sm_m[s * SPT_ROWS + lane];
#pragma unroll
        for (int c = 0; c < K; ++c) {
          const cplx mine = cmul(csub(r[c], acc[c]), d);
          cplx xs;
          xs.x = __shfl_sync(0xffffffffu, mine.x, s);
          xs.y = __shfl_sync(0xffffffffu, mine.y, s);
          if (lane == s) x[c] = xs;
          acc[c] = cfma(ms, xs, acc[c]);
        }
      }
      if (live) {
#pragma unroll
        for (int c = 0; c < K; ++c) out[(int64_t)c * ldo + i] = x[c];
      }
      __threadfence();
      __syncwarp();
      if (lane == 0) spt_st_release(&flags[b * SPT_FLAG_STRIDE], epoch);
    }
    __syncthreads();
  }
}
