// Shifted sparse products: ShiftedMat mul! (src/types/RLSMatrices.jl:24-64).
//   forward:  Y = C X + s·X[1:n_, :]            (C m × n, X n × b, Y m × b)
//   adjoint:  Y = Cᴴ X + conj(s)·X[1:n_, :]     (X m × b, Y n × b),  n_ = min(m, n)
// C arrives in the reference's CSC layout and is kept on the device twice, as the CSR of C
// and the CSR of Cᴴ (conjugated values), so both products stream their matrix row by row.
// X is first copied row-major (k_rows_major), so a nonzero's B values of X are contiguous.
// A group of G threads (a power of two up to 4, from the mean row length) owns one output
// row: the group's lanes stride over the row's nonzeros and reduce with shuffles inside the
// group.  HBM bound: each nonzero (16-byte value + 4-byte column) is read once per B columns.
#pragma once
#include "common.cuh"

struct CsrDev {
  int64_t rows = 0, cols = 0, nnz = 0;
  int64_t* rowptr = nullptr;   // rows + 1
  int32_t* col = nullptr;      // nnz
  cplx* val = nullptr;         // nnz
  int group = 1;               // threads per row
};

// X (n × B, column-major, ld ldx) → Xr (row-major: row r at Xr + r·B), so that the B values a
// nonzero multiplies sit in one or two cache lines.
template <int B>
__global__ void __launch_bounds__(256) k_rows_major(int64_t n, const cplx* __restrict__ X, int64_t ldx,
                                                    cplx* __restrict__ Xr) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
#pragma unroll
  for (int c = 0; c < B; ++c) Xr[r * B + c] = X[(int64_t)c * ldx + r];
}

// Y (column-major, ld ldy) = A·X + s·X on the first nshift rows, X given row-major (Xr) for the
// product and column-major (X, ld ldx) for the shift term.  A group of G threads per row.
template <int B>
__global__ void __launch_bounds__(256) k_spmm_shifted(CsrDev A, cplx s, int64_t nshift, const cplx* __restrict__ Xr,
                                                      const cplx* __restrict__ X, int64_t ldx, cplx* __restrict__ Y,
                                                      int64_t ldy) {
  const int G = A.group;
  const int64_t row = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / G;
  const int sub = threadIdx.x & (G - 1);
  cplx acc[B];
#pragma unroll
  for (int c = 0; c < B; ++c) acc[c] = czero();
  if (row < A.rows) {
    const int64_t j1 = A.rowptr[row + 1];
    int64_t j = A.rowptr[row] + sub;
    for (; j + 3 * G < j1; j += 4 * G) {   // four nonzeros in flight per thread
      int64_t cj[4];
      cplx aj[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        cj[u] = A.col[j + u * G];
        aj[u] = A.val[j + u * G];
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const cplx* xr = Xr + cj[u] * B;
#pragma unroll
        for (int c = 0; c < B; ++c) acc[c] = cfma(aj[u], __ldg(&xr[c]), acc[c]);
      }
    }
    for (; j < j1; j += G) {
      const cplx a = A.val[j];
      const cplx* xr = Xr + (int64_t)A.col[j] * B;
#pragma unroll
      for (int c = 0; c < B; ++c) acc[c] = cfma(a, __ldg(&xr[c]), acc[c]);
    }
  }
  for (int o = G >> 1; o > 0; o >>= 1) {
#pragma unroll
    for (int c = 0; c < B; ++c) {
      acc[c].x += __shfl_xor_sync(0xffffffffu, acc[c].x, o);
      acc[c].y += __shfl_xor_sync(0xffffffffu, acc[c].y, o);
    }
  }
  if (sub == 0 && row < A.rows) {
#pragma unroll
    for (int c = 0; c < B; ++c) {
      cplx y = acc[c];
      if (row < nshift) y = cfma(s, X[(int64_t)c * ldx + row], y);
      Y[(int64_t)c * ldy + row] = y;
    }
  }
}
