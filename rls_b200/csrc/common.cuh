// Shared device helpers for the σ_min(C − zI) engine: complex FP64 arithmetic on
// double2, warp/block reductions, status codes and launch checks.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>

#ifndef RLS_HD
#define RLS_HD __host__ __device__ __forceinline__
#endif

typedef double2 cplx;  // (re, im), 16 bytes, layout-compatible with rls_c64

RLS_HD cplx cmk(double re, double im) { return make_double2(re, im); }
RLS_HD cplx czero() { return make_double2(0.0, 0.0); }
RLS_HD cplx cadd(cplx a, cplx b) { return make_double2(a.x + b.x, a.y + b.y); }
RLS_HD cplx csub(cplx a, cplx b) { return make_double2(a.x - b.x, a.y - b.y); }
RLS_HD cplx cneg(cplx a) { return make_double2(-a.x, -a.y); }
RLS_HD cplx cconj(cplx a) { return make_double2(a.x, -a.y); }
RLS_HD cplx cscale(cplx a, double s) { return make_double2(a.x * s, a.y * s); }
RLS_HD cplx cmul(cplx a, cplx b) { return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
// conj(a) * b
RLS_HD cplx cmulc(cplx a, cplx b) { return make_double2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x); }
RLS_HD double cabs2(cplx a) { return a.x * a.x + a.y * a.y; }
// c + a*b
RLS_HD cplx cfma(cplx a, cplx b, cplx c) {
  c.x = fma(a.x, b.x, c.x); c.x = fma(-a.y, b.y, c.x);
  c.y = fma(a.x, b.y, c.y); c.y = fma(a.y, b.x, c.y);
  return c;
}
// c + conj(a)*b
RLS_HD cplx cfmac(cplx a, cplx b, cplx c) {
  c.x = fma(a.x, b.x, c.x); c.x = fma(a.y, b.y, c.x);
  c.y = fma(a.x, b.y, c.y); c.y = fma(-a.y, b.x, c.y);
  return c;
}
// c - a*b
RLS_HD cplx cfms(cplx a, cplx b, cplx c) {
  c.x = fma(-a.x, b.x, c.x); c.x = fma(a.y, b.y, c.x);
  c.y = fma(-a.x, b.y, c.y); c.y = fma(-a.y, b.x, c.y);
  return c;
}
RLS_HD cplx cdiv(cplx a, cplx b) {
  // Smith's algorithm (Smith 1962) for a/b.
  if (fabs(b.x) >= fabs(b.y)) {
    double t = b.y / b.x, d = b.x + b.y * t;
    return make_double2((a.x + a.y * t) / d, (a.y - a.x * t) / d);
  } else {
    double t = b.x / b.y, d = b.x * t + b.y;
    return make_double2((a.x * t + a.y) / d, (a.y * t - a.x) / d);
  }
}
RLS_HD cplx cinv(cplx b) { return cdiv(make_double2(1.0, 0.0), b); }

// 1/q by the hardware reciprocal estimate refined with two Newton–Raphson steps
// (r ← r + r(1 − q r)); the relative error is far below what a Sturm count needs.
__device__ __forceinline__ double recip_nr(double q) {
  double r;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(q));
  double e = fma(-q, r, 1.0);
  r = fma(r, e, r);
  e = fma(-q, r, 1.0);
  return fma(r, e, r);
}

// 16-byte global→shared copies issued without waiting (cp.async, L2 only); a thread's
// copies are complete after cp_async_wait_all(), visible to the block after a barrier.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ cplx warp_sum(cplx v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
    v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
  }
  return v;
}

// Block-wide sum; `red` must hold blockDim.x/32 doubles.  All threads get the result.
__device__ __forceinline__ double block_sum(double v, double* red) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) red[w] = v;
  __syncthreads();
  double s = 0.0;
  for (int i = 0; i < nw; ++i) s += red[i];
  return s;
}
__device__ __forceinline__ cplx block_sum(cplx v, cplx* red) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) red[w] = v;
  __syncthreads();
  cplx s = czero();
  for (int i = 0; i < nw; ++i) s = cadd(s, red[i]);
  return s;
}

// Status codes shared with include/rls_b200.h.
enum {
  RLS_OK_ = 0,
  RLS_ERR_ARG_ = -1,
  RLS_ERR_DIM_ = -2,
  RLS_ERR_CUDA_ = -3,
  RLS_ERR_NOMEM_ = -4,
  RLS_ERR_TIMEOUT_ = -5,
  RLS_ERR_BREAKDOWN_ = -6,
  RLS_ERR_STATE_ = -7,
};

// Device-side error word bits (set by kernels, read by the host after a step).
enum {
  DEVERR_SPIN_TIMEOUT = 1,
  DEVERR_NONFINITE = 2,
  DEVERR_SIZE = 4,
  DEVERR_BREAKDOWN = 8,
  DEVERR_POSDEF = 16,     // a Cholesky factorisation without a shift rule met a non-positive pivot
};

// Spin limit for dataflow waits: far above any legitimate wait (a wait of this
// length means a producer never ran), small enough to return in well under a second.
#ifndef RLS_SPIN_LIMIT
#define RLS_SPIN_LIMIT (1 << 22)
#endif
