// Householder QR of a banded shifted matrix on the device: the R factor that sparse psTriRecy
// solves with at a refine point (get_R_factor!, src/core/psTriRecy.jl:222-234, which calls
// SPQR's qr(M − zS).R on the host).
//
// The matrix is A = B − zI with B = PᵀCP, where the symmetric permutation P keeps C's entries
// within lower bandwidth l and upper bandwidth u.  R does not depend on the row order of the
// matrix it factors (QR of ΠA is (ΠQ)R), so R of PᵀCP − zI = Pᵀ(CP − zP) is the R of the
// reference's M − zS with M = C[:, p], S = I[:, p], up to unit-modulus row phases that no
// singular value or right singular vector sees.
//
// Storage (LAPACK band layout with room for the fill): kd = l + u is R's upper bandwidth;
// column j keeps rows j−kd..j+l at AB[j·ldab + (i − j + kd)], ldab = kd + l + 1.  After the
// factorisation R occupies rows j−kd..j of column j (its diagonal real, LAPACK zlarfg's β) and
// the reflector tails rows j+1..j+l.
//
// Blocked right-looking QR with panels of w ≤ W columns (W = 16 where a 16-column panel fits
// in shared memory, else 8):
//   * k_bqr_panel<W>: one CTA of W warps, the panel (rows c0..c0+mp−1, mp ≤ w + l) in shared
//     memory, warp q owning column q.  Step s: warp s forms reflector s with zlarfg's
//     conventions (β = −sign(Re α)·‖x‖, τ = (β − α)/β, v = x/(α − β)), leaving v below the
//     diagonal of its column and β on it; after one barrier warps q > s apply H_sᴴ =
//     I − conj(τ)vvᴴ to their columns and warps q < s form v_qᴴv_s.  Column s is final after
//     step s, so one barrier per step suffices.  Then lane q of warp 0 builds row q of the
//     forward block-reflector factor T (zlarft: T[s][s] = τ_s, T[0:s, s] =
//     −τ_s·T[0:s, 0:s]·(V[:, 0:s]ᴴv_s)), so that H_0 H_1 … H_{w−1} = I − V T Vᴴ.
//   * k_bqr_update: the trailing columns c0+w .. min(n, c0+mp+u)−1 (every column with a
//     nonzero in the panel's rows) get C ← (I − V T Vᴴ)ᴴ C = C − V·Tᴴ·(VᴴC): eight columns per
//     CTA, a warp per column streaming its rows from L2 twice (VᴴC, then the update) with V
//     staged in shared memory.
//   Entries above a column's band (row < j − kd) are never filled: a reflector of the panel
//   reaches row c0+s only if its column has a nonzero at or below c0+s+l, i.e. j − u ≤ c0+s+l.
#pragma once
#include "common.cuh"
#include "sparse.cuh"
#include "blas.cuh"

#define BQR_WMAX 16                   // widest panel (one warp per column)
#define BQR_MAXL 1008                 // largest lower bandwidth: mp ≤ 1016 rows at W = 8
#define BQR_MAXROWS 1024              // row stride of the panel's reflector array
#define BQR_UCOLS 8                   // trailing columns per update CTA (a warp each)

// A ← 0, then the entries of B (CSR, rows of PᵀCP) in band layout, then A[j][j] −= z.
__global__ void k_band_scatter(int64_t n, int64_t kd, int64_t ldab, CsrDev B, cplx* __restrict__ AB) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  for (int64_t e = B.rowptr[i]; e < B.rowptr[i + 1]; ++e) {
    const int64_t j = B.col[e];
    AB[j * ldab + (i - j + kd)] = cadd(AB[j * ldab + (i - j + kd)], B.val[e]);   // duplicates sum
  }
}

// The shift comes from device memory, so a captured factorisation serves every z.
__global__ void k_band_shift(int64_t n, int64_t kd, int64_t ldab, const cplx* __restrict__ zp, cplx* __restrict__ AB) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const cplx z = *zp;
  if (j < n) AB[j * ldab + kd] = csub(AB[j * ldab + kd], z);
}

// Σ over the lane's rows of a·b (two accumulators, then the warp sum), rows lo + lane, step 32.
template <bool CONJ_A>
__device__ __forceinline__ cplx warp_dot(const cplx* __restrict__ a, const cplx* __restrict__ b, int lo, int hi,
                                         int lane) {
  cplx s0 = czero(), s1 = czero();
  int i = lo + lane;
  for (; i + 32 < hi; i += 64) {
    s0 = cfma(CONJ_A ? cconj(a[i]) : a[i], b[i], s0);
    s1 = cfma(CONJ_A ? cconj(a[i + 32]) : a[i + 32], b[i + 32], s1);
  }
  if (i < hi) s0 = cfma(CONJ_A ? cconj(a[i]) : a[i], b[i], s0);
  cplx d = cadd(s0, s1);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    d.x += __shfl_xor_sync(0xffffffffu, d.x, o);
    d.y += __shfl_xor_sync(0xffffffffu, d.y, o);
  }
  return d;
}

// Dynamic shared memory: w·mp cplx (column q at P + q·mp).  Tm: W × W, column-major, ld W.
// The reflector tails stay unscaled in P during the panel (v_s = (1, scl_s·x_s)); they are
// scaled on the way out.  No block-wide barrier per reflector: warp q applies reflectors
// 0..q−1 to its column as each is published (a flag in shared memory, set after a block fence),
// accumulating its tail norm while it applies the last one, then forms and publishes its own
// reflector.  The chain of owners is the critical path; the other warps catch up beside it.
// Every wait is bounded (RLS_SPIN_LIMIT, then DEVERR_SPIN_TIMEOUT); a warp only waits on
// reflectors of lower-numbered warps of the same block, which never wait on it.
template <int W>
__global__ void __launch_bounds__(32 * W) k_bqr_panel(int64_t l, int64_t kd, int64_t ldab, cplx* __restrict__ AB,
                                                      int64_t c0, int w, int mp, cplx* __restrict__ Vp,
                                                      cplx* __restrict__ Tm, int* err) {
  extern __shared__ cplx P[];
  __shared__ cplx taus[W], scl[W];
  __shared__ cplx Y[W][W + 1];   // Y[q][s] = v_qᴴ v_s (q < s)
  __shared__ int ready[W];
  const int lane = threadIdx.x & 31, q = threadIdx.x >> 5;
  auto valid = [&](int i, int qq) { return (int64_t)(i - qq) <= l && (int64_t)(qq - i) <= kd; };
  auto iend_of = [&](int s) { return (int)min((int64_t)mp, (int64_t)s + l + 1); };   // reflector s: rows s..iend−1
  if (threadIdx.x < W) ready[threadIdx.x] = 0;
  for (int e = threadIdx.x; e < w * mp; e += blockDim.x) {   // all copies in flight at once
    const int qq = e / mp, i = e % mp;
    if (valid(i, qq)) cp_async16(&P[e], &AB[(c0 + qq) * ldab + (i - qq + kd)]);
    else P[e] = czero();
  }
  cp_async_wait_all();
  __syncthreads();
  if (q < w) {
    cplx* Pq = P + (size_t)q * mp;
    double xn2 = 0.0;   // ‖tail‖² of this column when it is this warp's turn
    if (q == 0) {
      const int e0 = iend_of(0);
      double t0 = 0.0, t1 = 0.0;
      int i = 1 + lane;
      for (; i + 32 < e0; i += 64) { t0 += cabs2(Pq[i]); t1 += cabs2(Pq[i + 32]); }
      if (i < e0) t0 += cabs2(Pq[i]);
      xn2 = t0 + t1;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) xn2 += __shfl_xor_sync(0xffffffffu, xn2, o);
    }
    for (int s = 0; s < q; ++s) {
      // wait for reflector s (every lane observes the flag itself, then a block fence)
      int spins = 0;
      while (*(volatile int*)&ready[s] == 0) {
        if (++spins > RLS_SPIN_LIMIT) {
          if (lane == 0) atomicOr(err, DEVERR_SPIN_TIMEOUT);
          break;
        }
      }
      __threadfence_block();
      const cplx* Ps = P + (size_t)s * mp;
      const int iend = iend_of(s);
      // H_sᴴ on column q: a ← a − conj(τ)·v·(vᴴa), v = (1, sc·x)
      const cplx sc = scl[s];
      const cplx d = cadd(Pq[s], cmul(cconj(sc), warp_dot<true>(Ps, Pq, s + 1, iend, lane)));
      const cplx f = cmul(cconj(taus[s]), d);
      const cplx g = cmul(sc, f);
      __syncwarp();   // every lane has read a_s
      if (s == q - 1) {   // the last one before this warp's turn: update and sum the new tail
        const int e1 = iend_of(q);
        double t = 0.0;
        for (int i = s + 1 + lane; i < e1; i += 32) {
          cplx v = Pq[i];
          if (i < iend) {
            v = cfms(Ps[i], g, v);
            Pq[i] = v;
          }
          if (i > q) t += cabs2(v);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
        xn2 = t;
      } else {
        for (int i = s + 1 + lane; i < iend; i += 32) Pq[i] = cfms(Ps[i], g, Pq[i]);
      }
      if (lane == 0) Pq[s] = csub(Pq[s], f);
      __syncwarp();
    }
    // this warp's reflector (zlarfg: β = −sign(Re α)·‖(α, x)‖, τ = (β − α)/β, tail scale 1/(α − β))
    const cplx alpha = Pq[q];
    cplx tau = czero(), sc = czero();
    double beta = alpha.x;
    if (xn2 > 0.0 || alpha.y != 0.0) {
      const double nrm = sqrt(alpha.x * alpha.x + alpha.y * alpha.y + xn2);
      beta = (alpha.x >= 0.0) ? -nrm : nrm;
      const double ib = recip_nr(beta);                      // reciprocals refined by Newton–Raphson
      tau = cmk((beta - alpha.x) * ib, -alpha.y * ib);
      const double ar = alpha.x - beta, ai = alpha.y;        // sc = 1 / (α − β)
      const double id = recip_nr(ar * ar + ai * ai);
      sc = cmk(ar * id, -ai * id);
    }
    __syncwarp();   // every lane has read α
    if (lane == 0) {
      Pq[q] = cmk(beta, 0.0);
      taus[q] = tau;
      scl[q] = sc;
      if (!isfinite(beta)) atomicOr(err, DEVERR_NONFINITE);
      __threadfence_block();   // column q, τ and the scale before the flag
      *(volatile int*)&ready[q] = 1;
    }
  }
  __syncthreads();
  // Y[k][s] = v_kᴴ v_s = conj(scl_k)·(conj(x_k,s) + scl_s·Σ_{i>s} conj(x_k,i)·x_s,i), pairs k < s
  // spread over the warps
  const int npairs = w * (w - 1) / 2;
  for (int pidx = q; pidx < npairs; pidx += W) {
    int s = 1, k = pidx;
    while (k >= s) { k -= s; ++s; }   // pidx = s(s−1)/2 + k, 0 ≤ k < s
    const cplx* Pk = P + (size_t)k * mp;
    const cplx* Ps = P + (size_t)s * mp;
    const cplx y = warp_dot<true>(Pk, Ps, s + 1, iend_of(s), lane);
    if (lane == 0) Y[k][s] = cmul(cconj(scl[k]), cadd(cconj(Pk[s]), cmul(scl[s], y)));
  }
  __syncthreads();
  // write back: R rows ≤ q and the scaled reflector tails in place; V (unit diagonal, zero
  // above) for the trailing update
  for (int e = threadIdx.x; e < w * mp; e += blockDim.x) {
    const int qq = e / mp, i = e % mp;
    cplx v = P[e];
    if (i > qq) v = cmul(v, scl[qq]);
    if (valid(i, qq)) AB[(c0 + qq) * ldab + (i - qq + kd)] = v;
    Vp[(int64_t)qq * BQR_MAXROWS + i] = (i < qq) ? czero() : (i == qq ? cmk(1.0, 0.0) : v);
  }
  if (q == 0 && lane < W) {   // lane = row of T
    cplx trow[W];
#pragma unroll
    for (int s = 0; s < W; ++s) {
      cplx tv = czero();
      if (s < w) {
        if (lane == s) {
          tv = taus[s];
        } else if (lane < s) {
          cplx acc = czero();
#pragma unroll
          for (int k = 0; k < s; ++k)
            if (k >= lane) acc = cfma(trow[k], Y[k][s], acc);
          tv = cneg(cmul(taus[s], acc));
        }
      }
      trow[s] = tv;
      Tm[(int64_t)s * W + lane] = tv;
    }
  }
}

// Strided partial dot over rows lo + off, lo + off + step, ... < hi (two accumulators), then the
// warp sum.
template <bool CONJ_A>
__device__ __forceinline__ cplx strided_dot(const cplx* __restrict__ a, const cplx* __restrict__ b, int lo, int hi,
                                            int off, int step) {
  cplx s0 = czero(), s1 = czero();
  int i = lo + off;
  for (; i + step < hi; i += 2 * step) {
    s0 = cfma(CONJ_A ? cconj(a[i]) : a[i], b[i], s0);
    s1 = cfma(CONJ_A ? cconj(a[i + step]) : a[i + step], b[i + step], s1);
  }
  if (i < hi) s0 = cfma(CONJ_A ? cconj(a[i]) : a[i], b[i], s0);
  cplx d = cadd(s0, s1);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    d.x += __shfl_xor_sync(0xffffffffu, d.x, o);
    d.y += __shfl_xor_sync(0xffffffffu, d.y, o);
  }
  return d;
}

__device__ __forceinline__ void group_bar(int id, int nthreads) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

// The same panel with G warps per column (W·G = 32 warps, 1024 threads): the G warps of column
// q split its rows (warp g takes rows ≡ 32g + lane mod 32G), and their partial sums meet in
// shared memory behind a named barrier of the column's G warps (id 1 + q), summed in a fixed
// order.  Per reflector a column's chain is a quarter (G = 4) of the rows per lane; the flags
// and everything else are those of k_bqr_panel.
template <int W, int G>
__global__ void __launch_bounds__(32 * W * G) k_bqr_panel_g(int64_t l, int64_t kd, int64_t ldab,
                                                            cplx* __restrict__ AB, int64_t c0, int w, int mp,
                                                            cplx* __restrict__ Vp, cplx* __restrict__ Tm, int* err) {
  static_assert(W * G == 32 && W <= 15, "32 warps, at most 15 named column barriers");
  extern __shared__ cplx P[];
  __shared__ cplx taus[W], scl[W], alph[W];
  __shared__ cplx part[W][G];
  __shared__ double npart[W][G];
  __shared__ cplx Y[W][W + 1];
  __shared__ int ready[W];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int q = wid / G, g = wid % G;          // column, and this warp's share of its rows
  const int off = 32 * g + lane, step = 32 * G;
  auto valid = [&](int i, int qq) { return (int64_t)(i - qq) <= l && (int64_t)(qq - i) <= kd; };
  auto iend_of = [&](int s) { return (int)min((int64_t)mp, (int64_t)s + l + 1); };
  if (threadIdx.x < W) ready[threadIdx.x] = 0;
  for (int e = threadIdx.x; e < w * mp; e += blockDim.x) {
    const int qq = e / mp, i = e % mp;
    if (valid(i, qq)) cp_async16(&P[e], &AB[(c0 + qq) * ldab + (i - qq + kd)]);
    else P[e] = czero();
  }
  cp_async_wait_all();
  __syncthreads();
  if (q < w) {
    cplx* Pq = P + (size_t)q * mp;
    double xn2 = 0.0;
    if (q == 0) {   // tail norm and α of column 0
      const int e0 = iend_of(0);
      double t = 0.0;
      for (int i = 1 + off; i < e0; i += step) t += cabs2(Pq[i]);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
      if (lane == 0) npart[0][g] = t;
      if (g == 0 && lane == 0) alph[0] = Pq[0];
      group_bar(1 + q, 32 * G);
#pragma unroll
      for (int h = 0; h < G; ++h) xn2 += npart[0][h];
    }
    for (int s = 0; s < q; ++s) {
      int spins = 0;
      while (*(volatile int*)&ready[s] == 0) {
        if (++spins > RLS_SPIN_LIMIT) {
          if (lane == 0) atomicOr(err, DEVERR_SPIN_TIMEOUT);
          break;
        }
      }
      __threadfence_block();
      const cplx* Ps = P + (size_t)s * mp;
      const int iend = iend_of(s);
      const cplx dp = strided_dot<true>(Ps, Pq, s + 1, iend, off, step);
      if (lane == 0) part[q][g] = dp;
      const cplx as = Pq[s];   // read by every warp of the group before the barrier
      group_bar(1 + q, 32 * G);
      cplx dsum = czero();
#pragma unroll
      for (int h = 0; h < G; ++h) dsum = cadd(dsum, part[q][h]);
      const cplx sc = scl[s];
      const cplx f = cmul(cconj(taus[s]), cadd(as, cmul(cconj(sc), dsum)));
      const cplx gg = cmul(sc, f);
      if (s == q - 1) {   // the last one before this column's turn: update, sum the new tail, α
        const int e1 = iend_of(q);
        double t = 0.0;
        for (int i = s + 1 + off; i < e1; i += step) {
          cplx v = Pq[i];
          if (i < iend) {
            v = cfms(Ps[i], gg, v);
            Pq[i] = v;
          }
          if (i > q) t += cabs2(v);
          if (i == q) alph[q] = v;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
        if (lane == 0) npart[q][g] = t;
        if (g == 0 && lane == 0) Pq[s] = csub(as, f);
        group_bar(1 + q, 32 * G);
        xn2 = 0.0;
#pragma unroll
        for (int h = 0; h < G; ++h) xn2 += npart[q][h];
      } else {
        for (int i = s + 1 + off; i < iend; i += step) Pq[i] = cfms(Ps[i], gg, Pq[i]);
        if (g == 0 && lane == 0) Pq[s] = csub(as, f);
        // the next reflector's partial sums go to part[q][·] again: every warp of the group has
        // read this one's before any rewrites it
        group_bar(1 + q, 32 * G);
      }
    }
    // this column's reflector, formed redundantly by the G warps from the same sums
    const cplx alpha = alph[q];
    cplx tau = czero(), sc = czero();
    double beta = alpha.x;
    if (xn2 > 0.0 || alpha.y != 0.0) {
      const double nrm = sqrt(alpha.x * alpha.x + alpha.y * alpha.y + xn2);
      beta = (alpha.x >= 0.0) ? -nrm : nrm;
      const double ib = recip_nr(beta);                      // reciprocals refined by Newton–Raphson
      tau = cmk((beta - alpha.x) * ib, -alpha.y * ib);
      const double ar = alpha.x - beta, ai = alpha.y;        // sc = 1 / (α − β)
      const double id = recip_nr(ar * ar + ai * ai);
      sc = cmk(ar * id, -ai * id);
    }
    if (g == 0 && lane == 0) {
      Pq[q] = cmk(beta, 0.0);
      taus[q] = tau;
      scl[q] = sc;
      if (!isfinite(beta)) atomicOr(err, DEVERR_NONFINITE);
      __threadfence_block();
      *(volatile int*)&ready[q] = 1;
    }
  }
  __syncthreads();
  // Y[k][s] = v_kᴴ v_s, pairs k < s spread over the warps
  const int npairs = w * (w - 1) / 2;
  for (int pidx = wid; pidx < npairs; pidx += 32) {
    int s = 1, k = pidx;
    while (k >= s) { k -= s; ++s; }
    const cplx* Pk = P + (size_t)k * mp;
    const cplx* Ps = P + (size_t)s * mp;
    const cplx y = warp_dot<true>(Pk, Ps, s + 1, iend_of(s), lane);
    if (lane == 0) Y[k][s] = cmul(cconj(scl[k]), cadd(cconj(Pk[s]), cmul(scl[s], y)));
  }
  __syncthreads();
  for (int e = threadIdx.x; e < w * mp; e += blockDim.x) {
    const int qq = e / mp, i = e % mp;
    cplx v = P[e];
    if (i > qq) v = cmul(v, scl[qq]);
    if (valid(i, qq)) AB[(c0 + qq) * ldab + (i - qq + kd)] = v;
    Vp[(int64_t)qq * BQR_MAXROWS + i] = (i < qq) ? czero() : (i == qq ? cmk(1.0, 0.0) : v);
  }
  if (wid == 0 && lane < W) {
    cplx trow[W];
#pragma unroll
    for (int s = 0; s < W; ++s) {
      cplx tv = czero();
      if (s < w) {
        if (lane == s) {
          tv = taus[s];
        } else if (lane < s) {
          cplx acc = czero();
#pragma unroll
          for (int k = 0; k < s; ++k)
            if (k >= lane) acc = cfma(trow[k], Y[k][s], acc);
          tv = cneg(cmul(taus[s], acc));
        }
      }
      trow[s] = tv;
      Tm[(int64_t)s * W + lane] = tv;
    }
  }
}

inline size_t bqr_panel_smem(int w, int mp) { return (size_t)w * mp * sizeof(cplx); }

// C ← C − V·Tᴴ·(VᴴC) on the trailing columns jb .. je−1 (jb = c0 + w), rows c0 .. c0+mp−1.
// Grid: ⌈(je − jb)/8⌉ CTAs of 8 warps, warp c on column jb + 8·blockIdx.x + c; the column's rows
// (at most 32·RPL) are loaded into registers at once, used for VᴴC and updated in place.
// Dynamic shared memory: mp·(W+1) cplx of V (row i at Vs + i·(W+1): the odd row stride keeps a
// warp's lanes, which read one column at consecutive rows, on distinct banks).
template <int W, int RPL>
__global__ void __launch_bounds__(32 * BQR_UCOLS) k_bqr_update(int64_t l, int64_t kd, int64_t ldab,
                                                               cplx* __restrict__ AB, int64_t c0, int w, int mp,
                                                               int64_t je, const cplx* __restrict__ Vp,
                                                               const cplx* __restrict__ Tm) {
  extern __shared__ cplx Vs[];
  __shared__ cplx Ts[W * W];
  for (int e = threadIdx.x; e < mp * W; e += blockDim.x) {   // coalesced along the rows of V, all in flight
    const int a = e / mp, i = e % mp;
    if (a < w) cp_async16(&Vs[i * (W + 1) + a], &Vp[(int64_t)a * BQR_MAXROWS + i]);
    else Vs[i * (W + 1) + a] = czero();
  }
  for (int e = threadIdx.x; e < W * W; e += blockDim.x) cp_async16(&Ts[e], &Tm[e]);
  const int lane = threadIdx.x & 31, c = threadIdx.x >> 5;
  const int64_t jj = c0 + w + (int64_t)blockIdx.x * BQR_UCOLS + c;
  // rows of column jj inside its band: c0 + i ∈ [jj − kd, jj + l]
  const int ilo = (jj < je) ? (int)max((int64_t)0, jj - kd - c0) : 0;
  const int ihi = (jj < je) ? (int)min((int64_t)mp, jj + l + 1 - c0) : 0;
  cplx* col = AB + jj * ldab + (c0 - jj + kd);   // col[i] = A[c0 + i][jj]
  cplx x[RPL];
#pragma unroll
  for (int t = 0; t < RPL; ++t) {
    const int i = ilo + lane + 32 * t;
    x[t] = (i < ihi) ? col[i] : czero();
  }
  cp_async_wait_all();
  __syncthreads();
  if (jj >= je) return;
  cplx d[W];
#pragma unroll
  for (int a = 0; a < W; ++a) d[a] = czero();
#pragma unroll
  for (int t = 0; t < RPL; ++t) {
    const int i = ilo + lane + 32 * t;
    if (i < ihi) {
#pragma unroll
      for (int a = 0; a < W; ++a) d[a] = cfma(cconj(Vs[i * (W + 1) + a]), x[t], d[a]);
    }
  }
#pragma unroll
  for (int a = 0; a < W; ++a) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      d[a].x += __shfl_xor_sync(0xffffffffu, d[a].x, o);
      d[a].y += __shfl_xor_sync(0xffffffffu, d[a].y, o);
    }
  }
  // Wc = Tᴴ (VᴴC): Wc[a] = Σ_{k ≤ a} conj(T[k][a]) d[k]   (T column-major, ld W)
  cplx Wc[W];
#pragma unroll
  for (int a = 0; a < W; ++a) {
    cplx acc = czero();
#pragma unroll
    for (int k = 0; k <= a; ++k) acc = cfma(cconj(Ts[a * W + k]), d[k], acc);
    Wc[a] = acc;
  }
#pragma unroll
  for (int t = 0; t < RPL; ++t) {
    const int i = ilo + lane + 32 * t;
    if (i < ihi) {
      cplx v = x[t];
#pragma unroll
      for (int a = 0; a < W; ++a) v = cfms(Vs[i * (W + 1) + a], Wc[a], v);
      col[i] = v;
    }
  }
}

inline size_t bqr_update_smem(int W, int mp) { return (size_t)mp * (W + 1) * sizeof(cplx); }

// Band tiles of R for the dataflow solve: tile (I, J), J − I ≤ bw, at slot tile_index_bw.
// Grid: tile_slots(nb, bw) CTAs (unused slots return), 256 threads.
__global__ void __launch_bounds__(256) k_band_tiles(int nb, int bw, int64_t n, int64_t kd, int64_t ldab,
                                                    const cplx* __restrict__ AB, cplx* __restrict__ T) {
  const int64_t idx = blockIdx.x;
  int I, J;
  if (bw >= nb - 1) {   // packed triangle: idx = J(J+1)/2 + I
    J = (int)((sqrt(8.0 * (double)idx + 1.0) - 1.0) * 0.5);
    while ((int64_t)J * (J + 1) / 2 > idx) --J;
    while ((int64_t)(J + 1) * (J + 2) / 2 <= idx) ++J;
    I = (int)(idx - (int64_t)J * (J + 1) / 2);
  } else {
    J = (int)(idx / (bw + 1));
    I = J - (int)(idx % (bw + 1));
    if (I < 0) return;
  }
  cplx* tp = T + idx * (TILE * TILE);
  for (int e = threadIdx.x; e < TILE * TILE; e += blockDim.x) {
    const int rr = e % TILE, cc = e / TILE;
    const int64_t gi = (int64_t)I * TILE + rr, gj = (int64_t)J * TILE + cc;
    const bool in = gi < n && gj < n && gi <= gj && gj - gi <= kd;
    tp[e] = in ? AB[gj * ldab + (gi - gj + kd)] : czero();
  }
}
