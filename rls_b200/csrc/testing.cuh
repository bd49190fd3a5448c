// Kernel-level entry points for parity tests (declared in include/rls_b200_testing.h).
// Each copies host inputs to the device, runs one device routine of the engine on the
// context's stream and copies the result back.  Included at the end of engine.cu so
// the kernels stay in one translation unit.
#pragma once

namespace {

struct DevTmp {
  rls_ctx* ctx;
  std::vector<void*> ptrs;
  explicit DevTmp(rls_ctx* c) : ctx(c) {}
  ~DevTmp() {
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    for (void* p : ptrs) cudaFree(p);
  }
  template <class T>
  T* alloc(size_t count) {
    void* p = nullptr;
    if (cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T)) != cudaSuccess) return nullptr;
    cudaMemsetAsync(p, 0, std::max<size_t>(count, 1) * sizeof(T), ctx->stream);
    ptrs.push_back(p);
    return static_cast<T*>(p);
  }
};

int need_space(rls_ctx* ctx) {
  if (!ctx) return RLS_ERR_ARG;
  if (!ctx->T || !ctx->V) {
    set_err(ctx, "test entry point needs rls_set_schur and rls_test_setup first");
    return RLS_ERR_STATE;
  }
  return RLS_OK;
}

}  // namespace

extern "C" int rls_test_lltp_plan_dense(int64_t n, const int64_t* colptr, const int64_t* rowval,
                                        const rls_c64* nzval, int base, int op, rls_c64* dense,
                                        int64_t* singular_at, int* levels) {
  std::string why;
  int st = lltp_check_csc(n, colptr, rowval, nzval, base, why);
  if (st != RLS_OK) {
    g_create_err = "rls_test_lltp_plan_dense: " + why;
    return st;
  }
  if ((op != 0 && op != 1) || (dense && n > 4096)) {
    g_create_err = "rls_test_lltp_plan_dense: invalid arguments";
    return RLS_ERR_ARG;
  }
  TriHost h[2];
  const int64_t sing = lltp_plan(n, colptr, rowval, nzval, base, h);
  const TriHost& o = h[op];
  auto fail = [&](const std::string& what) {
    g_create_err = "rls_test_lltp_plan_dense: plan invariant broken: " + what;
    return RLS_ERR_STATE;
  };
  const int64_t nblk = (n + SPT_ROWS - 1) / SPT_ROWS;
  if (o.nblk != nblk || (int64_t)o.rowptr.size() != n + 1 || o.rowptr[0] != 0 ||
      o.rowptr[(size_t)n] != (int64_t)o.col.size() || o.col.size() != o.val.size() ||
      (int64_t)o.blk.size() != nblk * SPT_ROWS * SPT_ROWS || (int64_t)o.dinv.size() != n)
    return fail("sizes");
  for (int64_t i = 0; i < n; ++i) {
    if (o.rowptr[(size_t)i + 1] < o.rowptr[(size_t)i]) return fail("row pointers");
    for (int64_t e = o.rowptr[(size_t)i]; e < o.rowptr[(size_t)i + 1]; ++e) {
      const int64_t j = o.col[(size_t)e];
      if (j < 0 || j >= n) return fail("column range");
      if (op == 0 ? (j / SPT_ROWS >= i / SPT_ROWS) : (j / SPT_ROWS <= i / SPT_ROWS)) return fail("block order");
      if (e > o.rowptr[(size_t)i] && (op == 0 ? j < o.col[(size_t)e - 1] : j > o.col[(size_t)e - 1]))
        return fail("entry order");
    }
  }
  for (int64_t b = 0; b < nblk; ++b)
    for (int s = 0; s < SPT_ROWS; ++s)
      for (int r = 0; r < SPT_ROWS; ++r) {
        const cplx v = o.blk[(size_t)((b * SPT_ROWS + s) * SPT_ROWS + r)];
        if (v.x == 0.0 && v.y == 0.0) continue;
        if (b * SPT_ROWS + r >= n || b * SPT_ROWS + s >= n || (op == 0 ? s >= r : s <= r)) return fail("block terms");
      }
  // dependency lists and segments: every row's terms are covered, segment by segment, and
  // each segment holds exactly the terms from its block row
  if ((int64_t)o.depptr.size() != nblk + 1 || o.depptr[0] != 0 || o.depptr[(size_t)nblk] != (int64_t)o.deps.size() ||
      o.segend.size() != o.deps.size() * SPT_ROWS)
    return fail("dependency list sizes");
  for (int64_t b = 0; b < nblk; ++b) {
    const int64_t k0 = o.depptr[(size_t)b], k1 = o.depptr[(size_t)b + 1];
    if (k1 < k0) return fail("dependency pointers");
    for (int64_t k = k0; k < k1; ++k) {
      const int64_t d = o.deps[(size_t)k];
      if (d < 0 || d >= nblk || (op == 0 ? d >= b : d <= b)) return fail("dependency block order");
      if (k > k0 && (op == 0 ? d <= o.deps[(size_t)k - 1] : d >= o.deps[(size_t)k - 1])) return fail("dependency order");
    }
    for (int r = 0; r < SPT_ROWS; ++r) {
      const int64_t i = b * SPT_ROWS + r;
      int64_t e = i < n ? o.rowptr[(size_t)i] : 0;
      for (int64_t k = k0; k < k1; ++k) {
        const int64_t z = o.segend[(size_t)(k * SPT_ROWS + r)];
        if (i >= n) {
          if (z != 0) return fail("segments of padding rows");
          continue;
        }
        if (z < e || z > o.rowptr[(size_t)i + 1]) return fail("segment ends");
        for (; e < z; ++e)
          if (o.col[(size_t)e] / SPT_ROWS != o.deps[(size_t)k]) return fail("segment contents");
      }
      if (i < n && e != o.rowptr[(size_t)i + 1]) return fail("uncovered terms");
    }
  }
  if (singular_at) *singular_at = sing;
  if (levels) *levels = o.levels;
  if (!dense) return RLS_OK;
  for (int64_t q = 0; q < n * n; ++q) dense[q] = rls_c64{0.0, 0.0};
  auto add = [&](int64_t row, int64_t x, cplx v) {
    dense[x * n + row].re += v.x;
    dense[x * n + row].im += v.y;
  };
  for (int64_t i = 0; i < n; ++i) {
    const cplx d = o.dinv[(size_t)i];
    if (d.x != 0.0 || d.y != 0.0) add(i, i, cinv(d));
    for (int64_t e = o.rowptr[(size_t)i]; e < o.rowptr[(size_t)i + 1]; ++e) add(i, o.col[(size_t)e], o.val[(size_t)e]);
  }
  for (int64_t b = 0; b < nblk; ++b)
    for (int s = 0; s < SPT_ROWS; ++s)
      for (int r = 0; r < SPT_ROWS; ++r) {
        const cplx v = o.blk[(size_t)((b * SPT_ROWS + s) * SPT_ROWS + r)];
        if (v.x != 0.0 || v.y != 0.0) add(b * SPT_ROWS + r, b * SPT_ROWS + s, v);
      }
  if (singular_at) *singular_at = sing;
  if (levels) *levels = o.levels;
  return RLS_OK;
}

extern "C" int rls_test_setup(rls_ctx* ctx, int r, int p_max) {
  if (!ctx || !ctx->T) return RLS_ERR_STATE;
  if (r < 1 || r > 8 || p_max < 1) return RLS_ERR_ARG;
  return setup_space(ctx, r, p_max);
}

extern "C" int rls_test_trsm(rls_ctx* ctx, rls_c64 z, int adj, int k, const rls_c64* B, rls_c64* X) {
  RET(need_space(ctx));
  if (k < 1 || k > 64 || !B || !X) return RLS_ERR_ARG;
  DevTmp t(ctx);
  const int64_t np = ctx->n_pad, n = ctx->n;
  cplx* d = t.alloc<cplx>((size_t)np * k);
  cplx* dx = t.alloc<cplx>((size_t)np * k);
  if (!d || !dx) return RLS_ERR_NOMEM;
  CK(cudaMemcpy2DAsync(d, np * sizeof(cplx), B, n * sizeof(cplx), n * sizeof(cplx), k, cudaMemcpyHostToDevice,
                       ctx->stream));
  RET(trsm(ctx, cmk(z.re, z.im), adj, d, dx, np, k));
  CK(cudaMemcpy2DAsync(X, n * sizeof(cplx), dx, np * sizeof(cplx), n * sizeof(cplx), k, cudaMemcpyDeviceToHost,
                       ctx->stream));
  return sync_and_check(ctx);
}

extern "C" int rls_test_trmm(rls_ctx* ctx, int adj, int k, const rls_c64* X, rls_c64* Y) {
  RET(need_space(ctx));
  if (k < 1 || k > 16 || !X || !Y) return RLS_ERR_ARG;
  DevTmp t(ctx);
  const int64_t np = ctx->n_pad, n = ctx->n;
  cplx* dx = t.alloc<cplx>((size_t)np * k);
  cplx* dy = t.alloc<cplx>((size_t)np * k);
  if (!dx || !dy) return RLS_ERR_NOMEM;
  CK(cudaMemcpy2DAsync(dx, np * sizeof(cplx), X, n * sizeof(cplx), n * sizeof(cplx), k, cudaMemcpyHostToDevice,
                       ctx->stream));
  RET(trmm(ctx, adj, dx, dy, np, k));
  CK(cudaMemcpy2DAsync(Y, n * sizeof(cplx), dy, np * sizeof(cplx), n * sizeof(cplx), k, cudaMemcpyDeviceToHost,
                       ctx->stream));
  return sync_and_check(ctx);
}

// R (k×k) of the QR of A (m×k, m <= n_pad), and optionally Q (m×k) by orth_qr.
extern "C" int rls_test_qr(rls_ctx* ctx, int64_t m, int k, const rls_c64* A, rls_c64* R, rls_c64* Q) {
  RET(need_space(ctx));
  if (m < k || m > ctx->n_pad || k < 1 || k > ctx->small_dim || !A || !R) return RLS_ERR_ARG;
  DevTmp t(ctx);
  const int64_t np = ctx->n_pad;
  cplx* d = t.alloc<cplx>((size_t)np * k);
  cplx* dR = t.alloc<cplx>((size_t)k * k);
  if (!d || !dR) return RLS_ERR_NOMEM;
  CK(cudaMemcpy2DAsync(d, np * sizeof(cplx), A, m * sizeof(cplx), m * sizeof(cplx), k, cudaMemcpyHostToDevice,
                       ctx->stream));
  if (Q) {
    if (k > 64) return RLS_ERR_ARG;
    RET(orth_qr(ctx, np, d, np, k, dR));
    CK(cudaMemcpy2DAsync(Q, m * sizeof(cplx), d, np * sizeof(cplx), m * sizeof(cplx), k, cudaMemcpyDeviceToHost,
                         ctx->stream));
  } else {
    RET(tsqr_r(ctx, np, d, np, k, dR));
  }
  CK(cudaMemcpyAsync(R, dR, sizeof(cplx) * k * k, cudaMemcpyDeviceToHost, ctx->stream));
  return sync_and_check(ctx);
}

extern "C" int rls_test_svd_rr(rls_ctx* ctx, int nS, int r, int sideL, int lq, const rls_c64* R, double* sigma,
                               double* lam, rls_c64* G) {
  RET(need_space(ctx));
  if (nS < 1 || nS > 512 || r < 1 || r > nS || !R || !sigma || !lam || !G) return RLS_ERR_ARG;
  if (lq && nS > r && 2 * r > nS) return RLS_ERR_ARG;
  DevTmp t(ctx);
  cplx* dR = t.alloc<cplx>((size_t)nS * nS);
  cplx* dG = t.alloc<cplx>((size_t)nS * nS);
  double* ds = t.alloc<double>((size_t)nS);
  double* dl = t.alloc<double>((size_t)nS);
  if (!dR || !dG || !ds || !dl) return RLS_ERR_NOMEM;
  CK(cudaMemcpyAsync(dR, R, sizeof(cplx) * nS * nS, cudaMemcpyHostToDevice, ctx->stream));
  const bool glob = nS > 80 || svd_rr_smem_bytes(nS, r, false) > kSvdSmemShared;
  cplx* gA = glob ? t.alloc<cplx>((size_t)nS * nS) : nullptr;
  cplx* gV = glob ? t.alloc<cplx>((size_t)nS * nS) : nullptr;
  k_svd_rr<<<1, 256, svd_rr_smem_bytes(nS, r, glob), ctx->stream>>>(nS, r, sideL, lq, dR, nS, ds, dl, dG, nS, gA, gV);
  RET(check_launch(ctx, "k_svd_rr"));
  CK(cudaMemcpyAsync(sigma, ds, sizeof(double) * nS, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaMemcpyAsync(lam, dl, sizeof(double) * r, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaMemcpyAsync(G, dG, sizeof(cplx) * nS * nS, cudaMemcpyDeviceToHost, ctx->stream));
  return sync_and_check(ctx);
}

// find_rr_dim on Hz built from H1, H2 (pr×pr, column-major); G gets pr × rr.
extern "C" int rls_test_heev_rr(rls_ctx* ctx, int pr, int r, const rls_c64* H1, const rls_c64* H2, rls_c64 z,
                                double shift, double tau, int* rr, double* lam, rls_c64* G, long long* clk) {
  RET(need_space(ctx));
  if (pr < 1 || pr > ctx->pr_max || r < 1 || !H1 || !H2 || !rr || !G) return RLS_ERR_ARG;
  DevTmp t(ctx);
  cplx* d1 = t.alloc<cplx>((size_t)pr * pr);
  cplx* d2 = t.alloc<cplx>((size_t)pr * pr);
  if (!d1 || !d2) return RLS_ERR_NOMEM;
  CK(cudaMemcpyAsync(d1, H1, sizeof(cplx) * pr * pr, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(d2, H2, sizeof(cplx) * pr * pr, cudaMemcpyHostToDevice, ctx->stream));
  cplx zz = cmk(z.re, z.im);
  CK(cudaMemcpyAsync(ctx->zdev, &zz, sizeof(cplx), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(ctx->taudev, &tau, sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  const HeevPlan plan = heev_plan(pr, ctx->heev_smem_avail);
  long long* dclk = clk ? t.alloc<long long>(8) : nullptr;
  k_heev_rr<<<1, HEEV_THREADS, plan.bytes, ctx->stream>>>(
      pr, r, d1, d2, pr, ctx->zdev, ctx->taudev, shift, ctx->heev, ctx->pr_max, ctx->Gheev, ctx->pr_max,
      (int64_t)ctx->pr_max * ctx->pr_max, ctx->rr_dev, ctx->lam_dev, ctx->derr, plan, dclk);
  RET(check_launch(ctx, "k_heev_rr"));
  RET(d2h(ctx, rr, ctx->rr_dev, 1));
  if (lam) CK(cudaMemcpyAsync(lam, ctx->lam_dev, sizeof(double) * pr, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaMemcpy2DAsync(G, pr * sizeof(cplx), ctx->Gheev, ctx->pr_max * sizeof(cplx), pr * sizeof(cplx), *rr,
                       cudaMemcpyDeviceToHost, ctx->stream));
  if (clk) CK(cudaMemcpyAsync(clk, dclk, sizeof(long long) * 6, cudaMemcpyDeviceToHost, ctx->stream));
  return sync_and_check(ctx);
}

// updateRecycledSpace!(M, S, z, recySp, X; τ, r_sub = 1, force_add) on the device space.
extern "C" int rls_test_space_update(rls_ctx* ctx, rls_c64 z, const rls_c64* X, double tau, int force_add,
                                     int p_min) {
  RET(need_space(ctx));
  if (!X) return RLS_ERR_ARG;
  const int64_t np = ctx->n_pad, n = ctx->n;
  const int r = ctx->r;
  CK(cudaMemsetAsync(ctx->S, 0, sizeof(cplx) * np * r, ctx->stream));
  CK(cudaMemcpy2DAsync(ctx->S, np * sizeof(cplx), X, n * sizeof(cplx), n * sizeof(cplx), r, cudaMemcpyHostToDevice,
                       ctx->stream));
  RET(update_recycled_space(ctx, cmk(z.re, z.im), ctx->S, tau, force_add != 0, p_min));
  return sync_and_check(ctx);
}

// Copies out the device space: p, V (n × p r), J1, J2, J5 and L, H1, H2 (p r × p r).
// Any output pointer may be NULL.
extern "C" int rls_test_space_get(rls_ctx* ctx, int* p, rls_c64* V, rls_c64* J1, rls_c64* J2, rls_c64* J5,
                                  rls_c64* L, rls_c64* H1, rls_c64* H2) {
  RET(need_space(ctx));
  const int64_t np = ctx->n_pad, n = ctx->n;
  const int pr = ctx->p * ctx->r, ld = ctx->pr_max;
  if (p) *p = ctx->p;
  if (pr == 0) return RLS_OK;
  const cplx* tall[4] = {ctx->V, ctx->J1, ctx->J2, ctx->J5};
  rls_c64* tout[4] = {V, J1, J2, J5};
  for (int i = 0; i < 4; ++i)
    if (tout[i])
      CK(cudaMemcpy2DAsync(tout[i], n * sizeof(cplx), tall[i], np * sizeof(cplx), n * sizeof(cplx), pr,
                           cudaMemcpyDeviceToHost, ctx->stream));
  const cplx* sq[3] = {ctx->L, ctx->H1, ctx->H2};
  rls_c64* sout[3] = {L, H1, H2};
  for (int i = 0; i < 3; ++i)
    if (sout[i])
      CK(cudaMemcpy2DAsync(sout[i], pr * sizeof(cplx), sq[i], ld * sizeof(cplx), pr * sizeof(cplx), pr,
                           cudaMemcpyDeviceToHost, ctx->stream));
  return sync_and_check(ctx);
}

// fastSvdRaylRitz_implicit! on the device space: Ritz dimension, σ (r), X and W (n × r).
extern "C" int rls_test_recycle(rls_ctx* ctx, rls_c64 z, double shift, double gap_tau, int* rr, double* sigma,
                                rls_c64* X, rls_c64* W, double* w0norm) {
  RET(need_space(ctx));
  if (ctx->p < 1) return RLS_ERR_STATE;
  const int64_t np = ctx->n_pad, n = ctx->n;
  const int r = ctx->r;
  RecycleResult res{};
  RET(recycle_step(ctx, cmk(z.re, z.im), shift, gap_tau, &res));
  if (rr) *rr = res.rr;
  if (w0norm) *w0norm = res.w0norm;
  if (sigma) CK(cudaMemcpyAsync(sigma, ctx->sig_rec, sizeof(double) * r, cudaMemcpyDeviceToHost, ctx->stream));
  if (X)
    CK(cudaMemcpy2DAsync(X, n * sizeof(cplx), ctx->S, np * sizeof(cplx), n * sizeof(cplx), r, cudaMemcpyDeviceToHost,
                         ctx->stream));
  if (W)
    CK(cudaMemcpy2DAsync(W, n * sizeof(cplx), ctx->S + np * r, np * sizeof(cplx), n * sizeof(cplx), r,
                         cudaMemcpyDeviceToHost, ctx->stream));
  return sync_and_check(ctx);
}

namespace {
__global__ void k_test_recip(int64_t n, const double* q, double* r_nr, double* r_div) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    r_nr[i] = recip_nr(q[i]);
    r_div[i] = 1.0 / q[i];
  }
}
}  // namespace

// recip_nr (the Sturm-count reciprocal: hardware estimate + two Newton steps) beside CUDA's
// correctly rounded 1.0/q, for the same inputs.
extern "C" int rls_test_recip(rls_ctx* ctx, int64_t n, const double* q, double* r_nr, double* r_div) {
  if (!ctx || n < 1 || !q || !r_nr || !r_div) return RLS_ERR_ARG;
  DevTmp t(ctx);
  double* dq = t.alloc<double>((size_t)n);
  double* d1 = t.alloc<double>((size_t)n);
  double* d2 = t.alloc<double>((size_t)n);
  if (!dq || !d1 || !d2) return RLS_ERR_NOMEM;
  CK(cudaMemcpyAsync(dq, q, sizeof(double) * n, cudaMemcpyHostToDevice, ctx->stream));
  const unsigned blocks = (unsigned)std::min<int64_t>((n + 255) / 256, 1024);
  k_test_recip<<<blocks, 256, 0, ctx->stream>>>(n, dq, d1, d2);
  RET(check_launch(ctx, "k_test_recip"));
  CK(cudaMemcpyAsync(r_nr, d1, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaMemcpyAsync(r_div, d2, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->stream));
  return sync_and_check(ctx);
}

extern "C" int rls_test_band_r(rls_ctx* ctx, rls_c64 z, rls_c64* R, int64_t ldr, int64_t* l, int64_t* u) {
  if (!ctx || !R) return RLS_ERR_ARG;
  if (!ctx->band.on) {
    set_err(ctx, "rls_test_band_r: no sparse operator (call rls_set_sparse_tri first)");
    return RLS_ERR_STATE;
  }
  const int64_t n = ctx->n;
  if (ldr < n) return RLS_ERR_DIM;
  CK(cudaSetDevice(ctx->device));
  ctx->z_dinv = cmk(NAN, NAN);
  RET(ensure_dinv(ctx, cmk(z.re, z.im)));
  const int nb = ctx->nb, bw = ctx->tile_bw;
  const size_t slots = (size_t)tile_slots(nb, bw);
  std::vector<cplx> h(slots * TILE * TILE);
  CK(cudaMemcpyAsync(h.data(), ctx->T, sizeof(cplx) * h.size(), cudaMemcpyDeviceToHost, ctx->stream));
  RET(sync_and_check(ctx));
  for (int64_t j = 0; j < n; ++j)
    for (int64_t i = 0; i < n; ++i) R[j * ldr + i] = rls_c64{0.0, 0.0};
  for (int J = 0; J < nb; ++J)
    for (int I = std::max(0, J - bw); I <= J; ++I) {
      const cplx* tp = h.data() + tile_index_bw(I, J, nb, bw) * TILE * TILE;
      for (int cc = 0; cc < TILE; ++cc)
        for (int rr = 0; rr < TILE; ++rr) {
          const int64_t gi = (int64_t)I * TILE + rr, gj = (int64_t)J * TILE + cc;
          if (gi < n && gj < n) R[gj * ldr + gi] = rls_c64{tp[cc * TILE + rr].x, tp[cc * TILE + rr].y};
        }
    }
  if (l) *l = ctx->band.l;
  if (u) *u = ctx->band.u;
  return RLS_OK;
}

extern "C" int rls_test_band_factor(rls_ctx* ctx, rls_c64 z) {
  if (!ctx) return RLS_ERR_ARG;
  if (!ctx->band.on) {
    set_err(ctx, "rls_test_band_factor: no sparse operator (call rls_set_sparse_tri first)");
    return RLS_ERR_STATE;
  }
  CK(cudaSetDevice(ctx->device));
  ctx->z_dinv = cmk(NAN, NAN);
  RET(ensure_dinv(ctx, cmk(z.re, z.im)));
  return sync_and_check(ctx);
}
