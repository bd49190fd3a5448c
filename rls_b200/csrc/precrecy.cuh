// psPrecRecy on the device: the preconditioned two-space grid solver of
// src/core/psPrecRecy.jl:617-1033, with the operator-generic block LOBPCG
// (src/core/lobpcgSvd.jl:365-477) it needs.  Included at the end of engine.cu.
//
// Layout of one run (one context):
//   * C (sparse, CSR of C and of Cᴴ) in ctx->sp; the main recycled space (r_main, p_main;
//     orth_S = true, so J3 = J5, J4 = J6 = V as in psTriRecy) in the context's space arrays,
//     with ctx->op_sparse set so that its products M·V and Mᴴ·[J5 V] use C;
//   * the IC factor of the current preconditioner in ctx->lltp (built on the host by
//     rls_ic_factor, uploaded by rls_lltp_upload at start-up and at every rebuild);
//   * the prediction space (r_pred, p_pred; orth_S = false, implict_update = true), its LOBPCG
//     keep, E_pred and the eigensolver's work arrays in PrecState.
// Operators are applied to device blocks with leading dimension n_pad (rows ≥ n stay zero):
//   Cz = C − zI            spmm_dev (s = −z)
//   invF = P·L⁻ᴴ           backward block solve on Lᴴ, then the row gather X[invp]
//   invFᴴ = L⁻¹·Pᴴ         forward block solve with the gather B[p] fused
//   Cz_pred = Cz·invF      (the pred stage's operator and _compute_λ_n's, :405-422)
//   L⁻¹ (InvMat(K.L))      _compute_γ's operator (:388-402)
//   K_ad⁻¹ = K⁻¹ + E·GramE⁻¹·Eᴴ   SparseLLTP_AD ldiv! (RLSPreconditioner.jl:229-262)
#pragma once
#include <functional>
#include <map>

struct PrecState {
  int64_t n = 0;
  // prediction recycled space (recySpace.jl:40-120 with orth_S = false)
  int r = 0, p_max = 0, pr_max = 0, p = 0, p_min = 1;
  std::vector<rls_c64> pts;
  cplx *V = nullptr, *J1 = nullptr, *J2 = nullptr, *J3 = nullptr, *J4 = nullptr, *J5 = nullptr, *J6 = nullptr;
  cplx *L = nullptr, *H1 = nullptr, *H2 = nullptr, *H3 = nullptr, *Hs = nullptr;
  cplx *Ulist = nullptr, *rot_ws = nullptr;
  // LOBPCG keep of the pred stage (S, CS n_pad × 3r; G, R 3r × 3r; σ, λ 3r) and E_pred
  cplx *S = nullptr, *CS = nullptr, *G = nullptr, *R = nullptr;
  double *sig = nullptr, *lam = nullptr;
  cplx *E = nullptr, *X0 = nullptr;
  // keep of the r = 1 bound estimates
  cplx *bS = nullptr, *bCS = nullptr, *bG = nullptr, *bR = nullptr, *bX0 = nullptr;
  double *bsig = nullptr, *blam = nullptr;
  // eigensolver of fastRaylRitz! (pr ≤ pr_max)
  cplx *hA = nullptr, *hv[2] = {nullptr, nullptr}, *hy = nullptr, *hpart = nullptr, *htau = nullptr;
  double *hd = nullptr, *he = nullptr, *he2 = nullptr, *hlu = nullptr;
  cplx* hG = nullptr;        // pr_max × r eigenvectors
  cplx* hz = nullptr;        // the shift, read by the captured sequence
  // the eigensolve's launch sequence for each order pr, captured once and replayed (its
  // 2·(pr − 1) + 4 launches are fixed by pr; z is read from hz)
  std::map<int, cudaGraphExec_t> heev_graphs;
  void drop_graphs() {
    for (auto& g : heev_graphs) cudaGraphExecDestroy(g.second);
    heev_graphs.clear();
  }
  ~PrecState() { drop_graphs(); }
  // two-level preconditioner: GramE (r × r), its Cholesky inverse, coefficients
  cplx *gram = nullptr, *grinv = nullptr, *coef = nullptr, *coef2 = nullptr, *chol_ws = nullptr;
  // LOBPCG scratch (lob_scratch): shifted Cholesky-QR work for up to qcap columns, operator
  // temporaries (n_pad × opt_cols), column norms
  cplx *qW = nullptr, *qRinv = nullptr, *qRtot = nullptr, *qws = nullptr, *qRG = nullptr;
  cplx *opt1 = nullptr, *opt2 = nullptr;
  int opt_cols = 0, qcap = 0;
  int64_t opt_np = 0;
  double* norms = nullptr;
  // keep of rls_lobpcg_svd (block size lr)
  int lr = 0;
  int64_t l_np = 0;
  cplx *lS = nullptr, *lCS = nullptr, *lG = nullptr, *lR = nullptr;
  double *lsig = nullptr, *llam = nullptr;
  // Schur vectors Q (n_pad × n_pad, rls_set_schur_vectors) and [u v Qu Qv] for ∂σ/∂C
  cplx *Qdev = nullptr, *Qws = nullptr;
  int64_t Q_np = 0, Q_n = 0;
  // host copy of C (for the IC rebuilds) and the column order
  std::vector<int64_t> colptr, rowval, p0;
  std::vector<rls_c64> nzval;
  // run state carried across range calls (psPrecRecy.jl:646-664)
  bool active = false;
  int64_t next = 0, nZ = 0;
  cplx z_dagger{0, 0};
  double lam_dagger_n = 0.0, gamma = 0.0, lam_lower = 0.0, lam_upper = 0.0;
  bool have_failed_main = false, have_failed_pred = false;
  rls_c64 last_failed_main{0, 0}, last_failed_pred{0, 0};
  double thresh = 0.0;
  bool pred_x0_given = false;
};

void prec_state_delete(PrecState* s) { delete s; }

namespace {

// A device buffer owned by one host call: freed (after the stream drains) when it goes out
// of scope.  For per-call inputs whose size the call's arguments fix.
template <class T>
struct DevTmpBuf {
  rls_ctx* ctx;
  T* p = nullptr;
  explicit DevTmpBuf(rls_ctx* c) : ctx(c) {}
  int alloc(size_t count) {
    if (cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T)) != cudaSuccess) {
      p = nullptr;
      set_err(ctx, "device allocation of %zu bytes failed", std::max<size_t>(count, 1) * sizeof(T));
      return RLS_ERR_NOMEM;
    }
    return RLS_OK;
  }
  ~DevTmpBuf() {
    if (p) {
      cudaStreamSynchronize(ctx->stream);
      cudaFree(p);
    }
  }
};

// ---- small building blocks ---------------------------------------------------------------

// R (k×k, ld k, may be null) and X ← Q of the shifted Cholesky-QR of X (nrows × k)
// (_rls_qr_shiftchol!, RLSLinearAlgebra.jl:725-796): up to three sweeps, each stopping test
// ‖XᴴX − I‖_F < 2√k·eps read back on the host.
int qr_shiftchol(rls_ctx* ctx, int64_t nrows, cplx* X, int64_t ldx, int k, cplx* R) {
  PrecState& ps = *ctx->prec;
  RET(gram(ctx, nrows, X, ldx, k, X, ldx, k, ps.qW, k));
  const double conv = 2.0 * std::sqrt((double)k) * kEps;
  for (int it = 1; it <= 3; ++it) {
    k_shiftchol_sweep<<<1, 256, 0, ctx->stream>>>(k, nrows, ps.qW, ps.qRinv, ps.qRtot, it == 1 ? 1 : 0, ps.qws,
                                                  ctx->derr);
    RET(check_launch(ctx, "k_shiftchol_sweep"));
    RET(gemm_rows(ctx, nrows, one_src(X), ldx, k, ps.qRinv, k, k, X, ldx));
    RET(gram(ctx, nrows, X, ldx, k, X, ldx, k, ps.qW, k));
    k_dist_identity2<<<1, 256, 0, ctx->stream>>>(k, ps.qW, ctx->dscal);
    RET(check_launch(ctx, "k_dist_identity2"));
    double d2 = 0.0;
    RET(d2h(ctx, &d2, ctx->dscal, 1));
    if (std::sqrt(d2) < conv) break;
  }
  if (R) CK(cudaMemcpyAsync(R, ps.qRtot, sizeof(cplx) * k * k, cudaMemcpyDeviceToDevice, ctx->stream));
  return RLS_OK;
}

// rls_qr!(X, R; type): orth = 0 :lapack (TSQR + R⁻¹ + CholQR pass), 1 :shiftchol.
int qr_typed(rls_ctx* ctx, int64_t nrows, cplx* X, int64_t ldx, int k, cplx* R, int orth) {
  if (orth == 1) return qr_shiftchol(ctx, nrows, X, ldx, k, R);
  return orth_qr(ctx, nrows, X, ldx, k, R);
}

// rls_orth!(V, X; type) (RLSLinearAlgebra.jl:1127-1160): two block CGS passes of X against V.
int orth_typed(rls_ctx* ctx, int64_t nrows, const cplx* V, int64_t ldv, int nV, cplx* X, int64_t ldx, int nX,
               int orth) {
  if (orth == 0) return orth_twice(ctx, nrows, V, ldv, nV, X, ldx, nX);
  cplx* W = ctx->small[5];
  for (int pass = 0; pass < 2; ++pass) {
    RET(gram(ctx, nrows, V, ldv, nV, X, ldx, nX, W, nV));
    RET(gemm_rows(ctx, nrows, one_src(V), ldv, nV, W, nV, nX, X, ldx, cmk(-1, 0), cmk(1, 0)));
    RET(qr_typed(ctx, nrows, X, ldx, nX, nullptr, orth));
  }
  return RLS_OK;
}

// Column norms ‖A[:, j]‖ for j < k read to the host.
int col_norms(rls_ctx* ctx, const cplx* A, int64_t lda, int k, double* out) {
  k_colnorm2<<<k, 256, 0, ctx->stream>>>(ctx->n_pad, A, lda, ctx->prec->norms);
  RET(check_launch(ctx, "k_colnorm2"));
  RET(d2h(ctx, out, ctx->prec->norms, (size_t)k));
  for (int j = 0; j < k; ++j) out[j] = std::sqrt(out[j]);
  return RLS_OK;
}

// ---- the preconditioner's triangular pieces ------------------------------------------------

// out = L⁻¹·(gather ? B[p] : B) (op 0) or Lᴴ⁻¹·B (op 1), b columns in chunks of 8; out ≠ B.
int lltp_tri(rls_ctx* ctx, int op, bool gather_p, int b, const cplx* B, int64_t ldb, cplx* out, int64_t ldo) {
  auto& F = ctx->lltp;
  if (!F.op[0].rowptr) {
    set_err(ctx, "no preconditioner factor uploaded");
    return RLS_ERR_STATE;
  }
  if (F.singular_at) {
    set_err(ctx, "SingularException(%lld): the factor's diagonal entry %lld is zero", (long long)F.singular_at,
            (long long)F.singular_at);
    return RLS_ERR_SINGULAR;
  }
  const int64_t nblk = F.op[0].nblk;
  const unsigned grid = (unsigned)std::min<int64_t>(nblk, 148 * 4);
  for (int c0 = 0; c0 < b; c0 += 8) {
    const int kk = std::min(8, b - c0);
    F.epoch += 1;
    if (F.epoch > (1 << 30)) {
      F.epoch = 1;
      CK(cudaMemsetAsync(F.flags, 0, sizeof(int) * 2 * nblk * SPT_FLAG_STRIDE, ctx->stream));
    }
    int* tk = F.ticket + op;
    int* fl = F.flags + (op ? nblk * SPT_FLAG_STRIDE : 0);
    CK(cudaMemsetAsync(tk, 0, sizeof(int), ctx->stream));
    const cplx* Bc = B + (int64_t)c0 * ldb;
    cplx* Oc = out + (int64_t)c0 * ldo;
    const int64_t* gat = (op == 0 && gather_p) ? F.p : nullptr;
#define RLS_TRI_CASE(K)                                                                                         \
  case K:                                                                                                       \
    if (op == 0)                                                                                                \
      k_sptrsv_wide<K, false><<<grid, 32 * SPW_WARPS, 0, ctx->stream>>>(F.op[0], Bc, ldb, gat, Oc, ldo, tk, fl, \
                                                                          F.epoch, ctx->derr);                  \
    else                                                                                                        \
      k_sptrsv_wide<K, true><<<grid, 32 * SPW_WARPS, 0, ctx->stream>>>(F.op[1], Bc, ldb, nullptr, Oc, ldo, tk,  \
                                                                         fl, F.epoch, ctx->derr);               \
    break;
    switch (kk) {
      RLS_TRI_CASE(1) RLS_TRI_CASE(2) RLS_TRI_CASE(3) RLS_TRI_CASE(4)
      RLS_TRI_CASE(5) RLS_TRI_CASE(6) RLS_TRI_CASE(7) RLS_TRI_CASE(8)
    }
#undef RLS_TRI_CASE
    RET(check_launch(ctx, "k_sptrsv_wide"));
  }
  return RLS_OK;
}

// Y = invF·X = (Lᴴ⁻¹X)[invp, :]  (b ≤ opt_cols columns)
int invF_mul(rls_ctx* ctx, int b, const cplx* X, cplx* Y) {
  PrecState& ps = *ctx->prec;
  const int64_t np = ctx->n_pad;
  RET(lltp_tri(ctx, 1, false, b, X, np, ps.opt2, np));
  const int64_t nf = ctx->lltp.n;   // the factor's order (ps.n is set only by a psPrecRecy run)
  const unsigned gg = (unsigned)((nf + 255) / 256);
  for (int c0 = 0; c0 < b; c0 += 8) {
    const int kk = std::min(8, b - c0);
    const cplx* W = ps.opt2 + (int64_t)c0 * np;
    cplx* Yc = Y + (int64_t)c0 * np;
#define RLS_G_CASE(K) \
  case K: k_gather_rows<K><<<gg, 256, 0, ctx->stream>>>(nf, ctx->lltp.invp, W, np, Yc, np); break;
    switch (kk) {
      RLS_G_CASE(1) RLS_G_CASE(2) RLS_G_CASE(3) RLS_G_CASE(4)
      RLS_G_CASE(5) RLS_G_CASE(6) RLS_G_CASE(7) RLS_G_CASE(8)
    }
#undef RLS_G_CASE
    RET(check_launch(ctx, "k_gather_rows"));
  }
  return RLS_OK;
}

// X = invFᴴ·Y = L⁻¹·Y[p, :]
int invF_adj(rls_ctx* ctx, int b, const cplx* Y, cplx* X) {
  return lltp_tri(ctx, 0, true, b, Y, ctx->n_pad, X, ctx->n_pad);
}

// A linear operator on device blocks of b columns (ld n_pad); out must not alias in.
struct DevOp {
  std::function<int(const cplx*, cplx*, int)> mul, mul_adj;
};

DevOp op_shifted(rls_ctx* ctx, cplx z) {   // ShiftedMat(C, −z)
  DevOp o;
  o.mul = [ctx, z](const cplx* X, cplx* Y, int b) {
    return spmm_dev(ctx, cneg(z), 0, b, X, ctx->n_pad, Y, ctx->n_pad);
  };
  o.mul_adj = [ctx, z](const cplx* X, cplx* Y, int b) {
    return spmm_dev(ctx, cneg(z), 1, b, X, ctx->n_pad, Y, ctx->n_pad);
  };
  return o;
}

DevOp op_pred(rls_ctx* ctx, cplx z) {      // MulChainMat(ShiftedMat(C, −z), invF)
  DevOp o;
  o.mul = [ctx, z](const cplx* X, cplx* Y, int b) {
    PrecState& ps = *ctx->prec;
    RET(invF_mul(ctx, b, X, ps.opt1));
    return spmm_dev(ctx, cneg(z), 0, b, ps.opt1, ctx->n_pad, Y, ctx->n_pad);
  };
  o.mul_adj = [ctx, z](const cplx* Y, cplx* X, int b) {
    PrecState& ps = *ctx->prec;
    RET(spmm_dev(ctx, cneg(z), 1, b, Y, ctx->n_pad, ps.opt1, ctx->n_pad));
    return invF_adj(ctx, b, ps.opt1, X);
  };
  return o;
}

DevOp op_invL(rls_ctx* ctx) {              // InvMat(K.L)
  DevOp o;
  o.mul = [ctx](const cplx* X, cplx* Y, int b) { return lltp_tri(ctx, 0, false, b, X, ctx->n_pad, Y, ctx->n_pad); };
  o.mul_adj = [ctx](const cplx* X, cplx* Y, int b) {
    return lltp_tri(ctx, 1, false, b, X, ctx->n_pad, Y, ctx->n_pad);
  };
  return o;
}

// ldiv!(K_ad, W) in place on b columns: W ← K⁻¹W + E·GramE⁻¹·(EᴴW) (RLSPreconditioner.jl:229-262)
int ldiv_ad(rls_ctx* ctx, cplx* W, int b) {
  PrecState& ps = *ctx->prec;
  const int64_t np = ctx->n_pad;
  const int rp = ps.r;
  RET(gram(ctx, np, ps.E, np, rp, W, np, b, ps.coef, rp));                                   // EᴴW
  RET(small_gemm(ctx, rp, b, rp, cmk(1, 0), ps.grinv, rp, 1, ps.coef, rp, 0, cmk(0, 0), ps.coef2, rp));  // R⁻ᴴ·
  RET(small_gemm(ctx, rp, b, rp, cmk(1, 0), ps.grinv, rp, 0, ps.coef2, rp, 0, cmk(0, 0), ps.coef, rp));  // R⁻¹·
  RET(lltp_ldiv_dev(ctx, b, W, np, ps.opt1, np));                                            // K⁻¹W
  RET(gemm_rows(ctx, np, one_src(ps.E), np, rp, ps.coef, rp, b, ps.opt1, np, cmk(1, 0), cmk(1, 0)));
  return copy_cols(ctx, ps.opt1, W, b);
}

// ---- operator-generic block LOBPCG (lobpcgSvd.jl:365-477) -------------------------------

struct LobKeep {
  cplx *S, *CS, *G, *R;   // n_pad × 3r, n_pad × 3r, 3r × 3r (ld 3r), 3r × 3r (ld 3r)
  double *sig, *lam;      // 3r
  int r;
};

struct LobCtl {
  int64_t maxit = 2000;
  double tol = 1e-3;
  bool sideL = false;
  double normC = 1.0;
  int orth = 0;           // 0 :lapack, 1 :shiftchol
  int conv_type = 0;      // conv_thresh_type
  int conv_first = 1, conv_last = 1;   // 1-based conv_range
};

// svdRaylRitz! (lobpcgSvd.jl:126-184) on CSv (n_pad × nS): R of its QR (CSv untouched for
// :lapack; CSv ← Q for :shiftchol), then k_svd_rr.  Sets *cs_is_q.
int svd_rr_gen(rls_ctx* ctx, LobKeep& k, cplx* CSv, int nS, const LobCtl& c, bool* cs_is_q) {
  const int64_t np = ctx->n_pad;
  const int r = k.r;
  if (c.orth == 1) {
    RET(qr_shiftchol(ctx, np, CSv, np, nS, k.R));
    *cs_is_q = true;
  } else {
    RET(tsqr_r(ctx, np, CSv, np, nS, k.R));
    *cs_is_q = false;
  }
  // A and V in shared memory while they fit beside the r-wide work arrays (to 80 columns at
  // small r), else in the global scratch
  const bool glob = nS > 80 || svd_rr_smem_bytes(nS, r, false) > kSvdSmemShared;
  k_svd_rr<<<1, 256, svd_rr_smem_bytes(nS, r, glob), ctx->stream>>>(nS, r, c.sideL ? 1 : 0, 1, k.R, nS, k.sig, k.lam,
                                                                   k.G, 3 * r, glob ? ctx->svdA : nullptr,
                                                                   glob ? ctx->svdV : nullptr);
  return check_launch(ctx, "k_svd_rr");
}

// basisUpdate! (lobpcgSvd.jl:195-220): V ← S·G[:, 0:m], CV ← CS·(R·G[:, 0:m]) (= CS_orig·G).
int basis_update_gen(rls_ctx* ctx, LobKeep& k, int nS, int m, bool cs_is_q) {
  const int64_t np = ctx->n_pad;
  const int ldg = 3 * k.r;
  RET(gemm_rows(ctx, np, one_src(k.S), np, nS, k.G, ldg, m, k.S, np));
  if (cs_is_q) {
    PrecState& ps = *ctx->prec;
    RET(small_gemm(ctx, nS, m, nS, cmk(1, 0), k.R, nS, 0, k.G, ldg, 0, cmk(0, 0), ps.qRG, nS));
    return gemm_rows(ctx, np, one_src(k.CS), np, nS, ps.qRG, nS, m, k.CS, np);
  }
  return gemm_rows(ctx, np, one_src(k.CS), np, nS, k.G, ldg, m, k.CS, np);
}

// residual! (lobpcgSvd.jl:227-248): W = Cᴴ(CX), then W −= X·λ ('S') or W = W·λ − X ('L').
int residual_gen(rls_ctx* ctx, const DevOp& C, LobKeep& k, cplx* W, const LobCtl& c) {
  const int64_t np = ctx->n_pad;
  RET(C.mul_adj(k.CS, W, k.r));
  const int blocks = (int)((np + 255) / 256);
  k_residual_fix<<<blocks, 256, 0, ctx->stream>>>(np, W, np, k.S, np, k.r, k.lam, c.sideL ? 1 : 0, nullptr);
  return check_launch(ctx, "k_residual_fix");
}

// check_conv_svd (lobpcgSvd.jl:317-357) on W's columns: one read of the norms and σ.
int check_conv_gen(rls_ctx* ctx, LobKeep& k, const cplx* W, const LobCtl& c, bool* conv) {
  const int r = k.r;
  std::vector<double> nrm((size_t)r), sg((size_t)r);
  k_colnorm2<<<r, 256, 0, ctx->stream>>>(ctx->n_pad, W, ctx->n_pad, ctx->prec->norms);
  RET(check_launch(ctx, "k_colnorm2"));
  {
    D2HBatch rd(ctx);
    RET(rd.add(nrm.data(), ctx->prec->norms, (size_t)r));
    RET(rd.add(sg.data(), k.sig, (size_t)r));
    RET(rd.finish());
  }
  for (auto& v : nrm) v = std::sqrt(v);
  if (c.sideL) {
    *conv = nrm[0] < c.tol;
    return RLS_OK;
  }
  const double floor_ = c.normC * c.normC * std::sqrt(2.0) * kEps;
  *conv = true;
  for (int j = c.conv_first - 1; j < c.conv_last; ++j) {
    const double th = (c.conv_type == 0) ? std::max(c.normC * sg[j] * c.tol, floor_)
                                         : std::max(c.normC * c.normC * c.tol, floor_);
    if (!(nrm[j] < th)) {
      *conv = false;
      break;
    }
  }
  return RLS_OK;
}

// lobpcgSvd(C, X0 = k.S[:, 0:r], K, keep, control).  Returns σ (side 'S': σ[1]; side 'L':
// 1/σ[1] of the inverted values, i.e. the largest singular value of C) and the iteration count.
int lobpcg_gen(rls_ctx* ctx, const DevOp& C, const std::function<int(cplx*, int)>* ldiv, LobKeep& k, const LobCtl& c,
               double* sigma, int64_t* it_out) {
  const int64_t np = ctx->n_pad;
  const int r = k.r;
  cplx *X = k.S, *P = k.S + np * r, *W = k.S + 2 * np * r;
  cplx *CX = k.CS, *CP = k.CS + np * r, *CW = k.CS + 2 * np * r;
  bool csq = false;
  RET(qr_typed(ctx, np, X, np, r, nullptr, c.orth));
  RET(C.mul(X, CX, r));
  RET(svd_rr_gen(ctx, k, CX, r, c, &csq));
  RET(basis_update_gen(ctx, k, r, r, csq));
  RET(residual_gen(ctx, C, k, P, c));
  if (ldiv) RET((*ldiv)(P, r));
  RET(orth_typed(ctx, np, X, np, r, P, np, r, c.orth));
  RET(C.mul(P, CP, r));
  for (int64_t i = 1; i <= c.maxit; ++i) {
    const int nS = (i == 1) ? 2 * r : 3 * r;
    RET(svd_rr_gen(ctx, k, k.CS, nS, c, &csq));
    RET(basis_update_gen(ctx, k, nS, 2 * r, csq));
    RET(residual_gen(ctx, C, k, W, c));
    bool conv = false;
    RET(check_conv_gen(ctx, k, W, c, &conv));
    if (conv) {
      double s0 = 0.0;
      RET(d2h(ctx, &s0, k.sig, 1));
      *sigma = c.sideL ? 1.0 / s0 : s0;
      *it_out = i;
      return RLS_OK;
    }
    if (ldiv) RET((*ldiv)(W, r));
    RET(orth_typed(ctx, np, k.S, np, 2 * r, W, np, r, c.orth));
    RET(C.mul(W, CW, r));
  }
  double s0 = 0.0;
  RET(d2h(ctx, &s0, k.sig, 1));
  *sigma = c.sideL ? 1.0 / s0 : s0;
  *it_out = c.maxit;
  return RLS_OK;
}

// ---- prediction recycled space ------------------------------------------------------------

// Ritz pairs 1..nvec of Hz = H1 − zH2 − z̄H2ᴴ + |z|²H3 (pr × pr): λ into lam, G (pr × nvec, ld
// pr_max) into ps.hG.  Householder tridiagonalisation, two launches per column (pred.cuh).  The
// launch sequence depends on pr only (z is read from ps.hz), so it is captured into a CUDA graph
// the first time an order pr occurs and replayed after that: one graph launch instead of
// 2·(pr − 1) + 4 kernel launches.
int pred_heev_launches(rls_ctx* ctx, int pr, int nvec, double* lam) {
  PrecState& ps = *ctx->prec;
  const int ld = ps.pr_max;
  cplx* A = ps.hA;
  k_hz_build<<<std::max(1, std::min(1024, (pr * pr + 255) / 256)), 256, 0, ctx->stream>>>(
      pr, ps.H1, ps.H2, ps.H3, ld, ps.hz, 0.0, A, pr);
  RET(check_launch(ctx, "k_hz_build"));
  if (pr > 1) {
    k_trd_first<<<1, 32, 0, ctx->stream>>>(pr, A, pr, ps.hv[0], ps.htau, ps.hd, ps.he);
    RET(check_launch(ctx, "k_trd_first"));
    for (int k = 0; k < pr - 1; ++k) {
      const int rows = pr - (k + 1);
      const int gs = std::max(1, std::min(148 * 2, (rows + 7) / 8));
      const int gu = std::max(1, std::min(148 * 2, rows));
      k_trd_symv<<<gs, 256, 0, ctx->stream>>>(k, pr, A, pr, ps.hv[k & 1], ps.htau, ps.hy, ps.hpart);
      k_trd_update<<<gu, 256, 0, ctx->stream>>>(k, pr, A, pr, ps.hv[k & 1], ps.htau, ps.hy, ps.hpart, gs,
                                               ps.hv[(k + 1) & 1], ps.hd, ps.he);
    }
    RET(check_launch(ctx, "k_trd_update"));
  } else {
    k_trd_first<<<1, 32, 0, ctx->stream>>>(1, A, 1, ps.hv[0], ps.htau, ps.hd, ps.he);   // d[0] only
    RET(check_launch(ctx, "k_trd_first"));
  }
  k_trd_eigvecs<<<1, 512, 0, ctx->stream>>>(pr, ps.hd, ps.he, nvec, lam, ps.hG, ld, ps.hlu, ps.he2, ctx->derr);
  RET(check_launch(ctx, "k_trd_eigvecs"));
  if (pr > 1) {
    k_trd_backtransform<<<(nvec + 15) / 16, 256, 0, ctx->stream>>>(pr, A, pr, ps.htau, ps.hG, ld, nvec);
    RET(check_launch(ctx, "k_trd_backtransform"));
  }
  return RLS_OK;
}

int pred_heev(rls_ctx* ctx, int pr, cplx z, int nvec, double* lam) {
  PrecState& ps = *ctx->prec;
  CK(cudaMemcpyAsync(ps.hz, &z, sizeof(cplx), cudaMemcpyHostToDevice, ctx->stream));
  auto it = ps.heev_graphs.find(pr);
  if (it == ps.heev_graphs.end()) {
    cudaGraph_t g = nullptr;
    CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    const int st = pred_heev_launches(ctx, pr, nvec, lam);
    const cudaError_t ce = cudaStreamEndCapture(ctx->stream, &g);
    if (st != RLS_OK) {
      if (g) cudaGraphDestroy(g);
      return st;
    }
    CK(ce);
    cudaGraphExec_t ex = nullptr;
    const cudaError_t ie = cudaGraphInstantiate(&ex, g, 0);
    cudaGraphDestroy(g);
    CK(ie);
    it = ps.heev_graphs.emplace(pr, ex).first;
  }
  cudaEvent_t e0 = nullptr;
  prof_begin(ctx, KP_HEEV, &e0);
  CK(cudaGraphLaunch(it->second, ctx->stream));
  ctx->launches += (pr > 1) ? 2 * (pr - 1) + 4 : 3;
  prof_end(ctx, KP_HEEV, e0, 16.0 / 3.0 * (double)pr * pr * pr);
  return RLS_OK;
}

// fastRaylRitz! (fastRaylRitz.jl:382-427): X_pred = V·G, E = J6·G, W = work·G − X·Λ with
// work = J1 − zJ2 − z̄J3 + |z|²J4; λ[1:r] into the keep's λ (λ_recy_pred is a view of it).
int pred_rayl_ritz(rls_ctx* ctx, cplx z) {
  PrecState& ps = *ctx->prec;
  const int r = ps.r, pr = ps.p * r;
  const int64_t np = ctx->n_pad;
  RET(pred_heev(ctx, pr, z, r, ps.lam));
  cplx* X = ps.S;
  cplx* W = ps.S + np * r;
  RET(gemm_rows(ctx, np, one_src(ps.V), np, pr, ps.hG, ps.pr_max, r, X, np));
  RET(gemm_rows(ctx, np, one_src(ps.J6), np, pr, ps.hG, ps.pr_max, r, ps.E, np));
  CombSrc w{};
  w.a[0] = ps.J1; w.coef[0] = cmk(1, 0);
  w.a[1] = ps.J2; w.coef[1] = cneg(z);
  w.a[2] = ps.J3; w.coef[2] = cneg(cconj(z));
  w.a[3] = ps.J4; w.coef[3] = cmk(z.x * z.x + z.y * z.y, 0);
  w.nsrc = 4;
  RET(gemm_rows(ctx, np, w, np, pr, ps.hG, ps.pr_max, r, W, np));
  const int blocks = (int)((np + 255) / 256);
  k_residual_fix<<<blocks, 256, 0, ctx->stream>>>(np, W, np, X, np, r, ps.lam, 0, nullptr);
  return check_launch(ctx, "k_residual_fix");
}

int pred_shift_blocks(rls_ctx* ctx, int l) {   // _shift_blocks! (recySpace.jl:290-340)
  PrecState& ps = *ctx->prec;
  const int p = ps.p, r = ps.r, nk = (p - l) * r;
  const int64_t np = ctx->n_pad;
  const int ld = ps.pr_max;
  for (int i = 0; i < p - l; ++i) ps.pts[i] = ps.pts[i + l];
  for (cplx* A : {ps.V, ps.J1, ps.J2, ps.J3, ps.J4, ps.J5, ps.J6}) {
    // column ranges do not overlap once l·r ≥ nk; otherwise go through the scratch
    RET(copy_cols(ctx, A + (int64_t)l * r * np, ctx->tall_tmp, nk));
    RET(copy_cols(ctx, ctx->tall_tmp, A, nk));
  }
  for (cplx* M : {ps.L, ps.H1, ps.H2, ps.H3}) {
    CK(cudaMemcpy2DAsync(ps.Hs, ld * sizeof(cplx), M + (int64_t)l * r * ld + l * r, ld * sizeof(cplx),
                         nk * sizeof(cplx), nk, cudaMemcpyDeviceToDevice, ctx->stream));
    CK(cudaMemcpy2DAsync(M, ld * sizeof(cplx), ps.Hs, ld * sizeof(cplx), nk * sizeof(cplx), nk,
                         cudaMemcpyDeviceToDevice, ctx->stream));
  }
  ps.p = p - l;
  return RLS_OK;
}

// _add_blocks! (recySpace.jl:344-453) with M = C·invF, S = invF (mul_coupled_ms! computes
// F·V_new once, RLSPreconditioner.jl:50-76), implicit cache with orth_S = false.
int pred_add_blocks(rls_ctx* ctx, const cplx* Xin, cplx z) {
  PrecState& ps = *ctx->prec;
  const int p = ps.p, r = ps.r, pr = p * r;
  const int64_t np = ctx->n_pad;
  const int ld = ps.pr_max;
  const int64_t off = (int64_t)pr * np;
  cplx *Vn = ps.V + off, *J1n = ps.J1 + off, *J2n = ps.J2 + off, *J3n = ps.J3 + off, *J4n = ps.J4 + off,
       *J5n = ps.J5 + off, *J6n = ps.J6 + off;
  RET(copy_cols(ctx, Xin, Vn, r));
  cplx* Lnn = ps.L + (int64_t)pr * ld + pr;
  if (p > 0) {
    RET(orth_robust(ctx, np, ps.V, np, pr, Vn, np, r, ctx->owW, ctx->owR));
    CK(cudaMemcpy2DAsync(ps.L + (int64_t)pr * ld, ld * sizeof(cplx), ctx->owW, pr * sizeof(cplx), pr * sizeof(cplx),
                         r, cudaMemcpyDeviceToDevice, ctx->stream));
  } else {
    RET(orth_qr(ctx, np, Vn, np, r, ctx->owR));
  }
  CK(cudaMemcpy2DAsync(Lnn, ld * sizeof(cplx), ctx->owR, r * sizeof(cplx), r * sizeof(cplx), r,
                       cudaMemcpyDeviceToDevice, ctx->stream));
  RET(invF_mul(ctx, r, Vn, J6n));                                            // J6 = S·V = F·V
  RET(spmm_dev(ctx, czero(), 0, r, J6n, np, J5n, np));                       // J5 = M·V = C·(F·V)
  RET(spmm_dev(ctx, czero(), 1, r, J5n, np, ps.opt1, np));                   // J1 = Fᴴ·Cᴴ·J5
  RET(invF_adj(ctx, r, ps.opt1, J1n));
  RET(spmm_dev(ctx, czero(), 1, r, J6n, np, ps.opt1, np));                   // J2 = Fᴴ·Cᴴ·J6
  RET(invF_adj(ctx, r, ps.opt1, J2n));
  RET(invF_adj(ctx, r, J5n, J3n));                                           // J3 = Sᴴ·J5
  RET(invF_adj(ctx, r, J6n, J4n));                                           // J4 = Sᴴ·J6
  RET(gram(ctx, np, Vn, np, r, J1n, np, r, ps.H1 + (int64_t)pr * ld + pr, ld));
  RET(gram(ctx, np, Vn, np, r, J2n, np, r, ps.H2 + (int64_t)pr * ld + pr, ld));
  RET(gram(ctx, np, Vn, np, r, J4n, np, r, ps.H3 + (int64_t)pr * ld + pr, ld));
  if (p > 0) {
    RET(gram(ctx, np, ps.J1, np, pr, Vn, np, r, ps.H1 + (int64_t)pr * ld, ld));   // H1[old,new]
    RET(gram(ctx, np, ps.J3, np, pr, Vn, np, r, ps.H2 + (int64_t)pr * ld, ld));   // H2[old,new]
    RET(gram(ctx, np, ps.J4, np, pr, Vn, np, r, ps.H3 + (int64_t)pr * ld, ld));   // H3[old,new]
    k_conj_transpose<<<64, 256, 0, ctx->stream>>>(pr, r, ps.H1 + (int64_t)pr * ld, ld, ps.H1 + pr, ld);
    RET(check_launch(ctx, "k_conj_transpose"));
    k_conj_transpose<<<64, 256, 0, ctx->stream>>>(pr, r, ps.H3 + (int64_t)pr * ld, ld, ps.H3 + pr, ld);
    RET(check_launch(ctx, "k_conj_transpose"));
    RET(gram(ctx, np, ps.J2, np, pr, Vn, np, r, ctx->small[4], pr));             // (J2_oldᴴ V_new)
    k_conj_transpose<<<64, 256, 0, ctx->stream>>>(pr, r, ctx->small[4], pr, ps.H2 + pr, ld);
    RET(check_launch(ctx, "k_conj_transpose"));
  }
  ps.pts[p] = rls_c64{z.x, z.y};
  ps.p = p + 1;
  return RLS_OK;
}

// _block_unitary_update! (recySpace.jl:226-286) with implict_update = true and orth_S = false:
// every cached block rotates (V, J1..J6; H1..H3 on both sides; L from the left).
int pred_block_update(rls_ctx* ctx) {
  PrecState& ps = *ctx->prec;
  const int p = ps.p, r = ps.r;
  if (p <= 1) return RLS_OK;
  const int pr = p * r;
  k_blockrot_coeffs_g<<<1, 256, 0, ctx->stream>>>(p, r, ps.L, ps.pr_max, ps.Ulist, ps.rot_ws);
  RET(check_launch(ctx, "k_blockrot_coeffs_g"));
  RotArraysG arr{};
  cplx* tall[7] = {ps.V, ps.J1, ps.J2, ps.J3, ps.J4, ps.J5, ps.J6};
  for (int q = 0; q < 7; ++q) { arr.a[q] = tall[q]; arr.nrows[q] = ctx->n_pad; arr.ld[q] = ctx->n_pad; }
  cplx* hs[3] = {ps.H1, ps.H2, ps.H3};
  for (int q = 0; q < 3; ++q) { arr.a[7 + q] = hs[q]; arr.nrows[7 + q] = pr; arr.ld[7 + q] = ps.pr_max; }
  const size_t sm = blockrot_g_smem(r);
  dim3 grid((unsigned)((ctx->n_pad + BR_ROWS - 1) / BR_ROWS), 10);
  k_blockrot_apply_g<<<grid, 256, sm, ctx->stream>>>(p, r, arr, ps.Ulist);
  RET(check_launch(ctx, "k_blockrot_apply_g"));
  RotMatsG mats{};
  mats.m[0] = ps.L; mats.m[1] = ps.H1; mats.m[2] = ps.H2; mats.m[3] = ps.H3;
  dim3 grid2((unsigned)((pr + BR_ROWS - 1) / BR_ROWS), 4);
  k_blockrot_left_g<<<grid2, 256, sm, ctx->stream>>>(p, r, mats, ps.pr_max, ps.Ulist);
  return check_launch(ctx, "k_blockrot_left_g");
}

// Block Frobenius norms of W (nV × nX, ld nV) in blocks of r rows, and ‖R‖_F² (nX × nX):
// out[b] for b < nV/r, out[nV/r] for R.  One CTA per output.
__global__ void k_block_fro2(int nV, int nX, int r, const cplx* __restrict__ W, const cplx* __restrict__ R,
                             double* out) {
  __shared__ double red[32];
  const int b = blockIdx.x, nb = nV / r;
  double s = 0.0;
  if (b < nb) {
    for (int q = threadIdx.x; q < r * nX; q += blockDim.x) s += cabs2(W[(int64_t)(q / r) * nV + b * r + (q % r)]);
  } else {
    for (int q = threadIdx.x; q < nX * nX; q += blockDim.x) s += cabs2(R[q]);
  }
  s = block_sum(s, red);
  if (threadIdx.x == 0) out[b] = s;
}

// updateRecycledSpace!(M_pred, S_pred, z, recySp_pred, X_pred; τ, r_sub, force_add)
// (recySpace.jl:160-223).  The residual scan uses one robust orthogonalisation of X[:, 1:r_sub]
// against all blocks: with X_sub = V·W + Q·R, dropping the first i blocks leaves the residual
// ‖[W_1; …; W_i; R]‖_F (the dropped blocks and Q are orthonormal), which is the Frobenius norm
// of the R factor the reference recomputes for each i.
int pred_update(rls_ctx* ctx, cplx z, double tau, int r_sub, bool force_add) {
  PrecState& ps = *ctx->prec;
  const int r = ps.r;
  const int64_t np = ctx->n_pad;
  const cplx* X = ps.S;
  if (ps.p > 0) {
    const int p = ps.p, pr = p * r;
    cplx* x = ctx->tall_tmp;
    RET(copy_cols(ctx, X, x, r_sub));
    RET(orth_robust(ctx, np, ps.V, np, pr, x, np, r_sub, ctx->owW, ctx->owR));
    k_block_fro2<<<p + 1, 256, 0, ctx->stream>>>(pr, r_sub, r, ctx->owW, ctx->owR, ps.norms);
    RET(check_launch(ctx, "k_block_fro2"));
    std::vector<double> f((size_t)p + 1);
    RET(d2h(ctx, f.data(), ps.norms, f.size()));
    const double rho2 = f[(size_t)p];
    const double res0 = std::sqrt(rho2);
    int l = 0;
    if (!force_add) {
      const int l_max = std::min(p - 1, p + 1 - ps.p_min);
      l = l_max;
      double acc = rho2;
      for (int i = 1; i <= l_max + 1; ++i) {
        acc += f[(size_t)i - 1];
        if (std::sqrt(acc) / res0 > tau) {
          l = i - 1;
          break;
        }
      }
    }
    if (l > 0) RET(pred_shift_blocks(ctx, l));
    if (l == 0 && p == ps.p_max) RET(pred_shift_blocks(ctx, 1));
  }
  RET(pred_add_blocks(ctx, X, z));
  return pred_block_update(ctx);
}

}  // namespace

namespace {

// The generic LOBPCG's scratch for blocks of up to k3 = 3r columns (grown, never shrunk).
int lob_scratch(rls_ctx* ctx, int k3) {
  PrecState& ps = *ctx->prec;
  const int64_t np = ctx->n_pad;
  if (ps.qcap < k3) {
    for (cplx** a : {&ps.qW, &ps.qRinv, &ps.qRtot, &ps.qRG, &ps.qws}) {
      dfree(ctx, *a);
      *a = nullptr;
    }
    dfree(ctx, ps.norms);
    ps.norms = nullptr;
    for (cplx** a : {&ps.qW, &ps.qRinv, &ps.qRtot, &ps.qRG}) RET(dalloc_t(ctx, a, (size_t)k3 * k3));
    RET(dalloc_t(ctx, &ps.qws, (size_t)2 * k3 * k3));
    RET(dalloc_t(ctx, &ps.norms, (size_t)k3 + 8));
    ps.qcap = k3;
  }
  const int oc = std::max((k3 + 2) / 3, 8);
  if (ps.opt_cols < oc || ps.opt_np != np) {
    dfree(ctx, ps.opt1);
    dfree(ctx, ps.opt2);
    ps.opt1 = ps.opt2 = nullptr;
    RET(dalloc_t(ctx, &ps.opt1, (size_t)np * oc));
    RET(dalloc_t(ctx, &ps.opt2, (size_t)np * oc));
    ps.opt_cols = oc;
    ps.opt_np = np;
  }
  return RLS_OK;
}

// Device memory of the prediction stage and the operator temporaries (allocated once per
// (n, r_pred, p_pred), reused by every grid point).
int prec_alloc(rls_ctx* ctx, int r, int p_max) {
  PrecState& ps = *ctx->prec;
  if (ps.V && ps.r == r && ps.p_max == p_max && ps.n == ctx->n) return RLS_OK;
  ps.drop_graphs();          // they hold the old arrays' addresses
  for (cplx** a : {&ps.V, &ps.J1, &ps.J2, &ps.J3, &ps.J4, &ps.J5, &ps.J6, &ps.L, &ps.H1, &ps.H2, &ps.H3, &ps.Hs,
                   &ps.hA, &ps.Ulist, &ps.rot_ws, &ps.S, &ps.CS, &ps.G, &ps.R, &ps.E, &ps.X0, &ps.bS, &ps.bCS, &ps.bG,
                   &ps.bR, &ps.bX0, &ps.hv[0], &ps.hv[1], &ps.hy, &ps.hpart, &ps.htau, &ps.hG, &ps.gram, &ps.grinv,
                   &ps.chol_ws, &ps.coef, &ps.coef2, &ps.hz}) {
    dfree(ctx, *a);
    *a = nullptr;
  }
  for (double** a : {&ps.sig, &ps.lam, &ps.bsig, &ps.blam, &ps.hd, &ps.he, &ps.he2, &ps.hlu}) {
    dfree(ctx, *a);
    *a = nullptr;
  }
  const int64_t np = ctx->n_pad;
  const int prm = r * p_max, r3 = 3 * r;
  ps.r = r;
  ps.p_max = p_max;
  ps.pr_max = prm;
  ps.n = ctx->n;
  for (cplx** a : {&ps.V, &ps.J1, &ps.J2, &ps.J3, &ps.J4, &ps.J5, &ps.J6}) RET(dalloc_t(ctx, a, (size_t)np * prm));
  for (cplx** a : {&ps.L, &ps.H1, &ps.H2, &ps.H3, &ps.Hs, &ps.hA}) RET(dalloc_t(ctx, a, (size_t)prm * prm));
  RET(dalloc_t(ctx, &ps.Ulist, (size_t)std::max(p_max - 1, 1) * 4 * r * r));
  RET(dalloc_t(ctx, &ps.rot_ws, (size_t)prm * r + (size_t)2 * r * r + (size_t)4 * r * r + 3 * (size_t)r + 64));
  RET(dalloc_t(ctx, &ps.S, (size_t)np * r3));
  RET(dalloc_t(ctx, &ps.CS, (size_t)np * r3));
  RET(dalloc_t(ctx, &ps.G, (size_t)r3 * r3));
  RET(dalloc_t(ctx, &ps.R, (size_t)r3 * r3));
  RET(dalloc_t(ctx, &ps.sig, (size_t)r3));
  RET(dalloc_t(ctx, &ps.lam, (size_t)std::max(r3, prm)));
  RET(dalloc_t(ctx, &ps.E, (size_t)np * r));
  RET(dalloc_t(ctx, &ps.X0, (size_t)np * r));
  RET(dalloc_t(ctx, &ps.bS, (size_t)np * 3));
  RET(dalloc_t(ctx, &ps.bCS, (size_t)np * 3));
  RET(dalloc_t(ctx, &ps.bG, 9));
  RET(dalloc_t(ctx, &ps.bR, 9));
  RET(dalloc_t(ctx, &ps.bX0, (size_t)np));
  RET(dalloc_t(ctx, &ps.bsig, 3));
  RET(dalloc_t(ctx, &ps.blam, 3));
  RET(dalloc_t(ctx, &ps.hv[0], (size_t)prm));
  RET(dalloc_t(ctx, &ps.hv[1], (size_t)prm));
  RET(dalloc_t(ctx, &ps.hy, (size_t)prm));
  RET(dalloc_t(ctx, &ps.hpart, (size_t)148 * 2));
  RET(dalloc_t(ctx, &ps.htau, (size_t)prm));
  RET(dalloc_t(ctx, &ps.hd, (size_t)prm));
  RET(dalloc_t(ctx, &ps.he, (size_t)prm));
  RET(dalloc_t(ctx, &ps.he2, (size_t)prm));
  RET(dalloc_t(ctx, &ps.hlu, (size_t)16 * 6 * prm));
  RET(dalloc_t(ctx, &ps.hG, (size_t)prm * r));
  RET(dalloc_t(ctx, &ps.hz, 1));
  RET(dalloc_t(ctx, &ps.gram, (size_t)r * r));
  RET(dalloc_t(ctx, &ps.grinv, (size_t)r * r));
  RET(dalloc_t(ctx, &ps.chol_ws, (size_t)r * r));
  RET(dalloc_t(ctx, &ps.coef, (size_t)r * 8 * 16));
  RET(dalloc_t(ctx, &ps.coef2, (size_t)r * 8 * 16));
  return lob_scratch(ctx, std::max(r3, p_max + 2));
}

// X (n × k, host, may be null) into the device block D (ld n_pad): copied, or the fixed
// uniform [0, 1) sequence that stands for rand!.
int fill_x0(rls_ctx* ctx, const rls_c64* X0, int k, cplx* D, uint64_t seed) {
  const int64_t np = ctx->n_pad;
  if (X0) {
    CK(cudaMemsetAsync(D, 0, sizeof(cplx) * np * k, ctx->stream));
    CK(cudaMemcpy2DAsync(D, np * sizeof(cplx), X0, ctx->n * sizeof(cplx), ctx->n * sizeof(cplx), k,
                         cudaMemcpyHostToDevice, ctx->stream));
  } else {
    dim3 grid((unsigned)((np + 255) / 256), k);
    k_fill_rand<<<grid, 256, 0, ctx->stream>>>(ctx->n, np, k, D, seed);
    RET(check_launch(ctx, "k_fill_rand"));
  }
  return RLS_OK;
}

// _get_pred_precond! (psPrecRecy.jl:436-462): the IC factor of the shifted normal matrix at z
// (host, rls_ic_factor), uploaded; then λ_n = ‖Cz·invF‖₂² and γ = ‖L⁻¹‖₂ by r = 1 LOBPCG
// runs on the device (_compute_λ_n, _compute_γ, :388-422).
int prec_build(rls_ctx* ctx, const rls_psprecrecy_control* c, cplx z) {
  PrecState& ps = *ctx->prec;
  const int64_t n = ps.n;
  const int64_t lsz = std::min<int64_t>(std::max<int64_t>(0, c->hsl_icntl_1), n - 1);
  const int64_t cap = n + lsz * n;
  std::vector<int64_t> lcol((size_t)n + 1), lrow((size_t)std::max<int64_t>(cap, 1)), invp((size_t)n);
  std::vector<rls_c64> lval((size_t)std::max<int64_t>(cap, 1));
  double shift_used = 0.0;
  int st = rls_ic_factor(n, ps.colptr.data(), ps.rowval.data(), ps.nzval.data(), 0, rls_c64{z.x, z.y}, c->hsl_tol,
                         c->hsl_cntl_1, c->hsl_cntl_2, c->hsl_icntl_1, c->hsl_icntl_2, ps.p0.data(), cap,
                         lcol.data(), lrow.data(), lval.data(), invp.data(), &shift_used);
  if (st != RLS_OK) {
    set_err(ctx, "get_hsl_LLTP at z = %g%+gi: %s", z.x, z.y, rls_last_error(nullptr));
    return st;
  }
  RET(rls_lltp_upload(ctx, n, lcol.data(), lrow.data(), lval.data(), ps.p0.data(), invp.data(), 0));
  const int64_t np = ctx->n_pad;
  LobKeep kb{ps.bS, ps.bCS, ps.bG, ps.bR, ps.bsig, ps.blam, 1};
  LobCtl cl;
  cl.sideL = true;
  cl.normC = 1.0;
  cl.conv_first = cl.conv_last = 1;
  double sig_n = 0.0, gamma = 0.0;
  int64_t it = 0;
  cl.tol = c->lambda_n_tol;
  CK(cudaMemcpyAsync(ps.bS, ps.bX0, sizeof(cplx) * np, cudaMemcpyDeviceToDevice, ctx->stream));
  const DevOp pred = op_pred(ctx, z);
  RET(lobpcg_gen(ctx, pred, nullptr, kb, cl, &sig_n, &it));
  cl.tol = c->gamma_tol;
  CK(cudaMemcpyAsync(ps.bS, ps.bX0, sizeof(cplx) * np, cudaMemcpyDeviceToDevice, ctx->stream));
  const DevOp il = op_invL(ctx);
  RET(lobpcg_gen(ctx, il, nullptr, kb, cl, &gamma, &it));
  ps.lam_dagger_n = sig_n * sig_n;
  ps.gamma = gamma;
  return RLS_OK;
}

int check_prec_control(rls_ctx* ctx, const rls_psprecrecy_control* c) {
  auto bad = [&](const char* what) {
    set_err(ctx, "rls_psprecrecy: %s", what);
    return RLS_ERR_ARG;
  };
  if (c->r_main < 1 || c->r_main > 8) return bad("r_main must be in 1..8");
  if (c->r_pred < 1 || c->r_pred > 40) return bad("r_pred must be in 1..40");
  if (c->p_main < 1 || c->p_pred < 1 || c->p_pred * c->r_pred > 800 || c->p_main * c->r_main > 360)
    return bad("p_pred·r_pred must be <= 800 and p_main·r_main <= 360");
  if (c->p_min_main < 0 || c->p_min_main > c->p_main || c->p_min_pred < 0 || c->p_min_pred > c->p_pred)
    return bad("p_min must satisfy 0 <= p_min <= p_max");
  if (!c->main_implict_recycle || c->main_implict_update)
    return bad("only main_implict_recycle = true, main_implict_update = false is implemented");
  if (!c->pred_implict_recycle || !c->pred_implict_update)
    return bad("only pred_implict_recycle = true, pred_implict_update = true is implemented");
  if (c->pred_orth_type != 0 && c->pred_orth_type != 1) return bad("pred_orth_type must be :lapack or :shiftchol");
  if (c->pred_conv_thresh_type != 0 && c->pred_conv_thresh_type != 1) return bad("pred_conv_thresh_type must be 0 or 1");
  if (c->pred_conv_first >= 1 && !(c->pred_conv_first <= c->pred_conv_last && c->pred_conv_last <= c->r_pred))
    return bad("pred_conv_range must satisfy 1 <= first <= last <= r_pred");
  if (c->hsl_icntl_1 < 1) return bad("hsl_icntl_1 (lsize) must be at least 1");
  return RLS_OK;
}

}  // namespace

extern "C" int rls_psprecrecy_range(rls_ctx* ctx, int64_t n, const int64_t* colptr, const int64_t* rowval,
                                    const rls_c64* nzval, int base, const int64_t* p, const rls_c64* Z, int64_t nZ,
                                    const rls_grid* g, const rls_psprecrecy_control* c, const rls_c64* X0_main,
                                    const rls_c64* X0_pred, const rls_c64* X0_bound, int64_t i_begin, int64_t i_end,
                                    double* sigma_min, rls_psprecrecy_stats* st) {
  if (!ctx) return RLS_ERR_ARG;
  if (!Z || !g || !c || !sigma_min || nZ < 1 || i_begin < 0 || i_end < i_begin || i_end > nZ) {
    set_err(ctx, "rls_psprecrecy: invalid arguments");
    return RLS_ERR_ARG;
  }
  if (g->n_x < 2 || g->n_y < 2 || g->k < 1) {
    set_err(ctx, "rls_psprecrecy: invalid grid");
    return RLS_ERR_ARG;
  }
  RET(check_prec_control(ctx, c));
  CK(cudaSetDevice(ctx->device));
  ctx->grad_on = false;
  const int rm = (int)c->r_main, rp = (int)c->r_pred;
  rls_psprecrecy_stats dummy{};
  if (!st) st = &dummy;
  if (!ctx->prec) ctx->prec = new PrecState();
  PrecState& ps = *ctx->prec;
  if (i_begin == 0) {
    if (n < 2 || !colptr || !rowval || !nzval || (base != 0 && base != 1)) {
      set_err(ctx, "rls_psprecrecy: C must be a square CSC of order >= 2 with base 0 or 1");
      return RLS_ERR_ARG;
    }
    if (ctx->T && ctx->n != n && !ctx->band.on) {
      set_err(ctx, "rls_psprecrecy: the context holds a Schur operator of order %lld", (long long)ctx->n);
      return RLS_ERR_STATE;
    }
    // host copy of C (0-based, rows sorted and summed per column as SparseMatrixCSC keeps them)
    const int64_t nnz = colptr[n] - base;
    if (nnz < 0 || colptr[0] != base) {
      set_err(ctx, "rls_psprecrecy: invalid colptr");
      return RLS_ERR_ARG;
    }
    ps.colptr.assign((size_t)n + 1, 0);
    ps.rowval.resize((size_t)nnz);
    ps.nzval.resize((size_t)nnz);
    for (int64_t j = 0; j <= n; ++j) ps.colptr[(size_t)j] = colptr[j] - base;
    for (int64_t q = 0; q < nnz; ++q) {
      ps.rowval[(size_t)q] = rowval[q] - base;
      ps.nzval[(size_t)q] = nzval[q];
      if (ps.rowval[(size_t)q] < 0 || ps.rowval[(size_t)q] >= n) {
        set_err(ctx, "rls_psprecrecy: row index out of range");
        return RLS_ERR_DIM;
      }
    }
    ps.p0.resize((size_t)n);
    std::vector<char> seen((size_t)n, 0);
    for (int64_t i = 0; i < n; ++i) {
      const int64_t v = p ? p[i] - base : i;
      if (v < 0 || v >= n || seen[(size_t)v]) {
        set_err(ctx, "rls_psprecrecy: p is not a permutation of 1..n");
        return RLS_ERR_ARG;
      }
      seen[(size_t)v] = 1;
      ps.p0[(size_t)i] = v;
    }
    RET(rls_sparse_upload_csc(ctx, n, n, ps.colptr.data(), ps.rowval.data(), ps.nzval.data(), 0));
    if (!ctx->T) {
      ctx->n = n;
      ctx->n_pad = (n + 63) / 64 * 64;
      drop_lob_graph(ctx);
      dfree(ctx, ctx->colpart);     // per-CTA partial sums of the recycle step, sized by n_pad
      ctx->colpart = nullptr;
      RET(dalloc_t(ctx, &ctx->colpart, (size_t)(ctx->n_pad / 32 + 64)));
    }
    ctx->op_sparse = true;
    ctx->scratch_cols = std::max(rp * (int)c->p_pred, 3 * rp);
    RET(setup_space(ctx, rm, (int)c->p_main));
    RET(prec_alloc(ctx, rp, (int)c->p_pred));
    ps.p = 0;
    ps.p_min = (int)c->p_min_pred;
    ps.pts.assign((size_t)c->p_pred, rls_c64{0, 0});
    RET(upload_x0(ctx, X0_main, rm));
    RET(fill_x0(ctx, X0_pred, rp, ps.X0, 20260319ull));
    RET(fill_x0(ctx, X0_bound, 1, ps.bX0, 20260320ull));
    CK(cudaMemcpyAsync(ps.S, ps.X0, sizeof(cplx) * ctx->n_pad * rp, cudaMemcpyDeviceToDevice, ctx->stream));
    CK(cudaMemsetAsync(ps.E, 0, sizeof(cplx) * ctx->n_pad * rp, ctx->stream));
    double thresh = c->recycle_fail_dist_thresh;
    if (!std::isfinite(thresh)) {
      const double dx = std::fabs(g->x_ed - g->x_st) / (double)(g->n_x - 1);
      const double dy = std::fabs(g->y_ed - g->y_st) / (double)(g->n_y - 1);
      thresh = 1.01 * std::max(dx, dy);
    } else if (thresh < 0) {
      set_err(ctx, "recycle_fail_dist_thresh must be nonnegative, got %g", thresh);
      return RLS_ERR_ARG;
    }
    ps.thresh = thresh;
    ps.active = true;
    ps.next = 0;
    ps.nZ = nZ;
    ps.have_failed_main = ps.have_failed_pred = false;
    ps.lam_lower = ps.lam_upper = 0.0;
    ctx->spec_cur = std::min(8, ctx->spec_max);
    st->main_recycle_time_ns = st->main_refine_time_ns = st->main_update_time_ns = 0;
    st->pred_recycle_time_ns = st->pred_refine_time_ns = st->pred_update_time_ns = st->precond_time_ns = 0;
    st->n_it = st->n_pred_it = st->n_pts = st->n_pred_pts = st->n_precond_rebuild_pts = 0;
    // construct the preconditioner at z† = rec.Z[1] (:650-657)
    ps.z_dagger = cmk(Z[0].re, Z[0].im);
    const uint64_t t0 = now_ns();
    RET(prec_build(ctx, c, ps.z_dagger));
    st->precond_time_ns += now_ns() - t0;
    if (st->precond_rebuild_pts) st->precond_rebuild_pts[0] = Z[0];
    st->n_precond_rebuild_pts = 1;
    if (ctx->verbose >= 1)
      emit_log(ctx, "[pred-precond:init] z=%10.6f%+10.6fim λ_n=%9.3e γ=%9.3e", ps.z_dagger.x, ps.z_dagger.y,
               ps.lam_dagger_n, ps.gamma);
  } else if (!ps.active || ps.next != i_begin || ps.nZ != nZ || ctx->r != rm || ps.r != rp) {
    set_err(ctx, "range call does not continue the previous one (expected i_begin=%lld)", (long long)ps.next);
    return RLS_ERR_STATE;
  }
  const int64_t np = ctx->n_pad;
  auto record_precond = [&](rls_c64 z) {   // _record_pred_precond_point! (:352-366)
    const int64_t k = st->n_precond_rebuild_pts;
    if (k > 0 && st->precond_rebuild_pts && st->precond_rebuild_pts[k - 1].re == z.re &&
        st->precond_rebuild_pts[k - 1].im == z.im)
      return;
    if (st->precond_rebuild_pts) st->precond_rebuild_pts[k] = z;
    st->n_precond_rebuild_pts = k + 1;
  };
  auto main_ok = [&](double w0, double s0) {   // check_conv_svd type 0 on column 1 (:707-713)
    return w0 < std::max(c->main_normC * s0 * c->tol, c->main_normC * c->main_normC * std::sqrt(2.0) * kEps);
  };
  auto zero_counts = [&](int64_t i) {
    if (st->main_M_vec_apps) st->main_M_vec_apps[i] = 0;
    if (st->main_M_vec_apps_no_recycle) st->main_M_vec_apps_no_recycle[i] = 0;
    if (st->main_L_vec_apps) st->main_L_vec_apps[i] = 0;
    if (st->pred_M_vec_apps) st->pred_M_vec_apps[i] = 0;
    if (st->pred_L_vec_apps) st->pred_L_vec_apps[i] = 0;
    if (st->main_refine_it) st->main_refine_it[i] = 0;
    if (st->pred_refine_it) st->pred_refine_it[i] = 0;
  };
  auto accept = [&](int64_t i, double s0, int rr) {
    sigma_min[i] = s0;
    zero_counts(i);
    if (ctx->verbose >= 1)
      emit_log(ctx, "[%4lld/%4lld] z=%9.4f%+9.4fim | main: state=%-12s p=%3d r_svdrr=%3d σ=%9.3e",
               (long long)(i + 1), (long long)nZ, Z[i].re, Z[i].im, "recycled", ctx->p, rr, s0);
  };
  const int upd_m = 3 * rp, upd_l = 5 * rp;    // _psPrecRecy_pred_update_ml_apps, implicit (:82-105)
  // pred refine: lobpcgSvd(Cz_pred, X_pred, I, keep_pred, control_pred) (:780-788)
  auto pred_refine = [&](cplx z, int conv_last, double normC, int64_t* it) -> int {
    LobKeep kp{ps.S, ps.CS, ps.G, ps.R, ps.sig, ps.lam, rp};
    LobCtl cl;
    cl.sideL = false;
    cl.normC = normC;
    cl.tol = c->tol_pred * c->lobpcg_pred_tol_scale;
    cl.orth = (int)c->pred_orth_type;
    cl.conv_type = (int)c->pred_conv_thresh_type;
    cl.conv_first = 1;
    cl.conv_last = conv_last;
    double s = 0.0;
    const DevOp op = op_pred(ctx, z);
    return lobpcg_gen(ctx, op, nullptr, kp, cl, &s, it);
  };
  auto pred_idx = [&](int* idx) -> int {    // something(findlast(<(cutoff), λ[1:r]), r) (:752)
    std::vector<double> lam((size_t)rp);
    RET(d2h(ctx, lam.data(), ps.lam, (size_t)rp));
    *idx = rp;
    for (int j = rp - 1; j >= 0; --j)
      if (lam[(size_t)j] < c->idx_cutoff_pred) {
        *idx = j + 1;
        break;
      }
    return RLS_OK;
  };
  auto lam_at = [&](int j, double* v) -> int { return d2h(ctx, v, ps.lam + j, 1); };

  // Refine point i: the prediction stage, the two-level preconditioner, the main LOBPCG and
  // the main update (psPrecRecy.jl:725-991).
  auto refine = [&](int64_t i, int r_svdrr) -> int {
    const cplx z = cmk(Z[i].re, Z[i].im);
    const double dz = std::hypot(z.x - ps.z_dagger.x, z.y - ps.z_dagger.y);
    const double pred_normC = std::sqrt(ps.lam_dagger_n) + ps.gamma * dz;
    int64_t pM = 0, pL = 0, pit_total = 0;
    int idx_pred = rp;
    bool pred_recycled = false, pred_refined = false;
    if (ps.p > 0) {   // RecyProjSpace (:744-764)
      const uint64_t t0 = now_ns();
      RET(pred_rayl_ritz(ctx, z));
      RET(pred_idx(&idx_pred));
      std::vector<double> nrm((size_t)idx_pred);
      RET(col_norms(ctx, ps.S + np * rp, np, idx_pred, nrm.data()));
      const double th = std::max(pred_normC * pred_normC * c->tol_pred,
                                 pred_normC * pred_normC * std::sqrt(2.0) * kEps);
      pred_recycled = true;
      for (double v : nrm)
        if (!(v < th)) { pred_recycled = false; break; }
      st->pred_recycle_time_ns += now_ns() - t0;
    }
    if (pred_recycled) {
      RET(spmm_dev(ctx, cneg(z), 0, rp, ps.E, np, ps.CS, np));   // CX_pred = Cz·E_pred (:770)
      pM += rp;
      RET(lam_at(rp - 1, &ps.lam_lower));
    } else {
      pred_refined = true;
      const uint64_t t1 = now_ns();
      int64_t it = 0;
      RET(pred_refine(z, idx_pred, pred_normC, &it));
      st->pred_refine_time_ns += now_ns() - t1;
      st->n_pred_it += it;
      pit_total += it;
      const int64_t ops = it > 0 ? 2 * (it + 1) * rp : 0;
      const uint64_t t2 = now_ns();
      const bool force = ps.have_failed_pred &&
                         std::hypot(z.x - ps.last_failed_pred.re, z.y - ps.last_failed_pred.im) <= ps.thresh;
      RET(pred_update(ctx, z, c->pred_tau, idx_pred, force));
      RET(invF_mul(ctx, rp, ps.S, ps.E));                         // E_pred = invF·X_pred (:815)
      st->pred_update_time_ns += now_ns() - t2;
      pM += ops + upd_m;
      pL += ops + upd_l + rp;
      RET(lam_at(rp - 1, &ps.lam_lower));
    }
    ps.lam_upper = pred_normC * pred_normC;
    if (ps.lam_lower < c->lambda_lower_min || ps.lam_upper > c->lambda_upper_max) {   // rebuild (:825-908)
      record_precond(Z[i]);
      const uint64_t t0 = now_ns();
      RET(prec_build(ctx, c, z));
      st->precond_time_ns += now_ns() - t0;
      if (ctx->verbose >= 1)
        emit_log(ctx, "[pred-precond:rebuild] z=%10.6f%+10.6fim λ_n=%9.3e γ=%9.3e", z.x, z.y, ps.lam_dagger_n,
                 ps.gamma);
      ps.p = 0;
      CK(cudaMemcpyAsync(ps.S, ps.X0, sizeof(cplx) * np * rp, cudaMemcpyDeviceToDevice, ctx->stream));
      ps.lam_upper = ps.lam_dagger_n;
      pred_refined = true;
      const uint64_t t1 = now_ns();
      int64_t it = 0;
      RET(pred_refine(z, rp, std::sqrt(ps.lam_dagger_n), &it));
      st->pred_refine_time_ns += now_ns() - t1;
      st->n_pred_it += it;
      pit_total += it;
      const int64_t ops = it > 0 ? 2 * (it + 1) * rp : 0;
      RET(pred_idx(&idx_pred));
      const uint64_t t2 = now_ns();
      const bool force = ps.have_failed_pred &&
                         std::hypot(z.x - ps.last_failed_pred.re, z.y - ps.last_failed_pred.im) <= ps.thresh;
      RET(pred_update(ctx, z, c->pred_tau, idx_pred, force));
      RET(invF_mul(ctx, rp, ps.S, ps.E));
      st->pred_update_time_ns += now_ns() - t2;
      pM += ops + upd_m;
      pL += ops + upd_l + rp;
      RET(lam_at(rp - 1, &ps.lam_lower));
      ps.z_dagger = z;
    }
    if (st->pred_p_count) st->pred_p_count[i] = ps.p;
    if (pred_refined) {
      if (st->pred_pts) st->pred_pts[st->n_pred_pts] = Z[i];
      st->n_pred_pts += 1;
      ps.have_failed_pred = true;
      ps.last_failed_pred = Z[i];
    }
    // two-level preconditioner (_get_pred_precond_ad!, :465-485)
    const uint64_t tp = now_ns();
    RET(gram(ctx, np, ps.CS, np, rp, ps.CS, np, rp, ps.gram, rp));
    k_chol_plain<<<1, 256, 0, ctx->stream>>>(rp, ps.gram, nullptr, ps.grinv, ps.chol_ws, ctx->derr);
    RET(check_launch(ctx, "k_chol_plain"));
    st->precond_time_ns += now_ns() - tp;
    // main solve (:923-945): lobpcgSvd(Cz, X_main, K_ad, keep_main, control_main)
    const uint64_t t3 = now_ns();
    LobKeep km{ctx->S, ctx->CS, ctx->Gk, ctx->Rk, ctx->sig, ctx->lam, rm};
    LobCtl cm;
    cm.sideL = false;
    cm.normC = c->main_normC;
    cm.tol = c->lobpcg_tol_scale * c->tol;
    cm.orth = 0;
    cm.conv_type = 0;
    cm.conv_first = cm.conv_last = 1;
    const DevOp cz = op_shifted(ctx, z);
    const std::function<int(cplx*, int)> kad = [ctx](cplx* W, int b) { return ldiv_ad(ctx, W, b); };
    double s = 0.0;
    int64_t it = 0;
    RET(lobpcg_gen(ctx, cz, &kad, km, cm, &s, &it));
    st->main_refine_time_ns += now_ns() - t3;
    sigma_min[i] = s;
    st->n_it += it;
    if (st->pts) st->pts[st->n_pts] = Z[i];
    st->n_pts += 1;
    int64_t mM = 0, mL = 0;
    if (it > 0) {
      mM = 2 * (it + 1) * rm;
      mL = 2 * it * rm;
      const uint64_t t4 = now_ns();
      const bool force = ps.have_failed_main &&
                         std::hypot(z.x - ps.last_failed_main.re, z.y - ps.last_failed_main.im) <= ps.thresh;
      RET(update_recycled_space(ctx, z, ctx->S, c->main_tau, force, (int)c->p_min_main));
      RET(sync_and_check(ctx));
      st->main_update_time_ns += now_ns() - t4;
      mM += 3 * rm;
    }
    ps.have_failed_main = true;
    ps.last_failed_main = Z[i];
    if (st->main_M_vec_apps) st->main_M_vec_apps[i] = mM;
    if (st->main_M_vec_apps_no_recycle) st->main_M_vec_apps_no_recycle[i] = mM;
    if (st->main_L_vec_apps) st->main_L_vec_apps[i] = mL;
    if (st->pred_M_vec_apps) st->pred_M_vec_apps[i] = pM;
    if (st->pred_L_vec_apps) st->pred_L_vec_apps[i] = pL;
    if (st->main_refine_it) st->main_refine_it[i] = it;
    if (st->pred_refine_it) st->pred_refine_it[i] = pit_total;
    if (ctx->verbose >= 1) {
      char state[32];
      snprintf(state, sizeof state, "refine(%lld)", (long long)it);
      emit_log(ctx, "[%4lld/%4lld] z=%9.4f%+9.4fim | main: state=%-12s p=%3d r_svdrr=%3d σ=%9.3e", (long long)(i + 1),
               (long long)nZ, z.x, z.y, state, ctx->p, r_svdrr, s);
      emit_log(ctx, "%35s| pred: state=%-12s p=%3d λ_upper=%9.4f λ_lower=%9.4f", "",
               pred_recycled ? "recycled" : "refine", ps.p, ps.lam_upper, ps.lam_lower);
    }
    return RLS_OK;
  };

  int64_t i = i_begin;
  while (i < i_end) {
    if (st->p_count) st->p_count[i] = ctx->p;
    if (st->pred_p_count) st->pred_p_count[i] = ps.p;
    if (st->r_recy) st->r_recy[i] = 0;
    if (ctx->p == 0) {
      RET(refine(i, 0));
      ps.next = ++i;
      continue;
    }
    // main recycle steps, speculatively batched: an accepted point changes nothing, so the
    // points up to the first rejection are exactly those of the sequential loop
    const int B = (int)std::min<int64_t>(std::min(ctx->spec_cur, ctx->spec_max), i_end - i);
    cplx zs[BATCH_MAX];
    double taus[BATCH_MAX], sig0[BATCH_MAX], w0[BATCH_MAX];
    int rr[BATCH_MAX];
    int nb = 0;
    const uint64_t t0 = now_ns();
    if (B >= 2) {
      for (int b = 0; b < B; ++b) {
        zs[b] = cmk(Z[i + b].re, Z[i + b].im);
        taus[b] = c->gap_tau;
      }
      RET(recycle_batch(ctx, B, zs, taus, c->shift, rr, sig0, w0, nullptr));
      nb = B;
    }
    st->main_recycle_time_ns += now_ns() - t0;
    int b = 0;
    bool failed = false;
    for (; b < nb; ++b) {
      if (rr[b] == 0) break;    // Ritz dimension beyond the batch path: per point below
      if (st->p_count) st->p_count[i + b] = ctx->p;
      if (st->pred_p_count) st->pred_p_count[i + b] = ps.p;
      if (st->r_recy) st->r_recy[i + b] = rr[b];
      if (main_ok(w0[b], sig0[b])) {
        accept(i + b, sig0[b], rr[b]);
        continue;
      }
      failed = true;
      break;
    }
    if (failed) {
      const cplx* xw = ctx->bXW + (int64_t)b * 2 * np * rm;
      CK(cudaMemcpyAsync(ctx->S, xw, sizeof(cplx) * 2 * np * rm, cudaMemcpyDeviceToDevice, ctx->stream));
      RET(refine(i + b, rr[b]));
      i += b + 1;
      ctx->spec_cur = std::max(4, std::min(ctx->spec_max, b + 4));
    } else if (nb > 0 && b == nb) {
      i += b;
      ctx->spec_cur = std::min(ctx->spec_max, 2 * ctx->spec_cur);
    } else {
      i += b;
      const cplx z = cmk(Z[i].re, Z[i].im);
      if (st->p_count) st->p_count[i] = ctx->p;
      if (st->pred_p_count) st->pred_p_count[i] = ps.p;
      const uint64_t t1 = now_ns();
      RecycleResult rres{};
      RET(recycle_step(ctx, z, c->shift, c->gap_tau, &rres));
      st->main_recycle_time_ns += now_ns() - t1;
      if (st->r_recy) st->r_recy[i] = rres.rr;
      if (main_ok(rres.w0norm, rres.sigma0)) accept(i, rres.sigma0, rres.rr);
      else RET(refine(i, rres.rr));
      ++i;
    }
    ps.next = i;
  }
  ps.next = i;
  if (i_end == nZ) ps.active = false;
  return sync_and_check(ctx);
}

extern "C" int rls_psprecrecy(rls_ctx* ctx, int64_t n, const int64_t* colptr, const int64_t* rowval,
                              const rls_c64* nzval, int base, const int64_t* p, const rls_c64* Z, int64_t nZ,
                              const rls_grid* g, const rls_psprecrecy_control* c, const rls_c64* X0_main,
                              const rls_c64* X0_pred, const rls_c64* X0_bound, double* sigma_min,
                              rls_psprecrecy_stats* st) {
  return rls_psprecrecy_range(ctx, n, colptr, rowval, nzval, base, p, Z, nZ, g, c, X0_main, X0_pred, X0_bound, 0, nZ,
                              sigma_min, st);
}

extern "C" int rls_lobpcg_svd(rls_ctx* ctx, int op, rls_c64 z, int prec, const rls_c64* X0,
                              const rls_lobpcg_control* c, rls_c64* X_out, double* sigma_r, double* sigma,
                              int64_t* it) {
  if (!ctx || !c) return RLS_ERR_ARG;
  if (op < RLS_OP_INV_SCHUR || op > RLS_OP_INV_L || prec < RLS_PREC_NONE || prec > RLS_PREC_LLTP) {
    set_err(ctx, "rls_lobpcg_svd: unknown operator %d or preconditioner %d", op, prec);
    return RLS_ERR_ARG;
  }
  if (c->r < 1 || c->r > 40 || c->maxit < 0) {
    set_err(ctx, "rls_lobpcg_svd: block size r=%lld outside 1..40", (long long)c->r);
    return RLS_ERR_ARG;
  }
  if (!(1 <= c->conv_first && c->conv_first <= c->conv_last && c->conv_last <= c->r)) {
    set_err(ctx, "conv_range must satisfy 1 <= first <= last <= r");
    return RLS_ERR_ARG;
  }
  if ((c->side != 'L' && c->side != 'S') || (c->orth_type != 0 && c->orth_type != 1) ||
      (c->conv_thresh_type != 0 && c->conv_thresh_type != 1)) {
    set_err(ctx, "rls_lobpcg_svd: side must be 'L' or 'S', orth_type :lapack or :shiftchol, conv_thresh_type 0 or 1");
    return RLS_ERR_ARG;
  }
  CK(cudaSetDevice(ctx->device));
  const bool sparse_op = op != RLS_OP_INV_SCHUR;
  int64_t n = 0;
  if (!sparse_op) {
    if (!ctx->T) {
      set_err(ctx, "no Schur factor uploaded (call rls_set_schur first)");
      return RLS_ERR_STATE;
    }
    n = ctx->n;
  } else {
    if ((op == RLS_OP_SHIFTED || op == RLS_OP_PRED) && !ctx->sp[0].rowptr) {
      set_err(ctx, "no sparse matrix uploaded (call rls_sparse_upload_csc first)");
      return RLS_ERR_STATE;
    }
    if ((op == RLS_OP_PRED || op == RLS_OP_INV_L) && !ctx->lltp.op[0].rowptr) {
      set_err(ctx, "no preconditioner factor uploaded (call rls_lltp_upload first)");
      return RLS_ERR_STATE;
    }
    n = (op == RLS_OP_INV_L) ? ctx->lltp.n : ctx->sp[0].rows;
    if (ctx->sp[0].rowptr && (ctx->sp[0].rows != ctx->sp[0].cols || (op == RLS_OP_PRED && ctx->lltp.n != n))) {
      set_err(ctx, "rls_lobpcg_svd: the operator's factors have mismatched orders");
      return RLS_ERR_DIM;
    }
  }
  if (prec == RLS_PREC_LLTP && (!ctx->lltp.op[0].rowptr || ctx->lltp.n != n)) {
    set_err(ctx, "rls_lobpcg_svd: no preconditioner factor of order %lld uploaded", (long long)n);
    return RLS_ERR_STATE;
  }
  if (c->m != n || c->n != n) {
    set_err(ctx, "LobpcgSvdControl m, n (%lld, %lld) do not match the operator (%lld)", (long long)c->m,
            (long long)c->n, (long long)n);
    return RLS_ERR_DIM;
  }
  if (sparse_op && !ctx->T && ctx->n != n) {
    ctx->n = n;
    ctx->n_pad = (n + 63) / 64 * 64;
    drop_lob_graph(ctx);
    dfree(ctx, ctx->colpart);
    ctx->colpart = nullptr;
    RET(dalloc_t(ctx, &ctx->colpart, (size_t)(ctx->n_pad / 32 + 64)));
    release_space(ctx);
  } else if (sparse_op && ctx->T && ctx->n != n) {
    set_err(ctx, "rls_lobpcg_svd: the context holds a Schur operator of order %lld", (long long)ctx->n);
    return RLS_ERR_STATE;
  }
  const int r = (int)c->r;
  const int64_t np = ctx->n_pad;
  if (!ctx->prec) ctx->prec = new PrecState();
  PrecState& ps = *ctx->prec;
  ctx->scratch_cols = std::max(ctx->scratch_cols, 3 * r);
  if (!ctx->V || ctx->small_dim < 3 * r) RET(setup_space(ctx, ctx->r > 0 ? ctx->r : std::min(r, 8),
                                                         std::max(ctx->p_max, 1)));
  RET(lob_scratch(ctx, 3 * r));
  if (ps.lr != r || ps.l_np != np) {
    for (cplx** a : {&ps.lS, &ps.lCS, &ps.lG, &ps.lR}) {
      dfree(ctx, *a);
      *a = nullptr;
    }
    for (double** a : {&ps.lsig, &ps.llam}) {
      dfree(ctx, *a);
      *a = nullptr;
    }
    RET(dalloc_t(ctx, &ps.lS, (size_t)np * 3 * r));
    RET(dalloc_t(ctx, &ps.lCS, (size_t)np * 3 * r));
    RET(dalloc_t(ctx, &ps.lG, (size_t)9 * r * r));
    RET(dalloc_t(ctx, &ps.lR, (size_t)9 * r * r));
    RET(dalloc_t(ctx, &ps.lsig, (size_t)3 * r));
    RET(dalloc_t(ctx, &ps.llam, (size_t)3 * r));
    ps.lr = r;
    ps.l_np = np;
  }
  RET(fill_x0(ctx, X0, r, ps.lS, 20260321ull));
  const cplx zz = cmk(z.re, z.im);
  DevOp C;
  if (op == RLS_OP_INV_SCHUR) {
    C.mul = [ctx, zz](const cplx* X, cplx* Y, int b) { return trsm(ctx, zz, 1, X, Y, ctx->n_pad, b); };
    C.mul_adj = [ctx, zz](const cplx* X, cplx* Y, int b) { return trsm(ctx, zz, 0, X, Y, ctx->n_pad, b); };
  } else if (op == RLS_OP_SHIFTED) {
    C = op_shifted(ctx, zz);
  } else if (op == RLS_OP_PRED) {
    C = op_pred(ctx, zz);
  } else {
    C = op_invL(ctx);
  }
  const std::function<int(cplx*, int)> kl = [ctx](cplx* W, int b) {
    PrecState& p = *ctx->prec;
    RET(lltp_ldiv_dev(ctx, b, W, ctx->n_pad, p.opt1, ctx->n_pad));
    return copy_cols(ctx, p.opt1, W, b);
  };
  LobKeep k{ps.lS, ps.lCS, ps.lG, ps.lR, ps.lsig, ps.llam, r};
  LobCtl cl;
  cl.maxit = c->maxit;
  cl.tol = c->tol;
  cl.sideL = c->side == 'L';
  cl.normC = c->normC;
  cl.orth = c->orth_type;
  cl.conv_type = c->conv_thresh_type;
  cl.conv_first = (int)c->conv_first;
  cl.conv_last = (int)c->conv_last;
  double s = 0.0;
  int64_t its = 0;
  RET(lobpcg_gen(ctx, C, prec == RLS_PREC_LLTP ? &kl : nullptr, k, cl, &s, &its));
  if (X_out)
    CK(cudaMemcpy2DAsync(X_out, n * sizeof(cplx), ps.lS, np * sizeof(cplx), n * sizeof(cplx), r,
                         cudaMemcpyDeviceToHost, ctx->stream));
  if (sigma_r) CK(cudaMemcpyAsync(sigma_r, ps.lsig, r * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  RET(sync_and_check(ctx));
  if (sigma) *sigma = s;
  if (it) *it = its;
  return RLS_OK;
}

// ---- ∂σ/∂C on a sparsity pattern (the adjoint of σ with respect to C's entries) ------------

namespace {
// out[k] = Re(conj(Qu[rows[k]]) · Qv[cols[k]])  (Qu, Qv columns of QUV, ld ldq)
__global__ void k_grad_pattern(int64_t nnz, const int64_t* __restrict__ rows, const int64_t* __restrict__ cols,
                               int base, const cplx* __restrict__ Qu, const cplx* __restrict__ Qv, int64_t n,
                               double* out, int* err) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nnz; k += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = rows[k] - base, j = cols[k] - base;
    if (i < 0 || i >= n || j < 0 || j >= n) {
      atomicOr(err, DEVERR_SIZE);
      out[k] = 0.0;
      continue;
    }
    const cplx a = Qu[i], b = Qv[j];
    out[k] = a.x * b.x + a.y * b.y;          // Re(conj(a)·b)
  }
}
}  // namespace

extern "C" int rls_set_schur_vectors(rls_ctx* ctx, const rls_c64* Q, int64_t ldq) {
  if (!ctx) return RLS_ERR_ARG;
  if (!ctx->T) {
    set_err(ctx, "no Schur factor uploaded (call rls_set_schur first)");
    return RLS_ERR_STATE;
  }
  if (!Q || ldq < ctx->n) {
    set_err(ctx, "rls_set_schur_vectors: Q must be n × n with ldq >= n");
    return RLS_ERR_ARG;
  }
  CK(cudaSetDevice(ctx->device));
  if (!ctx->prec) ctx->prec = new PrecState();
  PrecState& ps = *ctx->prec;
  const int64_t np = ctx->n_pad, n = ctx->n;
  if (ps.Q_np != np) {
    dfree(ctx, ps.Qdev);
    dfree(ctx, ps.Qws);
    ps.Qdev = ps.Qws = nullptr;
    RET(dalloc_t(ctx, &ps.Qdev, (size_t)np * np));
    RET(dalloc_t(ctx, &ps.Qws, (size_t)4 * np));
    ps.Q_np = np;
  }
  CK(cudaMemsetAsync(ps.Qdev, 0, sizeof(cplx) * np * np, ctx->stream));
  CK(cudaMemcpy2DAsync(ps.Qdev, np * sizeof(cplx), Q, ldq * sizeof(cplx), n * sizeof(cplx), n,
                       cudaMemcpyHostToDevice, ctx->stream));
  ps.Q_n = n;
  return sync_and_check(ctx);
}

extern "C" int rls_sigma_grad_pattern(rls_ctx* ctx, const rls_c64* u, const rls_c64* v, int64_t nnz,
                                      const int64_t* rows, const int64_t* cols, int base, double* dsdC) {
  if (!ctx) return RLS_ERR_ARG;
  if (!ctx->prec || !ctx->prec->Qdev || ctx->prec->Q_n != ctx->n) {
    set_err(ctx, "no Schur vectors uploaded (call rls_set_schur_vectors first)");
    return RLS_ERR_STATE;
  }
  if (!u || !v || nnz < 0 || (nnz > 0 && (!rows || !cols || !dsdC)) || (base != 0 && base != 1)) {
    set_err(ctx, "rls_sigma_grad_pattern: invalid arguments");
    return RLS_ERR_ARG;
  }
  if (nnz == 0) return RLS_OK;
  CK(cudaSetDevice(ctx->device));
  if (!ctx->V) RET(setup_space(ctx, 1, 1));
  PrecState& ps = *ctx->prec;
  const int64_t np = ctx->n_pad, n = ctx->n;
  cplx* UV = ps.Qws;            // [u v] (Schur basis)
  cplx* QUV = ps.Qws + 2 * np;  // [Q u, Q v]
  CK(cudaMemsetAsync(UV, 0, sizeof(cplx) * 2 * np, ctx->stream));
  CK(cudaMemcpyAsync(UV, u, sizeof(cplx) * n, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(UV + np, v, sizeof(cplx) * n, cudaMemcpyHostToDevice, ctx->stream));
  RET(gemm_rows(ctx, np, one_src(ps.Qdev), np, (int)n, UV, np, 2, QUV, np));
  DevTmpBuf<int64_t> dr(ctx), dc(ctx);
  DevTmpBuf<double> dout(ctx);
  RET(dr.alloc((size_t)nnz));
  RET(dc.alloc((size_t)nnz));
  RET(dout.alloc((size_t)nnz));
  CK(cudaMemcpyAsync(dr.p, rows, sizeof(int64_t) * nnz, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(dc.p, cols, sizeof(int64_t) * nnz, cudaMemcpyHostToDevice, ctx->stream));
  const unsigned blocks = (unsigned)std::min<int64_t>((nnz + 255) / 256, 148 * 8);
  k_grad_pattern<<<blocks, 256, 0, ctx->stream>>>(nnz, dr.p, dc.p, base, QUV, QUV + np, n, dout.p, ctx->derr);
  RET(check_launch(ctx, "k_grad_pattern"));
  CK(cudaMemcpyAsync(dsdC, dout.p, sizeof(double) * nnz, cudaMemcpyDeviceToHost, ctx->stream));
  return sync_and_check(ctx);
}
