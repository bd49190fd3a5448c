// Sparse psTriRecy: the psTriRecy loop on a sparse C (the SparseMatrixCSC branch,
// src/core/psTriRecy.jl:47-61 pre_process, :222-234 get_R_factor!, :654-700 the keep).
//
// The reference orders the columns by AMD of CᴴC, keeps M = C[:, p] and S = I[:, p], runs the
// recycled space on (M, S) and, at every refine point, takes R = qr(M − zS).R from SPQR on the
// host for LOBPCG on InvMat(Rᴴ).  Here the caller's (or this library's) permutation P is
// applied to both sides, B = PᵀCP, and the loop runs on B with S = I:
//   * the recycled space on (B, I) equals the one on (M, S): MV = P·BV and SV = PV are unitary
//     images of BV and V, so every Gram quantity (H1, H2, L) and every Ritz vector agrees;
//     right singular vectors of B − zI = Pᵀ(M − zS) are those of M − zS, so X0, X and the
//     space are in the reference's frame;
//   * R is the R factor of B − zI (the R of M − zS up to row phases), computed on the device by
//     the banded Householder QR of bandqr.cuh and cut into band tiles for the dataflow solve;
//   * P is chosen for a narrow band (the better of the natural and the reverse Cuthill–McKee
//     order), not for SPQR's fill: a banded QR's fill is its band.
// rls_set_sparse_tri installs B as the context's operator; rls_pstrirecy_schur(_range) and
// the lane entry points then run the sparse branch (the space's products on the CSR of B, the
// refine on the band factor).

namespace {

void band_release(rls_ctx* ctx) {
  auto& B = ctx->band;
  if (B.graph) cudaGraphExecDestroy(B.graph);   // before the arrays its nodes address
  for (void* q : {(void*)B.AB, (void*)B.Vp, (void*)B.Tm, (void*)B.tmp, (void*)B.zdev}) dfree(ctx, q);
  B = rls_ctx::Band{};
}

// The factorisation's launches (captured once per operator, then replayed): B − zI into the
// band array (z from B.zdev), the panels and their trailing updates, R into band tiles.
template <int W>
int band_factor_launches(rls_ctx* ctx, int64_t* count) {
  auto& B = ctx->band;
  const int64_t n = ctx->n;
  int rpl = 8;   // the update's rows per lane: the panel's rows W + l over 32 lanes, in steps of 8
  while (32 * rpl < W + B.l) rpl += 8;
  CK(cudaMemsetAsync(B.AB, 0, sizeof(cplx) * (size_t)n * (size_t)B.ldab, ctx->stream));
  const unsigned gr = (unsigned)((n + 255) / 256);
  k_band_scatter<<<gr, 256, 0, ctx->stream>>>(n, B.kd, B.ldab, ctx->sp[0], B.AB);
  k_band_shift<<<gr, 256, 0, ctx->stream>>>(n, B.kd, B.ldab, B.zdev, B.AB);
  RET(check_launch(ctx, "k_band_scatter"));
  int64_t k = 2;
  for (int64_t c0 = 0; c0 < n; c0 += W) {
    const int w = (int)std::min<int64_t>(W, n - c0);
    const int mp = (int)std::min<int64_t>(n - c0, w + B.l);
    if (W == 8)   // 8 columns, 4 warps per column
      k_bqr_panel_g<8, 4><<<1, 1024, bqr_panel_smem(w, mp), ctx->stream>>>(B.l, B.kd, B.ldab, B.AB, c0, w, mp,
                                                                           B.Vp, B.Tm, ctx->derr);
    else
      k_bqr_panel<W><<<1, 32 * W, bqr_panel_smem(w, mp), ctx->stream>>>(B.l, B.kd, B.ldab, B.AB, c0, w, mp, B.Vp,
                                                                        B.Tm, ctx->derr);
    ++k;
    const int64_t je = std::min<int64_t>(n, c0 + mp + B.u);
    const int64_t ncw = je - (c0 + w);
    if (ncw > 0) {
      const unsigned g = (unsigned)((ncw + BQR_UCOLS - 1) / BQR_UCOLS);
      const size_t sm = bqr_update_smem(W, mp);
#define RLS_BQRU(R) \
  case R: k_bqr_update<W, R><<<g, 32 * BQR_UCOLS, sm, ctx->stream>>>(B.l, B.kd, B.ldab, B.AB, c0, w, mp, je, B.Vp, B.Tm); break;
      switch (rpl) {
        RLS_BQRU(8) RLS_BQRU(16) RLS_BQRU(24) RLS_BQRU(32)
        default: set_err(ctx, "band QR update: %d rows per lane", rpl); return RLS_ERR_STATE;
      }
#undef RLS_BQRU
      ++k;
    }
  }
  RET(check_launch(ctx, "k_bqr_panel/k_bqr_update"));
  k_band_tiles<<<(unsigned)tile_slots(ctx->nb, ctx->tile_bw), 256, 0, ctx->stream>>>(ctx->nb, ctx->tile_bw, n, B.kd,
                                                                                     B.ldab, B.AB, ctx->T);
  *count = k + 1;
  return check_launch(ctx, "k_band_tiles");
}

int band_capture(rls_ctx* ctx, int W, cudaGraphExec_t* ex, int64_t* cnt) {
  cudaGraph_t g = nullptr;
  CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
  const int st = (W == 16) ? band_factor_launches<16>(ctx, cnt) : band_factor_launches<8>(ctx, cnt);
  const cudaError_t ce = cudaStreamEndCapture(ctx->stream, &g);
  if (st != RLS_OK) {
    if (g) cudaGraphDestroy(g);
    return st;
  }
  CK(ce);
  const cudaError_t ie = cudaGraphInstantiate(ex, g, 0);
  cudaGraphDestroy(g);
  CK(ie);
  return RLS_OK;
}

// Panel width chosen by timing: one factorisation with 8- and one with 16-column panels (where
// 16 fits) on the first refine of an operator shape, the faster kept for every later context
// of the same shape on the device, so that lanes share one choice (and one rounding).
struct BandTuneCache {
  std::mutex m;
  std::map<std::tuple<int, int64_t, int64_t, int64_t>, int> w;
};
BandTuneCache& band_tune_cache() {
  static BandTuneCache c;
  return c;
}

int band_time_graph(rls_ctx* ctx, cudaGraphExec_t ex, double* ms) {
  cudaEvent_t a = nullptr, b = nullptr;
  CK(cudaEventCreate(&a));
  CK(cudaEventCreate(&b));
  CK(cudaEventRecord(a, ctx->stream));
  CK(cudaGraphLaunch(ex, ctx->stream));
  CK(cudaEventRecord(b, ctx->stream));
  CK(cudaEventSynchronize(b));
  float f = 0.f;
  CK(cudaEventElapsedTime(&f, a, b));
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  *ms = f;
  return sync_and_check(ctx);
}

// R(z) of B − zI into the band tiles T (kernels in bandqr.cuh): the shift goes to device
// memory, then one graph launch replays the captured sequence.
int band_factor(rls_ctx* ctx, cplx z) {
  auto& B = ctx->band;
  CK(cudaMemcpyAsync(B.zdev, &z, sizeof(cplx), cudaMemcpyHostToDevice, ctx->stream));
  if (!B.graph) {
    int w = ctx->band_panel;
    if (w == 16 && !B.w16_fits) w = 8;
    const auto key = std::make_tuple(ctx->device, ctx->n, B.l, B.u);
    auto& cache = band_tune_cache();
    std::unique_lock<std::mutex> lk(cache.m);
    if (!w) {
      auto it = cache.w.find(key);
      if (it != cache.w.end()) w = it->second;
    }
    if (!w && !B.w16_fits) w = 8;
    if (!w) {   // time both widths once
      cudaGraphExec_t e8 = nullptr, e16 = nullptr;
      int64_t c8 = 0, c16 = 0;
      RET(band_capture(ctx, 8, &e8, &c8));
      int st = band_capture(ctx, 16, &e16, &c16);
      double m8 = 0.0, m16 = 0.0;
      if (st == RLS_OK) st = band_time_graph(ctx, e8, &m8);
      if (st == RLS_OK) st = band_time_graph(ctx, e16, &m16);
      if (st != RLS_OK) {
        if (e8) cudaGraphExecDestroy(e8);
        if (e16) cudaGraphExecDestroy(e16);
        return st;
      }
      ctx->launches += c8 + c16;
      B.tune_ms8 = m8;
      B.tune_ms16 = m16;
      w = (m16 < m8) ? 16 : 8;
      cache.w[key] = w;
      B.graph = (w == 16) ? e16 : e8;
      B.graph_launches = (w == 16) ? c16 : c8;
      cudaGraphExecDestroy(w == 16 ? e8 : e16);
    } else {
      if (!ctx->band_panel) cache.w.emplace(key, w);
      RET(band_capture(ctx, w, &B.graph, &B.graph_launches));
    }
    B.w = w;
  }
  cudaEvent_t e0 = nullptr;
  prof_begin(ctx, KP_BANDQR, &e0);
  CK(cudaGraphLaunch(B.graph, ctx->stream));
  ctx->launches += B.graph_launches;
  // algorithmic flops: per column, a reflector of l + 1 rows onto l + u columns (dot + update)
  prof_end(ctx, KP_BANDQR, e0, 16.0 * (double)(B.l + 1) * (double)(B.l + B.u) * (double)ctx->n);
  return RLS_OK;
}

// Reverse Cuthill–McKee order (new → old) of the pattern of |C| + |Cᵀ|, each component from a
// pseudo-peripheral vertex (repeated breadth-first searches from a last-level vertex of least
// degree while the eccentricity grows), neighbours taken by increasing degree, then index.
std::vector<int64_t> rcm_order(int64_t n, const std::vector<int64_t>& ap, const std::vector<int64_t>& ai) {
  std::vector<int64_t> deg((size_t)n);
  for (int64_t v = 0; v < n; ++v) deg[(size_t)v] = ap[(size_t)v + 1] - ap[(size_t)v];
  std::vector<int64_t> order;
  order.reserve((size_t)n);
  std::vector<char> done((size_t)n, 0);
  std::vector<int64_t> level((size_t)n, -1), queue;
  auto bfs = [&](int64_t root, int64_t* last_min, int64_t* ecc) {
    queue.clear();
    queue.push_back(root);
    level[(size_t)root] = 0;
    for (size_t h = 0; h < queue.size(); ++h) {
      const int64_t v = queue[h];
      for (int64_t e = ap[(size_t)v]; e < ap[(size_t)v + 1]; ++e) {
        const int64_t w = ai[(size_t)e];
        if (level[(size_t)w] < 0) {
          level[(size_t)w] = level[(size_t)v] + 1;
          queue.push_back(w);
        }
      }
    }
    *ecc = level[(size_t)queue.back()];
    int64_t best = queue.back();
    for (int64_t v : queue)
      if (level[(size_t)v] == *ecc && (deg[(size_t)v] < deg[(size_t)best] || (deg[(size_t)v] == deg[(size_t)best] && v < best)))
        best = v;
    *last_min = best;
    for (int64_t v : queue) level[(size_t)v] = -1;
  };
  for (int64_t s0 = 0; s0 < n; ++s0) {
    if (done[(size_t)s0]) continue;
    // least-degree vertex of this component
    int64_t root = s0, ecc = 0, cand = 0;
    bfs(s0, &cand, &ecc);
    std::vector<int64_t> comp(queue);
    for (int64_t v : comp)
      if (deg[(size_t)v] < deg[(size_t)root] || (deg[(size_t)v] == deg[(size_t)root] && v < root)) root = v;
    int64_t e0 = -1;
    for (int it = 0; it < 8; ++it) {
      bfs(root, &cand, &ecc);
      if (ecc <= e0) break;
      e0 = ecc;
      if (cand == root) break;
      root = cand;
    }
    // Cuthill–McKee from root
    const size_t first = order.size();
    order.push_back(root);
    done[(size_t)root] = 1;
    std::vector<int64_t> nb;
    for (size_t h = first; h < order.size(); ++h) {
      const int64_t v = order[h];
      nb.clear();
      for (int64_t e = ap[(size_t)v]; e < ap[(size_t)v + 1]; ++e)
        if (!done[(size_t)ai[(size_t)e]]) nb.push_back(ai[(size_t)e]);
      std::sort(nb.begin(), nb.end(), [&](int64_t a, int64_t b) {
        return deg[(size_t)a] != deg[(size_t)b] ? deg[(size_t)a] < deg[(size_t)b] : a < b;
      });
      for (int64_t w : nb)
        if (!done[(size_t)w]) {
          done[(size_t)w] = 1;
          order.push_back(w);
        }
    }
  }
  std::reverse(order.begin(), order.end());
  return order;
}

// Lower and upper bandwidths of PᵀCP for the order perm (new → old, 0-based).
void band_widths(int64_t n, const int64_t* colptr, const int64_t* rowval, int base, const std::vector<int64_t>& perm,
                 int64_t* l, int64_t* u) {
  std::vector<int64_t> ip((size_t)n);
  for (int64_t k = 0; k < n; ++k) ip[(size_t)perm[(size_t)k]] = k;
  int64_t lo = 0, up = 0;
  for (int64_t j = 0; j < n; ++j)
    for (int64_t e = colptr[j] - base; e < colptr[j + 1] - base; ++e) {
      const int64_t d = ip[(size_t)(rowval[e] - base)] - ip[(size_t)j];
      lo = std::max(lo, d);
      up = std::max(up, -d);
    }
  *l = lo;
  *u = up;
}

int check_csc(int64_t n, const int64_t* colptr, const int64_t* rowval, int base, std::string* why) {
  if (n < 1 || !colptr || (base != 0 && base != 1) || n >= (1ll << 31)) {
    *why = "invalid arguments (n, colptr or base)";
    return RLS_ERR_ARG;
  }
  if (colptr[0] != base) {
    *why = "colptr[0] is not the index base";
    return RLS_ERR_DIM;
  }
  for (int64_t c = 0; c < n; ++c)
    if (colptr[c + 1] < colptr[c]) {
      *why = "column pointers decrease at column " + std::to_string(c + 1);
      return RLS_ERR_DIM;
    }
  const int64_t nnz = colptr[n] - base;
  if (nnz > 0 && !rowval) {
    *why = "no row indices";
    return RLS_ERR_ARG;
  }
  for (int64_t e = 0; e < nnz; ++e)
    if (rowval[e] - base < 0 || rowval[e] - base >= n) {
      *why = "row index " + std::to_string(rowval[e] - base + 1) + " out of range 1.." + std::to_string(n);
      return RLS_ERR_DIM;
    }
  return RLS_OK;
}

int pick_band_order(int64_t n, const int64_t* colptr, const int64_t* rowval, int base, std::vector<int64_t>* perm,
                    int64_t* l, int64_t* u) {
  // symmetric pattern without the diagonal, as CSR
  std::vector<int64_t> cnt((size_t)n + 1, 0);
  for (int64_t j = 0; j < n; ++j)
    for (int64_t e = colptr[j] - base; e < colptr[j + 1] - base; ++e) {
      const int64_t i = rowval[e] - base;
      if (i == j) continue;
      ++cnt[(size_t)i + 1];
      ++cnt[(size_t)j + 1];
    }
  for (int64_t v = 0; v < n; ++v) cnt[(size_t)v + 1] += cnt[(size_t)v];
  std::vector<int64_t> ai((size_t)cnt[(size_t)n]), pos(cnt.begin(), cnt.end() - 1);
  for (int64_t j = 0; j < n; ++j)
    for (int64_t e = colptr[j] - base; e < colptr[j + 1] - base; ++e) {
      const int64_t i = rowval[e] - base;
      if (i == j) continue;
      ai[(size_t)pos[(size_t)i]++] = j;
      ai[(size_t)pos[(size_t)j]++] = i;
    }
  std::vector<int64_t> ap((size_t)n + 1, 0);
  {   // sort and deduplicate each row
    std::vector<int64_t> out;
    out.reserve(ai.size());
    for (int64_t v = 0; v < n; ++v) {
      auto b = ai.begin() + cnt[(size_t)v], e = ai.begin() + cnt[(size_t)v + 1];
      std::sort(b, e);
      auto last = std::unique(b, e);
      out.insert(out.end(), b, last);
      ap[(size_t)v + 1] = (int64_t)out.size();
    }
    ai.swap(out);
  }
  std::vector<int64_t> nat((size_t)n);
  for (int64_t k = 0; k < n; ++k) nat[(size_t)k] = k;
  int64_t l0, u0, l1, u1;
  band_widths(n, colptr, rowval, base, nat, &l0, &u0);
  std::vector<int64_t> rcm = rcm_order(n, ap, ai);
  band_widths(n, colptr, rowval, base, rcm, &l1, &u1);
  // QR work ∝ n·l·(l + u); the band array ∝ n·(2l + u)
  const double c0 = (double)l0 * (double)(l0 + u0 + 1) + (double)(l0 + u0);
  const double c1 = (double)l1 * (double)(l1 + u1 + 1) + (double)(l1 + u1);
  if (c1 < c0) {
    *perm = std::move(rcm);
    *l = l1;
    *u = u1;
  } else {
    *perm = std::move(nat);
    *l = l0;
    *u = u0;
  }
  return RLS_OK;
}

}  // namespace

extern "C" int rls_band_order(int64_t n, const int64_t* colptr, const int64_t* rowval, int base, int64_t* perm,
                              int64_t* l, int64_t* u) {
  std::string why;
  int rc = check_csc(n, colptr, rowval, base, &why);
  if (rc != RLS_OK) {
    g_create_err = "rls_band_order: " + why;
    return rc;
  }
  if (!perm) {
    g_create_err = "rls_band_order: perm is NULL";
    return RLS_ERR_ARG;
  }
  std::vector<int64_t> p;
  int64_t lo = 0, up = 0;
  RET(pick_band_order(n, colptr, rowval, base, &p, &lo, &up));
  for (int64_t k = 0; k < n; ++k) perm[k] = p[(size_t)k] + base;
  if (l) *l = lo;
  if (u) *u = up;
  return RLS_OK;
}

extern "C" int rls_set_sparse_tri(rls_ctx* ctx, int64_t n, const int64_t* colptr, const int64_t* rowval,
                                  const rls_c64* nzval, int base, const int64_t* perm) {
  if (!ctx) return RLS_ERR_ARG;
  std::string why;
  int rc = check_csc(n, colptr, rowval, base, &why);
  if (rc != RLS_OK) {
    set_err(ctx, "rls_set_sparse_tri: %s", why.c_str());
    return rc;
  }
  const int64_t nnz = colptr[n] - base;
  if (nnz > 0 && !nzval) {
    set_err(ctx, "rls_set_sparse_tri: no values");
    return RLS_ERR_ARG;
  }
  std::vector<int64_t> p((size_t)n);
  int64_t l = 0, u = 0;
  if (perm) {
    std::vector<char> seen((size_t)n, 0);
    for (int64_t k = 0; k < n; ++k) {
      const int64_t v = perm[k] - base;
      if (v < 0 || v >= n || seen[(size_t)v]) {
        set_err(ctx, "rls_set_sparse_tri: perm is not a permutation of %d..%lld", base, (long long)(n - 1 + base));
        return RLS_ERR_ARG;
      }
      seen[(size_t)v] = 1;
      p[(size_t)k] = v;
    }
    band_widths(n, colptr, rowval, base, p, &l, &u);
  } else {
    RET(pick_band_order(n, colptr, rowval, base, &p, &l, &u));
  }
  if (l > BQR_MAXL) {
    set_err(ctx, "rls_set_sparse_tri: lower bandwidth %lld of the ordered matrix exceeds the band QR's %d",
            (long long)l, BQR_MAXL);
    return RLS_ERR_DIM;
  }
  // CSC of B = PᵀCP: entry (i, j) of C goes to (ip[i], ip[j])
  std::vector<int64_t> ip((size_t)n);
  for (int64_t k = 0; k < n; ++k) ip[(size_t)p[(size_t)k]] = k;
  std::vector<int64_t> bcp((size_t)n + 1, 0), bri((size_t)std::max<int64_t>(nnz, 1));
  std::vector<rls_c64> bv((size_t)std::max<int64_t>(nnz, 1));
  for (int64_t j = 0; j < n; ++j) bcp[(size_t)ip[(size_t)j] + 1] = colptr[j + 1] - colptr[j];
  for (int64_t j = 0; j < n; ++j) bcp[(size_t)j + 1] += bcp[(size_t)j];
  for (int64_t j = 0; j < n; ++j) {
    int64_t q = bcp[(size_t)ip[(size_t)j]];
    for (int64_t e = colptr[j] - base; e < colptr[j + 1] - base; ++e, ++q) {
      bri[(size_t)q] = ip[(size_t)(rowval[e] - base)];
      bv[(size_t)q] = nzval[e];
    }
  }
  RET(operator_drop(ctx));
  RET(rls_sparse_upload_csc(ctx, n, n, bcp.data(), bri.data(), bv.data(), 0));
  ctx->n = n;
  ctx->nb = (int)((n + TILE - 1) / TILE);
  ctx->n_pad = (int64_t)ctx->nb * TILE;
  const int nb = ctx->nb;
  auto& B = ctx->band;
  B.l = l;
  B.u = u;
  B.kd = l + u;
  B.ldab = B.kd + l + 1;
  ctx->tile_bw = (int)std::min<int64_t>(nb - 1, (B.kd + TILE - 1) / TILE);
  const size_t elems = (size_t)tile_slots(nb, ctx->tile_bw) * TILE * TILE;
  {
    cplx* q = nullptr;
    cudaError_t e = cudaMalloc(&q, elems * sizeof(cplx));
    if (e != cudaSuccess) {
      set_err(ctx, "device allocation of %zu bytes failed: %s", elems * sizeof(cplx), cudaGetErrorString(e));
      return RLS_ERR_NOMEM;
    }
    const int dev = ctx->device;
    ctx->T_buf = std::shared_ptr<cplx>(q, [dev](cplx* a) {
      int prev = 0;
      cudaGetDevice(&prev);
      cudaSetDevice(dev);
      cudaFree(a);
      cudaSetDevice(prev);
    });
    ctx->T = q;
  }
  RET(dalloc_t(ctx, &ctx->G, elems));
  RET(dalloc_t(ctx, &ctx->Dinv, (size_t)nb * TILE * TILE));
  RET(dalloc_t(ctx, &ctx->trsm_u, (size_t)ctx->n_pad * 8));
  RET(dalloc_t(ctx, &ctx->flags, (size_t)2 * nb));
  RET(dalloc_t(ctx, &ctx->ticket, 2));   // work counter, epoch of the last solve (k_trsm_half)
  RET(dalloc_t(ctx, &ctx->colpart, (size_t)(ctx->n_pad / 32 + 64)));
  RET(dalloc_t(ctx, &B.AB, (size_t)n * (size_t)B.ldab));
  // 16-column panels are a candidate where the panel (and the update's copy of V) fit in
  // 200 KB of shared memory; band_factor picks the width by timing
  B.w16_fits = bqr_panel_smem(16, (int)(16 + l)) <= 200 * 1024 && bqr_update_smem(16, (int)(16 + l)) <= 200 * 1024 &&
               16 + l <= BQR_MAXROWS;
  B.w = 0;
  RET(dalloc_t(ctx, &B.Vp, (size_t)BQR_MAXROWS * BQR_WMAX));
  RET(dalloc_t(ctx, &B.Tm, (size_t)BQR_WMAX * BQR_WMAX));
  RET(dalloc_t(ctx, &B.zdev, 1));
  RET(dalloc_t(ctx, &B.tmp, (size_t)ctx->n_pad));
  B.on = true;
  ctx->op_sparse = true;
  ctx->z_dinv = cmk(NAN, NAN);
  CK(cudaStreamSynchronize(ctx->stream));
  return RLS_OK;
}

extern "C" int rls_pstrirecy_sparse(rls_ctx* ctx, int64_t n, const int64_t* colptr, const int64_t* rowval,
                                    const rls_c64* nzval, int base, const int64_t* perm, const rls_c64* Z, int64_t nZ,
                                    const rls_grid* g, const rls_pstrirecy_control* ctl, const rls_c64* X0,
                                    double* sigma_min, rls_pstrirecy_stats* st) {
  if (!ctx) return RLS_ERR_ARG;
  RET(rls_set_sparse_tri(ctx, n, colptr, rowval, nzval, base, perm));
  return rls_pstrirecy_schur_range(ctx, Z, nZ, g, ctl, X0, 0, nZ, sigma_min, st);
}

extern "C" int rls_band_set_panel(rls_ctx* ctx, int w) {
  if (!ctx) return RLS_ERR_ARG;
  if (w != 0 && w != 8 && w != 16) {
    set_err(ctx, "rls_band_set_panel: width %d (0, 8 or 16)", w);
    return RLS_ERR_ARG;
  }
  ctx->band_panel = w;
  if (ctx->band.on && ctx->band.graph) {   // recapture at the next factorisation
    CK(cudaStreamSynchronize(ctx->stream));
    cudaGraphExecDestroy(ctx->band.graph);
    ctx->band.graph = nullptr;
    ctx->z_dinv = cmk(NAN, NAN);
  }
  return RLS_OK;
}

extern "C" int rls_band_info(const rls_ctx* ctx, int64_t* l, int64_t* u, int* w, double* ms_w8, double* ms_w16) {
  if (!ctx) return RLS_ERR_ARG;
  if (!ctx->band.on) return RLS_ERR_STATE;
  if (l) *l = ctx->band.l;
  if (u) *u = ctx->band.u;
  if (w) *w = ctx->band.w;
  if (ms_w8) *ms_w8 = ctx->band.tune_ms8;
  if (ms_w16) *ms_w16 = ctx->band.tune_ms16;
  return RLS_OK;
}
