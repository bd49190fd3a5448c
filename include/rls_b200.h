/*
 * rls_b200.h — C ABI of the B200 σ_min(C − zI) grid engine.
 *
 * Drop-in boundary for kuandeng/rls's per-grid-point engine.  Every entry
 * point names the reference interface it replaces (file:line in the reference
 * project).  Conventions, shared by all calls:
 *   - complex values are rls_c64 {re, im} (layout of Julia ComplexF64 and of
 *     C99 double complex); matrices are column-major with a leading dimension;
 *   - grid indices and permutations are 1-based, as in the Julia API; the
 *     sparse entry points take a base argument (0 or 1) for their CSC arrays;
 *   - calls are synchronous (rls_tsqr_r_noalloc and rls_spmm_shifted_dev only
 *     enqueue; see there); no exceptions cross the ABI; a negative return is an
 *     rls_status and rls_last_error() gives the message (rls_last_error(NULL)
 *     for the calls that take no context: rls_lane_offsets, rls_ic_factor,
 *     rls_band_order and rls_mtx_*; the grid calls return the status alone);
 *   - the library never frees or retains caller memory.
 */
#ifndef RLS_B200_H
#define RLS_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct { double re, im; } rls_c64;
typedef struct rls_ctx rls_ctx;

typedef enum {
  RLS_OK = 0,
  RLS_ERR_ARG = -1,        /* ArgumentError in the reference            */
  RLS_ERR_DIM = -2,        /* DimensionMismatch in the reference        */
  RLS_ERR_CUDA = -3,       /* CUDA runtime failure                      */
  RLS_ERR_NOMEM = -4,      /* device allocation failed                  */
  RLS_ERR_TIMEOUT = -5,    /* a bounded device wait gave up             */
  RLS_ERR_BREAKDOWN = -6,  /* numerical breakdown (LAPACK info != 0)    */
  RLS_ERR_STATE = -7,      /* call order (e.g. no operator uploaded)    */
  RLS_ERR_SINGULAR = -8    /* SingularException in the reference        */
} rls_status;

/* Grid description; mirrors the fields of `Recursion` (src/core/recuGrid.jl:1-12). */
typedef struct {
  double x_st, x_ed, y_st, y_ed;
  int64_t n_x, n_y, k;
} rls_grid;

/* Mirrors `PsTriRecyControl` (src/core/psTriRecy.jl:350-370), fields in order.
 * lobpcg_side is a Julia Char (UTF-32 code point: 'L' or 'S').  The default
 * of `shift` depends on normC at construction time, so callers pass it
 * explicitly.  inner_verbose_override < 0 stands for `nothing`. */
typedef struct {
  double tol;
  double normC;
  double shift;
  double gap_tau;
  double gap_tau_scale;
  double recy_tau;
  double recycle_fail_dist_thresh;   /* NaN or Inf = default (one grid step × 1.01) */
  int64_t r;
  int64_t p;
  int64_t p_min;
  double lobpcg_tol_scale;
  uint32_t lobpcg_side;
  uint8_t implict_update;
  uint8_t implict_recycle;
  uint8_t collect_timing;
  uint8_t _pad0;
  int64_t inner_verbose_override;
} rls_pstrirecy_control;

/* Mirrors `PsTriRecyStats` (src/core/psTriRecy.jl:257-272).  Array members are
 * caller-allocated with length nZ and may be NULL; refine_it is an addition
 * (LOBPCG iterations per point, 0 when the point was recycled), and so are the trailing
 * dsdx and dsdy: ∂σ/∂Re z and ∂σ/∂Im z at every point from the point's own singular pair
 * (the accepted Ritz pair of a recycled point; LOBPCG's converged pair of a refined one),
 * −Re(uᴴv) and Im(uᴴv) with u = (T − zI)v/σ.  Their accuracy is first order in the residual
 * the solver accepted; rls_sigma_grad refines one point further. */
typedef struct {
  int64_t* p_count;
  int64_t* r_recy;
  rls_c64* pts;
  int64_t* M_vec_apps;
  int64_t* M_vec_apps_no_recycle;
  int64_t* R_vec_apps;
  int64_t* refine_it;
  uint64_t preprocess_time_ns;
  uint64_t recycle_time_ns;
  uint64_t qr_time_ns;
  uint64_t refine_time_ns;
  uint64_t update_time_ns;
  uint8_t mv_stats_available;
  uint8_t _pad0[7];
  int64_t n_it;
  int64_t n_pts;
  double* dsdx;
  double* dsdy;
} rls_pstrirecy_stats;

/* Mirrors `LobpcgSvdControl` (src/core/lobpcgSvd.jl:1-13).  orth_type: 0 =
 * :lapack, 1 = :shiftchol.  conv_first/conv_last is the 1-based UnitRange
 * conv_range. */
typedef struct {
  int64_t m, n, r, maxit;
  double tol;
  uint32_t side;
  int32_t verbose;
  double normC;
  int32_t orth_type;
  int32_t conv_thresh_type;
  int64_t conv_first, conv_last;
} rls_lobpcg_control;

/* Mirrors `PsPrecRecyControl` (src/core/psPrecRecy.jl:220-261), fields in order.  Julia
 * Symbol pred_orth_type: 0 = :lapack, 1 = :shiftchol.  pred_conv_range (Union{Nothing,
 * UnitRange}) is the 1-based pair pred_conv_first..pred_conv_last, with pred_conv_first < 1
 * for `nothing`.  shift's default depends on main_normC, so callers pass it explicitly.
 * inner_verbose_override < 0 stands for `nothing`.  Bool fields are uint8 with explicit
 * padding. */
typedef struct {
  double tol;
  double lobpcg_tol_scale;
  double main_normC;
  double main_tau;
  double shift;
  double gap_tau;
  double recycle_fail_dist_thresh;   /* NaN or Inf = default (one grid step × 1.01) */
  double tol_pred;
  double lobpcg_pred_tol_scale;
  int64_t pred_conv_first, pred_conv_last;
  double pred_tau;
  double idx_cutoff_pred;
  int32_t pred_orth_type;
  int32_t _pad0;
  int64_t pred_conv_thresh_type;
  double lambda_lower_min;
  double lambda_upper_max;
  int64_t r_main, p_main, p_min_main;
  uint8_t main_implict_update, main_implict_recycle, _pad1[6];
  int64_t r_pred, p_pred, p_min_pred;
  uint8_t pred_implict_update, pred_implict_recycle, _pad2[6];
  double hsl_tol, hsl_cntl_1, hsl_cntl_2;
  int64_t hsl_icntl_1, hsl_icntl_2;
  double gamma_tol, lambda_n_tol;
  int64_t inner_verbose_override;
  uint8_t collect_timing, _pad3[7];
} rls_psprecrecy_control;

/* Mirrors `PsPrecRecyStats` (src/core/psPrecRecy.jl:318-341), fields in order.  Array members
 * are caller-allocated with length nZ and may be NULL; main_refine_it and pred_refine_it are
 * additions (LOBPCG iterations of each stage per point). */
typedef struct {
  int64_t* p_count;
  int64_t* pred_p_count;
  int64_t* r_recy;
  rls_c64* pts;
  rls_c64* pred_pts;
  rls_c64* precond_rebuild_pts;
  int64_t* main_M_vec_apps;
  int64_t* main_M_vec_apps_no_recycle;
  int64_t* main_L_vec_apps;
  int64_t* pred_M_vec_apps;
  int64_t* pred_L_vec_apps;
  uint64_t main_recycle_time_ns, main_refine_time_ns, main_update_time_ns;
  uint64_t pred_recycle_time_ns, pred_refine_time_ns, pred_update_time_ns;
  uint64_t precond_time_ns;
  int64_t n_it, n_pred_it, n_pts, n_pred_pts, n_precond_rebuild_pts;
  int64_t* main_refine_it;
  int64_t* pred_refine_it;
} rls_psprecrecy_stats;

/* Optional per-point log sink (the reference prints the same lines to `io`). */
typedef void (*rls_log_fn)(const char* line, void* user);

/* ---- context ---------------------------------------------------------------- */

/* One context per host thread: owns a CUDA stream, the device workspaces and
 * the uploaded operator.  No reference counterpart (Julia keeps this state in
 * PsTriRecyKeep, src/core/psTriRecy.jl:395-417). */
int rls_ctx_create(rls_ctx** out, int device);
void rls_ctx_destroy(rls_ctx* ctx);
const char* rls_last_error(const rls_ctx* ctx);
const char* rls_status_string(int status);
int rls_ctx_set_log(rls_ctx* ctx, rls_log_fn fn, void* user, int verbose);
/* The context's cudaStream_t (as void*), for callers that time or order work
 * around the engine.  No reference counterpart. */
void* rls_ctx_stream(rls_ctx* ctx);
/* Number of kernel launches this context has issued so far.  No reference counterpart. */
int64_t rls_ctx_launches(const rls_ctx* ctx);
/* Speculative batching of recycle steps: up to max_points consecutive grid points
 * (1..32) run their recycle step together against the current recycled space;
 * points up to the first rejection are accepted exactly as the sequential loop
 * would accept them (an accepted point does not change the space), the first
 * rejected point is refined from its own recycle output.  1 = one point at a time
 * (the plain per-point drop-in).  Default 16.  No reference counterpart. */
int rls_ctx_set_batch(rls_ctx* ctx, int max_points);

/* How the calling thread waits for the device when the engine needs a result on the host
 * (convergence tests, ranks, error word).  spin_us < 0 (the default): spin until the
 * stream is idle, the lowest latency for one traversal.  spin_us ≥ 0: poll for that many
 * microseconds, then sleep until the device is done, so that threads of concurrent lanes
 * (rls_pstrirecy_schur_lanes) that outnumber the host's cores do not take the cores of
 * the threads that are issuing work.  No reference counterpart. */
int rls_ctx_set_host_wait(rls_ctx* ctx, int spin_us);
/* Ritz basis of the recycle step when the Ritz dimension equals the space size
 * (r_ == p·r): 1 (default) forms X = V·G1·G2 as for r_ < p·r; 0 keeps the
 * reference's X = V·G2 (fastRaylRitz.jl:199-202), whose result depends on the
 * phases the eigensolver gives the columns of G1. */
int rls_ctx_set_ritz_basis(rls_ctx* ctx, int g1_always);
/* Per-kernel CUDA-event timing: kernel 0 = triangular solve, 1 = projected
 * eigensolve, 2 = recycle-step streaming product, 3 = triangular multiply.
 * set_profile resets the counters; profile_get returns launches, total device
 * milliseconds and algorithmic work (bytes; flops for kernel 1).  kernel 4
 * returns the host's blocking waits on the stream instead: their number and
 * total wall milliseconds (work = 0); kernel 5 is the sparse shifted product
 * (rls_spmm_shifted*); kernel 6 the preconditioner solve (rls_lltp_ldiv*); kernel 7 the
 * sparse branch's band QR of B − zI (work: 16·(l+1)·(l+u) flops per column).  No
 * reference counterpart (the reference times phases
 * with time_ns, psTriRecy.jl:306-309). */
int rls_ctx_set_profile(rls_ctx* ctx, int on);
int rls_ctx_profile_get(rls_ctx* ctx, int kernel, int64_t* count, double* total_ms, double* work);

/* ---- recursion grid (bit-exact) ------------------------------------------- */

/* recursion_grid / recursion_grid_zigzag (src/core/recuGrid.jl:68-73, :157-176).
 * Z has n_x*n_y entries. */
int rls_grid_zigzag(const rls_grid* g, rls_c64* Z);
/* recursion_grid_linear (src/core/recuGrid.jl:82-102). */
int rls_grid_linear(const rls_grid* g, rls_c64* Z);
/* recursion_grid_spiral (src/core/recuGrid.jl:109-148). */
int rls_grid_spiral(const rls_grid* g, rls_c64* Z);
/* recursion_natural_permutation (src/core/recuGrid.jl:196-208): perm is 1-based,
 * length n_x*n_y, and Z[perm] is in natural order. */
int rls_natural_perm(const rls_grid* g, const rls_c64* Z, int64_t nZ, int64_t* perm);
/* reorder_to_natural (src/core/recuGrid.jl:216-221) for Float64 vectors. */
int rls_reorder_to_natural(const rls_grid* g, const rls_c64* Z, int64_t nZ,
                           const double* v, double* out);
/* reorder_to_natural_grid (src/core/recuGrid.jl:229-232): out is the n_y × n_x
 * column-major matrix A with A[iy, ix] at grid point (x[ix], y[iy]). */
int rls_reorder_to_natural_grid(const rls_grid* g, const rls_c64* Z, int64_t nZ,
                                const double* v, double* out);

/* ---- MatrixMarket input (loaddata, src/utils/loadmtx.jl:1-28) -------------------------
 * The reference reads `data/<name>.mtx` with MatrixMarket.jl's mmread and converts it to
 * ComplexF64; these read a MatrixMarket file at `path` the same way (host only, no context).
 * Symmetric, hermitian and skew-symmetric storage is expanded, coordinate duplicates add up,
 * explicit zeros stay stored, pattern entries are 1.  A file that cannot be opened or parsed
 * returns RLS_ERR_ARG with the file, line and reason in rls_last_error(NULL).
 * rls_mtx_info: m × n, an upper bound of the stored entries after expansion (m·n for the
 * array format) and dense = 1 for the array format.  Any output may be NULL. */
int rls_mtx_info(const char* path, int64_t* m, int64_t* n, int64_t* nnz_max, int* dense);
/* The coordinate format as CSC with 0- or 1-based indices (base): colptr has n + 1 entries,
 * rowval and nzval room for cap entries (cap = nnz_max suffices); rows ascend within each
 * column; *nnz gets the number of stored entries (RLS_ERR_DIM when it exceeds cap). */
int rls_mtx_read_csc(const char* path, int base, int64_t cap, int64_t* colptr, int64_t* rowval,
                     rls_c64* nzval, int64_t* nnz);
/* The array format, column-major into A with leading dimension lda >= m. */
int rls_mtx_read_dense(const char* path, rls_c64* A, int64_t lda);

/* ---- operator upload ---------------------------------------------------------- */

/* Uploads the upper-triangular complex Schur factor T of C (C = Q T Qᴴ), i.e.
 * the M of `pre_process(C::Matrix)` (src/core/psTriRecy.jl:6-14; S = I).  Only
 * the upper triangle of T (n × n, column-major, leading dimension ldt) is read.
 * Host memory. */
int rls_set_schur(rls_ctx* ctx, int64_t n, const rls_c64* T, int64_t ldt);

/* The sparse branch of psTriRecy (pre_process(C::SparseMatrixCSC), src/core/psTriRecy.jl:47-61;
 * the refine's factor get_R_factor!, :222-234, SPQR's qr(M − zS).R with M = C[:, p], S = I[:, p]).
 * Installs the square sparse C (n × n, the reference's CSC layout, indices base 0 or 1) as the
 * context's operator in the form B = PᵀCP for the column order perm (new → old, base as the CSC;
 * NULL: rls_band_order's choice).  rls_pstrirecy_schur(_range) and the lane entry points then
 * run the sparse branch: the recycled space's products on B's CSR, and at each refine point R of
 * B − zI = Pᵀ(M − zS), the R of the reference's M − zS up to row phases, by a banded Householder
 * QR on the device, solved with the dataflow triangular solve on its band tiles.  σ, the Ritz
 * vectors, X0 and the space are in the reference's frame (right singular vectors of M − zS).
 * The lower bandwidth of B must be at most 1008 (RLS_ERR_DIM otherwise); device memory is about
 * n·(3l + 2u)·16 bytes for the band and twice that of R's band tiles.  rls_set_schur,
 * rls_sparse_upload_csc or rls_psprecrecy on the context drop this operator. */
int rls_set_sparse_tri(rls_ctx* ctx, int64_t n, const int64_t* colptr, const int64_t* rowval,
                       const rls_c64* nzval, int base, const int64_t* perm);

/* The symmetric order rls_set_sparse_tri takes when perm is NULL: the natural order or the
 * reverse Cuthill–McKee order of |C| + |Cᵀ|, whichever gives the smaller banded-QR work
 * l·(l + u); perm receives it (new → old, base as the CSC), *l and *u (may be NULL) the
 * bandwidths of PᵀCP.  It stands in for the reference's AMD order of CᴴC (psTriRecy.jl:52),
 * which serves SPQR's fill, where a banded QR's fill is its band.  Errors: rls_last_error(NULL). */
int rls_band_order(int64_t n, const int64_t* colptr, const int64_t* rowval, int base, int64_t* perm,
                   int64_t* l, int64_t* u);

/* The band QR's panel width (no reference counterpart): 8 or 16 columns, or 0 (default) for the
 * library's choice, made by timing one factorisation with each width (16 only where its panel
 * fits in shared memory) at the first refine point of an operator shape on the device and kept
 * for every later context of that shape, so lanes share one choice.  The setting outlives
 * rls_set_sparse_tri. */
int rls_band_set_panel(rls_ctx* ctx, int w);
/* The installed sparse operator's bandwidths l, u, the panel width in use (0 before the first
 * factorisation) and the two timed factorisations of the choice in ms (0 if not timed).
 * RLS_ERR_STATE without a sparse operator.  Any output may be NULL. */
int rls_band_info(const rls_ctx* ctx, int64_t* l, int64_t* u, int* w, double* ms_w8, double* ms_w16);

/* psTriRecy(C::SparseMatrixCSC, rec; control) (psTriRecy.jl:889-913): rls_set_sparse_tri then
 * rls_pstrirecy_schur over the whole traversal.  stats->qr_time_ns gets the factorisation time
 * when control->collect_timing is set (one extra stream synchronisation per refine point). */
int rls_pstrirecy_sparse(rls_ctx* ctx, int64_t n, const int64_t* colptr, const int64_t* rowval,
                         const rls_c64* nzval, int base, const int64_t* perm, const rls_c64* Z, int64_t nZ,
                         const rls_grid* g, const rls_pstrirecy_control* control, const rls_c64* X0,
                         double* sigma_min, rls_pstrirecy_stats* stats);

/* Installs on dst the operator already uploaded to src (same device).  The two contexts
 * share src's device tiles of T, which no call writes after the upload; the tiles are freed
 * with the last context that uses them, and a later rls_set_schur on either context gives
 * that context a new copy and leaves the other's operator as it was.  Lane contexts
 * (rls_pstrirecy_schur_lanes) thereby hold one copy of T between them.  No reference
 * counterpart. */
int rls_set_schur_copy(rls_ctx* dst, rls_ctx* src);

/* How many CTAs each triangular solve on T − zI occupies (the per-refine R⁻¹ / R⁻ᴴ of
 * InvMat, src/types/RLSMatrices.jl).  0 (the default) gives one CTA per 32-row half block
 * row, 2·ceil(n/64), the lowest latency for one traversal; a smaller number, at least 1,
 * makes each CTA solve several half block rows in dependency order and leaves SMs to
 * concurrent lanes.  Values above 2·ceil(n/64) act as 0.  No reference counterpart. */
int rls_set_trsm_ctas(rls_ctx* ctx, int ctas);
/* Longest back-off, in ns, between the triangular solve's polls of a dependency's flag (32 to
 * 2^20; default 32): polls start back-to-back and, after 64, sleep 32 ns doubling up to this
 * cap.  A longer cap lowers the L2 traffic of waiting CTAs at the cost of hand-off latency.  No
 * reference counterpart. */
int rls_set_trsm_backoff(rls_ctx* ctx, int max_ns);
/* CUDA-graph replay of the refine's steady LOBPCG iteration (on: 1, the default; off: 0).  From
 * the second iteration on, the previous iteration's orthogonalisation and solve and this one's
 * Rayleigh–Ritz and residual (≈30 launches) are one graph launch, captured once per space;
 * results are the same bit for bit.  Per-kernel profiling (rls_ctx_set_profile) runs the
 * launches directly.  No reference counterpart. */
int rls_ctx_set_graphs(rls_ctx* ctx, int on);

/* ---- solvers ------------------------------------------------------------------ */

/* psTriRecy on the uploaded Schur factor (src/core/psTriRecy.jl:708-881,
 * dense branch :580-650).  Z (nZ points, traversal order of `rec.Z`) and the
 * grid g (used for the recycle-failure distance, recySpace.jl:22-37, and the
 * forced-add gap budget, psTriRecy.jl:388-393) come from rls_grid_*.  X0 is
 * the n × r initial block the reference draws with rand!(X)
 * (psTriRecy.jl:607); NULL draws it on the device.  sigma_min receives nZ
 * values in Z order.  Controls: r in 1..8, lobpcg_side 'L', implict_recycle true and
 * implict_update false (RLS_ERR_ARG otherwise); the projected eigensolve keeps its work vectors
 * (144 bytes per row) in shared memory, so p·r is limited to about 1600 on a B200 (a launch
 * error beyond; the reference's drivers use p·r = 360). */
int rls_pstrirecy_schur(rls_ctx* ctx, const rls_c64* Z, int64_t nZ, const rls_grid* g,
                        const rls_pstrirecy_control* control, const rls_c64* X0,
                        double* sigma_min, rls_pstrirecy_stats* stats);

/* The same loop over points i_begin..i_end-1 only (0-based, end exclusive).  A
 * call with i_begin = 0 starts a run (space reset, X0 used); a call with
 * i_begin > 0 continues the run whose previous call ended at i_begin, carrying
 * the recycled space, as consecutive iterations of the reference's loop
 * (psTriRecy.jl:735-856).  Z, sigma_min and the stats arrays are the full-length
 * (nZ) arrays; only entries of the range are written.  No reference
 * counterpart: it lets a caller stream a long grid in pieces. */
int rls_pstrirecy_schur_range(rls_ctx* ctx, const rls_c64* Z, int64_t nZ, const rls_grid* g,
                              const rls_pstrirecy_control* control, const rls_c64* X0, int64_t i_begin,
                              int64_t i_end, double* sigma_min, rls_pstrirecy_stats* stats);

/* Concurrent grid lanes on one GPU.  No reference counterpart: the reference walks the
 * whole traversal with one recycled space.  The traversal Z (nZ points) is split into
 * nlanes contiguous, near-equal ranges that start on column boundaries of the zigzag
 * traversal (k points, one grid column of a strip; rls_lane_offsets gives the split), and
 * lane l runs psTriRecy on its
 * range from an empty recycled space on context ctxs[l] (its own stream, operator
 * uploaded with rls_set_schur), each lane in its own host thread.  Each lane is exactly
 * the reference's run on that sub-grid; lanes keep the GPU busy where one traversal's
 * latency-bound kernels leave most SMs idle.  sigma_min and the stats arrays are the
 * full-length arrays; the stats scalars are summed over lanes.  The _range form runs,
 * in every lane, the lane-local points j_begin..j_end-1 (a call with j_begin > 0
 * continues each lane's run).  A log sink set on a context is called from that lane's
 * thread.  Every lane needs a context of its own: a context listed twice returns
 * RLS_ERR_ARG before any work, with the message in rls_last_error(NULL). */
int rls_lane_offsets(const rls_grid* g, int64_t nZ, int nlanes, int64_t* offsets /* nlanes+1 */);
int rls_pstrirecy_schur_lanes(rls_ctx* const* ctxs, int nlanes, const rls_c64* Z, int64_t nZ,
                              const rls_grid* g, const rls_pstrirecy_control* control,
                              const rls_c64* X0, double* sigma_min, rls_pstrirecy_stats* stats);
int rls_pstrirecy_schur_lanes_range(rls_ctx* const* ctxs, int nlanes, const rls_c64* Z, int64_t nZ,
                                    const rls_grid* g, const rls_pstrirecy_control* control,
                                    const rls_c64* X0, int64_t j_begin, int64_t j_end,
                                    double* sigma_min, rls_pstrirecy_stats* stats);

/* lobpcgSvd (src/core/lobpcgSvd.jl:365-477) on C = InvMat(adjoint(T − zI)) with
 * K = I, as psTriRecy calls it at psTriRecy.jl:797-808.  X0 (n × r) may be
 * NULL.  X_out (n × r, may be NULL) receives keep.S[:, 1:r]; sigma_r (r
 * values, may be NULL) receives keep.σ[1:r].  *sigma gets the returned σ and
 * *it the iteration count. */
int rls_lobpcg_svd_invtri(rls_ctx* ctx, rls_c64 z, const rls_c64* X0,
                          const rls_lobpcg_control* control, rls_c64* X_out,
                          double* sigma_r, double* sigma, int64_t* it);

/* Operators of rls_lobpcg_svd, each built from what the context holds:
 *   RLS_OP_INV_SCHUR  InvMat(adjoint(T − zI)) on the Schur factor (rls_set_schur), as
 *                     psTriRecy calls it (psTriRecy.jl:797);
 *   RLS_OP_SHIFTED    ShiftedMat(C, −z) = C − zI on the sparse C (rls_sparse_upload_csc), as
 *                     psPrecRecy's main stage (psPrecRecy.jl:926);
 *   RLS_OP_PRED       MulChainMat(ShiftedMat(C, −z), invF), invF = P·L⁻ᴴ of the uploaded
 *                     SparseLLTP (rls_lltp_upload), the prediction stage's operator and
 *                     _compute_λ_n's (psPrecRecy.jl:27-41, :405-422);
 *   RLS_OP_INV_L      InvMat(L) of the uploaded factor, _compute_γ's operator (:388-402).
 * Preconditioners: RLS_PREC_NONE (IdentityMat) or RLS_PREC_LLTP (the uploaded SparseLLTP). */
enum { RLS_OP_INV_SCHUR = 0, RLS_OP_SHIFTED = 1, RLS_OP_PRED = 2, RLS_OP_INV_L = 3 };
enum { RLS_PREC_NONE = 0, RLS_PREC_LLTP = 1 };

/* lobpcgSvd(C, X0, K, keep, control) (src/core/lobpcgSvd.jl:365-477) on the operator `op` at
 * shift z (ignored by RLS_OP_INV_L), with K = `prec`: side 'L' (largest singular values of
 * C, returned inverted in keep.σ) or 'S' (smallest), orth_type :lapack or :shiftchol,
 * conv_thresh_type 0 or 1 and conv_range as LobpcgSvdControl holds them; 1 <= r <= 40.
 * X0 (n × r, may be NULL: the fixed uniform [0,1) fill) stands for the caller's X0 or rand!.
 * X_out (n × r, may be NULL) receives keep.S[:, 1:r], sigma_r (r, may be NULL) keep.σ[1:r],
 * *sigma the returned σ (side 'S': σ[1]; side 'L': 1/σ[1]) and *it the iteration count. */
int rls_lobpcg_svd(rls_ctx* ctx, int op, rls_c64 z, int prec, const rls_c64* X0,
                   const rls_lobpcg_control* control, rls_c64* X_out, double* sigma_r, double* sigma,
                   int64_t* it);

/* ---- sparse shifted product ------------------------------------------------------ */

/* Uploads a sparse m × n C in the layout of Julia's SparseMatrixCSC (colptr n+1, rowval and
 * nzval nnz; indices 1-based with base = 1, 0-based with base = 0).  The device keeps the
 * CSR of C and of Cᴴ.  Host memory.  Replaces the operand of `ShiftedMat`
 * (src/types/RLSMatrices.jl:24-64). */
int rls_sparse_upload_csc(rls_ctx* ctx, int64_t m, int64_t n, const int64_t* colptr,
                          const int64_t* rowval, const rls_c64* nzval, int base);
/* mul!(Y, ShiftedMat(C, s), X) (RLSMatrices.jl:47-56): Y = C X + s·X[1:min(m,n), :]
 * (adj = 0; X n × b, Y m × b) or, for adjoint(ShiftedMat) (:64-66),
 * Y = Cᴴ X + conj(s)·X[1:min(m,n), :] (adj = 1; X m × b, Y n × b).  Column-major
 * with leading dimensions ldx, ldy.  rls_spmm_shifted takes host buffers and returns
 * when Y is written; rls_spmm_shifted_dev takes device pointers and only enqueues the
 * product on the context's stream (rls_ctx_stream). */
int rls_spmm_shifted(rls_ctx* ctx, rls_c64 s, int adj, int b, const rls_c64* X, int64_t ldx,
                     rls_c64* Y, int64_t ldy);
int rls_spmm_shifted_dev(rls_ctx* ctx, rls_c64 s, int adj, int b, const rls_c64* X, int64_t ldx,
                         rls_c64* Y, int64_t ldy);

/* ---- incomplete-Cholesky preconditioner apply (psPrecRecy) ------------------------ */

/* Uploads the factor of a SparseLLTP (src/preconditioner/RLSPreconditioner.jl:8-26, built
 * by get_hsl_LLTP, hsl_preconditioner.jl:159-252): L, n × n in the reference's CSC layout
 * (colptr n+1, rowval and nzval nnz; only the lower triangle is used, as
 * LowerTriangular(L) does), the permutation p and its inverse invp as the struct holds
 * them.  Indices are base 0 or 1 (1 = Julia's SparseMatrixCSC and Vector{Int}).  A real L
 * is passed with zero imaginary parts.  Replaces any earlier factor of the context. */
int rls_lltp_upload(rls_ctx* ctx, int64_t n, const int64_t* colptr, const int64_t* rowval,
                    const rls_c64* nzval, const int64_t* p, const int64_t* invp, int base);

/* ldiv!(X, K, B) for the uploaded SparseLLTP (RLSPreconditioner.jl:79-116):
 * temp = B[p, :]; X = L \ temp; temp = Lᴴ \ X; X = temp[invp, :], i.e. X = P·L⁻ᴴ·L⁻¹·Pᴴ·B,
 * B and X n × b, column-major with leading dimensions ldb, ldx.  rls_lltp_ldiv takes host
 * buffers and may be given X == B (the reference's ldiv!(K, B)); rls_lltp_ldiv_dev takes
 * device pointers with X ≠ B.  Both return when X is written.  A zero or absent diagonal
 * entry of L gives RLS_ERR_SINGULAR, naming the first such index j as the reference's
 * SingularException(j) does. */
int rls_lltp_ldiv(rls_ctx* ctx, int b, const rls_c64* B, int64_t ldb, rls_c64* X, int64_t ldx);

/* get_hsl_LLTP(C, z, tau1, tau2, α, lsize, rsize, p) (hsl_preconditioner.jl:159-252) on the
 * host, no context: the threshold incomplete-Cholesky factor of the permuted, L2-scaled
 * lower((C − zI)ᴴ(C − zI)) that psPrecRecy builds at start-up and on every rebuild.  C is
 * n × n in the reference's CSC layout (rows strictly increasing in each column), p a
 * permutation; indices base 0 or 1, outputs in the same base.  Writes L (lcolptr n+1,
 * lrowval and lnzval of capacity cap ≥ n·(1 + min(lsize, n−1)); NULL lrowval / lnzval skip
 * the entries) and invp, and the diagonal shift α the factorisation succeeded with
 * (shift_used, may be NULL).  L, p, invp are the fields of the SparseLLTP to pass to
 * rls_lltp_upload.  Only the control get_hsl_LLTP sets is supported (L2 scaling, no
 * R·Rᴴ term); lsize < 1 (n > 1) is an ArgumentError, as the reference cannot run it.
 * The shift grows by 2× per breakdown, as the reference's, for at most 200 retries. */
int rls_ic_factor(int64_t n, const int64_t* colptr, const int64_t* rowval, const rls_c64* nzval, int base,
                  rls_c64 z, double tau1, double tau2, double alpha, int64_t lsize, int64_t rsize,
                  const int64_t* p, int64_t cap, int64_t* lcolptr, int64_t* lrowval, rls_c64* lnzval,
                  int64_t* invp, double* shift_used);
int rls_lltp_ldiv_dev(rls_ctx* ctx, int b, const rls_c64* B, int64_t ldb, rls_c64* X, int64_t ldx);

/* ---- psPrecRecy -------------------------------------------------------------------- */

/* psPrecRecy(C, rec; control) (src/core/psPrecRecy.jl:617-1033) on the device: C is n × n in
 * the reference's CSC layout (colptr n+1, rowval and nzval nnz; indices base 0 or 1, as
 * SparseMatrixCSC holds them with base = 1).  p is the column order the reference takes from
 * SPQR (qr(C).cpiv, psPrecRecy.jl:625), passed in by the caller (base as the CSC; NULL: the
 * identity).  The IC preconditioner is built on the host (get_hsl_LLTP, rls_ic_factor) at
 * rec.Z[1] and at every rebuild; everything per grid point runs on the GPU.  X0_main (n ×
 * r_main), X0_pred (n × r_pred) and X0_bound (n × 1) stand for the reference's rand! draws of
 * the two stages' start blocks (:547, :586; X0_pred again at every rebuild, :849) and of the
 * Ritz-bound estimates γ and λ_n (:388-422); NULL fills them on the device with a fixed
 * uniform [0, 1) sequence.  sigma_min receives nZ values in Z order.  Supported: the
 * configuration of the reference's drivers (main_implict_recycle = true, main_implict_update
 * = false, pred_implict_recycle = true, pred_implict_update = true), 1 <= r_main <= 8,
 * 1 <= r_pred <= 40, p_pred·r_pred <= 800; other settings return RLS_ERR_ARG.  A context
 * holding a Schur operator of another order returns RLS_ERR_STATE. */
int rls_psprecrecy(rls_ctx* ctx, int64_t n, const int64_t* colptr, const int64_t* rowval, const rls_c64* nzval,
                   int base, const int64_t* p, const rls_c64* Z, int64_t nZ, const rls_grid* g,
                   const rls_psprecrecy_control* control, const rls_c64* X0_main, const rls_c64* X0_pred,
                   const rls_c64* X0_bound, double* sigma_min, rls_psprecrecy_stats* stats);

/* The same loop over points i_begin..i_end-1 (0-based, end exclusive): i_begin = 0 starts a
 * run (C uploaded, preconditioner built, spaces reset); i_begin > 0 continues the run whose
 * previous call ended there, with C, p and the X0 arguments ignored.  No reference
 * counterpart: it lets a caller stream a long grid in pieces. */
int rls_psprecrecy_range(rls_ctx* ctx, int64_t n, const int64_t* colptr, const int64_t* rowval,
                         const rls_c64* nzval, int base, const int64_t* p, const rls_c64* Z, int64_t nZ,
                         const rls_grid* g, const rls_psprecrecy_control* control, const rls_c64* X0_main,
                         const rls_c64* X0_pred, const rls_c64* X0_bound, int64_t i_begin, int64_t i_end,
                         double* sigma_min, rls_psprecrecy_stats* stats);

/* ---- gradient -------------------------------------------------------------------- */

/* σ = σ_min(T − zI) = σ_min(C − zI) at one point and its derivatives with respect to
 * z = x + iy.  No counterpart in the reference.  From the right singular vector v of
 * R = T − zI (v0, n values, e.g. the first column of rls_lobpcg_svd_invtri's X_out,
 * polished by refine_steps steps of inverse iteration on RᴴR) and u = R v / σ:
 *   ∂σ/∂x = −Re(uᴴv),  ∂σ/∂y = Im(uᴴv).
 * u_out and v_out (n values each, may be NULL) receive u and v in the Schur basis; with
 * C = Q T Qᴴ the singular vectors of C − zI are Q u and Q v, and ∂σ/∂C_ij =
 * Re(conj((Qu)_i) (Qv)_j).  Host memory. */
int rls_sigma_grad(rls_ctx* ctx, rls_c64 z, const rls_c64* v0, int refine_steps, double* sigma,
                   double* dsdx, double* dsdy, rls_c64* u_out, rls_c64* v_out);

/* Uploads the Schur vectors Q of C = Q T Qᴴ (n × n, column-major, leading dimension ldq; host
 * memory) to the context that holds T, for rls_sigma_grad_pattern.  No reference counterpart. */
int rls_set_schur_vectors(rls_ctx* ctx, const rls_c64* Q, int64_t ldq);

/* ∂σ/∂C_ij = Re(conj((Qu)_i)·(Qv)_j) on the nnz index pairs (rows[k], cols[k]) (base 0 or 1) of
 * a sparsity pattern, from the Schur-basis singular pair u, v of T − zI (host vectors of n
 * values, e.g. rls_sigma_grad's u_out and v_out), on the device: Q·[u v] against the uploaded
 * Q, then one gather per nonzero.  dsdC (nnz values, host) receives the gradient.  No
 * counterpart in the reference. */
int rls_sigma_grad_pattern(rls_ctx* ctx, const rls_c64* u, const rls_c64* v, int64_t nnz, const int64_t* rows,
                           const int64_t* cols, int base, double* dsdC);

/* ---- allocation-free utility ---------------------------------------------------- */

/* R (k × k, upper triangular, leading dimension k) of the QR factorisation of the
 * device block A (m × k, leading dimension lda), by the engine's warp TSQR kernel.
 * No counterpart in the reference: it exists for callers that must not have this
 * library allocate device memory — applications whose own pool allocator already
 * holds the device's free memory, or that call it inside a hot loop where a
 * cudaMalloc/cudaFree would synchronise the device.  It takes no context and
 * allocates nothing: its reduction tree lives in a fixed 2.25 MiB device array
 * inside the library, one per device, reserved when the library's device code
 * is loaded.
 *   - Limits: 1 <= m <= 131072, 1 <= k <= 8, lda >= m; anything larger returns
 *     RLS_ERR_DIM and rls_last_error(NULL) says which limit was hit.
 *   - A and R are device pointers on the current device.  Unlike the other
 *     calls, this one only enqueues work on `stream` (a cudaStream_t; NULL is
 *     the legacy default stream) and returns; R is ready when the stream has
 *     reached that point.
 *   - The first call on a device, with that device current, looks up the
 *     array's address there (cudaGetSymbolAddress); make that first call before
 *     any stream capture begins on the device.  A device reset (cudaDeviceReset,
 *     or a reset of the primary context by the application) unloads the array;
 *     the first call made in the new context looks its address up again, so that
 *     call too belongs before any stream capture.
 *   - All calls on a device share the one array, and it keeps the last call's
 *     contents (nothing in it needs to start at zero).  Calls whose work
 *     overlaps on the GPU — issued on different streams, or from several host
 *     threads on one stream without ordering — race on it and give wrong
 *     results; calls in order on one stream are safe. */
int rls_tsqr_r_noalloc(const rls_c64* A, int64_t lda, int64_t m, int k, rls_c64* R, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* RLS_B200_H */
