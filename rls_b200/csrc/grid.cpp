// Recursion-grid construction and natural-order remap (src/core/recuGrid.jl).
//
// Bit-exact with the reference: compiled with -ffp-contract=off so that
// x_st + (ix-1)*dx is one rounded multiply and one rounded add, as Julia
// evaluates recuGrid.jl:42-43; Julia's round(Int, x) is round-half-to-even,
// which std::nearbyint gives in the default rounding mode.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../../include/rls_b200.h"

namespace {

struct GridMeta {
  double x_st, x_ed, y_st, y_ed, dx, dy;
  int64_t n_x, n_y, k;
};

int make_meta(const rls_grid* g, GridMeta* m) {
  if (!g) return RLS_ERR_ARG;
  if (g->n_x < 2 || g->n_y < 2 || g->k < 1) return RLS_ERR_ARG;  // recuGrid.jl:26-28
  m->x_st = g->x_st; m->x_ed = g->x_ed; m->y_st = g->y_st; m->y_ed = g->y_ed;
  m->n_x = g->n_x; m->n_y = g->n_y; m->k = g->k;
  m->dx = (m->x_ed - m->x_st) / static_cast<double>(m->n_x - 1);  // recuGrid.jl:34
  m->dy = (m->y_ed - m->y_st) / static_cast<double>(m->n_y - 1);  // recuGrid.jl:35
  return RLS_OK;
}

inline rls_c64 zpt(const GridMeta& m, int64_t ix, int64_t iy) {  // recuGrid.jl:41-45
  volatile double tx = static_cast<double>(ix - 1) * m.dx;
  volatile double ty = static_cast<double>(iy - 1) * m.dy;
  rls_c64 z;
  z.re = m.x_st + tx;
  z.im = m.y_st + ty;
  return z;
}

}  // namespace

extern "C" int rls_grid_zigzag(const rls_grid* g, rls_c64* Z) {
  GridMeta m;
  int st = make_meta(g, &m);
  if (st) return st;
  if (!Z) return RLS_ERR_ARG;
  if (m.n_y % m.k != 0) return RLS_ERR_ARG;  // recuGrid.jl:162
  int64_t block_id = 0;
  for (int64_t by = 1; by <= m.n_y / m.k; ++by) {  // recuGrid.jl:166-174
    const bool fwd = (by % 2 == 1);
    const int64_t iy0 = (by - 1) * m.k + 1;
    for (int64_t j = 1; j <= m.n_x; ++j) {
      const int64_t ix = fwd ? j : m.n_x + 1 - j;
      const bool down = (j % 2 == 1);
      const int64_t base = block_id * m.k;
      for (int64_t l = 1; l <= m.k; ++l) {  // _set_col_k! recuGrid.jl:48-60
        const int64_t iy = down ? iy0 + l - 1 : iy0 + (m.k - l);
        Z[base + l - 1] = zpt(m, ix, iy);
      }
      ++block_id;
    }
  }
  return RLS_OK;
}

extern "C" int rls_grid_linear(const rls_grid* g, rls_c64* Z) {
  GridMeta m;
  int st = make_meta(g, &m);
  if (st) return st;
  if (!Z) return RLS_ERR_ARG;
  int64_t idx = 0;
  for (int64_t iy = 1; iy <= m.n_y; ++iy) {  // recuGrid.jl:88-100
    for (int64_t j = 1; j <= m.n_x; ++j) {
      const int64_t ix = (iy % 2 == 1) ? j : m.n_x + 1 - j;
      Z[idx++] = zpt(m, ix, iy);
    }
  }
  return RLS_OK;
}

extern "C" int rls_grid_spiral(const rls_grid* g, rls_c64* Z) {
  GridMeta m;
  int st = make_meta(g, &m);
  if (st) return st;
  if (!Z) return RLS_ERR_ARG;
  int64_t left = 1, right = m.n_x, top = 1, bottom = m.n_y, idx = 0;  // recuGrid.jl:115-146
  while (left <= right && top <= bottom) {
    for (int64_t ix = left; ix <= right; ++ix) Z[idx++] = zpt(m, ix, top);
    ++top;
    if (top > bottom) break;
    for (int64_t iy = top; iy <= bottom; ++iy) Z[idx++] = zpt(m, right, iy);
    --right;
    if (left > right) break;
    for (int64_t ix = right; ix >= left; --ix) Z[idx++] = zpt(m, ix, bottom);
    --bottom;
    if (top > bottom) break;
    for (int64_t iy = bottom; iy >= top; --iy) Z[idx++] = zpt(m, left, iy);
    ++left;
  }
  return RLS_OK;
}

extern "C" int rls_natural_perm(const rls_grid* g, const rls_c64* Z, int64_t nZ, int64_t* perm) {
  GridMeta m;
  int st = make_meta(g, &m);
  if (st) return st;
  if (!Z || !perm) return RLS_ERR_ARG;
  const int64_t n = m.n_x * m.n_y;
  if (nZ != n) return RLS_ERR_DIM;
  std::memset(perm, 0, sizeof(int64_t) * static_cast<size_t>(n));
  for (int64_t i = 1; i <= n; ++i) {  // recuGrid.jl:199-203
    volatile double rx = (Z[i - 1].re - m.x_st) / m.dx;  // recuGrid.jl:180-183
    volatile double ry = (Z[i - 1].im - m.y_st) / m.dy;
    const double fx = std::nearbyint(rx), fy = std::nearbyint(ry);
    if (!(fx >= 0.0 && fx <= static_cast<double>(m.n_x - 1) && fy >= 0.0 &&
          fy <= static_cast<double>(m.n_y - 1)))
      return RLS_ERR_ARG;  // outside the grid bounds (recuGrid.jl:184-186)
    const int64_t ix = static_cast<int64_t>(fx) + 1, iy = static_cast<int64_t>(fy) + 1;
    const int64_t j = (iy - 1) * m.n_x + ix;
    if (perm[j - 1] != 0) return RLS_ERR_ARG;  // duplicate grid point (recuGrid.jl:201)
    perm[j - 1] = i;
  }
  for (int64_t j = 0; j < n; ++j)
    if (perm[j] <= 0) return RLS_ERR_ARG;  // missing grid point (recuGrid.jl:204-206)
  return RLS_OK;
}

extern "C" int rls_reorder_to_natural(const rls_grid* g, const rls_c64* Z, int64_t nZ,
                                      const double* v, double* out) {
  if (!v || !out) return RLS_ERR_ARG;
  std::vector<int64_t> perm(static_cast<size_t>(nZ > 0 ? nZ : 0));
  int st = rls_natural_perm(g, Z, nZ, perm.data());
  if (st) return st;
  for (int64_t j = 0; j < nZ; ++j) out[j] = v[perm[j] - 1];  // recuGrid.jl:220
  return RLS_OK;
}

extern "C" int rls_reorder_to_natural_grid(const rls_grid* g, const rls_c64* Z, int64_t nZ,
                                           const double* v, double* out) {
  if (!v || !out) return RLS_ERR_ARG;
  std::vector<double> nat(static_cast<size_t>(nZ > 0 ? nZ : 0));
  int st = rls_reorder_to_natural(g, Z, nZ, v, nat.data());
  if (st) return st;
  const int64_t nx = g->n_x, ny = g->n_y;
  // permutedims(reshape(v_nat, n_x, n_y), (2, 1)) stored column-major (n_y × n_x).
  for (int64_t ix = 0; ix < nx; ++ix)
    for (int64_t iy = 0; iy < ny; ++iy) out[ix * ny + iy] = nat[iy * nx + ix];
  return RLS_OK;
}
