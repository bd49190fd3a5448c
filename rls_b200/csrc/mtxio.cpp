// MatrixMarket reader: loaddata (src/utils/loadmtx.jl:1-28) reads a `.mtx` file with
// MatrixMarket.jl 0.5's mmread (a dependency not vendored in the reference) and converts it to
// ComplexF64.  This file restates the published NIST MatrixMarket exchange format that mmread
// implements:
//
//   %%MatrixMarket matrix <coordinate|array> <real|complex|integer|pattern>
//                         <general|symmetric|skew-symmetric|hermitian>
//   % comment lines
//   M N NNZ            (coordinate)   or   M N   (array)
//   i j [re [im]]      one stored entry per line, 1-based (coordinate)
//   re [im]            column-major values (array; the lower triangle column by column when
//                      symmetric or hermitian, the strictly lower one when skew-symmetric)
//
// Symmetric storage is expanded (a_ji = a_ij, conj(a_ij) or −a_ij for every stored i ≠ j);
// coordinate duplicates add up and explicit zeros stay stored, as SparseArrays.sparse does;
// pattern entries are 1.  Keywords are case-insensitive; blank lines are skipped.  The CSC has
// 64-bit indices: loaddata's narrowing to Int32 indices is a Julia storage choice with no
// counterpart in the C ABI.
#include <algorithm>
#include <cctype>
#include <cerrno>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <new>
#include <stdexcept>
#include <vector>

#include "../../include/rls_b200.h"
#include "host_err.h"

namespace {

enum Field { F_REAL = 0, F_COMPLEX = 1, F_INTEGER = 2, F_PATTERN = 3 };
enum Symm { S_GENERAL = 0, S_SYMMETRIC = 1, S_HERMITIAN = 2, S_SKEW = 3 };

struct MtxFile {
  FILE* f = nullptr;
  std::string path;
  int64_t line_no = 0;
  bool dense = false;
  int field = F_REAL, symm = S_GENERAL;
  int64_t m = 0, n = 0, entries = 0;   // entries: stored values in the file

  ~MtxFile() {
    if (f) fclose(f);
  }

  int fail(const std::string& what) {
    rls_host_error("rls_mtx: " + path + (line_no > 0 ? ":" + std::to_string(line_no) : std::string()) + ": " + what);
    return RLS_ERR_ARG;
  }

  // Next line into s (without the newline); false at end of file.
  bool getline(std::string& s) {
    s.clear();
    int c;
    bool any = false;
    while ((c = fgetc(f)) != EOF) {
      any = true;
      if (c == '\n') break;
      if (c != '\r') s.push_back(static_cast<char>(c));
    }
    if (!any) return false;
    ++line_no;
    return true;
  }

  static bool blank(const std::string& s) {
    for (char c : s)
      if (!std::isspace(static_cast<unsigned char>(c))) return false;
    return true;
  }

  static std::string lower(std::string s) {
    for (char& c : s) c = static_cast<char>(std::tolower(static_cast<unsigned char>(c)));
    return s;
  }

  // Banner, comments and the size line.
  int open_header(const char* p) {
    if (!p) {
      rls_host_error("rls_mtx: no path");
      return RLS_ERR_ARG;
    }
    path = p;
    f = fopen(p, "rb");
    if (!f) return fail(std::string("cannot open the file (") + std::strerror(errno) + ")");
    std::string s;
    if (!getline(s)) return fail("empty file");
    char w[5][64] = {};
    if (std::sscanf(s.c_str(), "%63s %63s %63s %63s %63s", w[0], w[1], w[2], w[3], w[4]) != 5 ||
        lower(w[0]) != "%%matrixmarket" || lower(w[1]) != "matrix")
      return fail("not a MatrixMarket matrix banner: '" + s + "'");
    const std::string fmt = lower(w[2]), fld = lower(w[3]), sym = lower(w[4]);
    if (fmt == "coordinate") dense = false;
    else if (fmt == "array") dense = true;
    else return fail("unknown format '" + fmt + "'");
    if (fld == "real" || fld == "double") field = F_REAL;
    else if (fld == "complex") field = F_COMPLEX;
    else if (fld == "integer") field = F_INTEGER;
    else if (fld == "pattern") field = F_PATTERN;
    else return fail("unknown field '" + fld + "'");
    if (sym == "general") symm = S_GENERAL;
    else if (sym == "symmetric") symm = S_SYMMETRIC;
    else if (sym == "hermitian") symm = S_HERMITIAN;
    else if (sym == "skew-symmetric") symm = S_SKEW;
    else return fail("unknown symmetry '" + sym + "'");
    if (dense && field == F_PATTERN) return fail("the array format has no pattern field");
    if (symm == S_HERMITIAN && field != F_COMPLEX) symm = S_SYMMETRIC;   // real hermitian = symmetric
    do {
      if (!getline(s)) return fail("no size line");
    } while (blank(s) || s[0] == '%');
    long long a = 0, b = 0, c = 0;
    char extra = 0;
    if (dense) {
      if (std::sscanf(s.c_str(), "%lld %lld %c", &a, &b, &extra) != 2) return fail("bad size line '" + s + "'");
    } else {
      if (std::sscanf(s.c_str(), "%lld %lld %lld %c", &a, &b, &c, &extra) != 3)
        return fail("bad size line '" + s + "'");
    }
    if (a < 0 || b < 0 || c < 0) return fail("negative size");
    if (a > 0 && b > INT64_MAX / a) return fail("m × n does not fit in 64 bits");
    if (c > INT64_MAX / 2) return fail("too many entries");
    m = a;
    n = b;
    if (symm != S_GENERAL && m != n) return fail("a " + sym + " matrix must be square");
    if (dense) {
      if (symm == S_GENERAL) entries = m * n;
      else if (symm == S_SKEW) entries = n * (n - 1) / 2;
      else entries = n * (n + 1) / 2;
    } else {
      entries = c;
    }
    return RLS_OK;
  }

  // Next non-blank data line split into numbers: k integers then v reals.
  int next_numbers(int k, int v, int64_t* ix, double* val, int64_t which) {
    std::string s;
    do {
      if (!getline(s))
        return fail("the file ends after " + std::to_string(which) + " of " + std::to_string(entries) + " entries");
    } while (blank(s) || s[0] == '%');
    const char* p = s.c_str();
    for (int q = 0; q < k; ++q) {
      char* e = nullptr;
      errno = 0;
      const long long x = std::strtoll(p, &e, 10);
      if (e == p || errno) return fail("bad index in '" + s + "'");
      ix[q] = x;
      p = e;
    }
    for (int q = 0; q < v; ++q) {
      char* e = nullptr;
      const double x = std::strtod(p, &e);
      if (e == p) return fail("bad value in '" + s + "'");
      val[q] = x;
      p = e;
    }
    while (*p && std::isspace(static_cast<unsigned char>(*p))) ++p;
    if (*p) return fail("trailing text in '" + s + "'");
    return RLS_OK;
  }

  int values_per_entry() const { return field == F_COMPLEX ? 2 : (field == F_PATTERN ? 0 : 1); }
};

rls_c64 mirror(int symm, rls_c64 a) {
  rls_c64 r = a;
  if (symm == S_HERMITIAN) r.im = -a.im;
  if (symm == S_SKEW) { r.re = -a.re; r.im = -a.im; }
  return r;
}

}  // namespace

static int mtx_info_impl(const char* path, int64_t* m, int64_t* n, int64_t* nnz_max, int* dense) {
  MtxFile mf;
  const int rc = mf.open_header(path);
  if (rc != RLS_OK) return rc;
  if (m) *m = mf.m;
  if (n) *n = mf.n;
  if (nnz_max) *nnz_max = mf.dense ? mf.m * mf.n : (mf.symm == S_GENERAL ? mf.entries : 2 * mf.entries);
  if (dense) *dense = mf.dense ? 1 : 0;
  return RLS_OK;
}

static int mtx_read_csc_impl(const char* path, int base, int64_t cap, int64_t* colptr, int64_t* rowval,
                             rls_c64* nzval, int64_t* nnz) {
  if ((base != 0 && base != 1) || !colptr || !nnz || cap < 0 || (cap > 0 && (!rowval || !nzval))) {
    rls_host_error("rls_mtx_read_csc: invalid arguments");
    return RLS_ERR_ARG;
  }
  MtxFile mf;
  int rc = mf.open_header(path);
  if (rc != RLS_OK) return rc;
  if (mf.dense) return mf.fail("array format: read it with rls_mtx_read_dense");
  struct Entry {
    int64_t col, row, seq;
    rls_c64 v;
  };
  std::vector<Entry> ent;
  // the size line is not trusted for the allocation: reserve at most 2^24 entries up front
  ent.reserve(static_cast<size_t>(std::min<int64_t>(mf.symm == S_GENERAL ? mf.entries : 2 * mf.entries,
                                                    int64_t(1) << 24)));
  const int nv = mf.values_per_entry();
  int64_t seq = 0;
  for (int64_t q = 0; q < mf.entries; ++q) {
    int64_t ix[2];
    double val[2] = {1.0, 0.0};
    rc = mf.next_numbers(2, nv, ix, val, q);
    if (rc != RLS_OK) return rc;
    const int64_t i = ix[0], j = ix[1];
    if (i < 1 || i > mf.m || j < 1 || j > mf.n)
      return mf.fail("entry (" + std::to_string(i) + ", " + std::to_string(j) + ") outside " + std::to_string(mf.m) +
                     " × " + std::to_string(mf.n));
    rls_c64 a;
    a.re = val[0];
    a.im = (nv == 2) ? val[1] : 0.0;
    ent.push_back({j - 1, i - 1, seq++, a});
    if (mf.symm != S_GENERAL && i != j) ent.push_back({i - 1, j - 1, seq++, mirror(mf.symm, a)});
  }
  // column-major order, rows ascending, duplicates in file order (then summed in that order)
  std::stable_sort(ent.begin(), ent.end(), [](const Entry& x, const Entry& y) {
    return x.col != y.col ? x.col < y.col : x.row < y.row;
  });
  std::vector<int64_t> cnt(static_cast<size_t>(mf.n) + 1, 0);
  int64_t k = 0;
  for (size_t q = 0; q < ent.size();) {
    size_t e = q + 1;
    rls_c64 s = ent[q].v;
    while (e < ent.size() && ent[e].col == ent[q].col && ent[e].row == ent[q].row) {
      s.re += ent[e].v.re;
      s.im += ent[e].v.im;
      ++e;
    }
    if (k < cap) {
      rowval[k] = ent[q].row + base;
      nzval[k] = s;
    }
    ++cnt[static_cast<size_t>(ent[q].col) + 1];
    ++k;
    q = e;
  }
  *nnz = k;
  if (k > cap) {
    rls_host_error("rls_mtx_read_csc: " + std::to_string(k) + " stored entries, capacity " + std::to_string(cap));
    return RLS_ERR_DIM;
  }
  colptr[0] = base;
  for (int64_t j = 0; j < mf.n; ++j) colptr[j + 1] = colptr[j] + cnt[static_cast<size_t>(j) + 1];
  return RLS_OK;
}

static int mtx_read_dense_impl(const char* path, rls_c64* A, int64_t lda) {
  MtxFile mf;
  int rc = mf.open_header(path);
  if (rc != RLS_OK) return rc;
  if (!mf.dense) return mf.fail("coordinate format: read it with rls_mtx_read_csc");
  if (lda < std::max<int64_t>(mf.m, 1) || (!A && mf.m * mf.n > 0)) {
    rls_host_error("rls_mtx_read_dense: invalid arguments");
    return RLS_ERR_ARG;
  }
  for (int64_t j = 0; j < mf.n; ++j)
    for (int64_t i = 0; i < mf.m; ++i) A[j * lda + i] = rls_c64{0.0, 0.0};
  const int nv = mf.values_per_entry();
  int64_t q = 0;
  for (int64_t j = 0; j < mf.n; ++j) {
    const int64_t i0 = (mf.symm == S_GENERAL) ? 0 : (mf.symm == S_SKEW ? j + 1 : j);
    for (int64_t i = i0; i < mf.m; ++i, ++q) {
      double val[2] = {0.0, 0.0};
      rc = mf.next_numbers(0, nv, nullptr, val, q);
      if (rc != RLS_OK) return rc;
      const rls_c64 a{val[0], nv == 2 ? val[1] : 0.0};
      A[j * lda + i] = a;
      if (mf.symm != S_GENERAL && i != j) A[i * lda + j] = mirror(mf.symm, a);
    }
  }
  return RLS_OK;
}

// The C entry points: no exception crosses the ABI (an allocation that fails, e.g. for a size
// line far beyond the memory, returns RLS_ERR_NOMEM).
template <class F>
static int guarded(const char* what, F&& f) {
  try {
    return f();
  } catch (const std::bad_alloc&) {
    rls_host_error(std::string(what) + ": out of host memory");
    return RLS_ERR_NOMEM;
  } catch (const std::exception& e) {
    rls_host_error(std::string(what) + ": " + e.what());
    return RLS_ERR_ARG;
  }
}

extern "C" int rls_mtx_info(const char* path, int64_t* m, int64_t* n, int64_t* nnz_max, int* dense) {
  return guarded("rls_mtx_info", [&] { return mtx_info_impl(path, m, n, nnz_max, dense); });
}

extern "C" int rls_mtx_read_csc(const char* path, int base, int64_t cap, int64_t* colptr, int64_t* rowval,
                                rls_c64* nzval, int64_t* nnz) {
  return guarded("rls_mtx_read_csc", [&] { return mtx_read_csc_impl(path, base, cap, colptr, rowval, nzval, nnz); });
}

extern "C" int rls_mtx_read_dense(const char* path, rls_c64* A, int64_t lda) {
  return guarded("rls_mtx_read_dense", [&] { return mtx_read_dense_impl(path, A, lda); });
}
