// psPrecRecy's incomplete-Cholesky preconditioner build on the host: get_hsl_LLTP
// (src/preconditioner/hsl_preconditioner.jl:159-252).  It runs on the CPU, as the reference
// runs it; its factor is then applied on the device (rls_lltp_upload / rls_lltp_ldiv).
//
//   1. A = lower((C − zI)ᴴ(C − zI))                       (_build_hsl_normal_eq, :147-157)
//   2. A ← PᵀAP with the caller's permutation p           (permute_lower_csc!, permute_matrix.jl)
//   3. S = diag(1/sqrt(‖row i of A‖₂))                     (compute_scaling!, scale.jl, iscale = 1)
//   4. SAS + αI ≈ L̃ L̃ᴴ by the limited-memory threshold IC of the HSL MI28/MI35 codes (Scott &
//      Tůma) with a Tismenetsky–Kaporin R part (ictkl3_new!, ictkl3_new.jl), α grown on
//      breakdown                                          (ichsd, ichsd.jl:116-262)
//   5. L = S⁻¹ L̃ with the diagonal stored as is           (hsl_preconditioner.jl:238-246)
//
// Column j of L̃ is formed left-looking: its scaled column of A, minus (L̃ + R)·conj(L̃[j, :])
// and L̃·conj(R[j, :]) over earlier columns reached through per-row lists; the largest lsize
// (plus unused budget) entries of magnitude ≥ τ₁ stay in L̃ and subtract their squares from
// the later diagonals, the next largest rsize (> τ₂) go to R, the rest are dropped.  Which
// entries survive a magnitude tie depends on the scatter order and on the partition scheme,
// so both follow the reference step for step (and the CPU restatement in oracle/icfact.py
// follows the same steps): this code is compiled with -ffp-contract=off and gives the same
// bits.  Only the default control of get_hsl_LLTP is supported (iscale = 1, rrt = false,
// small = 1e-20, lowalpha = 1e-3 unless α > 0, shift factor 2).
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <string>
#include <thread>
#include <vector>

#include "../../include/rls_b200.h"
#include "host_err.h"

namespace {

using cd = std::complex<double>;
// a·b as Julia's `*` on Complex{Float64} forms it, (ac − bd) + i(ad + bc): the same bits as
// std::complex's operator* whenever that is not NaN, without its Annex G recovery call.
inline cd mulc(cd a, cd b) {
  return cd(a.real() * b.real() - a.imag() * b.imag(), a.real() * b.imag() + a.imag() * b.real());
}

constexpr double kSmall = 1e-20;
constexpr double kLowAlpha = 1e-3;
constexpr double kShiftFactor = 2.0;
constexpr int kMaxShifts = 200;   // the reference retries without limit; 2^200 is past any scale

struct Csc {   // 0-based
  std::vector<int64_t> ptr, row;
  std::vector<cd> val;
};

// lower((C − zI)ᴴ(C − zI)), accumulated as SparseArrays' sparse product does; every diagonal
// entry of C − zI is stored.
Csc normal_lower(int64_t n, const Csc& C, cd z) {
  Csc cz;
  cz.ptr.assign((size_t)n + 1, 0);
  for (int64_t j = 0; j < n; ++j) {
    bool diag = false;
    for (int64_t q = C.ptr[(size_t)j]; q < C.ptr[(size_t)j + 1]; ++q) {
      const int64_t r = C.row[(size_t)q];
      if (!diag && r > j) {
        cz.row.push_back(j);
        cz.val.push_back(-z);
        diag = true;
      }
      cz.row.push_back(r);
      cz.val.push_back(r == j ? C.val[(size_t)q] - z : C.val[(size_t)q]);
      if (r == j) diag = true;
    }
    if (!diag) {
      cz.row.push_back(j);
      cz.val.push_back(-z);
    }
    cz.ptr[(size_t)j + 1] = (int64_t)cz.row.size();
  }
  // (C − zI)ᴴ: column k holds (j, conj(Cz[k, j])) for ascending j
  Csc h;
  h.ptr.assign((size_t)n + 1, 0);
  for (int64_t q = 0; q < (int64_t)cz.row.size(); ++q) ++h.ptr[(size_t)cz.row[(size_t)q] + 1];
  for (int64_t k = 0; k < n; ++k) h.ptr[(size_t)k + 1] += h.ptr[(size_t)k];
  h.row.resize(cz.row.size());
  h.val.resize(cz.row.size());
  std::vector<int64_t> cur(h.ptr.begin(), h.ptr.end() - 1);
  for (int64_t j = 0; j < n; ++j)
    for (int64_t q = cz.ptr[(size_t)j]; q < cz.ptr[(size_t)j + 1]; ++q) {
      const int64_t k = cz.row[(size_t)q];
      const int64_t at = cur[(size_t)k]++;
      h.row[(size_t)at] = j;
      h.val[(size_t)at] = std::conj(cz.val[(size_t)q]);
    }
  // columns are independent: contiguous column ranges on host threads, each column summed in
  // the same order as a single thread would, then concatenated
  const int64_t nthreads = std::max<int64_t>(1, std::min<int64_t>((int64_t)std::thread::hardware_concurrency(),
                                                                  std::min<int64_t>(16, n / 256 + 1)));
  std::vector<Csc> part((size_t)nthreads);
  auto run = [&](int64_t t) {
    const int64_t j0 = n * t / nthreads, j1 = n * (t + 1) / nthreads;
    Csc& a = part[(size_t)t];
    a.ptr.assign((size_t)(j1 - j0) + 1, 0);
    std::vector<int64_t> seen((size_t)n, -1);
    std::vector<cd> x((size_t)n);
    std::vector<int64_t> touched;
    for (int64_t j = j0; j < j1; ++j) {
      touched.clear();
      for (int64_t qb = cz.ptr[(size_t)j]; qb < cz.ptr[(size_t)j + 1]; ++qb) {
        const int64_t k = cz.row[(size_t)qb];
        const cd b = cz.val[(size_t)qb];
        for (int64_t qa = h.ptr[(size_t)k]; qa < h.ptr[(size_t)k + 1]; ++qa) {
          const int64_t i = h.row[(size_t)qa];
          const cd t2 = mulc(h.val[(size_t)qa], b);
          if (seen[(size_t)i] != j) {
            seen[(size_t)i] = j;
            x[(size_t)i] = t2;
            touched.push_back(i);
          } else {
            x[(size_t)i] += t2;
          }
        }
      }
      std::sort(touched.begin(), touched.end());
      for (int64_t i : touched)
        if (i >= j) {
          a.row.push_back(i);
          a.val.push_back(x[(size_t)i]);
        }
      a.ptr[(size_t)(j - j0) + 1] = (int64_t)a.row.size();
    }
  };
  std::vector<std::thread> pool;
  for (int64_t t = 1; t < nthreads; ++t) pool.emplace_back(run, t);
  run(0);
  for (auto& th : pool) th.join();
  Csc a;
  a.ptr.assign((size_t)n + 1, 0);
  for (int64_t t = 0; t < nthreads; ++t) {
    const int64_t j0 = n * t / nthreads, j1 = n * (t + 1) / nthreads;
    const int64_t base = (int64_t)a.row.size();
    a.row.insert(a.row.end(), part[(size_t)t].row.begin(), part[(size_t)t].row.end());
    a.val.insert(a.val.end(), part[(size_t)t].val.begin(), part[(size_t)t].val.end());
    for (int64_t j = j0; j < j1; ++j) a.ptr[(size_t)j + 1] = base + part[(size_t)t].ptr[(size_t)(j - j0) + 1];
  }
  return a;
}

// PᵀAP of a lower CSC matrix: entry (i, j) moves to (newidx[i], newidx[j]) and is reflected
// (conjugated) into the lower triangle; each column keeps its diagonal first and the other
// entries in the order they are scattered.
Csc permute_lower(int64_t n, const Csc& A, const std::vector<int64_t>& newidx) {
  std::vector<int64_t> cnt((size_t)n, 0);
  for (int64_t j = 0; j < n; ++j)
    for (int64_t q = A.ptr[(size_t)j]; q < A.ptr[(size_t)j + 1]; ++q) {
      const int64_t i2 = newidx[(size_t)A.row[(size_t)q]], j2 = newidx[(size_t)j];
      ++cnt[(size_t)(i2 < j2 ? i2 : j2)];
    }
  Csc P;
  P.ptr.assign((size_t)n + 1, 0);
  std::vector<int64_t> cur((size_t)n);
  for (int64_t j = 0; j < n; ++j) {
    P.ptr[(size_t)j + 1] = P.ptr[(size_t)j] + cnt[(size_t)j];
    cur[(size_t)j] = P.ptr[(size_t)j] + 1;
  }
  P.row.assign((size_t)P.ptr[(size_t)n], 0);
  P.val.assign((size_t)P.ptr[(size_t)n], cd(0.0, 0.0));
  for (int64_t j = 0; j < n; ++j) {
    const int64_t j2 = newidx[(size_t)j];
    for (int64_t q = A.ptr[(size_t)j]; q < A.ptr[(size_t)j + 1]; ++q) {
      const int64_t i2 = newidx[(size_t)A.row[(size_t)q]];
      if (i2 == j2) {
        P.row[(size_t)P.ptr[(size_t)j2]] = j2;
        P.val[(size_t)P.ptr[(size_t)j2]] = A.val[(size_t)q];
      } else if (i2 < j2) {
        const int64_t at = cur[(size_t)i2]++;
        P.row[(size_t)at] = j2;
        P.val[(size_t)at] = std::conj(A.val[(size_t)q]);
      } else {
        const int64_t at = cur[(size_t)j2]++;
        P.row[(size_t)at] = i2;
        P.val[(size_t)at] = A.val[(size_t)q];
      }
    }
  }
  return P;
}

// 1/sqrt(‖row i‖₂) of the symmetric matrix held by its lower triangle (1 for an empty row).
std::vector<double> l2_scaling(int64_t n, const Csc& A) {
  std::vector<double> s((size_t)n, 0.0);
  for (int64_t i = 0; i < n; ++i)
    for (int64_t q = A.ptr[(size_t)i]; q < A.ptr[(size_t)i + 1]; ++q) {
      const int64_t k = A.row[(size_t)q];
      const double m = std::abs(A.val[(size_t)q]);
      const double t2 = m * m;
      s[(size_t)k] += t2;
      if (k != i) s[(size_t)i] += t2;
    }
  for (auto& v : s) v = std::sqrt(v);
  for (auto& v : s) v = v > 0.0 ? 1.0 / std::sqrt(v) : 1.0;
  return s;
}

// Partial partition of ix[0, n) by mag[ix] (each candidate's |w|, computed once per column):
// afterwards positions ncut..n (1-based) hold the n − ncut + 1 largest (a quickselect with
// the last element as pivot, larger values moved to the right end; the scheme of split2!,
// ictkl3.jl:9-44).
void partition_largest(int64_t n, int64_t ncut, std::vector<int64_t>& ix, const std::vector<double>& mag) {
  if (n <= 1 || ncut <= 0 || ncut > n) return;
  int64_t first = 1, last = n;
  while (first < last) {
    int64_t mid = last;
    const double pivot = mag[(size_t)ix[(size_t)mid - 1]];
    for (int64_t j = last - 1; j >= first; --j)
      if (mag[(size_t)ix[(size_t)j - 1]] > pivot) {
        --mid;
        std::swap(ix[(size_t)mid - 1], ix[(size_t)j - 1]);
      }
    std::swap(ix[(size_t)mid - 1], ix[(size_t)last - 1]);
    if (mid > ncut) last = mid - 1;
    else if (mid < ncut) first = mid + 1;
    else break;
  }
}

struct Factor {
  std::vector<int64_t> lp, lr, rp, rr;
  std::vector<cd> lv, rv;
};

// One attempt on the scaled, shifted matrix (diagonal d); 0, or −j (1-based column) on
// breakdown.  The L diagonal holds 1/sqrt(d_j).
int64_t ic_attempt(int64_t n, const Csc& A, const std::vector<double>& scale, std::vector<double>& d, int64_t lsize,
                   int64_t rsize, double tau1, double tau2, Factor& F) {
  F.lp.assign((size_t)n + 1, 0);
  F.rp.assign((size_t)n + 1, 0);
  F.lr.clear();
  F.lv.clear();
  F.rr.clear();
  F.rv.clear();
  // per-row lists of earlier columns whose next unread entry lies in that row (L and R)
  std::vector<int64_t> headl((size_t)n, -1), nextl((size_t)n, -1), headr((size_t)n, -1), nextr((size_t)n, -1);
  std::vector<int64_t> posl((size_t)n, 0), posr((size_t)n, 0);
  std::vector<cd> w((size_t)n, cd(0.0, 0.0));
  std::vector<double> mag((size_t)n, 0.0);
  std::vector<char> mark((size_t)n, 0);
  std::vector<int64_t> lst;
  lst.reserve((size_t)n);
  std::vector<std::pair<int64_t, cd>> seg;
  int64_t saved = 0, savedr = 0;
  auto add = [&](int64_t k, cd t) {
    if (mark[(size_t)k]) {
      w[(size_t)k] += t;
    } else {
      lst.push_back(k);
      mark[(size_t)k] = 1;
      w[(size_t)k] = t;
    }
  };
  for (int64_t j = 0; j < n; ++j) {
    const double dj = d[(size_t)j];
    if (dj < kSmall) return -(j + 1);
    lst.clear();
    for (int64_t q = A.ptr[(size_t)j] + 1; q < A.ptr[(size_t)j + 1]; ++q) {
      const int64_t i = A.row[(size_t)q];
      w[(size_t)i] = A.val[(size_t)q] * (scale[(size_t)i] * scale[(size_t)j]);
      mark[(size_t)i] = 1;
      lst.push_back(i);
    }
    // updates from earlier L columns with an entry in row j: their L and R parts
    for (int64_t c = headl[(size_t)j]; c != -1;) {
      const int64_t cn = nextl[(size_t)c];
      const int64_t ks = posl[(size_t)c];
      const cd ljc = std::conj(F.lv[(size_t)ks]);
      const int64_t i0 = ks + 1, i1 = F.lp[(size_t)c + 1];
      if (i0 < i1) {
        posl[(size_t)c] = i0;
        const int64_t r = F.lr[(size_t)i0];
        nextl[(size_t)c] = headl[(size_t)r];
        headl[(size_t)r] = c;
      }
      for (int64_t q = i0; q < i1; ++q) add(F.lr[(size_t)q], -mulc(F.lv[(size_t)q], ljc));
      for (int64_t q = posr[(size_t)c]; q < F.rp[(size_t)c + 1]; ++q) {
        const int64_t k = F.rr[(size_t)q];
        if (k > j) add(k, -mulc(F.rv[(size_t)q], ljc));
      }
      c = cn;
    }
    // updates from earlier R columns with an entry in row j: their L parts
    for (int64_t c = headr[(size_t)j]; c != -1;) {
      const int64_t cn = nextr[(size_t)c];
      const int64_t ks = posr[(size_t)c];
      const cd rjc = std::conj(F.rv[(size_t)ks]);
      const int64_t r0 = ks + 1, r1 = F.rp[(size_t)c + 1];
      if (r0 < r1) {
        posr[(size_t)c] = r0;
        const int64_t r = F.rr[(size_t)r0];
        nextr[(size_t)c] = headr[(size_t)r];
        headr[(size_t)r] = c;
      }
      for (int64_t q = posl[(size_t)c]; q < F.lp[(size_t)c + 1]; ++q) {
        const int64_t k = F.lr[(size_t)q];
        if (k > j) add(k, -mulc(F.lv[(size_t)q], rjc));
      }
      c = cn;
    }
    const double djt = 1.0 / std::sqrt(dj);
    F.lr.push_back(j);
    F.lv.push_back(cd(djt, 0.0));
    const int64_t nw = (int64_t)lst.size();
    for (int64_t k : lst) {
      w[(size_t)k] = w[(size_t)k] * djt;
      mag[(size_t)k] = std::abs(w[(size_t)k]);
      mark[(size_t)k] = 0;
    }
    const int64_t jsize = std::min(lsize + saved, nw);
    saved += lsize - jsize;
    const int64_t largep = nw - jsize + 1;   // 1-based start of the kept candidates
    if (nw >= 1) {
      partition_largest(nw, largep, lst, mag);
      std::sort(lst.begin() + (largep - 1), lst.end());
      int64_t indr = largep;
      for (int64_t pos = largep; pos <= nw; ++pos) {
        const int64_t k = lst[(size_t)pos - 1];
        const cd t = w[(size_t)k];
        const double m = mag[(size_t)k];
        if (m >= tau1) {
          d[(size_t)k] -= t.real() * t.real() + t.imag() * t.imag();
          if (d[(size_t)k] <= kSmall && k > j) return -(j + 1);
          F.lv.push_back(t);
          F.lr.push_back(k);
        } else if (m > 0.0 && m > tau2) {
          lst[(size_t)indr - 1] = k;
          ++indr;
        }
      }
      const int64_t radd = std::min(indr - 1, rsize + savedr);
      const int64_t larger = (indr - 1) - radd + 1;
      partition_largest(indr - 1, larger, lst, mag);
      savedr += rsize - radd;
      seg.clear();
      for (int64_t pos = larger; pos <= indr - 1; ++pos) {
        const int64_t k = lst[(size_t)pos - 1];
        const cd t = w[(size_t)k];
        w[(size_t)k] = cd(0.0, 0.0);
        if (tau2 == 0.0 || mag[(size_t)k] > tau2) seg.emplace_back(k, t);
      }
      for (int64_t pos = 1; pos < larger; ++pos) w[(size_t)lst[(size_t)pos - 1]] = cd(0.0, 0.0);
      std::sort(seg.begin(), seg.end(), [](const auto& x, const auto& y) { return x.first < y.first; });
      for (const auto& e : seg) {
        F.rr.push_back(e.first);
        F.rv.push_back(e.second);
      }
    }
    F.lp[(size_t)j + 1] = (int64_t)F.lr.size();
    F.rp[(size_t)j + 1] = (int64_t)F.rr.size();
    posl[(size_t)j] = F.lp[(size_t)j] + 1;
    if (F.lp[(size_t)j + 1] > F.lp[(size_t)j] + 1) {
      const int64_t r = F.lr[(size_t)F.lp[(size_t)j] + 1];
      nextl[(size_t)j] = headl[(size_t)r];
      headl[(size_t)r] = j;
    }
    if (F.rp[(size_t)j + 1] > F.rp[(size_t)j]) {
      posr[(size_t)j] = F.rp[(size_t)j];
      const int64_t r = F.rr[(size_t)F.rp[(size_t)j]];
      nextr[(size_t)j] = headr[(size_t)r];
      headr[(size_t)r] = j;
    } else {
      posr[(size_t)j] = F.rp[(size_t)j] + 1;
    }
  }
  return 0;
}

}  // namespace

extern "C" int rls_ic_factor(int64_t n, const int64_t* colptr, const int64_t* rowval, const rls_c64* nzval, int base,
                             rls_c64 z, double tau1, double tau2, double alpha, int64_t lsize, int64_t rsize,
                             const int64_t* p, int64_t cap, int64_t* lcolptr, int64_t* lrowval, rls_c64* lnzval,
                             int64_t* invp, double* shift_used) {
  if (n < 1 || !colptr || !p || !lcolptr || !invp || (base != 0 && base != 1)) {
    rls_host_error("rls_ic_factor: invalid arguments");
    return RLS_ERR_ARG;
  }
  if (!std::isfinite(z.re) || !std::isfinite(z.im) || !std::isfinite(alpha) || !std::isfinite(tau1) ||
      !std::isfinite(tau2)) {
    rls_host_error("rls_ic_factor: the shift z, α and the drop tolerances must be finite");
    return RLS_ERR_ARG;
  }
  if (rsize < 0 || (n > 1 && lsize < 1)) {
    rls_host_error("rls_ic_factor: lsize must be at least 1 and rsize at least 0 (lsize=" + std::to_string(lsize) +
                   ", rsize=" + std::to_string(rsize) + ")");
    return RLS_ERR_ARG;
  }
  const int64_t nnz = colptr[n] - base;
  if (colptr[0] != base || nnz < 0 || (nnz > 0 && (!rowval || !nzval))) {
    rls_host_error("rls_ic_factor: inconsistent column pointers");
    return RLS_ERR_DIM;
  }
  Csc C;
  C.ptr.resize((size_t)n + 1);
  for (int64_t j = 0; j <= n; ++j) C.ptr[(size_t)j] = colptr[j] - base;
  C.row.resize((size_t)nnz);
  C.val.resize((size_t)nnz);
  for (int64_t j = 0; j < n; ++j) {
    if (C.ptr[(size_t)j + 1] < C.ptr[(size_t)j]) {
      rls_host_error("rls_ic_factor: column pointers decrease at column " + std::to_string(j + 1));
      return RLS_ERR_DIM;
    }
    for (int64_t q = C.ptr[(size_t)j]; q < C.ptr[(size_t)j + 1]; ++q) {
      const int64_t r = rowval[q] - base;
      if (r < 0 || r >= n) {
        rls_host_error("rls_ic_factor: row index " + std::to_string(r + 1) + " out of range 1.." + std::to_string(n));
        return RLS_ERR_DIM;
      }
      if (q > C.ptr[(size_t)j] && r <= C.row[(size_t)q - 1]) {
        rls_host_error("rls_ic_factor: row indices of column " + std::to_string(j + 1) +
                       " are not strictly increasing (SparseMatrixCSC order)");
        return RLS_ERR_ARG;
      }
      if (!std::isfinite(nzval[q].re) || !std::isfinite(nzval[q].im)) {
        rls_host_error("rls_ic_factor: non-finite entry in column " + std::to_string(j + 1));
        return RLS_ERR_ARG;
      }
      C.row[(size_t)q] = r;
      C.val[(size_t)q] = cd(nzval[q].re, nzval[q].im);
    }
  }
  std::vector<int64_t> inv((size_t)n, -1);
  for (int64_t i = 0; i < n; ++i) {
    const int64_t v = p[i] - base;
    if (v < 0 || v >= n || inv[(size_t)v] != -1) {
      rls_host_error("rls_ic_factor: p is not a permutation of 1.." + std::to_string(n));
      return RLS_ERR_ARG;
    }
    inv[(size_t)v] = i;
  }
  const int64_t lsz = std::min<int64_t>(std::max<int64_t>(0, lsize), n - 1);
  if (cap < n + lsz * n) {
    rls_host_error("rls_ic_factor: capacity " + std::to_string(cap) + " below n·(1 + lsize) = " +
                   std::to_string(n + lsz * n));
    return RLS_ERR_DIM;
  }
  const Csc A = permute_lower(n, normal_lower(n, C, cd(z.re, z.im)), inv);
  const std::vector<double> scale = l2_scaling(n, A);
  // the initial shift (ichsd.jl:17-45)
  const double alpha_in = std::max(0.0, alpha);
  const double lowalpha = alpha_in > 0.0 ? alpha_in : kLowAlpha;
  double a = alpha_in;
  if (a == 0.0) {
    for (int64_t i = 0; i < n; ++i) {
      const cd di = A.val[(size_t)A.ptr[(size_t)i]];
      const double sca = scale[(size_t)i] * scale[(size_t)i];
      if (std::abs(di) == 0.0) a = lowalpha;
      else if (di.real() < 0.0) a = std::max(a, -di.real() * sca);
    }
    if (a > 0.0) a = std::max(a, lowalpha);
  }
  Factor F;
  std::vector<double> d((size_t)n);
  int64_t flag = 0;
  for (int tries = 0;; ++tries) {
    if (tries > kMaxShifts) {
      rls_host_error("rls_ic_factor: the factorisation broke down at every diagonal shift up to " + std::to_string(a));
      return RLS_ERR_BREAKDOWN;
    }
    const int64_t flag_prev = flag;
    for (int64_t i = 0; i < n; ++i) {
      const double sc = scale[(size_t)i] * scale[(size_t)i];
      d[(size_t)i] = A.val[(size_t)A.ptr[(size_t)i]].real() * sc + a;
    }
    flag = ic_attempt(n, A, scale, d, lsz, rsize, tau1, tau2, F);
    if (flag < 0) {
      a = std::max(kShiftFactor * a, lowalpha);
      if (flag_prev != 0 && std::llabs(flag - flag_prev) <= n / 10 && n + flag >= n / 10)
        a = std::max(kShiftFactor * a, lowalpha);
      continue;
    }
    break;
  }
  // the stored diagonal 1/sqrt(d_j) becomes sqrt(d_j) (as 1/(1/sqrt(d_j))), then rows are
  // scaled back by S⁻¹
  for (int64_t j = 0; j < n; ++j) {
    cd& v = F.lv[(size_t)F.lp[(size_t)j]];
    v = cd(1.0 / v.real(), 0.0);
  }
  const int64_t nl = (int64_t)F.lr.size();
  for (int64_t q = 0; q < nl; ++q) {
    const cd v = F.lv[(size_t)q] * (1.0 / scale[(size_t)F.lr[(size_t)q]]);
    if (lrowval) lrowval[q] = F.lr[(size_t)q] + base;
    if (lnzval) lnzval[q] = rls_c64{v.real(), v.imag()};
  }
  for (int64_t j = 0; j <= n; ++j) lcolptr[j] = F.lp[(size_t)j] + base;
  for (int64_t i = 0; i < n; ++i) invp[i] = inv[(size_t)i] + base;
  if (shift_used) *shift_used = a;
  return RLS_OK;
}
