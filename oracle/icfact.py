"""CPU restatement of get_hsl_LLTP, psPrecRecy's incomplete-Cholesky preconditioner build —
test infrastructure only.

get_hsl_LLTP (src/preconditioner/hsl_preconditioner.jl:159-252) forms the lower triangle of the
shifted normal matrix (C − zI)ᴴ(C − zI) (_build_hsl_normal_eq, :147-157), permutes it
symmetrically (permute_lower_csc!, permute_matrix.jl:5-69), scales it by inverse square roots
of its row 2-norms (compute_scaling!, scale.jl:14-81, iscale = 1), and factors it with the
limited-memory threshold incomplete Cholesky of the HSL MI28/MI35 codes (Scott & Tůma) with a
Tismenetsky–Kaporin R part, retried with a growing diagonal shift on breakdown (ichsd,
ichsd.jl:116-262; ictkl3_new!, ictkl3_new.jl:1-291).  The stored factor's diagonal is then
inverted and its rows scaled back (:238-246), so that PᵀAP ≈ L Lᴴ.

The step order below is the reference's own (which entries survive a magnitude tie depends on
the scatter order and the partition scheme of split2!, ictkl3.jl:9-44), so that the C++ build
(rls_ic_factor) can be held to it bit for bit.  Pure Python: small n only.
"""
from __future__ import annotations

import math

import numpy as np
import scipy.sparse as sp

SMALL = 1e-20          # mi35_control.small
LOWALPHA = 1e-3        # ALPHAM
SHIFT_FACTOR = 2.0     # SF_DEFAULT


def normal_lower(C, z):
    """lower((C − zI)ᴴ(C − zI)) as 0-based CSC lists (ptr, row, val), rows ascending, with
    the product accumulated as SparseArrays' spmatmul does (column j: for each stored (k, b)
    of Cz[:, j], for each stored (i, a) of Czᴴ[:, k]: x[i] += a·b).  Cz stores every diagonal
    entry (C[i, i] − z)."""
    A = sp.csc_matrix(C, dtype=np.complex128)
    A.sort_indices()
    n = A.shape[0]
    z = complex(z)
    # Cz columns
    cz = []
    for j in range(n):
        rows = [int(r) for r in A.indices[A.indptr[j]:A.indptr[j + 1]]]
        vals = [complex(v) for v in A.data[A.indptr[j]:A.indptr[j + 1]]]
        if j in rows:
            q = rows.index(j)
            vals[q] = vals[q] - z
        else:
            q = 0
            while q < len(rows) and rows[q] < j:
                q += 1
            rows.insert(q, j)
            vals.insert(q, -z)
        cz.append((rows, vals))
    # Czᴴ columns: column k holds (j, conj(Cz[k, j])) for ascending j
    czh = [([], []) for _ in range(n)]
    for j in range(n):
        for r, v in zip(*cz[j]):
            czh[r][0].append(j)
            czh[r][1].append(v.conjugate())
    ptr, row, val = [0], [], []
    for j in range(n):
        x = {}
        for k, b in zip(*cz[j]):
            for i, a in zip(*czh[k]):
                if i in x:
                    x[i] = x[i] + a * b
                else:
                    x[i] = a * b
        for i in sorted(x):
            if i >= j:
                row.append(i)
                val.append(x[i])
        ptr.append(len(row))
    return ptr, row, val


def permute_lower(n, ptr, row, val, newidx):
    """P'AP of a lower CSC matrix (permute_lower_csc!): entry (i, j) goes to (newidx[i],
    newidx[j]), reflected (and conjugated) into the lower triangle; the diagonal first in
    each column, the other entries in scatter order."""
    cnt = [0] * n
    for j in range(n):
        j2 = newidx[j]
        for q in range(ptr[j], ptr[j + 1]):
            i2 = newidx[row[q]]
            cnt[i2 if i2 < j2 else j2] += 1
    pp = [0] * (n + 1)
    cur = [0] * n
    for j in range(n):
        pp[j + 1] = pp[j] + cnt[j]
        cur[j] = pp[j] + 1
    rp = [0] * pp[n]
    vp = [0j] * pp[n]
    for j in range(n):
        j2 = newidx[j]
        for q in range(ptr[j], ptr[j + 1]):
            i2 = newidx[row[q]]
            if i2 == j2:
                rp[pp[j2]] = j2
                vp[pp[j2]] = val[q]
            elif i2 < j2:
                rp[cur[i2]] = j2
                vp[cur[i2]] = val[q].conjugate()
                cur[i2] += 1
            else:
                rp[cur[j2]] = i2
                vp[cur[j2]] = val[q]
                cur[j2] += 1
    return pp, rp, vp


def l2_scaling(n, ptr, row, val):
    """1/sqrt(‖row i‖₂) of the symmetric matrix held by its lower triangle (1 where zero)."""
    s = [0.0] * n
    for i in range(n):
        for q in range(ptr[i], ptr[i + 1]):
            k = row[q]
            m = abs(val[q])
            t2 = m * m
            s[k] += t2
            if k != i:
                s[i] += t2
    s = [math.sqrt(v) for v in s]
    return [1.0 / math.sqrt(v) if v > 0.0 else 1.0 for v in s]


def _split2(n, ncut, ix, w):
    """Partial partition of ix[0:n] by |w[ix]| so that positions ncut..n (1-based) hold the
    n − ncut + 1 largest (split2!, ictkl3.jl:9-44)."""
    if n <= 1 or ncut <= 0 or ncut > n:
        return
    first, last = 1, n
    while first < last:
        mid = last
        midval = abs(w[ix[mid - 1]])
        for j in range(last - 1, first - 1, -1):
            if abs(w[ix[j - 1]]) > midval:
                mid -= 1
                ix[mid - 1], ix[j - 1] = ix[j - 1], ix[mid - 1]
        ix[mid - 1], ix[last - 1] = ix[last - 1], ix[mid - 1]
        if mid > ncut:
            last = mid - 1
        elif mid < ncut:
            first = mid + 1
        else:
            break


def _ic_trial(n, ptr, row, val, scale, d, lsize, rsize, tau1, tau2):
    """One factorisation attempt (ictkl3_new!, rrt = false).  Returns (info, Lptr, Lrow, Lval)
    with info = −j (1-based column) on breakdown; the L diagonal holds 1/sqrt(d_j)."""
    LP = [0] * (n + 1)
    LR, LV = [], []
    RP = [0] * (n + 1)
    RR, RV = [], []
    nextl = [-1] * n      # next column in the same row list (L)
    headl = [-1] * n      # first column waiting at row r (L)
    nextr = [-1] * n
    headr = [-1] * n
    posl = [0] * n        # next unread L entry of column c
    posr = [0] * n
    w = [0j] * n
    mark = [False] * n
    saved = savedr = 0
    for j in range(n):
        dj = d[j]
        if dj < SMALL:
            return -(j + 1), None, None, None
        lst = []
        for q in range(ptr[j] + 1, ptr[j + 1]):
            i = row[q]
            w[i] = val[q] * (scale[i] * scale[j])
            mark[i] = True
            lst.append(i)

        def acc(k, t):
            if mark[k]:
                w[k] = w[k] + t
            else:
                lst.append(k)
                mark[k] = True
                w[k] = t

        c = headl[j]
        while c != -1:
            cn = nextl[c]
            ks = posl[c]
            temp = LV[ks]
            i0, i1 = ks + 1, LP[c + 1]
            if i0 < i1:
                posl[c] = i0
                r = LR[i0]
                nextl[c] = headl[r]
                headl[r] = c
            for q in range(i0, i1):
                acc(LR[q], -(LV[q] * temp.conjugate()))
            for q in range(posr[c], RP[c + 1]):
                k = RR[q]
                if k > j:
                    acc(k, -(RV[q] * temp.conjugate()))
            c = cn
        c = headr[j]
        while c != -1:
            cn = nextr[c]
            ks = posr[c]
            temp = RV[ks]
            r0, r1 = ks + 1, RP[c + 1]
            if r0 < r1:
                posr[c] = r0
                r = RR[r0]
                nextr[c] = headr[r]
                headr[r] = c
            for q in range(posl[c], LP[c + 1]):
                k = LR[q]
                if k > j:
                    acc(k, -(LV[q] * temp.conjugate()))
            c = cn
        djt = 1.0 / math.sqrt(dj)
        LR.append(j)
        LV.append(complex(djt, 0.0))
        nw = len(lst)
        for k in lst:
            w[k] = w[k] * djt
            mark[k] = False
        jsize = min(lsize + saved, nw)
        saved += lsize - jsize
        largep = nw - jsize + 1
        if nw >= 1:
            _split2(nw, largep, lst, w)
            lst[largep - 1:nw] = sorted(lst[largep - 1:nw])
            indr = largep
            for pos in range(largep, nw + 1):
                k = lst[pos - 1]
                temp = w[k]
                a = abs(temp)
                if a >= tau1:
                    d[k] -= temp.real * temp.real + temp.imag * temp.imag
                    if d[k] <= SMALL and k > j:
                        return -(j + 1), None, None, None
                    LV.append(temp)
                    LR.append(k)
                elif a > 0.0 and a > tau2:
                    lst[indr - 1] = k
                    indr += 1
            radd = min(indr - 1, rsize + savedr)
            larger = (indr - 1) - radd + 1
            _split2(indr - 1, larger, lst, w)
            savedr += rsize - radd
            rstart = len(RR)
            for pos in range(larger, indr):
                k = lst[pos - 1]
                temp = w[k]
                w[k] = 0j
                if tau2 == 0.0 or abs(temp) > tau2:
                    RV.append(temp)
                    RR.append(k)
            for pos in range(1, larger):
                w[lst[pos - 1]] = 0j
            seg = sorted(zip(RR[rstart:], RV[rstart:]), key=lambda t: t[0])
            RR[rstart:] = [t[0] for t in seg]
            RV[rstart:] = [t[1] for t in seg]
        LP[j + 1] = len(LR)
        RP[j + 1] = len(RR)
        posl[j] = LP[j] + 1
        if LP[j + 1] > LP[j] + 1:
            r = LR[LP[j] + 1]
            nextl[j] = headl[r]
            headl[r] = j
        if RP[j + 1] > RP[j]:
            posr[j] = RP[j]
            r = RR[RP[j]]
            nextr[j] = headr[r]
            headr[r] = j
        else:
            posr[j] = RP[j] + 1
    return 0, LP, LR, LV


def ic_factor(C, z, tau1, tau2, alpha, lsize, rsize, p):
    """get_hsl_LLTP(C, z, tau1, tau2, α, lsize, rsize, p) with 0-based p: returns (L as a CSC
    matrix, invp, the diagonal shift used)."""
    n = C.shape[0]
    p = [int(v) for v in p]
    invp = [0] * n
    for i in range(n):
        invp[p[i]] = i
    ptr, row, val = normal_lower(C, z)
    pp, rp, vp = permute_lower(n, ptr, row, val, invp)
    scale = l2_scaling(n, pp, rp, vp)
    lsize = min(max(0, lsize), n - 1)
    # initial shift (_initial_mi35_shift, ichsd.jl:17-45)
    alpha_in = max(0.0, alpha)
    lowalpha = alpha_in if alpha_in > 0.0 else LOWALPHA
    a = alpha_in
    if a == 0.0:
        for i in range(n):
            di = vp[pp[i]]
            sca = scale[i] * scale[i]
            if abs(di) == 0.0:
                a = lowalpha
            elif di.real < 0.0:
                a = max(a, -di.real * sca)
        if a > 0.0:
            a = max(a, lowalpha)
    flag = 0
    while True:
        flag_prev = flag
        d = [vp[pp[i]].real * (scale[i] * scale[i]) + a for i in range(n)]
        flag, LP, LR, LV = _ic_trial(n, pp, rp, vp, scale, d, lsize, rsize, tau1, tau2)
        if flag < 0:
            a = max(SHIFT_FACTOR * a, lowalpha)
            if flag_prev != 0:
                if abs(flag - flag_prev) <= n // 10 and n + flag >= n // 10:
                    a = max(SHIFT_FACTOR * a, lowalpha)
            continue
        break
    # invert the diagonal, scale rows back (hsl_preconditioner.jl:238-246)
    for j in range(n):
        q = LP[j]
        LV[q] = 1.0 / LV[q]
    LV = [v * (1.0 / scale[r]) for r, v in zip(LR, LV)]
    L = sp.csc_matrix((np.array(LV, dtype=np.complex128), np.array(LR, dtype=np.int64),
                       np.array(LP, dtype=np.int64)), shape=(n, n))
    return L, np.array(invp, dtype=np.int64), a
