"""Exact (rational) WENO-JS coefficients for arbitrary cell boundaries --
the checker of the library's weno_sb_coefficients (test infrastructure).

Written independently of the library's long-double generator: every
quantity is a Fraction, the candidate values come from solving the moment
system of the stencil polynomial (not the primitive-function Lagrange
form), the linear weights from Gaussian elimination over all 2R-1 cells of
the big stencil (asserting the over-determined system is consistent), and
beta from the Jiang-Shu integrals of the same polynomials.  Coordinates are
the physical ones (no rescaling): beta_r = sum_l h_j^(2l-1) int (p^(l))^2.
"""
from fractions import Fraction


def _solve(A, b):
    """Exact solution of the square system A x = b (lists of Fractions)."""
    n = len(A)
    M = [list(A[r]) + [b[r]] for r in range(n)]
    for c in range(n):
        p = next(r for r in range(c, n) if M[r][c] != 0)
        M[c], M[p] = M[p], M[c]
        pv = M[c][c]
        M[c] = [x / pv for x in M[c]]
        for r in range(n):
            if r != c and M[r][c] != 0:
                f = M[r][c]
                M[r] = [a - f * bb for a, bb in zip(M[r], M[c])]
    return [M[r][n] for r in range(n)]


def _poly(bounds):
    """Polynomial coefficients (in x) of the stencil polynomial as linear
    forms over its cells: coef[i][m]."""
    R = len(bounds) - 1
    A = [[(bounds[m + 1] ** (i + 1) - bounds[m] ** (i + 1)) / ((i + 1) * (bounds[m + 1] - bounds[m]))
          for i in range(R)] for m in range(R)]
    cols = []
    for m in range(R):
        e = [Fraction(int(k == m)) for k in range(R)]
        cols.append(_solve(A, e))          # coefficients for a unit average in cell m
    return [[cols[m][i] for m in range(R)] for i in range(R)]


def _value(coef, x0):
    R = len(coef)
    return [sum(coef[i][m] * x0 ** i for i in range(R)) for m in range(R)]


def _diff(lin):
    """Descending-difference coefficients of a zero-sum form over R cells."""
    R = len(lin)
    asc = []
    acc = Fraction(0)
    for k in range(R - 1):
        acc += lin[k]
        asc.append(-acc)
    return asc[::-1]


def face(xb, j, order):
    """(pL, pR, dL, dR, bq) of core cell j for cell boundaries xb (Fractions),
    per stencil r (cells j-r .. j-r+R-1); d indexed by stencil."""
    R = (order + 1) // 2
    h = xb[j + 1] - xb[j]
    xl, xr = xb[j], xb[j + 1]
    pL, pR, bq, S = [], [], [], []
    for r in range(R):
        c0 = j - r
        bnd = [xb[c0 + i] for i in range(R + 1)]
        coef = _poly(bnd)
        wl, wr = _value(coef, xl), _value(coef, xr)
        S.append((wl, wr))
        for w, out in ((wl, pL), (wr, pR)):
            lin = [w[m] - (1 if c0 + m == j else 0) for m in range(R)]
            out.append(_diff(lin))
        # beta: sum_l h^(2l-1) int_{xl}^{xr} (p^(l))^2 dx as a quadratic form
        # over the descending differences
        ad = {i: _diff(coef[i]) for i in range(1, R)}
        nd = R - 1
        Q = [[Fraction(0)] * nd for _ in range(nd)]
        for l in range(1, R):
            for i1 in range(l, R):
                for i2 in range(l, R):
                    f1 = f2 = 1
                    for q in range(i1 - l + 1, i1 + 1):
                        f1 *= q
                    for q in range(i2 - l + 1, i2 + 1):
                        f2 *= q
                    e = (i1 - l) + (i2 - l)
                    integ = (xr ** (e + 1) - xl ** (e + 1)) / (e + 1)
                    for a in range(nd):
                        for b in range(nd):
                            Q[a][b] += h ** (2 * l - 1) * f1 * f2 * integ * ad[i1][a] * ad[i2][b]
        row = []
        for a in range(nd):
            for b in range(a, nd):
                row.append(Q[a][a] if a == b else Q[a][b] + Q[b][a])
        bq.append(row)
    ds = []
    b0 = j - (R - 1)
    big = _poly([xb[b0 + i] for i in range(2 * R)])
    for side, x0 in ((0, xl), (1, xr)):
        W = _value(big, x0)
        rows = []
        for m in range(2 * R - 1):
            cell = b0 + m
            rows.append([S[r][side][cell - (j - r)] if 0 <= cell - (j - r) < R else Fraction(0) for r in range(R)]
                        + [W[m]])
        # eliminate over all rows; the extra rows must reduce to 0 = 0
        A = [list(rw) for rw in rows]
        n = R
        for c in range(n):
            p = next(r for r in range(c, len(A)) if A[r][c] != 0)
            A[c], A[p] = A[p], A[c]
            pv = A[c][c]
            A[c] = [x / pv for x in A[c]]
            for r in range(len(A)):
                if r != c and A[r][c] != 0:
                    f = A[r][c]
                    A[r] = [a - f * bb for a, bb in zip(A[r], A[c])]
        assert all(all(x == 0 for x in A[r]) for r in range(n, len(A))), "linear weights do not exist"
        ds.append([A[r][n] for r in range(R)])
    return pL, pR, ds[0], ds[1], bq
