"""Input generators for the WENO path (host side, numpy, Fortran order).

* harness_field / harness_coefficients: the reference harness's own
  synthetic data (wilfonba/WenoStandalone inputs/weno_standalone.f90:221-279),
  used by the driver, the golden checksums and the bench's drop-in case.
* smooth_jump_field: seeded smooth-plus-jump field (a sinusoid per variable,
  +-1e-3 uniform noise, a +1 Heaviside jump at x > 1/2 on odd variables).
* sinusoid_shock_field: modes 1..8 around a mean of 1 plus one planar shock
  of jump ratio 5 at a seeded orientation (the mixed-precision workload).
* uniform_weno_coefficients: the true uniform-grid WENO-JS polynomial,
  ideal-weight and smoothness-indicator coefficients, in the reference's
  array layouts, derived in exact rational arithmetic.

Random numbers come from a splitmix64 stream: element number k (0-based, in
Fortran order of the array) uses splitmix64(seed + (k+1) * 0x9E3779B97F4A7C15)
mapped to [0, 1) by its top 53 bits.
"""
from __future__ import annotations

from fractions import Fraction

import numpy as np

_GOLDEN = np.uint64(0x9E3779B97F4A7C15)


def splitmix64_uniform(seed: int, n: int, offset: int = 0) -> np.ndarray:
    """n uniform doubles in [0, 1): element k is mix(seed + (offset+k+1)*golden)."""
    with np.errstate(over="ignore"):
        k = np.arange(offset + 1, offset + n + 1, dtype=np.uint64)
        z = np.uint64(seed) + k * _GOLDEN
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def vf_shape(m, n, p, nv, buff):
    return (m + 2 * buff + 7, n + 2 * buff + 7, p + 2 * buff + 7, nv)


def harness_field(m, n, p, nv, buff) -> np.ndarray:
    """f90:221-244: v_vf(i,j,k,l) = sin(2.1 x l) + cos(3.7 y) + 0.25 sin(4.3 z)
    + 0.02 (i + 2j - k + l), x = (i - is1_beg + 1)/(is1_end - is1_beg + 3)."""
    isb = -buff
    ie = [m + buff, n + buff, p + buff]
    idx = [np.arange(isb - 3, e + 4) for e in ie]
    den = [float(max(1, e - isb + 3)) for e in ie]
    x = (idx[0] - isb + 1) / den[0]
    y = (idx[1] - isb + 1) / den[1]
    z = (idx[2] - isb + 1) / den[2]
    out = np.empty(vf_shape(m, n, p, nv, buff), order="F")
    cy = np.cos(3.7 * y)
    sz = 0.25 * np.sin(4.3 * z)
    for l in range(1, nv + 1):
        sx = np.sin(2.1 * x * float(l))
        lin = 0.02 * (idx[0][:, None, None] + 2 * idx[1][None, :, None] - idx[2][None, None, :] + l)
        out[:, :, :, l - 1] = ((sx[:, None, None] + cy[None, :, None]) + sz[None, None, :]) + lin
    return out


def harness_coefficients(nc: int, offset: float):
    """f90:246-279: synthetic (polyL, polyR, dL, dR, beta_coef) for one direction;
    x/y/z use offset 0.03/0.05/0.07 (f90:190-192)."""
    baseL = np.array([0.30, 0.27, 0.20, 0.14, 0.09])
    baseR = np.array([0.09, 0.14, 0.20, 0.27, 0.30])
    r = np.arange(5)
    s = np.arange(3)
    pL = np.empty((nc, 5, 3), order="F")
    pR = np.empty((nc, 5, 3), order="F")
    pL[:] = (offset + 0.015 * ((r[:, None] + 1) * (s[None, :] + 1)))[None]
    pR[:] = (-offset + 0.012 * (2 * r[:, None] + s[None, :] + 1))[None]
    dL = np.empty((5, nc), order="F")
    dR = np.empty((5, nc), order="F")
    dL[:] = (baseL + offset * 0.10)[:, None]
    dR[:] = (baseR + offset * 0.10)[:, None]
    bc = np.zeros((nc, 5, 6), order="F")
    bc[:, :, 0] = (0.8 + offset) + 0.05 * (r + 1)
    bc[:, :, 2] = (0.9 + offset) + 0.04 * (r + 1)
    bc[:, :, 3] = (1.0 + offset) + 0.03 * (r + 1)
    bc[:, :, 5] = (1.1 + offset) + 0.02 * (r + 1)
    return pL, pR, dL, dR, bc


def _cell_centres(cells: int, buff: int) -> np.ndarray:
    """Cell centres (i + 1/2)/(cells) for i = -buff-3 .. cells-1+buff+3."""
    i = np.arange(-buff - 3, cells + buff + 3)
    return (i + 0.5) / cells


def smooth_jump_field(m, n, p, nv, buff, seed=0, noise=1e-3, jump=1.0) -> np.ndarray:
    """q(x,y,z) = 1 + 0.5 sin(2 pi (q+1) x) cos(2 pi y) sin(2 pi z) + U(-noise, noise)
    (+ jump for x > 1/2 on odd q), at cell centres x = (i+1/2)/(m+1) continued
    into the halo; q is the 0-based variable index."""
    x = _cell_centres(m + 1, buff)
    y = _cell_centres(n + 1, buff)
    z = _cell_centres(p + 1, buff)
    shp = vf_shape(m, n, p, nv, buff)
    out = np.empty(shp, order="F")
    per = shp[0] * shp[1] * shp[2]
    cyz = np.cos(2 * np.pi * y)[:, None] * np.sin(2 * np.pi * z)[None, :]
    for q in range(nv):
        sx = np.sin(2 * np.pi * (q + 1) * x)
        f = 1.0 + 0.5 * sx[:, None, None] * cyz[None, :, :]
        u = splitmix64_uniform(seed, per, offset=q * per).reshape(shp[:3], order="F")
        f = f + (-noise + 2.0 * noise * u)
        if q % 2 == 1:
            f = f + jump * (x > 0.5)[:, None, None]
        out[:, :, :, q] = f
    return out


def sinusoid_shock_field(m, n, p, nv, buff, seed=0, ratio=5.0, shock=True) -> np.ndarray:
    """1 + 0.5 * mean over modes k=1..8 of sin(2 pi k (c_k . X) + phi_k), with
    seeded unit directions c_k and phases phi_k per variable, times `ratio`
    on the far side of a plane through the domain centre with a seeded normal."""
    x = _cell_centres(m + 1, buff)
    y = _cell_centres(n + 1, buff)
    z = _cell_centres(p + 1, buff)
    X, Y, Zc = np.meshgrid(x, y, z, indexing="ij")
    shp = vf_shape(m, n, p, nv, buff)
    out = np.empty(shp, order="F")
    rnd = splitmix64_uniform(seed ^ 0x5EED, 4 * 8 * nv + 3)
    nrm = rnd[-3:] * 2.0 - 1.0
    nrm = nrm / max(np.linalg.norm(nrm), 1e-12)
    side = (nrm[0] * (X - 0.5) + nrm[1] * (Y - 0.5) + nrm[2] * (Zc - 0.5)) > 0.0
    for q in range(nv):
        f = np.zeros(shp[:3])
        for k in range(1, 9):
            base = 4 * (8 * q + (k - 1))
            c = rnd[base:base + 3] * 2.0 - 1.0
            c = c / max(np.linalg.norm(c), 1e-12)
            phi = 2 * np.pi * rnd[base + 3]
            f += np.sin(2 * np.pi * k * (c[0] * X + c[1] * Y + c[2] * Zc) + phi)
        f = 1.0 + 0.5 * f / 8.0
        if shock:
            f = np.where(side, f * ratio, f)
        out[:, :, :, q] = f
    return out


# ---------------------------------------------------------------------------
# True uniform-grid WENO-JS coefficients in the reference's layouts.
# ---------------------------------------------------------------------------
def _poly_mul(a, b):
    out = [Fraction(0)] * (len(a) + len(b) - 1)
    for i, x in enumerate(a):
        for j, y in enumerate(b):
            out[i + j] += x * y
    return out


def _reconstruction_weights(cells, x0):
    """Weights w_m (cell m in `cells`, unit cells [m-1/2, m+1/2]) of the
    degree-(len-1) polynomial with those cell averages, evaluated at x0."""
    R = len(cells)
    pts = [Fraction(2 * cells[0] - 1, 2) + i for i in range(R + 1)]  # interfaces
    # primitive P(pts[i]) = sum_{m < i} v_m ; p(x0) = P'(x0) = sum_i L_i'(x0) P_i
    dL = []
    for i in range(R + 1):
        # derivative of the Lagrange basis L_i at x0
        tot = Fraction(0)
        for k in range(R + 1):
            if k == i:
                continue
            term = Fraction(1, 1) / (pts[i] - pts[k])
            for l in range(R + 1):
                if l in (i, k):
                    continue
                term *= (x0 - pts[l]) / (pts[i] - pts[l])
            tot += term
        dL.append(tot)
    # P_i = sum_{m < i} v_m  ->  w_m = sum_{i > m} dL_i
    return [sum(dL[i] for i in range(m + 1, R + 1)) for m in range(R)]


def _poly_of_stencil(cells):
    """Coefficients (in x, cell j at x in [-1/2, 1/2]) of the polynomial with the
    given cell averages, as lists over x^i of linear forms {cell: coef}."""
    R = len(cells)
    # Solve moments: for basis x^i, average over cell m = ((m+1/2)^{i+1} - (m-1/2)^{i+1})/(i+1)
    A = [[(Fraction(2 * m + 1, 2) ** (i + 1) - Fraction(2 * m - 1, 2) ** (i + 1)) / (i + 1)
          for i in range(R)] for m in cells]
    # invert A (R x R) exactly
    n = R
    M = [row[:] + [Fraction(int(r == c)) for c in range(n)] for r, row in enumerate(A)]
    for col in range(n):
        piv = next(r for r in range(col, n) if M[r][col] != 0)
        M[col], M[piv] = M[piv], M[col]
        pv = M[col][col]
        M[col] = [x / pv for x in M[col]]
        for r in range(n):
            if r != col and M[r][col] != 0:
                fct = M[r][col]
                M[r] = [a - fct * b for a, b in zip(M[r], M[col])]
    inv = [row[n:] for row in M]  # coef_i = sum_m inv[i][m] v_m
    return [{cells[m]: inv[i][m] for m in range(R)} for i in range(R)]


def _to_differences(lin, j, ks):
    """Rewrite a linear form over cell values that sums to zero as one over
    the differences D_k = v_{k+1} - v_k for k in ks: returns [coef per k]."""
    # sum_m w_m v_m with sum w = 0: coefficient of D_k is -sum_{m <= k} w_m
    out = []
    for k in ks:
        out.append(-sum((w for m, w in lin.items() if m <= k), Fraction(0)))
    return out


def uniform_weno_coefficients(order: int, nc: int):
    """(polyL, polyR, dL, dR, beta_coef) of uniform-grid WENO-JS for order
    3, 5 or 7 in the harness layouts.  "L" is the state at the left face of
    cell j (x_{j-1/2}) and "R" the state at its right face (x_{j+1/2}): the
    MP limiter's bounds (f90:1573-1583) place vL between v_{j-1} and v_j."""
    R = (order + 1) // 2
    j = 0
    rows = []
    for r in range(R):
        cells = list(range(j - r, j - r + R))
        ks = list(range(j - r + R - 2, j - r - 1, -1))  # descending differences
        rows.append((cells, ks))
    pL = np.zeros((5, 3))
    pR = np.zeros((5, 3))
    beta = np.zeros((5, 6))
    for r, (cells, ks) in enumerate(rows):
        for side, x0, tgt in (("L", Fraction(-1, 2), pL), ("R", Fraction(1, 2), pR)):
            w = _reconstruction_weights(cells, x0)
            # q - v_j = sum_m w_m (v_m - v_j): linear form with zero sum
            lin = {m: wm for m, wm in zip(cells, w)}
            lin[j] = lin.get(j, Fraction(0)) - 1
            c = _to_differences(lin, j, ks)
            for s, val in enumerate(c):
                tgt[r, s] = float(val)
        # smoothness indicator: sum_l int_{-1/2}^{1/2} (p^{(l)})^2 dx
        coefs = _poly_of_stencil(cells)
        # express each polynomial coefficient in the difference basis
        cd = []
        for lin in coefs[1:]:
            cd.append(_to_differences(lin, j, ks))
        nd = len(ks)
        Q = [[Fraction(0)] * nd for _ in range(nd)]
        deg = R - 1
        for l in range(1, deg + 1):
            # p^{(l)}(x) = sum_{i>=l} i!/(i-l)! a_i x^{i-l}
            terms = []
            for i in range(l, deg + 1):
                fac = Fraction(1)
                for t in range(i - l + 1, i + 1):
                    fac *= t
                terms.append((i - l, fac, cd[i - 1]))
            for (e1, f1, v1) in terms:
                for (e2, f2, v2) in terms:
                    e = e1 + e2
                    integ = (Fraction(1, 2) ** (e + 1) - Fraction(-1, 2) ** (e + 1)) / (e + 1)
                    for a in range(nd):
                        for b in range(nd):
                            Q[a][b] += f1 * f2 * integ * v1[a] * v2[b]
        # pack as (aa, ab, [ae], bb, [be], [ee]) in descending-difference order
        k = 0
        for a in range(nd):
            for b in range(a, nd):
                beta[r, k] = float(Q[a][a] if a == b else Q[a][b] + Q[b][a])
                k += 1
    # ideal weights: sum_r d_r q_r = big-stencil reconstruction
    big = list(range(j - (R - 1), j + R))
    dvals = {}
    for side, x0 in (("L", Fraction(-1, 2)), ("R", Fraction(1, 2))):
        W = {m: w for m, w in zip(big, _reconstruction_weights(big, x0))}
        S = [{m: w for m, w in zip(cells, _reconstruction_weights(cells, x0))} for cells, _ in rows]
        # solve for d over the R equations from the first R cells of the big stencil
        eqs = []
        for m in big:
            eqs.append(([S[r].get(m, Fraction(0)) for r in range(R)], W[m]))
        # least-squares-free: pick a square, nonsingular subset by elimination
        A = [e[0][:] + [e[1]] for e in eqs]
        n = R
        for col in range(n):
            piv = next(r for r in range(col, len(A)) if A[r][col] != 0)
            A[col], A[piv] = A[piv], A[col]
            pv = A[col][col]
            A[col] = [x / pv for x in A[col]]
            for r2 in range(len(A)):
                if r2 != col and A[r2][col] != 0:
                    fct = A[r2][col]
                    A[r2] = [a - fct * b for a, b in zip(A[r2], A[col])]
        d = [A[r][n] for r in range(R)]
        assert all(all(x == 0 for x in A[r][:n]) and A[r][n] == 0 for r in range(n, len(A)))
        dvals[side] = d
    dL = np.zeros(5)
    dR = np.zeros(5)
    for q in range(R):
        # WENO3/5 pair d(q) with coefficient row q; WENO7 pairs d(q) with row 3-q
        row = (R - 1 - q) if order == 7 else q
        dL[q] = float(dvals["L"][row])
        dR[q] = float(dvals["R"][row])
    polyL = np.empty((nc, 5, 3), order="F")
    polyR = np.empty((nc, 5, 3), order="F")
    polyL[:] = pL[None]
    polyR[:] = pR[None]
    dLa = np.empty((5, nc), order="F")
    dRa = np.empty((5, nc), order="F")
    dLa[:] = dL[:, None]
    dRa[:] = dR[:, None]
    bca = np.empty((nc, 5, 6), order="F")
    bca[:] = beta[None]
    return polyL, polyR, dLa, dRa, bca


# ---------------------------------------------------------------------------
# Device-side generators (torch) for large benchmark inputs: the same
# formulas as above, evaluated on the GPU in FP64; the noise comes from a
# seeded torch generator instead of splitmix64, so values match the numpy
# generators in distribution, not bit for bit.  Returned flat in Fortran
# order (x fastest), shape (N1+6)(N2+6)(N3+6)V.
# ---------------------------------------------------------------------------
def _centres_t(cells, buff, device):
    import torch
    i = torch.arange(-buff - 3, cells + buff + 3, dtype=torch.float64, device=device)
    return (i + 0.5) / cells


def sinusoid_shock_field_dev(m, n, p, nv, buff, seed=0, ratio=5.0, shock=True, device="cuda"):
    """Device version of sinusoid_shock_field (same modes, directions, phases
    and shock plane for a given seed)."""
    import torch
    x = _centres_t(m + 1, buff, device)
    y = _centres_t(n + 1, buff, device)
    z = _centres_t(p + 1, buff, device)
    Zc, Y, X = torch.meshgrid(z, y, x, indexing="ij")  # C order (z, y, x): x fastest
    rnd = splitmix64_uniform(seed ^ 0x5EED, 4 * 8 * nv + 3)
    nrm = rnd[-3:] * 2.0 - 1.0
    nrm = nrm / max(np.linalg.norm(nrm), 1e-12)
    out = torch.empty((nv,) + tuple(X.shape), dtype=torch.float64, device=device)
    side = (float(nrm[0]) * (X - 0.5) + float(nrm[1]) * (Y - 0.5) + float(nrm[2]) * (Zc - 0.5)) > 0.0
    for q in range(nv):
        f = torch.zeros_like(X)
        for k in range(1, 9):
            base = 4 * (8 * q + (k - 1))
            c = rnd[base:base + 3] * 2.0 - 1.0
            c = c / max(np.linalg.norm(c), 1e-12)
            phi = 2 * np.pi * rnd[base + 3]
            f += torch.sin(2 * np.pi * k * (float(c[0]) * X + float(c[1]) * Y + float(c[2]) * Zc) + phi)
        f = 1.0 + 0.5 * f / 8.0
        if shock:
            f = torch.where(side, f * ratio, f)
        out[q] = f
    return out.reshape(-1)


def smooth_jump_field_dev(m, n, p, nv, buff, seed=0, noise=1e-3, jump=1.0, device="cuda"):
    """Device version of smooth_jump_field (noise from a seeded torch
    generator)."""
    import torch
    x = _centres_t(m + 1, buff, device)
    y = _centres_t(n + 1, buff, device)
    z = _centres_t(p + 1, buff, device)
    gen = torch.Generator(device=device).manual_seed(int(seed))
    cyz = torch.sin(2 * np.pi * z)[:, None, None] * torch.cos(2 * np.pi * y)[None, :, None]
    out = torch.empty((nv, z.numel(), y.numel(), x.numel()), dtype=torch.float64, device=device)
    for q in range(nv):
        sx = torch.sin(2 * np.pi * (q + 1) * x)[None, None, :]
        u = torch.rand(out.shape[1:], generator=gen, dtype=torch.float64, device=device)
        f = 1.0 + 0.5 * sx * cyz + noise * (2.0 * u - 1.0)
        if q % 2 == 1:
            f = f + jump * (x > 0.5).to(torch.float64)[None, None, :]
        out[q] = f
    return out.reshape(-1)
