"""weno_sb_coefficients: WENO-JS coefficients for arbitrary cell widths
(MFC's s_compute_weno_coefficients, which the reference harness replaces
with synthetic values, f90:246-279).  CPU only.

* on a uniform grid they are the uniform-grid coefficients the rest of the
  suite uses (fields.uniform_weno_coefficients);
* on stretched grids every coefficient matches an exact rational
  computation (tests/coef_exact.py, an independent formulation);
* the candidate stencils reproduce polynomials of degree R-1 at both faces,
  the ideal weights polynomials of degree 2R-2, and beta of a linear field
  is h_j^2 times its slope squared;
* with these coefficients the oracle's WENO5-JS reconstruction of a smooth
  monotone profile converges at fifth order on a stretched grid.
"""
from fractions import Fraction

import numpy as np
import pytest

import coef_exact


@pytest.fixture(scope="module")
def api():
    from wenostandalone_b200 import build
    build.build_lib()
    from wenostandalone_b200 import api as a
    return a


def _random_boundaries(ns, seed, spread=0.6):
    rng = np.random.default_rng(seed)
    w = 1.0 + spread * (rng.random(ns) - 0.5) * 2.0
    return np.concatenate([[0.0], np.cumsum(w)]) * 0.01


@pytest.mark.parametrize("order", [3, 5, 7])
def test_uniform_grid_gives_the_uniform_coefficients(api, order):
    from wenostandalone_b200 import fields
    ns = 30
    x = np.arange(ns + 1, dtype=np.float64) * 0.25 + 2.0   # exactly uniform in binary
    got = api.weno_coefficients(order, x)
    ref = fields.uniform_weno_coefficients(order, ns - 6)
    for g, r in zip(got, ref):
        assert np.max(np.abs(g - r)) <= 1e-14 * max(1.0, np.max(np.abs(r)))


@pytest.mark.parametrize("order", [3, 5, 7])
@pytest.mark.parametrize("grid", ["random", "tanh"])
def test_stretched_grid_matches_exact_rationals(api, order, grid):
    ns = 24
    x = _random_boundaries(ns, seed=order) if grid == "random" else api.stretched_boundaries(ns - 12, 6, ratio=6.0)
    pL, pR, dL, dR, bc = api.weno_coefficients(order, x)
    xb = [Fraction(float(v)) for v in x]
    R = (order + 1) // 2
    nb = R * (R - 1) // 2
    for c in range(0, ns - 6, 3):
        eL, eR, edL, edR, ebq = coef_exact.face(xb, c + 3, order)
        for r in range(R):
            for s in range(R - 1):
                assert abs(pL[c, r, s] - float(eL[r][s])) <= 1e-13 * (1 + abs(float(eL[r][s])))
                assert abs(pR[c, r, s] - float(eR[r][s])) <= 1e-13 * (1 + abs(float(eR[r][s])))
            for q in range(nb):
                e = float(ebq[r][q])
                assert abs(bc[c, r, q] - e) <= 1e-12 * (1 + abs(e)), (c, r, q, bc[c, r, q], e)
        for q in range(R):
            row = (R - 1 - q) if order == 7 else q
            assert abs(dL[q, c] - float(edL[row])) <= 1e-13
            assert abs(dR[q, c] - float(edR[row])) <= 1e-13
        # unused entries stay zero
        assert not np.any(pL[c, R:, :]) and not np.any(pL[c, :, R - 1:]) and not np.any(dL[R:, c])


def _cell_averages(x, coeffs):
    """Exact cell averages of the polynomial sum_i coeffs[i] x^i."""
    P = np.polynomial.polynomial.polyint(coeffs)
    vals = np.polynomial.polynomial.polyval(x, P)
    return np.diff(vals) / np.diff(x)


@pytest.mark.parametrize("order", [3, 5, 7])
def test_polynomial_exactness_on_a_stretched_grid(api, order):
    ns = 26
    x = api.stretched_boundaries(ns - 12, 6, ratio=5.0)
    pL, pR, dL, dR, bc = api.weno_coefficients(order, x)
    R = (order + 1) // 2
    rng = np.random.default_rng(1)
    for deg, ideal in ((R - 1, False), (2 * R - 2, True)):
        a = rng.normal(size=deg + 1)
        v = _cell_averages(x, a)
        for c in range(ns - 6):
            j = c + 3
            for side, P, d, x0 in (("L", pL, dL, x[j]), ("R", pR, dR, x[j + 1])):
                exact = np.polynomial.polynomial.polyval(x0, a)
                cand = []
                for r in range(R):
                    cells = list(range(j - r, j - r + R))
                    D = [v[k + 1] - v[k] for k in range(cells[-2], cells[0] - 1, -1)]
                    cand.append(v[j] + sum(P[c, r, s] * D[s] for s in range(R - 1)))
                if not ideal:
                    assert np.allclose(cand, exact, rtol=0, atol=1e-11), (side, c, cand, exact)
                else:
                    rows = [(R - 1 - q) if order == 7 else q for q in range(R)]
                    comb = sum(d[q, c] * cand[rows[q]] for q in range(R))
                    assert abs(comb - exact) <= 1e-10, (side, c, comb, exact)
                    assert abs(sum(d[:R, c]) - 1.0) <= 1e-13


def test_beta_of_a_linear_field(api):
    ns = 22
    x = _random_boundaries(ns, seed=7)
    slope = 3.25
    v = _cell_averages(x, [0.4, slope])
    for order in (3, 5, 7):
        R = (order + 1) // 2
        pL, pR, dL, dR, bc = api.weno_coefficients(order, x)
        for c in range(ns - 6):
            j = c + 3
            h = x[j + 1] - x[j]
            for r in range(R):
                cells = list(range(j - r, j - r + R))
                D = [v[k + 1] - v[k] for k in range(cells[-2], cells[0] - 1, -1)]
                beta = 0.0
                q = 0
                for a in range(R - 1):
                    for b in range(a, R - 1):
                        beta += bc[c, r, q] * D[a] * D[b]
                        q += 1
                assert abs(beta - (h * slope) ** 2) <= 1e-10 * (h * slope) ** 2


def test_weno5_converges_at_fifth_order_on_a_stretched_grid(api, oracle_mod):
    """Reconstruct cell averages of tanh(4x - 2) + x on [0, 1] (smooth, no
    critical point) with the oracle's WENO5-JS using these coefficients;
    the max face error falls ~2^5 per halving of the cells."""
    errs = []
    for cells in (32, 64, 128):
        x = api.stretched_boundaries(cells, 6, ratio=3.0, centre=0.4, width=0.15)
        ns = x.size - 1
        F = lambda t: np.log(np.cosh(4 * t - 2)) / 4 + t * t / 2    # primitive of tanh(4t-2) + t
        f = lambda t: np.tanh(4 * t - 2) + t
        avg = np.diff(F(x)) / np.diff(x)
        rs = np.zeros((ns + 6, 1, 1, 1), order="F")
        rs[3:ns + 3, 0, 0, 0] = avg
        coefs = api.weno_coefficients(5, x)
        L, R = oracle_mod.reconstruct(rs, coefs, 5, eps=1e-40)
        core = slice(3, ns - 3)
        eL = np.abs(L[core, 0, 0, 0] - f(x[3:ns - 3]))
        eR = np.abs(R[core, 0, 0, 0] - f(x[4:ns - 2]))
        errs.append(max(eL.max(), eR.max()))
    rates = [np.log2(errs[k] / errs[k + 1]) for k in range(len(errs) - 1)]
    assert min(rates) >= 4.5, (errs, rates)
