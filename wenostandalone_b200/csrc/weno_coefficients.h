// weno_coefficients.h -- WENO reconstruction coefficients for arbitrary
// (stretched) cell widths, in the layouts the sweeps read.  Host code.
//
// The reference harness fills its coefficient arrays with synthetic values
// (inputs/weno_standalone.f90:246-279) in place of MFC's
// s_compute_weno_coefficients, which is not part of it.  This generator
// computes the true coefficients of WENO-JS reconstruction on a grid with
// any cell boundaries, following the published construction:
//
//  * C.-W. Shu, "Essentially non-oscillatory and weighted essentially
//    non-oscillatory schemes for hyperbolic conservation laws", ICASE
//    Report 97-65 (1997), section 2.1: the value at a cell face of the
//    degree R-1 polynomial with the cell averages of a stencil, through
//    the derivative of the Lagrange interpolant of the primitive function
//    at the stencil's R+1 cell boundaries; section 2.2: the linear (ideal)
//    weights that combine the R candidate stencils into the 2R-1 cell
//    stencil's value;
//  * G.-S. Jiang and C.-W. Shu, J. Comput. Phys. 126 (1996) 202-228: the
//    smoothness indicator beta_r = sum_{l=1}^{R-1} h_j^{2l-1}
//    int_{cell j} (d^l p_r / dx^l)^2 dx.
//
// Everything is formed in the cell's own coordinate xi = (x - x_j) / h_j, in
// which beta is free of h_j, with long double arithmetic, and then written
// in the difference form the harness's kernels evaluate (f90:535-550 for
// WENO5, f90:1455-1473 for WENO7, f90:422-431 for WENO3):
//   state_r = v_j + sum_s poly(c, r, s) * D_s,   D = descending differences
//             v_{k+1} - v_k of stencil r (cells j-r .. j-r+R-1)
//   beta_r  = sum over pairs (s <= t) of beta_coef(c, r, q) D_s D_t
//             (q runs aa, ab, [ae], bb, [be], [ee]) + eps
// with "L" the state at the left face of cell j (x_{j-1/2}) and "R" at its
// right face, the ideal weight d(q, c) of WENO3 / WENO5 paired with row q
// and that of WENO7 with row 3 - q (f90:1480-1488).
#pragma once

#include <cmath>
#include <cstdint>
#include <vector>

namespace wsb {
namespace coef {

typedef long double Real;

// Weights w_m of the cell averages (cells 0..R-1 of a stencil with
// boundaries t[0..R] in xi) in the stencil polynomial's value at x0.
inline void face_weights(const Real* t, int R, Real x0, Real* w) {
    // P(t_i) = sum_{m < i} v_m (t_{m+1} - t_m); p(x0) = sum_i L_i'(x0) P(t_i)
    Real dl[16];
    for (int i = 0; i <= R; ++i) {
        Real tot = 0;
        for (int k = 0; k <= R; ++k) {
            if (k == i) continue;
            Real term = 1.0L / (t[i] - t[k]);
            for (int l = 0; l <= R; ++l) {
                if (l == i || l == k) continue;
                term *= (x0 - t[l]) / (t[i] - t[l]);
            }
            tot += term;
        }
        dl[i] = tot;
    }
    for (int m = 0; m < R; ++m) {
        Real s = 0;
        for (int i = m + 1; i <= R; ++i) s += dl[i];
        w[m] = s * (t[m + 1] - t[m]);
    }
}

// Coefficients of the R descending differences D_k = v_{k+1} - v_k (k from
// the stencil's last pair down to its first) of the zero-sum linear form
// sum_m lin[m] v_m over the stencil's R cells.
inline void to_differences(const Real* lin, int R, Real* out) {
    // coefficient of D_k (k = 0..R-2 ascending) is -sum_{m <= k} lin[m]
    Real asc[8];
    Real acc = 0;
    for (int k = 0; k < R - 1; ++k) {
        acc += lin[k];
        asc[k] = -acc;
    }
    for (int s = 0; s < R - 1; ++s) out[s] = asc[R - 2 - s];
}

// Solve the R x R system A a = b in place (partial pivoting); false if
// singular.
inline bool solve(Real A[8][8], Real* b, int n) {
    for (int c = 0; c < n; ++c) {
        int p = c;
        for (int r = c + 1; r < n; ++r)
            if (fabsl(A[r][c]) > fabsl(A[p][c])) p = r;
        if (A[p][c] == 0) return false;
        if (p != c) {
            for (int k = 0; k < n; ++k) std::swap(A[p][k], A[c][k]);
            std::swap(b[p], b[c]);
        }
        for (int r = 0; r < n; ++r) {
            if (r == c) continue;
            const Real f = A[r][c] / A[c][c];
            if (f == 0) continue;
            for (int k = c; k < n; ++k) A[r][k] -= f * A[c][k];
            b[r] -= f * b[c];
        }
    }
    for (int r = 0; r < n; ++r) b[r] /= A[r][r];
    return true;
}

// One core face: cell j with boundaries xb[j], xb[j + 1] (xb indexed by
// cell), order 2R - 1.  Writes pL/pR[r][s], dL/dR[r] (indexed by stencil r)
// and bq[r][q].  False on a degenerate grid.
inline bool face(const double* xb, long long j, int R, Real pL[4][3], Real pR[4][3], Real dLr[4], Real dRr[4],
                 Real bq[4][6]) {
    const Real xc = 0.5L * ((Real)xb[j] + (Real)xb[j + 1]);
    const Real h = (Real)xb[j + 1] - (Real)xb[j];
    if (!(h > 0)) return false;
    auto X = [&](long long k) { return ((Real)xb[k] - xc) / h; };
    Real S[4][2][8];  // face weights of stencil r at side (0 = L, 1 = R), over its cells
    for (int r = 0; r < R; ++r) {
        const long long c0 = j - r;  // first cell of stencil r
        Real t[8];
        for (int i = 0; i <= R; ++i) {
            t[i] = X(c0 + i);
            if (i > 0 && !(t[i] > t[i - 1])) return false;
        }
        for (int side = 0; side < 2; ++side) {
            Real* w = S[r][side];
            face_weights(t, R, side == 0 ? -0.5L : 0.5L, w);
            Real lin[8];
            for (int m = 0; m < R; ++m) lin[m] = w[m] - ((c0 + m == j) ? 1.0L : 0.0L);
            Real dd[8];
            to_differences(lin, R, dd);
            for (int s = 0; s < R - 1; ++s) (side == 0 ? pL : pR)[r][s] = dd[s];
        }
        // smoothness indicator: polynomial sum_i a_i xi^i with the stencil's
        // cell averages, a = A^{-1} v, A[m][i] = int_cell xi^i / width
        Real inv[8][8];
        for (int col = 0; col < R; ++col) {
            Real A[8][8], b[8];
            for (int m = 0; m < R; ++m) {
                const Real a0 = t[m], a1 = t[m + 1];
                for (int i = 0; i < R; ++i)
                    A[m][i] = (powl(a1, i + 1) - powl(a0, i + 1)) / ((Real)(i + 1) * (a1 - a0));
                b[m] = (m == col) ? 1.0L : 0.0L;
            }
            if (!solve(A, b, R)) return false;
            for (int i = 0; i < R; ++i) inv[i][col] = b[i];
        }
        // a_i (i >= 1) as forms over the differences: a_i has zero sum over
        // the cells (a constant field has no slope or curvature)
        Real ad[8][8];
        for (int i = 1; i < R; ++i) {
            Real lin[8];
            for (int m = 0; m < R; ++m) lin[m] = inv[i][m];
            to_differences(lin, R, ad[i]);
        }
        const int nd = R - 1;
        Real Q[8][8] = {};
        for (int l = 1; l < R; ++l) {
            // p^(l)(xi) = sum_{i >= l} i!/(i-l)! a_i xi^(i-l)
            for (int i1 = l; i1 < R; ++i1)
                for (int i2 = l; i2 < R; ++i2) {
                    Real f1 = 1, f2 = 1;
                    for (int q = i1 - l + 1; q <= i1; ++q) f1 *= q;
                    for (int q = i2 - l + 1; q <= i2; ++q) f2 *= q;
                    const int e = (i1 - l) + (i2 - l);
                    const Real integ = (powl(0.5L, e + 1) - powl(-0.5L, e + 1)) / (Real)(e + 1);
                    for (int a = 0; a < nd; ++a)
                        for (int b = 0; b < nd; ++b) Q[a][b] += f1 * f2 * integ * ad[i1][a] * ad[i2][b];
                }
        }
        int k = 0;
        for (int a = 0; a < nd; ++a)
            for (int b = a; b < nd; ++b) bq[r][k++] = (a == b) ? Q[a][a] : Q[a][b] + Q[b][a];
    }
    // linear weights: sum_r d_r S_r = W (the 2R-1 cell stencil's weights),
    // solved from the right end of the big stencil, where cell j + R - 1 - r
    // is first reached by stencil r
    for (int side = 0; side < 2; ++side) {
        Real t[16];
        const long long b0 = j - (R - 1);
        for (int i = 0; i <= 2 * R - 1; ++i) t[i] = X(b0 + i);
        Real W[16];
        face_weights(t, 2 * R - 1, side == 0 ? -0.5L : 0.5L, W);
        Real* d = side == 0 ? dLr : dRr;
        for (int r = 0; r < R; ++r) {
            const long long cell = j + R - 1 - r;   // cell index
            Real rhs = W[cell - b0];
            for (int q = 0; q < r; ++q) rhs -= d[q] * S[q][side][cell - (j - q)];
            d[r] = rhs / S[r][side][cell - (j - r)];
        }
    }
    return true;
}

// All core faces of one sweep: ns cells with boundaries x_cb[0..ns], core
// faces c = 0..ns-7 at cells j = c + 3.  Arrays in the harness layouts
// (polyL/R (nc,5,3), d (5,nc), beta_coef (nc,5,6)); unused entries zero.
inline int generate(int order, long long ns, const double* x_cb, double* polyL, double* polyR, double* dL,
                    double* dR, double* beta) {
    const int R = (order + 1) / 2;
    const long long nc = ns - 6;
    for (long long i = 0; i < nc * 15; ++i) polyL[i] = polyR[i] = 0.0;
    for (long long i = 0; i < nc * 5; ++i) dL[i] = dR[i] = 0.0;
    for (long long i = 0; i < nc * 30; ++i) beta[i] = 0.0;
    for (long long c = 0; c < nc; ++c) {
        Real pL[4][3], pR[4][3], dl[4], dr[4], bq[4][6];
        if (!face(x_cb, c + 3, R, pL, pR, dl, dr, bq)) return -1;
        const int nb = R * (R - 1) / 2;
        for (int r = 0; r < R; ++r) {
            for (int s = 0; s < R - 1; ++s) {
                polyL[c + nc * (r + 5 * s)] = (double)pL[r][s];
                polyR[c + nc * (r + 5 * s)] = (double)pR[r][s];
            }
            for (int q = 0; q < nb; ++q) beta[c + nc * (r + 5 * q)] = (double)bq[r][q];
        }
        for (int q = 0; q < R; ++q) {
            const int row = (order == 7) ? (R - 1 - q) : q;
            dL[q + 5 * c] = (double)dl[row];
            dR[q + 5 * c] = (double)dr[row];
        }
    }
    return 0;
}

}  // namespace coef
}  // namespace wsb
