// weno_adjoint.cuh -- hand-written adjoint (VJP) of one reconstruction sweep.
//
// For every face the forward pass is recomputed from the field (nothing is
// stored by the forward sweep), then the cotangents gL, gR of the face's
// outputs are pulled back to the stencil cells:
//   * MP limiter (f90:1564-1608): piecewise linear.  The forward recompute
//     records which expression the limiter returned (the WENO value itself,
//     or one of v0, v_{j-1}, v_{j+1}, the upper limit UL, the median MD or
//     the curvature bound LC, with the minmod argument it picked) and the
//     cotangent goes to that expression's stencil weights.
//   * Weights: out = sum_r alpha_r p_r / S with S = sum alpha.
//       dout/dp_r = alpha_r / S,   dout/dalpha_r = (p_r - out) / S.
//     JS: alpha_r = d_r / beta_r^2, so dalpha_r/dbeta_r = -2 alpha_r / beta_r.
//     TENO: alpha_r = delta_r d_r with a cutoff delta that is constant
//     almost everywhere, so only the candidate polynomials carry
//     derivatives -- except the reference's WENO7 TENO, whose extra
//     alpha(4) = (1 + |eps - beta(3)|/eps)^6 (f90:1491-1506) depends on beta(3).
//   * Candidate polynomials and smoothness indicators are linear / quadratic
//     in the differences D_k = v_{k+1} - v_k.
// Cells receive contributions from the faces whose stencils contain them;
// the kernel gathers them tile by tile through shared memory (no atomics).
#pragma once

#include "weno_math.cuh"
#include "sweep_generic.cuh"

namespace wsb {

// Stencil layout of order 3/5/7 in the reference's coefficient rows:
// row r, term s uses D_{S-1-r-s} (D_k = v[k+1] - v[k]), S = R-1 terms,
// and pairs with weight index q(r) = r (WENO3/5) or 3 - r (WENO7).
template <int ORDER>
struct Shape {
    static constexpr int R = (ORDER + 1) / 2;
    static constexpr int S = R - 1;
    static constexpr int NB = S * (S + 1) / 2;
    static __device__ __forceinline__ int q_of(int r) { return ORDER == 7 ? 3 - r : r; }
    static __device__ __forceinline__ int dk(int r, int s) { return S - 1 - r - s; }  // D index
};

// Reads of the Coef<ORDER> register blocks in (row, term) form.
template <int ORDER>
__device__ __forceinline__ double cf_poly(const Coef<ORDER>& c, bool left, int r, int s) {
    constexpr int S = Shape<ORDER>::S;
    return left ? c.pL[r * S + s] : c.pR[r * S + s];
}
template <int ORDER>
__device__ __forceinline__ double cf_beta(const Coef<ORDER>& c, int r, int t) {
    constexpr int NB = Shape<ORDER>::NB;
    return c.b[r * NB + t];
}
template <int ORDER>
__device__ __forceinline__ double cf_d(const Coef<ORDER>& c, bool left, int q) {
    return left ? c.dL[q] : c.dR[q];
}

// ---------------------------------------------------------------------
// MP limiter: forward value and the stencil weights of the selected branch.
// w[0..4] receive d(out)/d(v[q-2]); the return value is d(out)/d(weno in).
// ---------------------------------------------------------------------
struct Grad5 {
    double g[5];  // q = -2..2 at g[q+2]
};

__device__ __forceinline__ void g5_zero(Grad5& a) {
#pragma unroll
    for (int i = 0; i < 5; ++i) a.g[i] = 0.0;
}

// minmod(dl, dr) of f90:1568-1571 with the gradient of the argument it returns
__device__ __forceinline__ double mp_minmod_grad(double dl, double dr, const Grad5& gdl, const Grad5& gdr,
                                                 Grad5& out) {
    // same decisions as mp_minmod: m = min(|dl|,|dr|), M = max, t = 4m - M
    const double a = fabs(dl), b = fabs(dr);
    const bool al = a < b;
    const double m = al ? a : b, M = al ? b : a;
    const double t = fma(4.0, m, -M);
    g5_zero(out);
    const bool same = ((__double2hiint(dl) ^ __double2hiint(dr)) >= 0) && (t > 0.0);
    if (!same) return 0.0;
    // result = copysign(min(t, m), dl): either 4 x_small - x_large or x_small
    const Grad5& gs = al ? gdl : gdr;
    const Grad5& gl = al ? gdr : gdl;
    const bool pick_t = t < m;
#pragma unroll
    for (int i = 0; i < 5; ++i) out.g[i] = pick_t ? 4.0 * gs.g[i] - gl.g[i] : gs.g[i];
    return copysign(pick_t ? t : m, dl);
}

// One side of the limiter (left: neighbour vn = v[-1], far = v[+1];
// right: vn = v[+1], far = v[-1]).  Returns d(out)/d(in) and adds
// d(out)/d(v) * g into acc.
__device__ __forceinline__ double mp_side_vjp(bool left, const double* v, double in, double mMD, double mLC,
                                              const Grad5& gMD, const Grad5& gLC, double g, Grad5& acc) {
    const double kBetaMP = 4.0 / 3.0;
    const double v0 = v[0], vn = left ? v[-1] : v[1], vf = left ? v[1] : v[-1];
    const int in_ = left ? 1 : 3, if_ = left ? 3 : 1;  // index of vn / vf in Grad5
    // expressions (same rounding as mp_limit) and their stencil weights
    const double dF = left ? vf - v0 : v0 - vf;  // dR1 (left) or dL1 (right)
    const double UL = left ? fma(-2.0, dF, v0) : fma(2.0, dF, v0);
    const double MD = ((v0 + vn) - mMD) * 0.5;
    const double LC = left ? fma(kBetaMP, mLC, fma(-0.5, dF, v0)) : fma(kBetaMP, mLC, fma(0.5, dF, v0));
    // candidates: 0 v0, 1 vn, 2 MD, 3 UL, 4 LC, carried as (value, code)
    // pairs through the min/max selections (no indexed array, so nothing
    // goes to local memory)
    const double dN = left ? v0 - vn : vn - v0;
    const bool vn_low = left ? (__double2hiint(dN) >= 0) : (__double2hiint(dN) < 0);  // vn <= v0
    const double vmn1 = vn_low ? vn : v0, vmx1 = vn_low ? v0 : vn;
    const int cmn1 = vn_low ? 1 : 0, cmx1 = vn_low ? 0 : 1;
    // min/max(v0, UL): UL <= v0 iff dF >= 0 (left), UL >= v0 iff dF >= 0 (right)
    const bool f_up = __double2hiint(dF) >= 0;
    const bool ul_low = left ? f_up : !f_up;
    const double vmn2 = ul_low ? UL : v0, vmx2 = ul_low ? v0 : UL;
    const int cmn2 = ul_low ? 3 : 0, cmx2 = ul_low ? 0 : 3;
    const bool la = MD < vmn1, lb = LC < vmn2;
    const double lo_av = la ? MD : vmn1, lo_bv = lb ? LC : vmn2;
    const int lo_ac = la ? 2 : cmn1, lo_bc = lb ? 4 : cmn2;
    const bool lsel = lo_av < lo_bv;  // max(lo_a, lo_b)
    const double lo_v = lsel ? lo_bv : lo_av;
    const int lo_c = lsel ? lo_bc : lo_ac;
    const bool ha = vmx1 < MD, hb = vmx2 < LC;
    const double hi_av = ha ? MD : vmx1, hi_bv = hb ? LC : vmx2;
    const int hi_ac = ha ? 2 : cmx1, hi_bc = hb ? 4 : cmx2;
    const bool hsel = hi_bv < hi_av;  // min(hi_a, hi_b)
    const double hi_v = hsel ? hi_bv : hi_av;
    const int hi_c = hsel ? hi_bc : hi_ac;
    // median(in, lo, hi) with lo <= hi: the input passes through unless it
    // lies outside the bounds
    if (!(in < lo_v) && !(hi_v < in)) return 1.0;
    const int pick = (in < lo_v) ? lo_c : hi_c;
    // stencil weights of the picked expression, times g
    switch (pick) {
        case 0: acc.g[2] += g; break;
        case 1: acc.g[in_] += g; break;
        case 2:
            acc.g[2] += 0.5 * g;
            acc.g[in_] += 0.5 * g;
#pragma unroll
            for (int i = 0; i < 5; ++i) acc.g[i] -= 0.5 * g * gMD.g[i];
            break;
        case 3:  // v0 -/+ 2 (vf - v0) -> 3 v0 - 2 vf
            acc.g[2] += 3.0 * g;
            acc.g[if_] -= 2.0 * g;
            break;
        default:  // v0 -/+ (vf - v0)/2 + beta mLC -> 1.5 v0 - 0.5 vf + beta mLC
            acc.g[2] += 1.5 * g;
            acc.g[if_] -= 0.5 * g;
#pragma unroll
            for (int i = 0; i < 5; ++i) acc.g[i] += kBetaMP * g * gLC.g[i];
            break;
    }
    return 0.0;
}

// ---------------------------------------------------------------------
// One face: v[-3..3] (entries outside the order's stencil are not read
// unless MP needs +-2), cotangents gL, gR of the face's final outputs;
// out[q+3] += d(outputs)/d(v[q]) . (gL, gR).
// ---------------------------------------------------------------------
template <int ORDER>
__device__ void face_vjp(const double* v, const Coef<ORDER>& cf, int scheme, double eps, double teno_ct, bool mp_on,
                         double gL, double gR, double* out) {
    using Sh = Shape<ORDER>;
    constexpr int R = Sh::R, S = Sh::S;
    double D[6];  // D_k at D[k+3], k = -3..2
#pragma unroll
    for (int k = -3; k <= 2; ++k) D[k + 3] = (k + 1 >= -Sh::R && k >= -Sh::R) ? v[k + 1] - v[k] : 0.0;
    // candidate terms and smoothness indicators
    double t[R][3], beta[R], pL[R], pR[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
#pragma unroll
        for (int s = 0; s < S; ++s) t[r][s] = D[Sh::dk(r, s) + 3];
        double b = 0.0;
        int idx = 0;
#pragma unroll
        for (int s1 = 0; s1 < S; ++s1)
#pragma unroll
            for (int s2 = s1; s2 < S; ++s2) b += cf_beta<ORDER>(cf, r, idx++) * t[r][s1] * t[r][s2];
        beta[r] = b + eps;
        double l = v[0], rr = v[0];
#pragma unroll
        for (int s = 0; s < S; ++s) {
            l += cf_poly<ORDER>(cf, true, r, s) * t[r][s];
            rr += cf_poly<ORDER>(cf, false, r, s) * t[r][s];
        }
        pL[r] = l;
        pR[r] = rr;
    }
    // weights for both sides: wL[r], wR[r] are the normalised weights
    double wL[R], wR[R];
    double a4 = 0.0, tau4 = 0.0;  // WENO7 TENO extra alpha (f90:1491-1506)
    double SL4 = 1.0, SR4 = 1.0;  // WENO7 TENO: the sums that include a4
    bool js_fast = false;
    // WENO3 keeps the reference's division form: its two-stencil weights
    // amplify the few-ulp rounding change of the one-reciprocal form.
    if (ORDER != 3 && scheme == JS) {
        // one-reciprocal form: w_r = d_r P_r / sum_m d_m P_m, P_r = prod_{m != r} beta_m^2
        double qq[R], P[R];
#pragma unroll
        for (int r = 0; r < R; ++r) qq[r] = beta[r] * beta[r];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            double p = 1.0;
#pragma unroll
            for (int m = 0; m < R; ++m)
                if (m != r) p *= qq[m];
            P[r] = p;
        }
        double aL[R], aR[R], SL = 0.0, SR = 0.0;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int q = Sh::q_of(r);
            aL[r] = cf_d<ORDER>(cf, true, q) * P[r];
            aR[r] = cf_d<ORDER>(cf, false, q) * P[r];
            SL += aL[r];
            SR += aR[r];
        }
        if (mid_range(SL) && mid_range(SR)) {
            const double rr = nr_rcp(SL * SR), gSL = SR * rr, gSR = SL * rr;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                wL[r] = aL[r] * gSL;
                wR[r] = aR[r] * gSR;
            }
            js_fast = true;
        }
    }
    if (!js_fast) {
        double aL[R], aR[R], SL = 0.0, SR = 0.0;
        double delta[R];
        if (scheme == TENO) {
            // cutoff exactly as the forward sweep decides it
            double al[R], s = 0.0, tau;
            if (ORDER == 7) {
                tau4 = fabs(eps - beta[0]);  // beta(3) of the reference is row 0 here
                tau = tau4;
            } else {
                tau = fabs(beta[R - 1] - beta[0]);
            }
            // (quotients here and below by Newton-refined reciprocals: an
            // FP64 division is a long instruction sequence, and these paths
            // had up to 5R + 1 of them per face)
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const double x = fma(tau, mid_range(beta[r]) ? nr_rcp(beta[r]) : 1.0 / beta[r], 1.0);
                if (ORDER == 7) {
                    const double a3 = ipow3(x);
                    al[r] = a3 * a3;
                } else {
                    al[r] = ipow6(x);
                }
            }
            if (ORDER == 7) {
                const double a3 = ipow3(fma(tau, nr_rcp(eps), 1.0));
                a4 = a3 * a3;
            }
            // reference sums in weight order q = 0..
#pragma unroll
            for (int q = 0; q < R; ++q) {
                int r = q;
                if (ORDER == 7) r = 3 - q;
                s += al[r];
            }
            if (ORDER == 7) s += a4;
            const double rs = mid_range(s) ? nr_rcp(s) : 1.0 / s;
#pragma unroll
            for (int r = 0; r < R; ++r) delta[r] = (al[r] * rs < teno_ct) ? 0.0 : 1.0;
        }
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int q = Sh::q_of(r);
            if (scheme == TENO) {
                aL[r] = delta[r] * cf_d<ORDER>(cf, true, q);
                aR[r] = delta[r] * cf_d<ORDER>(cf, false, q);
            } else {
                // d / beta^2 by one reciprocal shared by both sides (division
                // outside the reciprocal's range)
                const double q2 = beta[r] * beta[r];
                const double rq = mid_range(q2) ? nr_rcp(q2) : 1.0 / q2;
                aL[r] = cf_d<ORDER>(cf, true, q) * rq;
                aR[r] = cf_d<ORDER>(cf, false, q) * rq;
            }
            SL += aL[r];
            SR += aR[r];
        }
        if (ORDER == 7 && scheme == TENO) {
            SL += a4;
            SR += a4;
        }
        {
            const double rL = mid_range(SL) ? nr_rcp(SL) : 1.0 / SL, rR = mid_range(SR) ? nr_rcp(SR) : 1.0 / SR;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                wL[r] = aL[r] * rL;
                wR[r] = aR[r] * rR;
            }
        }
        SL4 = SL;
        SR4 = SR;
    }
    double Lw = 0.0, Rw = 0.0;
#pragma unroll
    for (int r = 0; r < R; ++r) {
        Lw += wL[r] * pL[r];
        Rw += wR[r] * pR[r];
    }

    // ---- MP (core faces only), pulled back first ----
    Grad5 acc;
    g5_zero(acc);
    double gLw = gL, gRw = gR;
    if (mp_on) {
        double Lv = Lw, Rv = Rw;
        Grad5 gdm1, gd0, gdp1, gA, gB;
        g5_zero(gdm1); g5_zero(gd0); g5_zero(gdp1);
        gdm1.g[2] += 1.0; gdm1.g[0] += 1.0; gdm1.g[1] -= 2.0;  // v0 + v-2 - 2 v-1
        gd0.g[3] += 1.0; gd0.g[1] += 1.0; gd0.g[2] -= 2.0;     // v1 + v-1 - 2 v0
        gdp1.g[4] += 1.0; gdp1.g[2] += 1.0; gdp1.g[3] -= 2.0;  // v2 + v0 - 2 v1
        const double dm1 = fma(-2.0, v[-1], v[0] + v[-2]);
        const double d0 = fma(-2.0, v[0], v[1] + v[-1]);
        const double dp1 = fma(-2.0, v[1], v[2] + v[0]);
        const double mA = mp_minmod_grad(dm1, d0, gdm1, gd0, gA);
        const double mB = mp_minmod_grad(d0, dp1, gd0, gdp1, gB);
        (void)Lv; (void)Rv;
        gLw = gL * mp_side_vjp(true, v, Lw, mA, mB, gA, gB, gL, acc);
        gRw = gR * mp_side_vjp(false, v, Rw, mB, mA, gB, gA, gR, acc);
    }

    // ---- weights and candidates ----
    // d out / d p_r = w_r;  d out / d beta_r = -2 w_r (p_r - out) / beta_r (JS)
    double inv_beta[R];
    if (scheme != TENO) {
        double B = 1.0;
#pragma unroll
        for (int r = 0; r < R; ++r) B *= beta[r];
        if (mid_range(B)) {
            const double rB = nr_rcp(B);
#pragma unroll
            for (int r = 0; r < R; ++r) {
                double p = rB;
#pragma unroll
                for (int m = 0; m < R; ++m)
                    if (m != r) p *= beta[m];
                inv_beta[r] = p;
            }
        } else {
#pragma unroll
            for (int r = 0; r < R; ++r) inv_beta[r] = 1.0 / beta[r];
        }
    }
    double gD[6] = {0, 0, 0, 0, 0, 0};
    double gv0 = 0.0;
    double gbeta[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const double gpL = gLw * wL[r], gpR = gRw * wR[r];
        gv0 += gpL + gpR;
#pragma unroll
        for (int s = 0; s < S; ++s)
            gD[Sh::dk(r, s) + 3] += cf_poly<ORDER>(cf, true, r, s) * gpL + cf_poly<ORDER>(cf, false, r, s) * gpR;
        gbeta[r] = (scheme == TENO) ? 0.0
                                    : -2.0 * (gpL * (pL[r] - Lw) + gpR * (pR[r] - Rw)) * inv_beta[r];
    }
    if (ORDER == 7 && scheme == TENO) {
        // alpha(4) = (1 + |eps - beta(3)|/eps)^6 sits in both sums
        const double re = nr_rcp(eps);
        const double ga4 = (gLw * (0.0 - Lw)) * nr_rcp(SL4) + (gRw * (0.0 - Rw)) * nr_rcp(SR4);
        const double base = fma(tau4, re, 1.0);
        const double b2 = base * base;
        const double da4 = 6.0 * (b2 * b2 * base) * re;   // d a4 / d tau
        const double sgn = (beta[0] - eps) >= 0.0 ? 1.0 : -1.0;
        gbeta[0] += ga4 * da4 * sgn;
    }
#pragma unroll
    for (int r = 0; r < R; ++r) {
        int idx = 0;
#pragma unroll
        for (int s1 = 0; s1 < S; ++s1)
#pragma unroll
            for (int s2 = s1; s2 < S; ++s2) {
                const double c = cf_beta<ORDER>(cf, r, idx++) * gbeta[r];
                gD[Sh::dk(r, s1) + 3] += c * t[r][s2];
                gD[Sh::dk(r, s2) + 3] += c * t[r][s1];
            }
    }
    // D_k = v[k+1] - v[k]
#pragma unroll
    for (int k = -3; k <= 2; ++k) {
        out[k + 1 + 3] += gD[k + 3];
        out[k + 3] -= gD[k + 3];
    }
    out[3] += gv0;
#pragma unroll
    for (int q = -2; q <= 2; ++q) out[q + 3] += acc.g[q + 2];
}

// ---------------------------------------------------------------------
// Kernel: one thread per column (a, b, v) of the sweep, marching along it.
// Face o reads cells o..o+6 of the column (sweep index J = o + 3 + q,
// q = -3..3) and contributes to the same cells; a cell has all its
// contributions once face o = J is done.  The thread keeps the 7-cell
// stencil window and the 7 pending cell sums in registers, so each step
// loads one new cell and the two cotangents and writes one finished cell:
// no shared memory, no barriers, no atomics.  Consecutive threads take
// consecutive columns, i.e. consecutive x for the folded y/z sweeps
// (coalesced); for sweeps along the contiguous axis the warp's 32 rows are
// read through L1, each 32-byte sector serving four consecutive steps.
// ---------------------------------------------------------------------
struct VjpArgs {
    SweepGeom g;
    const double* v;
    const double* gL;
    const double* gR;
    double* gv;
    CoefPtrs cp;
    UniCoefs uc;
    WenoParams wp;
    int mp;
    int accumulate;
};

// UNI: face-independent coefficients, read from the kernel-parameter bank.
template <int ORDER, bool UNI>
__global__ void __launch_bounds__(128) vjp_kernel(const VjpArgs a) {
    const long long ns = a.g.ns;
    for (long long col = (long long)blockIdx.x * blockDim.x + threadIdx.x; col < a.g.cols;
         col += (long long)gridDim.x * blockDim.x) {
        const long long av = col % a.g.c1;
        const long long tt = col / a.g.c1;
        const long long bv = tt % a.g.c2;
        const long long vv = tt / a.g.c2;
        const double* __restrict__ vin = a.v + a.g.in_off + av * a.g.sA + bv * a.g.sB + vv * a.g.sV;
        double* __restrict__ gout = a.gv + a.g.in_off + av * a.g.sA + bv * a.g.sB + vv * a.g.sV;
        const double* __restrict__ gLc = a.gL + ns * col;
        const double* __restrict__ gRc = a.gR + ns * col;
        const long long sJ = a.g.sJ;
        double w[7], acc[7];
#pragma unroll
        for (int q = 0; q < 6; ++q) w[q] = __ldg(vin + q * sJ);
#pragma unroll
        for (int q = 0; q < 7; ++q) acc[q] = 0.0;
        // the new cell, the two cotangents and (accumulating) the old
        // gradient of step o are loaded four steps earlier into slot o % 4 of
        // a register ring (the loop is unrolled four times, so no register
        // moves wait on a load in flight; each step's loads used at once,
        // the gradient's read-modify-write among them, left the kernel
        // waiting on memory latency at every step).  Only this thread touches
        // the column's cells in this launch, so the old gradient read ahead
        // is current.  Loads past the column's end read its last element and
        // are not used.
        const long long ncell = ns + 6;
        const bool acc_on = a.accumulate != 0;
        auto fetch = [&](long long o, double& x, double& l, double& r, double& q) {
            const long long jc = o + 6 < ncell ? o + 6 : ncell - 1;
            const long long oc = o < ns ? o : ns - 1;
            x = __ldg(vin + jc * sJ);
            l = __ldg(gLc + oc);
            r = __ldg(gRc + oc);
            q = acc_on ? gout[oc * sJ] : 0.0;
        };
        constexpr int P = 4;
        double px[P], pl[P], pr[P], pq[P];
#pragma unroll
        for (int k = 0; k < P; ++k) fetch(k, px[k], pl[k], pr[k], pq[k]);
        for (long long o0 = 0; o0 < ns; o0 += P) {
#pragma unroll
            for (int k = 0; k < P; ++k) {
                const long long o = o0 + k;
                if (o >= ns) break;
                w[6] = px[k];
                const double gLo = pl[k], gRo = pr[k], gvo = pq[k];
                fetch(o + P, px[k], pl[k], pr[k], pq[k]);
                const bool face_ok = (ORDER == 3) || (o >= 3 && o <= ns - 4);
                if (face_ok) {
                    const bool core = (o >= 3 && o <= ns - 4);
                    if constexpr (UNI) {
                        face_vjp<ORDER>(w + 3, *reinterpret_cast<const Coef<ORDER>*>(a.uc.v), a.wp.scheme, a.wp.eps,
                                        a.wp.teno_ct, a.mp && core, gLo, gRo, acc);
                    } else {
                        long long c = o - 3;
                        c = c < 0 ? 0 : (c > a.g.nc - 1 ? a.g.nc - 1 : c);
                        Coef<ORDER> cf;
                        cf.load(a.cp.polyL, a.cp.polyR, a.cp.dL, a.cp.dR, a.cp.beta, a.g.nc, c);
                        face_vjp<ORDER>(w + 3, cf, a.wp.scheme, a.wp.eps, a.wp.teno_ct, a.mp && core, gLo, gRo, acc);
                    }
                }
                // cell J = o is complete
                gout[o * sJ] = gvo + acc[0];
#pragma unroll
                for (int q = 0; q < 6; ++q) {
                    acc[q] = acc[q + 1];
                    w[q] = w[q + 1];
                }
                acc[6] = 0.0;
            }
        }
        // cells ns .. ns+5
#pragma unroll
        for (int q = 0; q < 6; ++q) {
            double* dst = gout + (ns + q) * sJ;
            if (a.accumulate) *dst += acc[q];
            else *dst = acc[q];
        }
    }
}

}  // namespace wsb
