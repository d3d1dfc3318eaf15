// weno_math.cuh -- per-face arithmetic of the WENO path, FP64 and FP32-bulk.
//
// Restates the per-point bodies of the reference harness
// (wilfonba/WenoStandalone inputs/weno_standalone.f90, "f90:"):
//   WENO3  f90:416-468     WENO5  f90:511-662     WENO7  f90:1448-1535
//   MP     f90:1564-1608
//
// Two forms of the nonlinear weights:
//  * "faithful": the reference's sequence (alpha_k = d_k/beta_k^2, then
//    omega_k = alpha_k/sum) for every weight family, used for
//    mapped / Z / TENO / none;
//  * "one-reciprocal JS": omega_k = d_k P_k / sum_m d_m P_m with
//    P_k = prod_{m != k} beta_m^2, which is the same rational function
//    multiplied through by prod beta_m^2.  The P_k are shared by the left
//    and right states, and both normalisations use one reciprocal,
//    1/(S_L S_R).  It rounds differently (a few ulp) and is exact in real
//    arithmetic; when a sum leaves [2^-498, 2^498) (extreme beta, or
//    eps < ~1e-37) the faithful form is used instead.
//
// The MP limiter is a continuous, piecewise-linear function of the stencil
// (min, max, minmod, median), so it may be evaluated in any form that is
// equal in exact arithmetic: a comparison that rounds the other way near a
// tie changes the result by a rounding only.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace wsb {

enum Scheme { JS = 0, MAPPED = 1, WZ = 2, TENO = 3, NONE = 4 };

// ---------------------------------------------------------------------
// Coefficient register blocks for one core face (index c).
// Layouts: poly(c,r,s) = p[c + nc*(r + 5*s)], d(r,c) = d[r + 5*c],
//          beta(c,r,s) = b[c + nc*(r + 5*s)].
// ---------------------------------------------------------------------
template <int ORDER>
struct Coef;

template <>
struct Coef<3> {
    double pL[2], pR[2], dL[2], dR[2], b[2];
    __device__ __forceinline__ void load(const double* __restrict__ polyL,
                                         const double* __restrict__ polyR,
                                         const double* __restrict__ d_L,
                                         const double* __restrict__ d_R,
                                         const double* __restrict__ beta, long long nc, long long c) {
#pragma unroll
        for (int r = 0; r < 2; ++r) {
            pL[r] = __ldg(polyL + c + nc * r);
            pR[r] = __ldg(polyR + c + nc * r);
            dL[r] = __ldg(d_L + r + 5 * c);
            dR[r] = __ldg(d_R + r + 5 * c);
            b[r] = __ldg(beta + c + nc * r);
        }
    }
};

template <>
struct Coef<5> {
    double pL[6], pR[6], dL[3], dR[3], b[9];
    __device__ __forceinline__ void load(const double* __restrict__ polyL,
                                         const double* __restrict__ polyR,
                                         const double* __restrict__ d_L,
                                         const double* __restrict__ d_R,
                                         const double* __restrict__ beta, long long nc, long long c) {
#pragma unroll
        for (int r = 0; r < 3; ++r) {
#pragma unroll
            for (int s = 0; s < 2; ++s) {
                pL[2 * r + s] = __ldg(polyL + c + nc * (r + 5 * s));
                pR[2 * r + s] = __ldg(polyR + c + nc * (r + 5 * s));
            }
#pragma unroll
            for (int s = 0; s < 3; ++s) b[3 * r + s] = __ldg(beta + c + nc * (r + 5 * s));
            dL[r] = __ldg(d_L + r + 5 * c);
            dR[r] = __ldg(d_R + r + 5 * c);
        }
    }
};

template <>
struct Coef<7> {
    double pL[12], pR[12], dL[4], dR[4], b[24];
    __device__ __forceinline__ void load(const double* __restrict__ polyL,
                                         const double* __restrict__ polyR,
                                         const double* __restrict__ d_L,
                                         const double* __restrict__ d_R,
                                         const double* __restrict__ beta, long long nc, long long c) {
#pragma unroll
        for (int r = 0; r < 4; ++r) {
#pragma unroll
            for (int s = 0; s < 3; ++s) {
                pL[3 * r + s] = __ldg(polyL + c + nc * (r + 5 * s));
                pR[3 * r + s] = __ldg(polyR + c + nc * (r + 5 * s));
            }
#pragma unroll
            for (int s = 0; s < 6; ++s) b[6 * r + s] = __ldg(beta + c + nc * (r + 5 * s));
            dL[r] = __ldg(d_L + r + 5 * c);
            dR[r] = __ldg(d_R + r + 5 * c);
        }
    }
};

// True when s is positive with 2^-498 <= s < 2^498 (an integer test on the
// exponent field, so it costs no FP64 issue slot).  Two such values have a
// product that is a normal number.
__device__ __forceinline__ bool mid_range(double s) {
    const unsigned hi = (unsigned)__double2hiint(s);
    return (hi - (525u << 20)) < (996u << 20);
}

// True when p is positive with 2^-996 <= p < 2^996: the product of two
// normalisation sums whose reciprocal and whose products with either sum
// stay normal.
__device__ __forceinline__ bool mid_range_prod(double p) {
    const unsigned hi = (unsigned)__double2hiint(p);
    return (hi - (27u << 20)) < (1992u << 20);
}

// Reciprocal of a normal positive double by Newton-Raphson refinement of the
// hardware seed (PTX rcp.approx.ftz.f64): r <- r + r (1 - s r), twice.  Each
// step squares the relative error, so any seed better than 2^-14 ends below
// 2^-53 plus rounding; the GPU tests check the result against IEEE division
// on random inputs.
__device__ __forceinline__ double nr_rcp(double s) {
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(s));
    double e = fma(-s, r, 1.0);
    r = fma(r, e, r);
    e = fma(-s, r, 1.0);
    return fma(r, e, r);
}

// The TENO weights' powers (f90:580-582: (1 + tau/beta)**6._wp; f90:1492:
// (alpha**3._wp)**2._wp) as products: x^6 = (x^2)^3, x^3 = x^2 x.  A double
// pow() with a real exponent goes through a logarithm and an exponential in
// extended precision (on the order of a hundred instructions); the products
// round differently by a few ulp, which moves the weights by as much.
__device__ __forceinline__ double ipow6(double x) {
    const double x2 = x * x;
    return x2 * x2 * x2;
}
__device__ __forceinline__ double ipow3(double x) { return x * x * x; }

// Mapped-WENO transform (f90:419-423, 557-568).
__device__ __forceinline__ double mapw(double d, double w) {
    return (d * (1.0 + d - 3.0 * w) + w * w) * (w / (d * d + w * (1.0 - 2.0 * d)));
}

// ---------------------------------------------------------------------
// WENO3 (f90:416-468).  v[-1..1] as doubles.
// ---------------------------------------------------------------------
__device__ __forceinline__ void weno3_face(const double vm1, const double v0, const double vp1,
                                           const Coef<3>& c, int scheme, double eps, double& oL,
                                           double& oR) {
    const double dvd0 = vp1 - v0;
    const double dvdm1 = v0 - vm1;
    const double beta0 = c.b[0] * dvd0 * dvd0 + eps;
    const double beta1 = c.b[1] * dvdm1 * dvdm1 + eps;
    const double pL0 = v0 + c.pL[0] * dvd0, pL1 = v0 + c.pL[1] * dvdm1;
    const double pR0 = v0 + c.pR[0] * dvd0, pR1 = v0 + c.pR[1] * dvdm1;
    if (scheme == JS) {
        const double P0 = beta1 * beta1, P1 = beta0 * beta0;
        const double aL0 = c.dL[0] * P0, aL1 = c.dL[1] * P1;
        const double aR0 = c.dR[0] * P0, aR1 = c.dR[1] * P1;
        const double SL = aL0 + aL1, SR = aR0 + aR1;
        if (mid_range(SL) && mid_range(SR)) {
            const double r = nr_rcp(SL * SR);
            oL = (aL0 * pL0 + aL1 * pL1) * (SR * r);
            oR = (aR0 * pR0 + aR1 * pR1) * (SL * r);
            return;
        }
    }
    double a0 = 0.0, a1 = 0.0, tau = 0.0, s, w0, w1;
    if (scheme == JS) {
        a0 = c.dL[0] / (beta0 * beta0);
        a1 = c.dL[1] / (beta1 * beta1);
    } else if (scheme == MAPPED) {
        a0 = c.dL[0] / (beta0 * beta0);
        a1 = c.dL[1] / (beta1 * beta1);
        s = a0 + a1;
        a0 = mapw(c.dL[0], a0 / s);
        a1 = mapw(c.dL[1], a1 / s);
    } else if (scheme == WZ) {
        tau = fabs(beta1 - beta0);
        a0 = c.dL[0] * (1.0 + tau / beta0);
        a1 = c.dL[1] * (1.0 + tau / beta1);
    }
    s = a0 + a1;
    w0 = a0 / s;
    w1 = a1 / s;
    oL = w0 * pL0 + w1 * pL1;
    if (scheme == JS) {
        a0 = c.dR[0] / (beta0 * beta0);
        a1 = c.dR[1] / (beta1 * beta1);
    } else if (scheme == MAPPED) {
        a0 = c.dR[0] / (beta0 * beta0);
        a1 = c.dR[1] / (beta1 * beta1);
        s = a0 + a1;
        a0 = mapw(c.dR[0], a0 / s);
        a1 = mapw(c.dR[1], a1 / s);
    } else if (scheme == WZ) {
        a0 = c.dR[0] * (1.0 + tau / beta0);
        a1 = c.dR[1] * (1.0 + tau / beta1);
    } else {
        a0 = 0.0;
        a1 = 0.0;
    }
    s = a0 + a1;
    w0 = a0 / s;
    w1 = a1 / s;
    oR = w0 * pR0 + w1 * pR1;
}

// ---------------------------------------------------------------------
// WENO5 (f90:511-662).  Differences and beta in FP64; PT is the type of the
// candidate polynomials (double, or float for FP32-bulk).
// ---------------------------------------------------------------------
template <typename PT>
__device__ __forceinline__ void weno5_face(const double vm2, const double vm1, const double v0,
                                           const double vp1, const double vp2, const Coef<5>& c,
                                           int scheme, double eps, double teno_ct, double& oL,
                                           double& oR) {
    const double dvd_p1 = vp2 - vp1;
    const double dvd_0 = vp1 - v0;
    const double dvd_m1 = v0 - vm1;
    const double dvd_m2 = vm1 - vm2;
    const double beta0 = c.b[0] * dvd_p1 * dvd_p1 + c.b[1] * dvd_p1 * dvd_0 + c.b[2] * dvd_0 * dvd_0 + eps;
    const double beta1 = c.b[3] * dvd_0 * dvd_0 + c.b[4] * dvd_0 * dvd_m1 + c.b[5] * dvd_m1 * dvd_m1 + eps;
    const double beta2 = c.b[6] * dvd_m1 * dvd_m1 + c.b[7] * dvd_m1 * dvd_m2 + c.b[8] * dvd_m2 * dvd_m2 + eps;

    const PT v0p = (PT)v0, fp1 = (PT)dvd_p1, f0 = (PT)dvd_0, fm1 = (PT)dvd_m1, fm2 = (PT)dvd_m2;
    const double pL0 = (double)(v0p + (PT)c.pL[0] * fp1 + (PT)c.pL[1] * f0);
    const double pL1 = (double)(v0p + (PT)c.pL[2] * f0 + (PT)c.pL[3] * fm1);
    const double pL2 = (double)(v0p + (PT)c.pL[4] * fm1 + (PT)c.pL[5] * fm2);
    const double pR0 = (double)(v0p + (PT)c.pR[0] * fp1 + (PT)c.pR[1] * f0);
    const double pR1 = (double)(v0p + (PT)c.pR[2] * f0 + (PT)c.pR[3] * fm1);
    const double pR2 = (double)(v0p + (PT)c.pR[4] * fm1 + (PT)c.pR[5] * fm2);

    if (scheme == JS) {
        const double q0 = beta0 * beta0, q1 = beta1 * beta1, q2 = beta2 * beta2;
        const double P0 = q1 * q2, P1 = q0 * q2, P2 = q0 * q1;
        const double aL0 = c.dL[0] * P0, aL1 = c.dL[1] * P1, aL2 = c.dL[2] * P2;
        const double aR0 = c.dR[0] * P0, aR1 = c.dR[1] * P1, aR2 = c.dR[2] * P2;
        const double SL = aL0 + aL1 + aL2, SR = aR0 + aR1 + aR2;
        if (mid_range(SL) && mid_range(SR)) {
            const double r = nr_rcp(SL * SR);
            oL = (aL0 * pL0 + aL1 * pL1 + aL2 * pL2) * (SR * r);
            oR = (aR0 * pR0 + aR1 * pR1 + aR2 * pR2) * (SL * r);
            return;
        }
    }
    double a0 = 0.0, a1 = 0.0, a2 = 0.0, s;
    double de0 = 0.0, de1 = 0.0, de2 = 0.0, tau = 0.0;
    if (scheme == JS) {
        a0 = c.dL[0] / (beta0 * beta0);
        a1 = c.dL[1] / (beta1 * beta1);
        a2 = c.dL[2] / (beta2 * beta2);
    } else if (scheme == MAPPED) {
        a0 = c.dL[0] / (beta0 * beta0);
        a1 = c.dL[1] / (beta1 * beta1);
        a2 = c.dL[2] / (beta2 * beta2);
        s = a0 + a1 + a2;
        const double w0 = a0 / s, w1 = a1 / s, w2 = a2 / s;
        a0 = mapw(c.dL[0], w0);
        a1 = mapw(c.dL[1], w1);
        a2 = mapw(c.dL[2], w2);
    } else if (scheme == WZ) {
        tau = fabs(beta2 - beta0);
        a0 = c.dL[0] * (1.0 + (tau / beta0));
        a1 = c.dL[1] * (1.0 + (tau / beta1));
        a2 = c.dL[2] * (1.0 + (tau / beta2));
    } else if (scheme == TENO) {
        tau = fabs(beta2 - beta0);
        a0 = ipow6(1.0 + tau / beta0);
        a1 = ipow6(1.0 + tau / beta1);
        a2 = ipow6(1.0 + tau / beta2);
        s = a0 + a1 + a2;
        de0 = (a0 / s < teno_ct) ? 0.0 : 1.0;
        de1 = (a1 / s < teno_ct) ? 0.0 : 1.0;
        de2 = (a2 / s < teno_ct) ? 0.0 : 1.0;
        a0 = de0 * c.dL[0];
        a1 = de1 * c.dL[1];
        a2 = de2 * c.dL[2];
    }
    s = a0 + a1 + a2;
    oL = (a0 / s) * pL0 + (a1 / s) * pL1 + (a2 / s) * pL2;
    if (scheme == JS) {
        a0 = c.dR[0] / (beta0 * beta0);
        a1 = c.dR[1] / (beta1 * beta1);
        a2 = c.dR[2] / (beta2 * beta2);
    } else if (scheme == MAPPED) {
        a0 = c.dR[0] / (beta0 * beta0);
        a1 = c.dR[1] / (beta1 * beta1);
        a2 = c.dR[2] / (beta2 * beta2);
        s = a0 + a1 + a2;
        const double w0 = a0 / s, w1 = a1 / s, w2 = a2 / s;
        a0 = mapw(c.dR[0], w0);
        a1 = mapw(c.dR[1], w1);
        a2 = mapw(c.dR[2], w2);
    } else if (scheme == WZ) {
        a0 = c.dR[0] * (1.0 + (tau / beta0));
        a1 = c.dR[1] * (1.0 + (tau / beta1));
        a2 = c.dR[2] * (1.0 + (tau / beta2));
    } else if (scheme == TENO) {
        a0 = de0 * c.dR[0];
        a1 = de1 * c.dR[1];
        a2 = de2 * c.dR[2];
    } else {
        a0 = a1 = a2 = 0.0;
    }
    s = a0 + a1 + a2;
    oR = (a0 / s) * pR0 + (a1 / s) * pR1 + (a2 / s) * pR2;
}

// WENO5-JS in the one-reciprocal form with no fallback inside: computes oL
// and oR unconditionally and returns false when a normalisation sum left
// the range where the form is valid, in which case the caller redoes the
// face with weno5_face.  Straight-line code, so two columns can interleave.
template <typename PT>
__device__ __forceinline__ bool weno5_js_fast(const double vm2, const double vm1, const double v0,
                                              const double vp1, const double vp2, const Coef<5>& c,
                                              double eps, double& oL, double& oR) {
    const double dvd_p1 = vp2 - vp1;
    const double dvd_0 = vp1 - v0;
    const double dvd_m1 = v0 - vm1;
    const double dvd_m2 = vm1 - vm2;
    const double beta0 = c.b[0] * dvd_p1 * dvd_p1 + c.b[1] * dvd_p1 * dvd_0 + c.b[2] * dvd_0 * dvd_0 + eps;
    const double beta1 = c.b[3] * dvd_0 * dvd_0 + c.b[4] * dvd_0 * dvd_m1 + c.b[5] * dvd_m1 * dvd_m1 + eps;
    const double beta2 = c.b[6] * dvd_m1 * dvd_m1 + c.b[7] * dvd_m1 * dvd_m2 + c.b[8] * dvd_m2 * dvd_m2 + eps;
    const PT v0p = (PT)v0, fp1 = (PT)dvd_p1, f0 = (PT)dvd_0, fm1 = (PT)dvd_m1, fm2 = (PT)dvd_m2;
    const double pL0 = (double)(v0p + (PT)c.pL[0] * fp1 + (PT)c.pL[1] * f0);
    const double pL1 = (double)(v0p + (PT)c.pL[2] * f0 + (PT)c.pL[3] * fm1);
    const double pL2 = (double)(v0p + (PT)c.pL[4] * fm1 + (PT)c.pL[5] * fm2);
    const double pR0 = (double)(v0p + (PT)c.pR[0] * fp1 + (PT)c.pR[1] * f0);
    const double pR1 = (double)(v0p + (PT)c.pR[2] * f0 + (PT)c.pR[3] * fm1);
    const double pR2 = (double)(v0p + (PT)c.pR[4] * fm1 + (PT)c.pR[5] * fm2);
    const double q0 = beta0 * beta0, q1 = beta1 * beta1, q2 = beta2 * beta2;
    const double P0 = q1 * q2, P1 = q0 * q2, P2 = q0 * q1;
    const double aL0 = c.dL[0] * P0, aL1 = c.dL[1] * P1, aL2 = c.dL[2] * P2;
    const double aR0 = c.dR[0] * P0, aR1 = c.dR[1] * P1, aR2 = c.dR[2] * P2;
    const double SL = aL0 + aL1 + aL2, SR = aR0 + aR1 + aR2;
    const bool ok = mid_range(SL) && mid_range(SR);
    const double r = nr_rcp(SL * SR);
    oL = (aL0 * pL0 + aL1 * pL1 + aL2 * pL2) * (SR * r);
    oR = (aR0 * pR0 + aR1 * pR1 + aR2 * pR2) * (SL * r);
    return ok;
}

// ---------------------------------------------------------------------
// WENO7 (f90:1448-1535).  v[-3..3].  The reference's arrays are sized 0:4
// with beta(4) = eps; its TENO branch keeps alpha(4) = (1+tau/eps)^6 in the
// final sum (f90:1491-1506), restated here as written.
// ---------------------------------------------------------------------
template <typename PT>
__device__ __forceinline__ void weno7_face(const double* v /* v[-3..3] */, const Coef<7>& c,
                                           int scheme, double eps, double teno_ct, double& oL,
                                           double& oR) {
    double D[6];  // D[k+3] = dvd(k), k = -3..2
    D[5] = v[3] - v[2];
    D[4] = v[2] - v[1];
    D[3] = v[1] - v[0];
    D[2] = v[0] - v[-1];
    D[1] = v[-1] - v[-2];
    D[0] = v[-2] - v[-3];
    double beta[5];
    // beta(3 - r) uses dvd(2-r), dvd(1-r), dvd(-r) with coefficient row r.
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        const double a = D[5 - r], b = D[4 - r], e = D[3 - r];
        beta[3 - r] = c.b[6 * r + 0] * a * a + c.b[6 * r + 1] * a * b + c.b[6 * r + 2] * a * e +
                      c.b[6 * r + 3] * b * b + c.b[6 * r + 4] * b * e + c.b[6 * r + 5] * e * e + eps;
    }
    beta[4] = eps;
    double pL[4], pR[4];
    const PT v0p = (PT)v[0];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        const PT a = (PT)D[5 - r], b = (PT)D[4 - r], e = (PT)D[3 - r];
        pL[3 - r] = (double)(v0p + (PT)c.pL[3 * r] * a + (PT)c.pL[3 * r + 1] * b + (PT)c.pL[3 * r + 2] * e);
        pR[3 - r] = (double)(v0p + (PT)c.pR[3 * r] * a + (PT)c.pR[3 * r + 1] * b + (PT)c.pR[3 * r + 2] * e);
    }
    if (scheme == JS) {
        const double q0 = beta[0] * beta[0], q1 = beta[1] * beta[1], q2 = beta[2] * beta[2],
                     q3 = beta[3] * beta[3];
        const double q01 = q0 * q1, q23 = q2 * q3;
        const double P0 = q1 * q23, P1 = q0 * q23, P2 = q01 * q3, P3 = q01 * q2;
        const double aL0 = c.dL[0] * P0, aL1 = c.dL[1] * P1, aL2 = c.dL[2] * P2, aL3 = c.dL[3] * P3;
        const double aR0 = c.dR[0] * P0, aR1 = c.dR[1] * P1, aR2 = c.dR[2] * P2, aR3 = c.dR[3] * P3;
        const double SL = aL0 + aL1 + aL2 + aL3, SR = aR0 + aR1 + aR2 + aR3;
        if (mid_range(SL) && mid_range(SR)) {
            const double r = nr_rcp(SL * SR);
            oL = (aL0 * pL[0] + aL1 * pL[1] + aL2 * pL[2] + aL3 * pL[3]) * (SR * r);
            oR = (aR0 * pR[0] + aR1 * pR[1] + aR2 * pR[2] + aR3 * pR[3]) * (SL * r);
            return;
        }
    }
    double alpha[5] = {0.0, 0.0, 0.0, 0.0, 0.0}, delta[4] = {0.0, 0.0, 0.0, 0.0};
    double tau = 0.0, s;
    if (scheme == JS || scheme == MAPPED) {
#pragma unroll
        for (int q = 0; q < 4; ++q) alpha[q] = c.dL[q] / (beta[q] * beta[q]);
        if (scheme == MAPPED) {
            s = alpha[0] + alpha[1] + alpha[2] + alpha[3] + alpha[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) alpha[q] = mapw(c.dL[q], alpha[q] / s);
        }
    } else if (scheme == WZ) {
        tau = fabs(beta[3] - beta[0]);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const double t = tau / beta[q];
            alpha[q] = c.dL[q] * (1.0 + t * t);
        }
    } else if (scheme == TENO) {
        tau = fabs(beta[4] - beta[3]);
#pragma unroll
        for (int q = 0; q < 5; ++q) {
            const double a3 = ipow3(1.0 + tau / beta[q]);
            alpha[q] = a3 * a3;
        }
        s = alpha[0] + alpha[1] + alpha[2] + alpha[3] + alpha[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            delta[q] = (alpha[q] / s < teno_ct) ? 0.0 : 1.0;
            alpha[q] = delta[q] * c.dL[q];
        }
    }
    s = alpha[0] + alpha[1] + alpha[2] + alpha[3] + alpha[4];
    oL = (alpha[0] / s) * pL[0] + (alpha[1] / s) * pL[1] + (alpha[2] / s) * pL[2] + (alpha[3] / s) * pL[3];
    if (scheme == JS || scheme == MAPPED) {
#pragma unroll
        for (int q = 0; q < 4; ++q) alpha[q] = c.dR[q] / (beta[q] * beta[q]);
        if (scheme == MAPPED) {
            s = alpha[0] + alpha[1] + alpha[2] + alpha[3] + alpha[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) alpha[q] = mapw(c.dR[q], alpha[q] / s);
        }
    } else if (scheme == WZ) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const double t = tau / beta[q];
            alpha[q] = c.dR[q] * (1.0 + t * t);
        }
    } else if (scheme == TENO) {
#pragma unroll
        for (int q = 0; q < 4; ++q) alpha[q] = delta[q] * c.dR[q];
    }
    s = alpha[0] + alpha[1] + alpha[2] + alpha[3] + alpha[4];
    oR = (alpha[0] / s) * pR[0] + (alpha[1] / s) * pR[1] + (alpha[2] / s) * pR[2] + (alpha[3] / s) * pR[3];
}

// ---------------------------------------------------------------------
// FP32-bulk WENO-JS without FP32 <-> FP64 conversion instructions.
//
// On B200 a conversion between float and double issues at a quarter of the
// FP64 FMA rate, so a per-face path that widens its stencil and narrows its
// weights with cvt instructions spends more on conversions than on the
// WENO arithmetic.  Here:
//  * the stencil values are widened by bit manipulation on the integer
//    pipe (f2d_bits): exact for normal floats; zero and subnormal floats
//    become values below 2^-126 in magnitude (immaterial next to eps in
//    beta), Inf/NaN become large finite values -- the float stencil sums
//    below still carry the Inf/NaN into the face state;
//  * the differences, beta (with eps) and the weight normalisation are
//    FP64, as in the FP64 path;
//  * the normalised weights (in [0, 1]) are narrowed by bit manipulation
//    with truncation (unit_d2f, relative error < 2^-23);
//  * the candidate polynomials and the weighted sum are FP32, written as
//    v0 + (small corrections): L = v0 + e1 + w0 (e0 - e1) + w2 (e2 - e1)
//    with e_k = p_k - v0 (and the WENO7 analogue), so the weights'
//    truncation multiplies only the small differences e_k - e1 and the
//    face state is rounded once, at the final add.
// ---------------------------------------------------------------------
__device__ __forceinline__ double f2d_bits(float x) {
    const unsigned u = __float_as_uint(x);
    const unsigned hi = ((((u & 0x7FFFFFFFu) >> 3) | (u & 0x80000000u)) + 0x38000000u);
    return __hiloint2double((int)hi, (int)(u << 29));
}

// w in [0, 1] (or NaN-free non-negative) to float, truncating; values below
// 2^-126 become 0.
__device__ __forceinline__ float unit_d2f(double w) {
    const unsigned hi = (unsigned)__double2hiint(w), lo = (unsigned)__double2loint(w);
    const unsigned t = __funnelshift_l(lo, hi, 3) + 0x40000000u;
    return (hi < 0x38100000u) ? 0.0f : __uint_as_float(t);
}

// Float copies of one face's polynomial coefficients (layout of Coef<ORDER>).
template <int ORDER>
struct PolyF {
    static constexpr int N = (ORDER == 7) ? 12 : (ORDER == 5 ? 6 : 2);
    float L[N], R[N];
    __device__ __forceinline__ void from(const Coef<ORDER>& c) {
#pragma unroll
        for (int i = 0; i < N; ++i) {
            L[i] = (float)c.pL[i];
            R[i] = (float)c.pR[i];
        }
    }
};

// WENO5-JS, FP32 in and out.  Returns false when a normalisation sum left
// the one-reciprocal range; the caller then redoes the face in FP64.
__device__ __forceinline__ bool weno5_js_mixed(float m2, float m1, float z0, float p1, float p2,
                                               const Coef<5>& c, const PolyF<5>& pf, double eps, float& L,
                                               float& R) {
    const double Dm2 = f2d_bits(m2), Dm1 = f2d_bits(m1), D0 = f2d_bits(z0), Dp1 = f2d_bits(p1),
                 Dp2 = f2d_bits(p2);
    const double dvd_p1 = Dp2 - Dp1, dvd_0 = Dp1 - D0, dvd_m1 = D0 - Dm1, dvd_m2 = Dm1 - Dm2;
    const double beta0 = c.b[0] * dvd_p1 * dvd_p1 + c.b[1] * dvd_p1 * dvd_0 + c.b[2] * dvd_0 * dvd_0 + eps;
    const double beta1 = c.b[3] * dvd_0 * dvd_0 + c.b[4] * dvd_0 * dvd_m1 + c.b[5] * dvd_m1 * dvd_m1 + eps;
    const double beta2 = c.b[6] * dvd_m1 * dvd_m1 + c.b[7] * dvd_m1 * dvd_m2 + c.b[8] * dvd_m2 * dvd_m2 + eps;
    const double q0 = beta0 * beta0, q1 = beta1 * beta1, q2 = beta2 * beta2;
    const double P0 = q1 * q2, P1 = q0 * q2, P2 = q0 * q1;
    const double aL0 = c.dL[0] * P0, aL1 = c.dL[1] * P1, aL2 = c.dL[2] * P2;
    const double aR0 = c.dR[0] * P0, aR1 = c.dR[1] * P1, aR2 = c.dR[2] * P2;
    const double SL = aL0 + aL1 + aL2, SR = aR0 + aR1 + aR2;
    const bool ok = mid_range(SL) && mid_range(SR);
    const double r = nr_rcp(SL * SR), gL = SR * r, gR = SL * r;
    const float wL0 = unit_d2f(aL0 * gL), wL2 = unit_d2f(aL2 * gL);
    const float wR0 = unit_d2f(aR0 * gR), wR2 = unit_d2f(aR2 * gR);
    const float fp1 = p2 - p1, f0 = p1 - z0, fm1 = z0 - m1, fm2 = m1 - m2;
    const float eL0 = fmaf(pf.L[0], fp1, pf.L[1] * f0), eL1 = fmaf(pf.L[2], f0, pf.L[3] * fm1),
                eL2 = fmaf(pf.L[4], fm1, pf.L[5] * fm2);
    const float eR0 = fmaf(pf.R[0], fp1, pf.R[1] * f0), eR1 = fmaf(pf.R[2], f0, pf.R[3] * fm1),
                eR2 = fmaf(pf.R[4], fm1, pf.R[5] * fm2);
    L = z0 + fmaf(wL0, eL0 - eL1, fmaf(wL2, eL2 - eL1, eL1));
    R = z0 + fmaf(wR0, eR0 - eR1, fmaf(wR2, eR2 - eR1, eR1));
    return ok;
}

// WENO7-JS, FP32 in and out (v[-3..3]); same contract as weno5_js_mixed.
__device__ __forceinline__ bool weno7_js_mixed(const float* v, const Coef<7>& c, const PolyF<7>& pf, double eps,
                                               float& L, float& R) {
    double V[7];
#pragma unroll
    for (int q = 0; q < 7; ++q) V[q] = f2d_bits(v[q - 3]);
    double D[6];  // D[k+3] = dvd(k), k = -3..2
#pragma unroll
    for (int k = 0; k < 6; ++k) D[k] = V[k + 1] - V[k];
    double beta[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        const double a = D[5 - r], b = D[4 - r], e = D[3 - r];
        beta[3 - r] = c.b[6 * r + 0] * a * a + c.b[6 * r + 1] * a * b + c.b[6 * r + 2] * a * e +
                      c.b[6 * r + 3] * b * b + c.b[6 * r + 4] * b * e + c.b[6 * r + 5] * e * e + eps;
    }
    const double q0 = beta[0] * beta[0], q1 = beta[1] * beta[1], q2 = beta[2] * beta[2], q3 = beta[3] * beta[3];
    const double q01 = q0 * q1, q23 = q2 * q3;
    const double P0 = q1 * q23, P1 = q0 * q23, P2 = q01 * q3, P3 = q01 * q2;
    const double aL0 = c.dL[0] * P0, aL1 = c.dL[1] * P1, aL2 = c.dL[2] * P2, aL3 = c.dL[3] * P3;
    const double aR0 = c.dR[0] * P0, aR1 = c.dR[1] * P1, aR2 = c.dR[2] * P2, aR3 = c.dR[3] * P3;
    const double SL = aL0 + aL1 + aL2 + aL3, SR = aR0 + aR1 + aR2 + aR3;
    const bool ok = mid_range(SL) && mid_range(SR);
    const double r = nr_rcp(SL * SR), gL = SR * r, gR = SL * r;
    // stencil 3 - r uses float differences F[5-r], F[4-r], F[3-r]
    float F[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) F[k] = v[k - 2] - v[k - 3];
    float eL[4], eR[4];
#pragma unroll
    for (int r2 = 0; r2 < 4; ++r2) {
        eL[3 - r2] = fmaf(pf.L[3 * r2], F[5 - r2], fmaf(pf.L[3 * r2 + 1], F[4 - r2], pf.L[3 * r2 + 2] * F[3 - r2]));
        eR[3 - r2] = fmaf(pf.R[3 * r2], F[5 - r2], fmaf(pf.R[3 * r2 + 1], F[4 - r2], pf.R[3 * r2 + 2] * F[3 - r2]));
    }
    // pivot on stencil 1: L = v0 + e1 + sum_{k != 1} w_k (e_k - e1)
    const float wL0 = unit_d2f(aL0 * gL), wL2 = unit_d2f(aL2 * gL), wL3 = unit_d2f(aL3 * gL);
    const float wR0 = unit_d2f(aR0 * gR), wR2 = unit_d2f(aR2 * gR), wR3 = unit_d2f(aR3 * gR);
    L = v[0] + fmaf(wL0, eL[0] - eL[1], fmaf(wL2, eL[2] - eL[1], fmaf(wL3, eL[3] - eL[1], eL[1])));
    R = v[0] + fmaf(wR0, eR[0] - eR[1], fmaf(wR2, eR[2] - eR[1], fmaf(wR3, eR[3] - eR[1], eR[1])));
    return ok;
}

// ---------------------------------------------------------------------
// MP limiter (f90:1564-1608), rounding exactly as the reference.
// ---------------------------------------------------------------------
// 4-argument minmod of (4dl-dr, dl, 4dr-dl, dr) (f90:1568-1571).  The
// reference's product of SIGN() sums is +-1 when all four arguments share a
// sign and 0 otherwise.  With m = min(|dl|,|dr|) and M = max(|dl|,|dr|) the
// four share a sign exactly when dl, dr do and 4m > M, and then the least
// magnitude is min(4m - M, m) (|4dr - dl| >= 3m > m for the other pair), so
// the result is copysign(min(4m - M, m), dl) or 0 with two comparisons.
__device__ __forceinline__ double mp_minmod(double dl, double dr) {
    const double a = fabs(dl), b = fabs(dr);
    const bool al = a < b;
    const double m = al ? a : b, M = al ? b : a;
    const double t = fma(4.0, m, -M);  // |4 dl - dr| or |4 dr - dl| of the smaller one
    const bool same = ((__double2hiint(dl) ^ __double2hiint(dr)) >= 0) && (t > 0.0);
    return same ? copysign(t < m ? t : m, dl) : 0.0;
}

__device__ __forceinline__ bool sign_clear(double x) { return __double2hiint(x) >= 0; }

// min / max as one comparison and a select (no NaN special-casing: the
// limiter's bound candidates are finite whenever the field is).
template <typename T>
__device__ __forceinline__ T smin(T a, T b) { return (b < a) ? b : a; }
template <typename T>
__device__ __forceinline__ T smax(T a, T b) { return (a < b) ? b : a; }
// median(x, lo, hi) for lo <= hi; a NaN x stays NaN, as in the reference.
template <typename T>
__device__ __forceinline__ T sclamp(T x, T lo, T hi) { return (x < lo) ? lo : ((hi < x) ? hi : x); }

// The limiter proper (f90:1564-1608).  Every step is continuous in the data
// (min, max, minmod, median), so roundings that differ from the reference's
// move the result by roundings only; the forms below are the reference's
// expressions rearranged in exact arithmetic:
//  * the final update x + (sign(1/2, lo-x) + sign(1/2, hi-x)) min(|lo-x|, |hi-x|)
//    is median(x, lo, hi), and lo <= v0 <= hi always (each term of lo is a
//    min over a set containing v0, each term of hi a max), so it is
//    max(lo, min(x, hi));
//  * min/max(v0, v0 -+ 2 dv) and min/max(v0, v_{j+-1}) follow from the sign
//    of the difference, without a comparison.
__device__ __forceinline__ void mp_limit(const double vm2, const double vm1, const double v0,
                                         const double vp1, const double vp2, double& L, double& R) {
    const double kBetaMP = 4.0 / 3.0;  // beta_mp (f90:1556)
    const double dm1 = fma(-2.0, vm1, v0 + vm2);
    const double d0 = fma(-2.0, v0, vp1 + vm1);
    const double dp1 = fma(-2.0, vp1, vp2 + v0);
    const double mA = mp_minmod(dm1, d0);  // d_MD of vL, d_LC of vR
    const double mB = mp_minmod(d0, dp1);  // d_LC of vL, d_MD of vR
    const double dR1 = vp1 - v0;           // >= 0  <=>  vp1 >= v0
    const double dL1 = v0 - vm1;           // >= 0  <=>  v0 >= vm1
    const bool up_r = sign_clear(dR1), up_l = sign_clear(dL1);
    {
        const double UL = fma(-2.0, dR1, v0);  // <= v0 iff dR1 >= 0
        const double MD = ((v0 + vm1) - mA) * 0.5;
        const double LC = fma(kBetaMP, mB, fma(-0.5, dR1, v0));
        const double mn1 = up_l ? vm1 : v0, mx1 = up_l ? v0 : vm1;  // min/max(v0, vm1)
        const double mn2 = up_r ? UL : v0, mx2 = up_r ? v0 : UL;    // min/max(v0, UL)
        const double lo = smax(smin(mn1, MD), smin(mn2, LC));
        const double hi = smin(smax(mx1, MD), smax(mx2, LC));
        L = sclamp(L, lo, hi);
    }
    {
        const double UL = fma(2.0, dL1, v0);   // >= v0 iff dL1 >= 0
        const double MD = ((v0 + vp1) - mB) * 0.5;
        const double LC = fma(kBetaMP, mA, fma(0.5, dL1, v0));
        const double mn1 = up_r ? v0 : vp1, mx1 = up_r ? vp1 : v0;  // min/max(v0, vp1)
        const double mn2 = up_l ? v0 : UL, mx2 = up_l ? UL : v0;    // min/max(v0, UL)
        const double lo = smax(smin(mn1, MD), smin(mn2, LC));
        const double hi = smin(smax(mx1, MD), smax(mx2, LC));
        R = sclamp(R, lo, hi);
    }
}

// FP32-bulk MP: the same limiter in FP32 on the FP32 field.
__device__ __forceinline__ float mp_minmod_f(float dl, float dr) {
    const float a = fabsf(dl), b = fabsf(dr);
    const bool al = a < b;
    const float m = al ? a : b, M = al ? b : a;
    const float t = fmaf(4.0f, m, -M);
    const bool same = ((__float_as_int(dl) ^ __float_as_int(dr)) >= 0) && (t > 0.0f);
    return same ? copysignf(t < m ? t : m, dl) : 0.0f;
}

// The same limiter for FP32-bulk, on the FP32 field, with every bound
// carried as an offset from v0: the first differences a, b, c, e of
// neighbouring values are exact for values within a factor of two of each
// other, the bounds minus v0 are sums of small terms, and the state is
// rounded once when v0 is added back.  In exact arithmetic this is the
// reference's median(x, lo, hi) shifted by v0.
__device__ __forceinline__ void mp_limit_f(const float vm2, const float vm1, const float v0, const float vp1,
                                           const float vp2, float& L, float& R) {
    const float kBetaMP = 4.0f / 3.0f;
    const float a = vm1 - vm2, b = v0 - vm1, c = vp1 - v0, e = vp2 - vp1;
    const float mA = mp_minmod_f(b - a, c - b);  // minmod(d_{j-1}, d_j)
    const float mB = mp_minmod_f(c - b, e - c);  // minmod(d_j, d_{j+1})
    {
        const float x = L - v0;
        const float oMD = -0.5f * (b + mA);           // (v0 + vm1 - mA)/2 - v0
        const float oLC = fmaf(kBetaMP, mB, -0.5f * c);  // v0 - c/2 + 4/3 mB - v0
        const float ul = -2.0f * c;                   // UL - v0
        const float lo = fmaxf(fminf(fminf(0.0f, -b), oMD), fminf(fminf(0.0f, ul), oLC));
        const float hi = fminf(fmaxf(fmaxf(0.0f, -b), oMD), fmaxf(fmaxf(0.0f, ul), oLC));
        L = v0 + sclamp(x, lo, hi);
    }
    {
        const float x = R - v0;
        const float oMD = 0.5f * (c - mB);            // (v0 + vp1 - mB)/2 - v0
        const float oLC = fmaf(kBetaMP, mA, 0.5f * b);   // v0 + b/2 + 4/3 mA - v0
        const float ul = 2.0f * b;                    // UL - v0
        const float lo = fmaxf(fminf(fminf(0.0f, c), oMD), fminf(fminf(0.0f, ul), oLC));
        const float hi = fminf(fmaxf(fmaxf(0.0f, c), oMD), fmaxf(fmaxf(0.0f, ul), oLC));
        R = v0 + sclamp(x, lo, hi);
    }
}

template <typename T>
struct MP;
template <>
struct MP<double> {
    static __device__ __forceinline__ void apply(double vm2, double vm1, double v0, double vp1,
                                                 double vp2, double& L, double& R) {
        mp_limit(vm2, vm1, v0, vp1, vp2, L, R);
    }
};
template <>
struct MP<float> {
    static __device__ __forceinline__ void apply(float vm2, float vm1, float v0, float vp1,
                                                 float vp2, float& L, float& R) {
        mp_limit_f(vm2, vm1, v0, vp1, vp2, L, R);
    }
};

}  // namespace wsb
