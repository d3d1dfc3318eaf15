/*
 * weno_oracle.c -- TEST INFRASTRUCTURE ONLY (see weno_oracle.h).
 *
 * A line-by-line CPU restatement of the device loops of the reference
 * harness wilfonba/WenoStandalone, file inputs/weno_standalone.f90 ("f90:"
 * below).  Every function cites the loop it follows.  Expressions keep the
 * Fortran evaluation order (left to right, no re-association) and the
 * recipe builds this file with -ffp-contract=off so no FMA is formed, which
 * is how the reference's CPU build (gfortran -O3, x86-64 without FMA)
 * rounds.  Fortran SIGN(a,b) is copysign(|a|,b); x**2._wp is x*x; real
 * exponents other than 2 go through pow().
 *
 * Parity pin: wo_harness_run() with all_mode=0 reproduces the committed
 * golden checksums tests/golden/weno5.txt of the reference (200^3 x 8,
 * WENO5-JS) -- see tests/test_oracle_golden.py.
 *
 * Deliberate, documented deviation: the reference's WENO3 loop runs over
 * the full is1 range but indexes coefficient arrays that exist only on the
 * core range (f90:413 vs f90:171-187), an out-of-bounds read whose result
 * is undefined.  Here (and in the CUDA library) the coefficient index is
 * clamped to the nearest core face.
 */
#include "weno_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

static int g_threads = 0; /* 0 = OpenMP default */

void wo_set_threads(int nthreads) { g_threads = nthreads; }

int wo_get_threads(void) {
#ifdef _OPENMP
    return g_threads > 0 ? g_threads : omp_get_max_threads();
#else
    return 1;
#endif
}

#define NTHR (wo_get_threads())

/* ------------------------------------------------------------------ */
/* f90:221-244  s_fill_input_field                                      */
/* ------------------------------------------------------------------ */
void wo_fill_input_field(int m, int n, int p, int nv, int buff, double *v_vf) {
    const int is1b = -buff, is1e = m + buff;
    const int is2b = -buff, is2e = n + buff;
    const int is3b = -buff, is3e = p + buff;
    const long long e1 = (long long)(is1e - is1b + 1) + 6;
    const long long e2 = (long long)(is2e - is2b + 1) + 6;
    const long long e3 = (long long)(is3e - is3b + 1) + 6;
    const double den1 = (double)((is1e - is1b + 3) > 1 ? (is1e - is1b + 3) : 1);
    const double den2 = (double)((is2e - is2b + 3) > 1 ? (is2e - is2b + 3) : 1);
    const double den3 = (double)((is3e - is3b + 3) > 1 ? (is3e - is3b + 3) : 1);
#pragma omp parallel for collapse(2) schedule(static) num_threads(NTHR)
    for (int l = 1; l <= nv; ++l) {
        for (long long kk = 0; kk < e3; ++kk) {
            const int k = (int)kk + is3b - 3;
            const double z = (double)(k - is3b + 1) / den3;
            for (long long jj = 0; jj < e2; ++jj) {
                const int j = (int)jj + is2b - 3;
                const double y = (double)(j - is2b + 1) / den2;
                double *row = v_vf + e1 * (jj + e2 * (kk + e3 * (long long)(l - 1)));
                for (long long ii = 0; ii < e1; ++ii) {
                    const int i = (int)ii + is1b - 3;
                    const double x = (double)(i - is1b + 1) / den1;
                    row[ii] = sin(2.1 * x * (double)l) + cos(3.7 * y) + 0.25 * sin(4.3 * z)
                              + 0.02 * (double)(i + 2 * j - k + l);
                }
            }
        }
    }
}

/* ------------------------------------------------------------------ */
/* f90:246-279  s_fill_coefficients                                     */
/* ------------------------------------------------------------------ */
void wo_fill_coefficients(int nc, double offset, double *polyL, double *polyR,
                          double *dL, double *dR, double *beta) {
    static const double baseL[5] = {0.30, 0.27, 0.20, 0.14, 0.09};
    static const double baseR[5] = {0.09, 0.14, 0.20, 0.27, 0.30};
    for (int c = 0; c < nc; ++c) {
        for (int r = 0; r <= 4; ++r) {
            dL[r + 5 * c] = baseL[r] + offset * 0.10;
            dR[r + 5 * c] = baseR[r] + offset * 0.10;
            for (int s = 0; s <= 2; ++s) {
                polyL[c + nc * (r + 5 * s)] = offset + 0.015 * (double)((r + 1) * (s + 1));
                polyR[c + nc * (r + 5 * s)] = -offset + 0.012 * (double)(2 * r + s + 1);
            }
            for (int s = 0; s < 6; ++s) beta[c + nc * (r + 5 * s)] = 0.0;
            beta[c + nc * (r + 5 * 0)] = 0.8 + offset + 0.05 * (double)(r + 1);
            beta[c + nc * (r + 5 * 2)] = 0.9 + offset + 0.04 * (double)(r + 1);
            beta[c + nc * (r + 5 * 3)] = 1.0 + offset + 0.03 * (double)(r + 1);
            beta[c + nc * (r + 5 * 5)] = 1.1 + offset + 0.02 * (double)(r + 1);
        }
    }
}

/* Extents of a direction's sweep arrays (general form of f90:150-187). */
static int sweep_extents(int m, int n, int p, int buff, int dir, long long *ns,
                         long long *c1, long long *c2) {
    const long long N1 = m + 2LL * buff + 1, N2 = n + 2LL * buff + 1, N3 = p + 2LL * buff + 1;
    if (dir == 0) { *ns = N1; *c1 = N2; *c2 = N3; }
    else if (dir == 1) { *ns = N2; *c1 = N1; *c2 = N3; }
    else if (dir == 2) { *ns = N3; *c1 = N2; *c2 = N1; }
    else return -1;
    return 0;
}

/* ------------------------------------------------------------------ */
/* f90:281-330  s_initialize_weno_{x,y,z}                               */
/*   x: v_rs_ws(k,l,q,j) = v_vf(k,l,q,j)                                */
/*   y: v_rs_ws(k,l,q,j) = v_vf(l,k,q,j)                                */
/*   z: v_rs_ws(k,l,q,j) = v_vf(q,l,k,j)                                */
/* k over the sweep axis with +-3 halo, (l,q) over the buffered block.  */
/* ------------------------------------------------------------------ */
int wo_reshape(int m, int n, int p, int nv, int buff, int dir,
               const double *v_vf, double *v_rs_ws) {
    long long ns, c1, c2;
    if (sweep_extents(m, n, p, buff, dir, &ns, &c1, &c2)) return -1;
    const long long E1 = m + 2LL * buff + 7, E2 = n + 2LL * buff + 7, E3 = p + 2LL * buff + 7;
    const long long ks = ns + 6;
#pragma omp parallel for collapse(2) schedule(static) num_threads(NTHR)
    for (long long jv = 0; jv < nv; ++jv) {
        for (long long q = 0; q < c2; ++q) {
            for (long long l = 0; l < c1; ++l) {
                double *out = v_rs_ws + ks * (l + c1 * (q + c2 * jv));
                for (long long k = 0; k < ks; ++k) {
                    /* (x,y,z) index into v_vf, 0-based incl. its 3-cell pad */
                    long long x, y, z;
                    if (dir == 0) { x = k; y = l + 3; z = q + 3; }
                    else if (dir == 1) { x = l + 3; y = k; z = q + 3; }
                    else { x = q + 3; y = l + 3; z = k; }
                    out[k] = v_vf[x + E1 * (y + E2 * (z + E3 * jv))];
                }
            }
        }
    }
    return 0;
}

/* ------------------------------------------------------------------ */
/* f90:332-390  s_order1_copy_{x,y,z}: vL = vR = permuted v_vf          */
/* ------------------------------------------------------------------ */
int wo_order1_copy(int m, int n, int p, int nv, int buff, int dir,
                   const double *v_vf, double *vL, double *vR) {
    long long ns, c1, c2;
    if (sweep_extents(m, n, p, buff, dir, &ns, &c1, &c2)) return -1;
    const long long E1 = m + 2LL * buff + 7, E2 = n + 2LL * buff + 7, E3 = p + 2LL * buff + 7;
#pragma omp parallel for collapse(2) schedule(static) num_threads(NTHR)
    for (long long iv = 0; iv < nv; ++iv) {
        for (long long l = 0; l < c2; ++l) {
            for (long long k = 0; k < c1; ++k) {
                const long long o = ns * (k + c1 * (l + c2 * iv));
                for (long long j = 0; j < ns; ++j) {
                    long long x, y, z;
                    if (dir == 0) { x = j + 3; y = k + 3; z = l + 3; }
                    else if (dir == 1) { x = k + 3; y = j + 3; z = l + 3; }
                    else { x = l + 3; y = k + 3; z = j + 3; }
                    const double val = v_vf[x + E1 * (y + E2 * (z + E3 * iv))];
                    vL[o + j] = val;
                    vR[o + j] = val;
                }
            }
        }
    }
    return 0;
}

/* Coefficient accessors: poly(c,r,s), d(r,c), beta(c,r,s). */
#define PC(a, c, r, s) (a)[(c) + nc * ((r) + 5 * (s))]
#define DC(a, r, c) (a)[(r) + 5 * (c)]
#define BC(a, c, r, s) (a)[(c) + nc * ((r) + 5 * (s))]

/* Mapped-WENO weight transform (f90:419-423, 557-568). */
static inline double mapw(double d, double w) {
    return (d * (1.0 + d - 3.0 * w) + w * w) * (w / (d * d + w * (1.0 - 2.0 * d)));
}

/* ------------------------------------------------------------------ */
/* f90:392-475  s_weno3_kernel (2 stencils, JS / mapped / Z; no TENO    */
/* branch in the reference, so TENO and "none" give alpha=0 -> NaN)    */
/* ------------------------------------------------------------------ */
static void weno3_point(const double *v, int c, long long nc, int scheme, double eps,
                        const double *polyL, const double *polyR, const double *dL,
                        const double *dR, const double *bc, double *oL, double *oR) {
    double dvd0, dvdm1, poly0, poly1, beta0, beta1, a0 = 0.0, a1 = 0.0, w0, w1, tau = 0.0, s;
    dvd0 = v[1] - v[0];
    dvdm1 = v[0] - v[-1];
    poly0 = v[0] + PC(polyL, c, 0, 0) * dvd0;
    poly1 = v[0] + PC(polyL, c, 1, 0) * dvdm1;
    beta0 = BC(bc, c, 0, 0) * dvd0 * dvd0 + eps;
    beta1 = BC(bc, c, 1, 0) * dvdm1 * dvdm1 + eps;
    if (scheme == WO_JS) {
        a0 = DC(dL, 0, c) / (beta0 * beta0);
        a1 = DC(dL, 1, c) / (beta1 * beta1);
    } else if (scheme == WO_MAPPED) {
        a0 = DC(dL, 0, c) / (beta0 * beta0);
        a1 = DC(dL, 1, c) / (beta1 * beta1);
        s = a0 + a1;
        w0 = a0 / s; w1 = a1 / s;
        a0 = mapw(DC(dL, 0, c), w0);
        a1 = mapw(DC(dL, 1, c), w1);
    } else if (scheme == WO_Z) {
        tau = fabs(beta1 - beta0);
        a0 = DC(dL, 0, c) * (1.0 + tau / beta0);
        a1 = DC(dL, 1, c) * (1.0 + tau / beta1);
    }
    s = a0 + a1;
    w0 = a0 / s; w1 = a1 / s;
    *oL = w0 * poly0 + w1 * poly1;

    poly0 = v[0] + PC(polyR, c, 0, 0) * dvd0;
    poly1 = v[0] + PC(polyR, c, 1, 0) * dvdm1;
    if (scheme == WO_JS) {
        a0 = DC(dR, 0, c) / (beta0 * beta0);
        a1 = DC(dR, 1, c) / (beta1 * beta1);
    } else if (scheme == WO_MAPPED) {
        a0 = DC(dR, 0, c) / (beta0 * beta0);
        a1 = DC(dR, 1, c) / (beta1 * beta1);
        s = a0 + a1;
        w0 = a0 / s; w1 = a1 / s;
        a0 = mapw(DC(dR, 0, c), w0);
        a1 = mapw(DC(dR, 1, c), w1);
    } else if (scheme == WO_Z) {
        a0 = DC(dR, 0, c) * (1.0 + tau / beta0);
        a1 = DC(dR, 1, c) * (1.0 + tau / beta1);
    }
    s = a0 + a1;
    w0 = a0 / s; w1 = a1 / s;
    *oR = w0 * poly0 + w1 * poly1;
}

/* ------------------------------------------------------------------ */
/* f90:477-669  s_weno5_kernel (also the math of the specialized        */
/* f90:671-1143 and split f90:1145-1397 variants)                       */
/* ------------------------------------------------------------------ */
static void weno5_point(const double *v, int c, long long nc, int scheme, double eps,
                        double teno_ct, const double *polyL, const double *polyR,
                        const double *dL, const double *dR, const double *bc,
                        double *oL, double *oR) {
    double a0 = 0.0, a1 = 0.0, a2 = 0.0, w0, w1, w2;
    double de0 = 0.0, de1 = 0.0, de2 = 0.0, tau = 0.0, s;
    const double vj = v[0], vjp2 = v[2], vjp1 = v[1], vjm1 = v[-1], vjm2 = v[-2];
    const double dvd_p1 = vjp2 - vjp1;
    const double dvd_0 = vjp1 - vj;
    const double dvd_m1 = vj - vjm1;
    const double dvd_m2 = vjm1 - vjm2;
    double poly0 = vj + PC(polyL, c, 0, 0) * dvd_p1 + PC(polyL, c, 0, 1) * dvd_0;
    double poly1 = vj + PC(polyL, c, 1, 0) * dvd_0 + PC(polyL, c, 1, 1) * dvd_m1;
    double poly2 = vj + PC(polyL, c, 2, 0) * dvd_m1 + PC(polyL, c, 2, 1) * dvd_m2;
    const double beta0 = BC(bc, c, 0, 0) * dvd_p1 * dvd_p1 + BC(bc, c, 0, 1) * dvd_p1 * dvd_0
                         + BC(bc, c, 0, 2) * dvd_0 * dvd_0 + eps;
    const double beta1 = BC(bc, c, 1, 0) * dvd_0 * dvd_0 + BC(bc, c, 1, 1) * dvd_0 * dvd_m1
                         + BC(bc, c, 1, 2) * dvd_m1 * dvd_m1 + eps;
    const double beta2 = BC(bc, c, 2, 0) * dvd_m1 * dvd_m1 + BC(bc, c, 2, 1) * dvd_m1 * dvd_m2
                         + BC(bc, c, 2, 2) * dvd_m2 * dvd_m2 + eps;
    if (scheme == WO_JS) {
        a0 = DC(dL, 0, c) / (beta0 * beta0);
        a1 = DC(dL, 1, c) / (beta1 * beta1);
        a2 = DC(dL, 2, c) / (beta2 * beta2);
    } else if (scheme == WO_MAPPED) {
        a0 = DC(dL, 0, c) / (beta0 * beta0);
        a1 = DC(dL, 1, c) / (beta1 * beta1);
        a2 = DC(dL, 2, c) / (beta2 * beta2);
        s = a0 + a1 + a2;
        w0 = a0 / s; w1 = a1 / s; w2 = a2 / s;
        a0 = mapw(DC(dL, 0, c), w0);
        a1 = mapw(DC(dL, 1, c), w1);
        a2 = mapw(DC(dL, 2, c), w2);
    } else if (scheme == WO_Z) {
        tau = fabs(beta2 - beta0);
        a0 = DC(dL, 0, c) * (1.0 + (tau / beta0));
        a1 = DC(dL, 1, c) * (1.0 + (tau / beta1));
        a2 = DC(dL, 2, c) * (1.0 + (tau / beta2));
    } else if (scheme == WO_TENO) {
        tau = fabs(beta2 - beta0);
        a0 = pow(1.0 + tau / beta0, 6.0);
        a1 = pow(1.0 + tau / beta1, 6.0);
        a2 = pow(1.0 + tau / beta2, 6.0);
        s = a0 + a1 + a2;
        w0 = a0 / s; w1 = a1 / s; w2 = a2 / s;
        de0 = (w0 < teno_ct) ? 0.0 : 1.0;
        de1 = (w1 < teno_ct) ? 0.0 : 1.0;
        de2 = (w2 < teno_ct) ? 0.0 : 1.0;
        a0 = de0 * DC(dL, 0, c);
        a1 = de1 * DC(dL, 1, c);
        a2 = de2 * DC(dL, 2, c);
    }
    s = a0 + a1 + a2;
    w0 = a0 / s; w1 = a1 / s; w2 = a2 / s;
    *oL = w0 * poly0 + w1 * poly1 + w2 * poly2;

    poly0 = vj + PC(polyR, c, 0, 0) * dvd_p1 + PC(polyR, c, 0, 1) * dvd_0;
    poly1 = vj + PC(polyR, c, 1, 0) * dvd_0 + PC(polyR, c, 1, 1) * dvd_m1;
    poly2 = vj + PC(polyR, c, 2, 0) * dvd_m1 + PC(polyR, c, 2, 1) * dvd_m2;
    if (scheme == WO_JS) {
        a0 = DC(dR, 0, c) / (beta0 * beta0);
        a1 = DC(dR, 1, c) / (beta1 * beta1);
        a2 = DC(dR, 2, c) / (beta2 * beta2);
    } else if (scheme == WO_MAPPED) {
        a0 = DC(dR, 0, c) / (beta0 * beta0);
        a1 = DC(dR, 1, c) / (beta1 * beta1);
        a2 = DC(dR, 2, c) / (beta2 * beta2);
        s = a0 + a1 + a2;
        w0 = a0 / s; w1 = a1 / s; w2 = a2 / s;
        a0 = mapw(DC(dR, 0, c), w0);
        a1 = mapw(DC(dR, 1, c), w1);
        a2 = mapw(DC(dR, 2, c), w2);
    } else if (scheme == WO_Z) {
        a0 = DC(dR, 0, c) * (1.0 + (tau / beta0));
        a1 = DC(dR, 1, c) * (1.0 + (tau / beta1));
        a2 = DC(dR, 2, c) * (1.0 + (tau / beta2));
    } else if (scheme == WO_TENO) {
        a0 = de0 * DC(dR, 0, c);
        a1 = de1 * DC(dR, 1, c);
        a2 = de2 * DC(dR, 2, c);
    }
    s = a0 + a1 + a2;
    w0 = a0 / s; w1 = a1 / s; w2 = a2 / s;
    *oR = w0 * poly0 + w1 * poly1 + w2 * poly2;
}

/* ------------------------------------------------------------------ */
/* f90:1419-1542  s_weno7_kernel (4 stencils, 6-term beta).  Arrays are */
/* sized 0:4 with beta(4)=eps, and TENO keeps alpha(4)=(1+tau/eps)^6 in */
/* the final normalisation (f90:1491-1506) -- restated as written.      */
/* ------------------------------------------------------------------ */
static void weno7_point(const double *v, int c, long long nc, int scheme, double eps,
                        double teno_ct, const double *polyL, const double *polyR,
                        const double *dL, const double *dR, const double *bc,
                        double *oL, double *oR) {
    double alpha[5] = {0, 0, 0, 0, 0}, omega[5] = {0, 0, 0, 0, 0};
    double delta[5] = {0, 0, 0, 0, 0}, beta[5] = {eps, eps, eps, eps, eps};
    double poly[4], dvd[6], tau = 0.0, s;
    double *D = dvd + 3; /* D[-3..2] */
    D[2] = v[3] - v[2];
    D[1] = v[2] - v[1];
    D[0] = v[1] - v[0];
    D[-1] = v[0] - v[-1];
    D[-2] = v[-1] - v[-2];
    D[-3] = v[-2] - v[-3];

#define POLY7(P)                                                                                  \
    poly[3] = v[0] + PC(P, c, 0, 0) * D[2] + PC(P, c, 0, 1) * D[1] + PC(P, c, 0, 2) * D[0];       \
    poly[2] = v[0] + PC(P, c, 1, 0) * D[1] + PC(P, c, 1, 1) * D[0] + PC(P, c, 1, 2) * D[-1];      \
    poly[1] = v[0] + PC(P, c, 2, 0) * D[0] + PC(P, c, 2, 1) * D[-1] + PC(P, c, 2, 2) * D[-2];     \
    poly[0] = v[0] + PC(P, c, 3, 0) * D[-1] + PC(P, c, 3, 1) * D[-2] + PC(P, c, 3, 2) * D[-3];
    POLY7(polyL)

#define BETA7(r, a, b, e)                                                                          \
    (BC(bc, c, r, 0) * a * a + BC(bc, c, r, 1) * a * b + BC(bc, c, r, 2) * a * e                 \
     + BC(bc, c, r, 3) * b * b + BC(bc, c, r, 4) * b * e + BC(bc, c, r, 5) * e * e + eps)
    beta[3] = BETA7(0, D[2], D[1], D[0]);
    beta[2] = BETA7(1, D[1], D[0], D[-1]);
    beta[1] = BETA7(2, D[0], D[-1], D[-2]);
    beta[0] = BETA7(3, D[-1], D[-2], D[-3]);

    if (scheme == WO_JS) {
        for (int q = 0; q <= 3; ++q) alpha[q] = DC(dL, q, c) / (beta[q] * beta[q]);
    } else if (scheme == WO_MAPPED) {
        for (int q = 0; q <= 3; ++q) alpha[q] = DC(dL, q, c) / (beta[q] * beta[q]);
        s = alpha[0] + alpha[1] + alpha[2] + alpha[3] + alpha[4];
        for (int q = 0; q <= 4; ++q) omega[q] = alpha[q] / s;
        for (int q = 0; q <= 3; ++q) alpha[q] = mapw(DC(dL, q, c), omega[q]);
    } else if (scheme == WO_Z) {
        tau = fabs(beta[3] - beta[0]);
        for (int q = 0; q <= 3; ++q) {
            const double t = tau / beta[q];
            alpha[q] = DC(dL, q, c) * (1.0 + t * t);
        }
    } else if (scheme == WO_TENO) {
        tau = fabs(beta[4] - beta[3]);
        for (int q = 0; q <= 4; ++q) alpha[q] = 1.0 + tau / beta[q];
        for (int q = 0; q <= 4; ++q) {
            const double a3 = pow(alpha[q], 3.0);
            alpha[q] = a3 * a3;
        }
        s = alpha[0] + alpha[1] + alpha[2] + alpha[3] + alpha[4];
        for (int q = 0; q <= 4; ++q) omega[q] = alpha[q] / s;
        for (int q = 0; q <= 3; ++q) {
            delta[q] = (omega[q] < teno_ct) ? 0.0 : 1.0;
            alpha[q] = delta[q] * DC(dL, q, c);
        }
    }
    s = alpha[0] + alpha[1] + alpha[2] + alpha[3] + alpha[4];
    for (int q = 0; q <= 4; ++q) omega[q] = alpha[q] / s;
    *oL = omega[0] * poly[0] + omega[1] * poly[1] + omega[2] * poly[2] + omega[3] * poly[3];

    POLY7(polyR)
    if (scheme == WO_JS) {
        for (int q = 0; q <= 3; ++q) alpha[q] = DC(dR, q, c) / (beta[q] * beta[q]);
    } else if (scheme == WO_MAPPED) {
        for (int q = 0; q <= 3; ++q) alpha[q] = DC(dR, q, c) / (beta[q] * beta[q]);
        s = alpha[0] + alpha[1] + alpha[2] + alpha[3] + alpha[4];
        for (int q = 0; q <= 4; ++q) omega[q] = alpha[q] / s;
        for (int q = 0; q <= 3; ++q) alpha[q] = mapw(DC(dR, q, c), omega[q]);
    } else if (scheme == WO_Z) {
        for (int q = 0; q <= 3; ++q) {
            const double t = tau / beta[q];
            alpha[q] = DC(dR, q, c) * (1.0 + t * t);
        }
    } else if (scheme == WO_TENO) {
        for (int q = 0; q <= 3; ++q) alpha[q] = delta[q] * DC(dR, q, c);
    }
    s = alpha[0] + alpha[1] + alpha[2] + alpha[3] + alpha[4];
    for (int q = 0; q <= 4; ++q) omega[q] = alpha[q] / s;
    *oR = omega[0] * poly[0] + omega[1] * poly[1] + omega[2] * poly[2] + omega[3] * poly[3];
#undef POLY7
#undef BETA7
}

int wo_reconstruct(int ns_, int c1_, int c2_, int nv_, int order, int scheme,
                   double eps, double teno_ct, const double *v_rs_ws,
                   const double *polyL, const double *polyR, const double *dL,
                   const double *dR, const double *beta, double *vL, double *vR) {
    const long long ns = ns_, c1 = c1_, c2 = c2_, nv = nv_;
    const long long nc = ns - 6;
    if (nc < 1 || c1 < 1 || c2 < 1 || nv < 1) return -1;
    if (order != 3 && order != 5 && order != 7) return -2;
    const long long rows = c1 * c2 * nv;
    /* WENO3 covers the full sweep range (f90:413), WENO5/7 the core
     * range (f90:509, 1444). */
    const long long jb = (order == 3) ? 0 : 3;
    const long long je = (order == 3) ? ns - 1 : ns - 4;
#pragma omp parallel for schedule(static) num_threads(NTHR)
    for (long long r = 0; r < rows; ++r) {
        const double *in = v_rs_ws + (ns + 6) * r;
        double *oL = vL + ns * r;
        double *oR = vR + ns * r;
        for (long long o = jb; o <= je; ++o) {
            const double *v = in + o + 3;
            long long c = o - 3;
            if (order == 3) {
                if (c < 0) c = 0;
                if (c > nc - 1) c = nc - 1;
                weno3_point(v, (int)c, nc, scheme, eps, polyL, polyR, dL, dR, beta, oL + o, oR + o);
            } else if (order == 5) {
                weno5_point(v, (int)c, nc, scheme, eps, teno_ct, polyL, polyR, dL, dR, beta,
                            oL + o, oR + o);
            } else {
                weno7_point(v, (int)c, nc, scheme, eps, teno_ct, polyL, polyR, dL, dR, beta,
                            oL + o, oR + o);
            }
        }
    }
    return 0;
}

/* ------------------------------------------------------------------ */
/* TENO cutoff margin (checker support, no reference counterpart): per   */
/* core face, min over the cutoff tests of |omega_q - CT| / CT, with     */
/* beta, alpha and omega formed exactly as weno5_point (f90:545-550,     */
/* 578-590) and weno7_point (f90:1462-1473, 1491-1506) form them.  A     */
/* GPU result may differ from the oracle's only where this margin is at  */
/* rounding level (the cutoff decision can go either way there).         */
/* Faces outside the core get +inf.                                      */
/* ------------------------------------------------------------------ */
int wo_teno_margin(int ns_, int c1_, int c2_, int nv_, int order, double eps, double teno_ct,
                   const double *v_rs_ws, const double *bc, double *margin) {
    const long long ns = ns_, c1 = c1_, c2 = c2_, nv = nv_;
    const long long nc = ns - 6;
    if (nc < 1 || c1 < 1 || c2 < 1 || nv < 1) return -1;
    if (order != 5 && order != 7) return -2;
    const long long rows = c1 * c2 * nv;
#pragma omp parallel for schedule(static) num_threads(NTHR)
    for (long long r = 0; r < rows; ++r) {
        const double *in = v_rs_ws + (ns + 6) * r;
        double *mg = margin + ns * r;
        for (long long o = 0; o < ns; ++o) mg[o] = INFINITY;
        for (long long o = 3; o <= ns - 4; ++o) {
            const double *v = in + o + 3;
            const long long c = o - 3;
            double best = INFINITY;
            if (order == 5) {
                const double dvd_p1 = v[2] - v[1], dvd_0 = v[1] - v[0];
                const double dvd_m1 = v[0] - v[-1], dvd_m2 = v[-1] - v[-2];
                const double b0 = BC(bc, c, 0, 0) * dvd_p1 * dvd_p1 + BC(bc, c, 0, 1) * dvd_p1 * dvd_0
                                  + BC(bc, c, 0, 2) * dvd_0 * dvd_0 + eps;
                const double b1 = BC(bc, c, 1, 0) * dvd_0 * dvd_0 + BC(bc, c, 1, 1) * dvd_0 * dvd_m1
                                  + BC(bc, c, 1, 2) * dvd_m1 * dvd_m1 + eps;
                const double b2 = BC(bc, c, 2, 0) * dvd_m1 * dvd_m1 + BC(bc, c, 2, 1) * dvd_m1 * dvd_m2
                                  + BC(bc, c, 2, 2) * dvd_m2 * dvd_m2 + eps;
                const double tau = fabs(b2 - b0);
                const double a[3] = {pow(1.0 + tau / b0, 6.0), pow(1.0 + tau / b1, 6.0),
                                     pow(1.0 + tau / b2, 6.0)};
                const double s = a[0] + a[1] + a[2];
                for (int q = 0; q < 3; ++q) {
                    const double m = fabs(a[q] / s - teno_ct) / teno_ct;
                    if (!(m >= best)) best = m;
                }
            } else {
                double D6[6];
                double *D = D6 + 3;
                D[2] = v[3] - v[2]; D[1] = v[2] - v[1]; D[0] = v[1] - v[0];
                D[-1] = v[0] - v[-1]; D[-2] = v[-1] - v[-2]; D[-3] = v[-2] - v[-3];
#define BETA7M(r, a, b, e)                                                                         \
    (BC(bc, c, r, 0) * a * a + BC(bc, c, r, 1) * a * b + BC(bc, c, r, 2) * a * e                 \
     + BC(bc, c, r, 3) * b * b + BC(bc, c, r, 4) * b * e + BC(bc, c, r, 5) * e * e + eps)
                double beta[5];
                beta[3] = BETA7M(0, D[2], D[1], D[0]);
                beta[2] = BETA7M(1, D[1], D[0], D[-1]);
                beta[1] = BETA7M(2, D[0], D[-1], D[-2]);
                beta[0] = BETA7M(3, D[-1], D[-2], D[-3]);
                beta[4] = eps;
#undef BETA7M
                const double tau = fabs(beta[4] - beta[3]);
                double alpha[5], s = 0.0;
                for (int q = 0; q <= 4; ++q) {
                    const double a3 = pow(1.0 + tau / beta[q], 3.0);
                    alpha[q] = a3 * a3;
                }
                s = alpha[0] + alpha[1] + alpha[2] + alpha[3] + alpha[4];
                for (int q = 0; q <= 3; ++q) {
                    const double m = fabs(alpha[q] / s - teno_ct) / teno_ct;
                    if (!(m >= best)) best = m;
                }
            }
            mg[o] = best;
        }
    }
    return 0;
}

/* ------------------------------------------------------------------ */
/* f90:1544-1615  s_preserve_monotonicity (core faces, in place)        */
/* ------------------------------------------------------------------ */
static inline double fsign(double a, double b) { return copysign(fabs(a), b); }
static inline double min3(double a, double b, double c) { return fmin(fmin(a, b), c); }
static inline double max3(double a, double b, double c) { return fmax(fmax(a, b), c); }

static inline double mp_minmod(double dl, double dr) {
    /* (f90:1568-1571): 4-argument minmod of (4dl-dr, dl, 4dr-dl, dr) */
    const double A = 4.0 * dl - dr;
    const double B = 4.0 * dr - dl;
    return (fsign(1.0, A) + fsign(1.0, B))
           * fabs((fsign(1.0, A) + fsign(1.0, dl)) * (fsign(1.0, A) + fsign(1.0, dr)))
           * fmin(fmin(fmin(fabs(A), fabs(dl)), fabs(B)), fabs(dr)) / 8.0;
}

int wo_preserve_monotonicity(int ns_, int c1_, int c2_, int nv_,
                             const double *v_rs_ws, double *vL, double *vR) {
    const long long ns = ns_, rows = (long long)c1_ * c2_ * nv_;
    if (ns < 7) return -1;
    const double alpha_mp = 2.0;
    const double beta_mp = 4.0 / 3.0;
#pragma omp parallel for schedule(static) num_threads(NTHR)
    for (long long r = 0; r < rows; ++r) {
        const double *in = v_rs_ws + (ns + 6) * r;
        double *oL = vL + ns * r;
        double *oR = vR + ns * r;
        for (long long o = 3; o <= ns - 4; ++o) {
            const double *v = in + o + 3;
            const double dm1 = v[0] + v[-2] - 2.0 * v[-1];
            const double d0 = v[1] + v[-1] - 2.0 * v[0];
            const double dp1 = v[2] + v[0] - 2.0 * v[1];
            double d_MD = mp_minmod(dm1, d0);
            double d_LC = mp_minmod(d0, dp1);
            const double vL_UL = v[0] - alpha_mp * (v[1] - v[0]);
            const double vL_MD = (v[0] + v[-1] - d_MD) * 5.e-1;
            const double vL_LC = v[0] - (v[1] - v[0]) * 5.e-1 + beta_mp * d_LC;
            const double vL_min = fmax(min3(v[0], v[-1], vL_MD), min3(v[0], vL_UL, vL_LC));
            const double vL_max = fmin(max3(v[0], v[-1], vL_MD), max3(v[0], vL_UL, vL_LC));
            const double l0 = oL[o];
            oL[o] = l0 + (fsign(5.e-1, vL_min - l0) + fsign(5.e-1, vL_max - l0))
                             * fmin(fabs(vL_min - l0), fabs(vL_max - l0));

            const double vR_UL = v[0] + alpha_mp * (v[0] - v[-1]);
            d_MD = mp_minmod(d0, dp1);
            d_LC = mp_minmod(dm1, d0);
            const double vR_MD = (v[0] + v[1] - d_MD) * 5.e-1;
            const double vR_LC = v[0] + (v[0] - v[-1]) * 5.e-1 + beta_mp * d_LC;
            const double vR_min = fmax(min3(v[0], v[1], vR_MD), min3(v[0], vR_UL, vR_LC));
            const double vR_max = fmin(max3(v[0], v[1], vR_MD), max3(v[0], vR_UL, vR_LC));
            const double r0 = oR[o];
            oR[o] = r0 + (fsign(5.e-1, vR_min - r0) + fsign(5.e-1, vR_max - r0))
                             * fmin(fabs(vR_min - r0), fabs(vR_max - r0));
        }
    }
    return 0;
}

/* ------------------------------------------------------------------ */
/* f90:1617-1620  f_checksum = sum(abs(arr)), in array order            */
/* ------------------------------------------------------------------ */
double wo_checksum(long long n, const double *a) {
    double s = 0.0;
    for (long long i = 0; i < n; ++i) s += fabs(a[i]);
    return s;
}

/* ------------------------------------------------------------------ */
/* The driver's default-scope paths (f90:1684-1730 and 1651-1682) on    */
/* the harness's synthetic data, one direction at a time, returning     */
/* Checksum X, Y, Z, T (f90:1836-1839).                                 */
/* all_mode=0: weno5 scope=full: reshape, order-1 copy, WENO5.          */
/* all_mode=1: reshape, copy, WENO3, WENO5, WENO7, MP.                  */
/* ------------------------------------------------------------------ */
int wo_harness_run(int m, int n, int p, int nv, int buff, double eps, int scheme,
                   double teno_ct, int all_mode, double out[4]) {
    const long long E1 = m + 2LL * buff + 7, E2 = n + 2LL * buff + 7, E3 = p + 2LL * buff + 7;
    double *v_vf = (double *)malloc(sizeof(double) * E1 * E2 * E3 * nv);
    if (!v_vf) return -3;
    wo_fill_input_field(m, n, p, nv, buff, v_vf);
    static const double offs[3] = {0.03, 0.05, 0.07};
    double total = 0.0;
    for (int dir = 0; dir < 3; ++dir) {
        long long ns, c1, c2;
        sweep_extents(m, n, p, buff, dir, &ns, &c1, &c2);
        const long long nc = ns - 6;
        const long long nin = (ns + 6) * c1 * c2 * nv, nout = ns * c1 * c2 * nv;
        double *rs = (double *)malloc(sizeof(double) * nin);
        double *L = (double *)malloc(sizeof(double) * nout);
        double *R = (double *)malloc(sizeof(double) * nout);
        double *pL = (double *)malloc(sizeof(double) * nc * 15);
        double *pR = (double *)malloc(sizeof(double) * nc * 15);
        double *dL = (double *)malloc(sizeof(double) * nc * 5);
        double *dR = (double *)malloc(sizeof(double) * nc * 5);
        double *bc = (double *)malloc(sizeof(double) * nc * 30);
        if (!rs || !L || !R || !pL || !pR || !dL || !dR || !bc) {
            free(rs); free(L); free(R); free(pL); free(pR); free(dL); free(dR); free(bc);
            free(v_vf);
            return -3;
        }
        wo_fill_coefficients((int)nc, offs[dir], pL, pR, dL, dR, bc);
        wo_reshape(m, n, p, nv, buff, dir, v_vf, rs);
        wo_order1_copy(m, n, p, nv, buff, dir, v_vf, L, R);
        if (all_mode)
            wo_reconstruct((int)ns, (int)c1, (int)c2, nv, 3, scheme, eps, teno_ct, rs, pL, pR, dL,
                           dR, bc, L, R);
        wo_reconstruct((int)ns, (int)c1, (int)c2, nv, 5, scheme, eps, teno_ct, rs, pL, pR, dL, dR,
                       bc, L, R);
        if (all_mode) {
            wo_reconstruct((int)ns, (int)c1, (int)c2, nv, 7, scheme, eps, teno_ct, rs, pL, pR, dL,
                           dR, bc, L, R);
            wo_preserve_monotonicity((int)ns, (int)c1, (int)c2, nv, rs, L, R);
        }
        out[dir] = wo_checksum(nout, L) + wo_checksum(nout, R);
        total += out[dir];
        free(rs); free(L); free(R); free(pL); free(pR); free(dL); free(dR); free(bc);
    }
    out[3] = out[0] + out[1] + out[2];
    (void)total;
    free(v_vf);
    return 0;
}
