// weno_oracle_ad.cpp -- TEST INFRASTRUCTURE ONLY.
//
// Forward-mode (dual-number) differentiation of the reference harness's
// per-face formulas (wilfonba/WenoStandalone inputs/weno_standalone.f90:
// WENO3 f90:416-468, WENO5 f90:511-662, WENO7 f90:1448-1535, MP
// f90:1564-1608), used to check the library's hand-written adjoint (VJP).
// The formulas are restated on a scalar type T (double or Dual) in the
// reference's own operation order; min/max/sign pick operands by value, so
// the derivative is that of the branch the reference takes.  Each face is
// evaluated once per stencil input with that input seeded, which gives the
// face's exact local Jacobian; wo_vjp then gathers
//   gv[J] = sum over faces f, sides s of d(out_s(f))/d(v[J]) * g_s(f).
#include <cmath>
#include <cstring>

namespace {

struct Dual {
    double v, d;
    Dual(double x = 0.0, double dx = 0.0) : v(x), d(dx) {}
};
inline Dual operator+(Dual a, Dual b) { return {a.v + b.v, a.d + b.d}; }
inline Dual operator-(Dual a, Dual b) { return {a.v - b.v, a.d - b.d}; }
inline Dual operator*(Dual a, Dual b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }
inline Dual operator/(Dual a, Dual b) { return {a.v / b.v, (a.d * b.v - a.v * b.d) / (b.v * b.v)}; }
inline bool operator<(Dual a, Dual b) { return a.v < b.v; }
inline double val(Dual a) { return a.v; }
inline double val(double a) { return a; }
inline Dual dabs(Dual a) { return a.v < 0.0 || (a.v == 0.0 && std::signbit(a.v)) ? Dual{-a.v, -a.d} : a; }
inline double dabs(double a) { return std::fabs(a); }
// Fortran SIGN(a, b) = |a| with the sign of b
inline Dual fsign(Dual a, Dual b) {
    const Dual m = dabs(a);
    return std::signbit(b.v) ? Dual{-m.v, -m.d} : m;
}
inline double fsign(double a, double b) { return std::copysign(std::fabs(a), b); }
inline Dual dmin(Dual a, Dual b) { return (b.v < a.v) ? b : a; }
inline Dual dmax(Dual a, Dual b) { return (a.v < b.v) ? b : a; }
inline double dmin(double a, double b) { return std::fmin(a, b); }
inline double dmax(double a, double b) { return std::fmax(a, b); }
inline Dual dpow(Dual x, double p) {
    const double f = std::pow(x.v, p);
    return {f, p * std::pow(x.v, p - 1.0) * x.d};
}
inline double dpow(double x, double p) { return std::pow(x, p); }

enum { JS = 0, MAPPED = 1, WZ = 2, TENO = 3, NONE = 4 };

struct CoefView {
    const double *pL, *pR, *dL, *dR, *bc;
    long long nc, c;
    double polyL(int r, int s) const { return pL[c + nc * (r + 5 * s)]; }
    double polyR(int r, int s) const { return pR[c + nc * (r + 5 * s)]; }
    double d_L(int r) const { return dL[r + 5 * c]; }
    double d_R(int r) const { return dR[r + 5 * c]; }
    double beta(int r, int s) const { return bc[c + nc * (r + 5 * s)]; }
};

template <class T>
T mapw(double d, T w) {
    return (T(d) * (T(1.0 + d) - T(3.0) * w) + w * w) * (w / (T(d * d) + w * T(1.0 - 2.0 * d)));
}

// f90:416-468
template <class T>
void weno3(const T* v, const CoefView& k, int scheme, double eps, T& oL, T& oR) {
    const T dvd0 = v[1] - v[0], dvdm1 = v[0] - v[-1];
    T poly0 = v[0] + T(k.polyL(0, 0)) * dvd0, poly1 = v[0] + T(k.polyL(1, 0)) * dvdm1;
    const T beta0 = T(k.beta(0, 0)) * dvd0 * dvd0 + T(eps);
    const T beta1 = T(k.beta(1, 0)) * dvdm1 * dvdm1 + T(eps);
    T a0(0.0), a1(0.0), tau(0.0), s;
    if (scheme == JS || scheme == MAPPED) {
        a0 = T(k.d_L(0)) / (beta0 * beta0);
        a1 = T(k.d_L(1)) / (beta1 * beta1);
        if (scheme == MAPPED) {
            s = a0 + a1;
            a0 = mapw(k.d_L(0), a0 / s);
            a1 = mapw(k.d_L(1), a1 / s);
        }
    } else if (scheme == WZ) {
        tau = dabs(beta1 - beta0);
        a0 = T(k.d_L(0)) * (T(1.0) + tau / beta0);
        a1 = T(k.d_L(1)) * (T(1.0) + tau / beta1);
    }
    s = a0 + a1;
    oL = (a0 / s) * poly0 + (a1 / s) * poly1;
    poly0 = v[0] + T(k.polyR(0, 0)) * dvd0;
    poly1 = v[0] + T(k.polyR(1, 0)) * dvdm1;
    if (scheme == JS || scheme == MAPPED) {
        a0 = T(k.d_R(0)) / (beta0 * beta0);
        a1 = T(k.d_R(1)) / (beta1 * beta1);
        if (scheme == MAPPED) {
            s = a0 + a1;
            a0 = mapw(k.d_R(0), a0 / s);
            a1 = mapw(k.d_R(1), a1 / s);
        }
    } else if (scheme == WZ) {
        a0 = T(k.d_R(0)) * (T(1.0) + tau / beta0);
        a1 = T(k.d_R(1)) * (T(1.0) + tau / beta1);
    } else {
        a0 = a1 = T(0.0);
    }
    s = a0 + a1;
    oR = (a0 / s) * poly0 + (a1 / s) * poly1;
}

// f90:511-662
template <class T>
void weno5(const T* v, const CoefView& k, int scheme, double eps, double ct, T& oL, T& oR) {
    const T dvd_p1 = v[2] - v[1], dvd_0 = v[1] - v[0], dvd_m1 = v[0] - v[-1], dvd_m2 = v[-1] - v[-2];
    T p0 = v[0] + T(k.polyL(0, 0)) * dvd_p1 + T(k.polyL(0, 1)) * dvd_0;
    T p1 = v[0] + T(k.polyL(1, 0)) * dvd_0 + T(k.polyL(1, 1)) * dvd_m1;
    T p2 = v[0] + T(k.polyL(2, 0)) * dvd_m1 + T(k.polyL(2, 1)) * dvd_m2;
    const T b0 = T(k.beta(0, 0)) * dvd_p1 * dvd_p1 + T(k.beta(0, 1)) * dvd_p1 * dvd_0 +
                 T(k.beta(0, 2)) * dvd_0 * dvd_0 + T(eps);
    const T b1 = T(k.beta(1, 0)) * dvd_0 * dvd_0 + T(k.beta(1, 1)) * dvd_0 * dvd_m1 +
                 T(k.beta(1, 2)) * dvd_m1 * dvd_m1 + T(eps);
    const T b2 = T(k.beta(2, 0)) * dvd_m1 * dvd_m1 + T(k.beta(2, 1)) * dvd_m1 * dvd_m2 +
                 T(k.beta(2, 2)) * dvd_m2 * dvd_m2 + T(eps);
    T a0(0.0), a1(0.0), a2(0.0), s, tau(0.0);
    double de0 = 0, de1 = 0, de2 = 0;
    auto js = [&](double d0, double d1, double d2) {
        a0 = T(d0) / (b0 * b0);
        a1 = T(d1) / (b1 * b1);
        a2 = T(d2) / (b2 * b2);
    };
    if (scheme == JS || scheme == MAPPED) {
        js(k.d_L(0), k.d_L(1), k.d_L(2));
        if (scheme == MAPPED) {
            s = a0 + a1 + a2;
            const T w0 = a0 / s, w1 = a1 / s, w2 = a2 / s;
            a0 = mapw(k.d_L(0), w0);
            a1 = mapw(k.d_L(1), w1);
            a2 = mapw(k.d_L(2), w2);
        }
    } else if (scheme == WZ) {
        tau = dabs(b2 - b0);
        a0 = T(k.d_L(0)) * (T(1.0) + (tau / b0));
        a1 = T(k.d_L(1)) * (T(1.0) + (tau / b1));
        a2 = T(k.d_L(2)) * (T(1.0) + (tau / b2));
    } else if (scheme == TENO) {
        tau = dabs(b2 - b0);
        a0 = dpow(T(1.0) + tau / b0, 6.0);
        a1 = dpow(T(1.0) + tau / b1, 6.0);
        a2 = dpow(T(1.0) + tau / b2, 6.0);
        s = a0 + a1 + a2;
        de0 = (val(a0 / s) < ct) ? 0.0 : 1.0;
        de1 = (val(a1 / s) < ct) ? 0.0 : 1.0;
        de2 = (val(a2 / s) < ct) ? 0.0 : 1.0;
        a0 = T(de0 * k.d_L(0));
        a1 = T(de1 * k.d_L(1));
        a2 = T(de2 * k.d_L(2));
    }
    s = a0 + a1 + a2;
    oL = (a0 / s) * p0 + (a1 / s) * p1 + (a2 / s) * p2;
    p0 = v[0] + T(k.polyR(0, 0)) * dvd_p1 + T(k.polyR(0, 1)) * dvd_0;
    p1 = v[0] + T(k.polyR(1, 0)) * dvd_0 + T(k.polyR(1, 1)) * dvd_m1;
    p2 = v[0] + T(k.polyR(2, 0)) * dvd_m1 + T(k.polyR(2, 1)) * dvd_m2;
    if (scheme == JS || scheme == MAPPED) {
        js(k.d_R(0), k.d_R(1), k.d_R(2));
        if (scheme == MAPPED) {
            s = a0 + a1 + a2;
            const T w0 = a0 / s, w1 = a1 / s, w2 = a2 / s;
            a0 = mapw(k.d_R(0), w0);
            a1 = mapw(k.d_R(1), w1);
            a2 = mapw(k.d_R(2), w2);
        }
    } else if (scheme == WZ) {
        a0 = T(k.d_R(0)) * (T(1.0) + (tau / b0));
        a1 = T(k.d_R(1)) * (T(1.0) + (tau / b1));
        a2 = T(k.d_R(2)) * (T(1.0) + (tau / b2));
    } else if (scheme == TENO) {
        a0 = T(de0 * k.d_R(0));
        a1 = T(de1 * k.d_R(1));
        a2 = T(de2 * k.d_R(2));
    } else {
        a0 = a1 = a2 = T(0.0);
    }
    s = a0 + a1 + a2;
    oR = (a0 / s) * p0 + (a1 / s) * p1 + (a2 / s) * p2;
}

// f90:1448-1535 (arrays 0:4, beta(4) = eps; TENO keeps alpha(4))
template <class T>
void weno7(const T* v, const CoefView& k, int scheme, double eps, double ct, T& oL, T& oR) {
    T D[6];  // D[q+3] = dvd(q)
    D[5] = v[3] - v[2];
    D[4] = v[2] - v[1];
    D[3] = v[1] - v[0];
    D[2] = v[0] - v[-1];
    D[1] = v[-1] - v[-2];
    D[0] = v[-2] - v[-3];
    T beta[5], poly[4], alpha[5], om[5];
    double delta[4] = {0, 0, 0, 0};
    for (int r = 0; r < 4; ++r) {
        const T a = D[5 - r], b = D[4 - r], e = D[3 - r];
        beta[3 - r] = T(k.beta(r, 0)) * a * a + T(k.beta(r, 1)) * a * b + T(k.beta(r, 2)) * a * e +
                      T(k.beta(r, 3)) * b * b + T(k.beta(r, 4)) * b * e + T(k.beta(r, 5)) * e * e + T(eps);
    }
    beta[4] = T(eps);
    auto polys = [&](bool left) {
        for (int r = 0; r < 4; ++r) {
            const T a = D[5 - r], b = D[4 - r], e = D[3 - r];
            const double c0 = left ? k.polyL(r, 0) : k.polyR(r, 0);
            const double c1 = left ? k.polyL(r, 1) : k.polyR(r, 1);
            const double c2 = left ? k.polyL(r, 2) : k.polyR(r, 2);
            poly[3 - r] = v[0] + T(c0) * a + T(c1) * b + T(c2) * e;
        }
    };
    T tau(0.0), s;
    for (int side = 0; side < 2; ++side) {
        const bool left = side == 0;
        polys(left);
        auto d = [&](int q) { return left ? k.d_L(q) : k.d_R(q); };
        if (left)
            for (int q = 0; q < 5; ++q) alpha[q] = T(0.0);
        if (scheme == JS || scheme == MAPPED) {
            for (int q = 0; q < 4; ++q) alpha[q] = T(d(q)) / (beta[q] * beta[q]);
            if (scheme == MAPPED) {
                s = alpha[0] + alpha[1] + alpha[2] + alpha[3] + alpha[4];
                for (int q = 0; q < 5; ++q) om[q] = alpha[q] / s;
                for (int q = 0; q < 4; ++q) alpha[q] = mapw(d(q), om[q]);
            }
        } else if (scheme == WZ) {
            if (left) tau = dabs(beta[3] - beta[0]);
            for (int q = 0; q < 4; ++q) {
                const T t = tau / beta[q];
                alpha[q] = T(d(q)) * (T(1.0) + t * t);
            }
        } else if (scheme == TENO) {
            if (left) {
                tau = dabs(beta[4] - beta[3]);
                for (int q = 0; q < 5; ++q) alpha[q] = T(1.0) + tau / beta[q];
                for (int q = 0; q < 5; ++q) {
                    const T a3 = dpow(alpha[q], 3.0);
                    alpha[q] = a3 * a3;
                }
                s = alpha[0] + alpha[1] + alpha[2] + alpha[3] + alpha[4];
                for (int q = 0; q < 4; ++q) delta[q] = (val(alpha[q] / s) < ct) ? 0.0 : 1.0;
            }
            for (int q = 0; q < 4; ++q) alpha[q] = T(delta[q] * d(q));
        }
        s = alpha[0] + alpha[1] + alpha[2] + alpha[3] + alpha[4];
        for (int q = 0; q < 5; ++q) om[q] = alpha[q] / s;
        const T out = om[0] * poly[0] + om[1] * poly[1] + om[2] * poly[2] + om[3] * poly[3];
        if (left) oL = out;
        else oR = out;
    }
}

template <class T>
T minmod4(T dl, T dr) {
    const T A = T(4.0) * dl - dr, B = T(4.0) * dr - dl;
    return (fsign(T(1.0), A) + fsign(T(1.0), B)) * dabs((fsign(T(1.0), A) + fsign(T(1.0), dl)) *
                                                      (fsign(T(1.0), A) + fsign(T(1.0), dr))) *
           dmin(dmin(dmin(dabs(A), dabs(dl)), dabs(B)), dabs(dr)) / T(8.0);
}

// f90:1564-1608 on one face; v[-2..2]
template <class T>
void mp(const T* v, T& L, T& R) {
    const T am(2.0), bm(4.0 / 3.0), h(5.e-1);
    const T dm1 = v[0] + v[-2] - T(2.0) * v[-1];
    const T d0 = v[1] + v[-1] - T(2.0) * v[0];
    const T dp1 = v[2] + v[0] - T(2.0) * v[1];
    T dMD = minmod4(dm1, d0), dLC = minmod4(d0, dp1);
    const T ULl = v[0] - am * (v[1] - v[0]);
    const T MDl = (v[0] + v[-1] - dMD) * h;
    const T LCl = v[0] - (v[1] - v[0]) * h + bm * dLC;
    const T lo = dmax(dmin(dmin(v[0], v[-1]), MDl), dmin(dmin(v[0], ULl), LCl));
    const T hi = dmin(dmax(dmax(v[0], v[-1]), MDl), dmax(dmax(v[0], ULl), LCl));
    L = L + (fsign(h, lo - L) + fsign(h, hi - L)) * dmin(dabs(lo - L), dabs(hi - L));
    const T ULr = v[0] + am * (v[0] - v[-1]);
    dMD = minmod4(d0, dp1);
    dLC = minmod4(dm1, d0);
    const T MDr = (v[0] + v[1] - dMD) * h;
    const T LCr = v[0] + (v[0] - v[-1]) * h + bm * dLC;
    const T lo2 = dmax(dmin(dmin(v[0], v[1]), MDr), dmin(dmin(v[0], ULr), LCr));
    const T hi2 = dmin(dmax(dmax(v[0], v[1]), MDr), dmax(dmax(v[0], ULr), LCr));
    R = R + (fsign(h, lo2 - R) + fsign(h, hi2 - R)) * dmin(dabs(lo2 - R), dabs(hi2 - R));
}

template <class T>
void face(const T* v, const CoefView& k, int order, int scheme, bool with_mp, bool core, double eps, double ct,
          T& L, T& R) {
    if (order == 3) weno3(v, k, scheme, eps, L, R);
    else if (order == 5) weno5(v, k, scheme, eps, ct, L, R);
    else weno7(v, k, scheme, eps, ct, L, R);
    if (with_mp && core) mp(v, L, R);
}

}  // namespace

extern "C" {

// gv (layout of v_rs_ws, (ns+6) x c1 x c2 x nv) = VJP of the sweep's
// (vL, vR) with cotangents (gL, gR); faces as the forward sweep: all faces
// for WENO3 (coefficient index clamped to the core), core faces otherwise;
// MP on core faces.
int wo_vjp(int ns_, int c1, int c2, int nv, int order, int scheme, int with_mp, double eps, double ct,
           const double* rs, const double* pL, const double* pR, const double* dL, const double* dR,
           const double* bc, const double* gL, const double* gR, double* gv) {
    const long long ns = ns_, nc = ns - 6, rows = (long long)c1 * c2 * nv;
    if (nc < 1 || (order != 3 && order != 5 && order != 7)) return -1;
    std::memset(gv, 0, sizeof(double) * (ns + 6) * rows);
    const long long ob = (order == 3) ? 0 : 3, oe = (order == 3) ? ns - 1 : ns - 4;
#pragma omp parallel for schedule(static)
    for (long long r = 0; r < rows; ++r) {
        const double* in = rs + (ns + 6) * r;
        double* out = gv + (ns + 6) * r;
        for (long long o = ob; o <= oe; ++o) {
            long long c = o - 3;
            c = c < 0 ? 0 : (c > nc - 1 ? nc - 1 : c);
            CoefView k{pL, pR, dL, dR, bc, nc, c};
            const bool core = (o >= 3 && o <= ns - 4);
            // seed every input of the 7-wide window; those outside the
            // face's stencil get a zero derivative
            for (int q = -3; q <= 3; ++q) {
                Dual w[7];
                for (int t = -3; t <= 3; ++t) {
                    const long long J = o + 3 + t;
                    w[t + 3] = Dual((J >= 0 && J < ns + 6) ? in[J] : 0.0, t == q ? 1.0 : 0.0);
                }
                Dual L, R;
                face(w + 3, k, order, scheme, with_mp != 0, core, eps, ct, L, R);
                out[o + 3 + q] += L.d * gL[ns * r + o] + R.d * gR[ns * r + o];
            }
        }
    }
    return 0;
}

}  // extern "C"
