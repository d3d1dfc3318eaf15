// sweep_generic.cuh -- general-stride reconstruction sweep.
//
// One thread per face along the sweep axis; the face's coefficients stay in
// registers while the thread walks over the cross-section columns.  It reads
// its stencil straight from global memory with arbitrary strides, so it
// serves every layout (v_rs_ws, or v_vf directly for the folded form) and
// every alignment.  The TMA-pipelined kernel (sweep_tma.cuh) is the fast
// path; this one is its fallback and its in-library cross-check.
#pragma once

#include "weno_math.cuh"

namespace wsb {

// Geometry of one sweep.  Input element (J, a, b, v), J in [0, ns+6) along
// the sweep (J = face index + 3), at  in + in_off + J*sJ + a*sA + b*sB + v*sV.
// Output element (o, a, b, v) at out + o + ns*(a + c1*(b + c2*v)).
struct SweepGeom {
    long long ns, nc, c1, c2, nv, cols;
    long long sJ, sA, sB, sV, in_off;
};

struct CoefPtrs {
    const double *polyL, *polyR, *dL, *dR, *beta;
};

struct WenoParams {
    int scheme;
    double eps, teno_ct;
};

// Face-independent coefficients passed by value (laid out as Coef<ORDER>);
// used when the coefficient pointers are null.
struct UniCoefs {
    double v[56];
};

template <typename T>
__device__ __forceinline__ double ld(const T* p) { return (double)__ldg(p); }

// ORDER in {3,5,7}; ORDER == 0 is the standalone MP limiter (reads vL/vR).
template <int ORDER, bool MPF, typename T>
__global__ void __launch_bounds__(128) sweep_generic_kernel(SweepGeom g, const T* __restrict__ in,
                                                            T* __restrict__ vL, T* __restrict__ vR,
                                                            CoefPtrs cp, WenoParams wp, const UniCoefs uc) {
    using PT = T;  // polynomial sums in the storage precision
    const long long o0 = (ORDER == 3) ? 0 : 3;
    const long long nf = (ORDER == 3) ? g.ns : g.nc;
    const long long f = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nf) return;
    const long long o = o0 + f;
    long long c = o - 3;
    c = c < 0 ? 0 : (c > g.nc - 1 ? g.nc - 1 : c);

    Coef<(ORDER == 0 ? 3 : ORDER)> cf;
    if constexpr (ORDER != 0) {
        if (cp.polyL) cf.load(cp.polyL, cp.polyR, cp.dL, cp.dR, cp.beta, g.nc, c);
        else cf = *reinterpret_cast<const Coef<ORDER>*>(uc.v);
    }

    for (long long col = blockIdx.y; col < g.cols; col += gridDim.y) {
        const long long a = col % g.c1;
        const long long t = col / g.c1;
        const long long b = t % g.c2;
        const long long v = t / g.c2;
        const T* __restrict__ p = in + g.in_off + (o + 3) * g.sJ + a * g.sA + b * g.sB + v * g.sV;
        const long long oi = o + g.ns * col;
        if constexpr (ORDER == 3) {
            double L, R;
            weno3_face(ld(p - g.sJ), ld(p), ld(p + g.sJ), cf, wp.scheme, wp.eps, L, R);
            T Lt = (T)L, Rt = (T)R;
            if (MPF && o >= 3 && o <= g.ns - 4)
                MP<T>::apply(__ldg(p - 2 * g.sJ), __ldg(p - g.sJ), __ldg(p), __ldg(p + g.sJ),
                             __ldg(p + 2 * g.sJ), Lt, Rt);
            vL[oi] = Lt;
            vR[oi] = Rt;
        } else if constexpr (ORDER == 5 || ORDER == 0) {
            const T m2 = __ldg(p - 2 * g.sJ), m1 = __ldg(p - g.sJ), z0 = __ldg(p), p1 = __ldg(p + g.sJ),
                    p2 = __ldg(p + 2 * g.sJ);
            T Lt, Rt;
            if constexpr (ORDER == 5) {
                double L, R;
                weno5_face<PT>((double)m2, (double)m1, (double)z0, (double)p1, (double)p2, cf,
                               wp.scheme, wp.eps, wp.teno_ct, L, R);
                Lt = (T)L;
                Rt = (T)R;
            } else {
                Lt = vL[oi];
                Rt = vR[oi];
            }
            if (MPF || ORDER == 0) MP<T>::apply(m2, m1, z0, p1, p2, Lt, Rt);
            vL[oi] = Lt;
            vR[oi] = Rt;
        } else {
            double s[7];
#pragma unroll
            for (int k = 0; k < 7; ++k) s[k] = ld(p + (k - 3) * g.sJ);
            double L, R;
            weno7_face<PT>(s + 3, cf, wp.scheme, wp.eps, wp.teno_ct, L, R);
            T Lt = (T)L, Rt = (T)R;
            if (MPF)
                MP<T>::apply(__ldg(p - 2 * g.sJ), __ldg(p - g.sJ), __ldg(p), __ldg(p + g.sJ),
                             __ldg(p + 2 * g.sJ), Lt, Rt);
            vL[oi] = Lt;
            vR[oi] = Rt;
        }
    }
}

}  // namespace wsb
