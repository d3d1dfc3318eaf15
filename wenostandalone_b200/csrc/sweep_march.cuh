// sweep_march.cuh -- WENO5-JS (+MP) sweep that marches along the sweep axis.
//
// The face-parallel kernels (sweep_pipe.cuh, sweep_tma.cuh) give every
// thread one face and recompute, for each face, everything its stencil
// shares with the neighbouring faces: 4 differences, the products in the 3
// smoothness indicators, 3 second differences and 2 minmods of the MP
// limiter (and, for FP32-bulk storage, 5 widenings to FP64).  Consecutive
// faces overlap in 4 of their 5 stencil cells, so here a thread owns one
// column of the sweep and walks along it: per face it loads one new cell,
// forms one new difference (FP64, plus its FP32 twin for FP32-bulk), one
// new square and one new cross product, one new second difference and one
// new minmod, and slides the rest along in registers.
//
// Work item: 32 adjacent columns (one warp; lanes take consecutive values
// of the cross axis with unit stride when the sweep is strided, so the
// folded y/z sweeps load 32 consecutive x per instruction) by a segment of
// faces.  Face states go to a per-warp shared-memory tile [F faces][33] and
// leave as F-face row segments, one coalesced store per column pair, so
// the face-fastest vL/vR layout is written contiguously.  Only warp-level
// synchronisation is used; nothing waits on another warp.
//
// Coefficients are face-independent (uniform grids, weno_sb_weno_uniform_dev)
// and come from the kernel-parameter bank.  Arithmetic per face follows
// weno_math.cuh: FP64 differences, beta and the one-reciprocal JS weights
// (faithful fallback outside its range); FP64 or FP32 (FP32-bulk)
// candidate polynomials; the MP limiter in the storage precision.
#pragma once

#include <cuda_runtime.h>

#include "weno_math.cuh"
#include "sweep_generic.cuh"

namespace wsb {

struct MarchArgs {
    const void* in;
    void* vL;
    void* vR;
    WenoParams wp;
    long long ns, nc;
    // input element (J, u, w, v) at in + in_off + J*sJ + u*sU + w*sW + v*sV
    long long sJ, sU, sW, sV, in_off;
    // output element (o, u, w, v) at o + u*oU + w*oW + v*oV
    long long oU, oW, oV;
    int Nu, Nw, NV;
    int n_ut;        // 32-column tiles along u
    int seg;         // faces per segment (multiple of the flush size)
    int n_seg;       // segments per column
    long long n_items;
    double ucf[56];  // Coef<5> layout
    float ucf32[12]; // float copies of polyL[0..5], polyR[0..5]
};

// Second-order minmod of the MP limiter (same decisions as mp_minmod /
// mp_minmod_f), for the storage type.
__device__ __forceinline__ double mm_t(double a, double b) { return mp_minmod(a, b); }
__device__ __forceinline__ float mm_t(float a, float b) { return mp_minmod_f(a, b); }

// MP limiter (f90:1564-1608) from precomputed pieces, FP64: v0, its
// neighbours, the first differences dL1 = v0 - vm1, dR1 = vp1 - v0 and the
// two minmods.  Same expressions as mp_limit.
__device__ __forceinline__ void mp_core(double vm1, double v0, double vp1, double dL1, double dR1, double mA,
                                        double mB, double& L, double& R) {
    const double kBetaMP = 4.0 / 3.0;
    const bool up_r = sign_clear(dR1), up_l = sign_clear(dL1);
    {
        const double UL = fma(-2.0, dR1, v0);
        const double MD = ((v0 + vm1) - mA) * 0.5;
        const double LC = fma(kBetaMP, mB, fma(-0.5, dR1, v0));
        const double mn1 = up_l ? vm1 : v0, mx1 = up_l ? v0 : vm1;
        const double mn2 = up_r ? UL : v0, mx2 = up_r ? v0 : UL;
        const double lo = smax(smin(mn1, MD), smin(mn2, LC));
        const double hi = smin(smax(mx1, MD), smax(mx2, LC));
        L = sclamp(L, lo, hi);
    }
    {
        const double UL = fma(2.0, dL1, v0);
        const double MD = ((v0 + vp1) - mB) * 0.5;
        const double LC = fma(kBetaMP, mA, fma(0.5, dL1, v0));
        const double mn1 = up_r ? v0 : vp1, mx1 = up_r ? vp1 : v0;
        const double mn2 = up_l ? v0 : UL, mx2 = up_l ? UL : v0;
        const double lo = smax(smin(mn1, MD), smin(mn2, LC));
        const double hi = smin(smax(mx1, MD), smax(mx2, LC));
        R = sclamp(R, lo, hi);
    }
}

// FP32 form (offsets from v0, as mp_limit_f): b = v0 - vm1, c = vp1 - v0.
__device__ __forceinline__ void mp_core(float vm1, float v0, float vp1, float b, float c, float mA, float mB,
                                        float& L, float& R) {
    (void)vm1;
    (void)vp1;
    const float kBetaMP = 4.0f / 3.0f;
    {
        const float oMD = -0.5f * (b + mA);
        const float oLC = fmaf(kBetaMP, mB, -0.5f * c);
        const float ul = -2.0f * c;
        const float lo = fmaxf(fminf(fminf(0.0f, -b), oMD), fminf(fminf(0.0f, ul), oLC));
        const float hi = fminf(fmaxf(fmaxf(0.0f, -b), oMD), fmaxf(fmaxf(0.0f, ul), oLC));
        L = v0 + sclamp(L - v0, lo, hi);
    }
    {
        const float oMD = 0.5f * (c - mB);
        const float oLC = fmaf(kBetaMP, mA, 0.5f * b);
        const float ul = 2.0f * b;
        const float lo = fmaxf(fminf(fminf(0.0f, c), oMD), fminf(fminf(0.0f, ul), oLC));
        const float hi = fminf(fmaxf(fmaxf(0.0f, c), oMD), fmaxf(fmaxf(0.0f, ul), oLC));
        R = v0 + sclamp(R - v0, lo, hi);
    }
}

// Widening of one stored value to FP64 (exact).
__device__ __forceinline__ double widen(double x) { return x; }
__device__ __forceinline__ double widen(float x) { return (double)x; }

// Sliding window of one column at face centre J (cells J-2 .. J+2).
template <typename T>
struct MarchWin {
    T vm2, vm1, v0, vp1, vp2;       // stored values
    double Dp2;                     // FP64 value of vp2
    double dm2, dm1, d0, dp1;       // FP64 differences v[k+1]-v[k], k = J-2 .. J+1
    double sm2, sm1, s0, sp1;       // their squares
    double cm, c0, cp;              // dm2*dm1, dm1*d0, d0*dp1
    T fm2, fm1, f0, fp1;            // the same differences in the storage type
    T e2m, e20, e2p;                // second differences at J-1, J, J+1
    T mA;                           // minmod(e2m, e20)
    T mB;                           // minmod(e20, e2p)

    // Fill the window for centre J from the five cells.
    __device__ __forceinline__ void init(T a, T b, T c, T d, T e) {
        vm2 = a; vm1 = b; v0 = c; vp1 = d; vp2 = e;
        const double A = widen(a), B = widen(b), C = widen(c), D = widen(d);
        Dp2 = widen(e);
        dm2 = B - A; dm1 = C - B; d0 = D - C; dp1 = Dp2 - D;
        sm2 = dm2 * dm2; sm1 = dm1 * dm1; s0 = d0 * d0; sp1 = dp1 * dp1;
        cm = dm2 * dm1; c0 = dm1 * d0; cp = d0 * dp1;
        if constexpr (sizeof(T) == 8) {
            fm2 = dm2; fm1 = dm1; f0 = d0; fp1 = dp1;
        } else {
            fm2 = b - a; fm1 = c - b; f0 = d - c; fp1 = e - d;
        }
        e2m = fm1 - fm2; e20 = f0 - fm1; e2p = fp1 - f0;
        mA = mm_t(e2m, e20);
        mB = mm_t(e20, e2p);
    }
    // Advance the centre by one cell; `n` is cell J+3.
    __device__ __forceinline__ void push(T n) {
        const double Dn = widen(n);
        vm2 = vm1; vm1 = v0; v0 = vp1; vp1 = vp2; vp2 = n;
        dm2 = dm1; dm1 = d0; d0 = dp1; dp1 = Dn - Dp2; Dp2 = Dn;
        sm2 = sm1; sm1 = s0; s0 = sp1; sp1 = dp1 * dp1;
        cm = c0; c0 = cp; cp = d0 * dp1;
        fm2 = fm1; fm1 = f0; f0 = fp1;
        if constexpr (sizeof(T) == 8) fp1 = dp1;
        else fp1 = vp2 - vp1;
        e2m = e20; e20 = e2p; e2p = fp1 - f0;
        mA = mB;
        mB = mm_t(e20, e2p);
    }
};

// Reconstruct the face at the window's centre: WENO5-JS, then MP.
template <bool MPF, typename T>
__device__ __forceinline__ void march_face(const MarchWin<T>& w, const Coef<5>& c, const float* pf, double eps,
                                           T& Lo, T& Ro) {
    const double beta0 = fma(c.b[0], w.sp1, fma(c.b[1], w.cp, fma(c.b[2], w.s0, eps)));
    const double beta1 = fma(c.b[3], w.s0, fma(c.b[4], w.c0, fma(c.b[5], w.sm1, eps)));
    const double beta2 = fma(c.b[6], w.sm1, fma(c.b[7], w.cm, fma(c.b[8], w.sm2, eps)));
    const double q0 = beta0 * beta0, q1 = beta1 * beta1, q2 = beta2 * beta2;
    const double P0 = q1 * q2, P1 = q0 * q2, P2 = q0 * q1;
    const double aL0 = c.dL[0] * P0, aL1 = c.dL[1] * P1, aL2 = c.dL[2] * P2;
    const double aR0 = c.dR[0] * P0, aR1 = c.dR[1] * P1, aR2 = c.dR[2] * P2;
    const double SL = aL0 + aL1 + aL2, SR = aR0 + aR1 + aR2;
    if (mid_range(SL) && mid_range(SR)) {
        const double r = nr_rcp(SL * SR), gL = SR * r, gR = SL * r;
        if constexpr (sizeof(T) == 8) {
            const double v0 = w.v0;
            const double pL0 = fma(c.pL[1], w.d0, fma(c.pL[0], w.dp1, v0));
            const double pL1 = fma(c.pL[3], w.dm1, fma(c.pL[2], w.d0, v0));
            const double pL2 = fma(c.pL[5], w.dm2, fma(c.pL[4], w.dm1, v0));
            const double pR0 = fma(c.pR[1], w.d0, fma(c.pR[0], w.dp1, v0));
            const double pR1 = fma(c.pR[3], w.dm1, fma(c.pR[2], w.d0, v0));
            const double pR2 = fma(c.pR[5], w.dm2, fma(c.pR[4], w.dm1, v0));
            Lo = (aL0 * pL0 + aL1 * pL1 + aL2 * pL2) * gL;
            Ro = (aR0 * pR0 + aR1 * pR1 + aR2 * pR2) * gR;
        } else {
            // v0 + e1 + w0 (e0 - e1) + w2 (e2 - e1), e_k = p_k - v0 in FP32
            const float wL0 = unit_d2f(aL0 * gL), wL2 = unit_d2f(aL2 * gL);
            const float wR0 = unit_d2f(aR0 * gR), wR2 = unit_d2f(aR2 * gR);
            const float eL0 = fmaf(pf[0], w.fp1, pf[1] * w.f0), eL1 = fmaf(pf[2], w.f0, pf[3] * w.fm1),
                        eL2 = fmaf(pf[4], w.fm1, pf[5] * w.fm2);
            const float eR0 = fmaf(pf[6], w.fp1, pf[7] * w.f0), eR1 = fmaf(pf[8], w.f0, pf[9] * w.fm1),
                        eR2 = fmaf(pf[10], w.fm1, pf[11] * w.fm2);
            Lo = w.v0 + fmaf(wL0, eL0 - eL1, fmaf(wL2, eL2 - eL1, eL1));
            Ro = w.v0 + fmaf(wR0, eR0 - eR1, fmaf(wR2, eR2 - eR1, eR1));
        }
    } else {
        double L, R;
        weno5_face<T>(widen(w.vm2), widen(w.vm1), widen(w.v0), widen(w.vp1), widen(w.vp2), c, JS, eps, 0.0, L, R);
        Lo = (T)L;
        Ro = (T)R;
    }
    if constexpr (MPF) {
        if constexpr (sizeof(T) == 8) mp_core(w.vm1, w.v0, w.vp1, w.dm1, w.d0, w.mA, w.mB, Lo, Ro);
        else mp_core(w.vm1, w.v0, w.vp1, w.fm1, w.f0, w.mA, w.mB, Lo, Ro);
    }
}

// Faces per shared-memory flush (F) and cells per load chunk (CH).
template <typename T>
struct MarchFlush {
    static constexpr int F = (sizeof(T) == 8) ? 16 : 32;
    static constexpr int CH = 4;
};

template <bool MPF, typename T>
__global__ void __launch_bounds__(128) sweep_march_kernel(const MarchArgs a) {
    constexpr int F = MarchFlush<T>::F;
    __shared__ T tile[4][2][F][33];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const Coef<5>& cf = *reinterpret_cast<const Coef<5>*>(a.ucf);
    const T* __restrict__ in = (const T*)a.in;
    T* __restrict__ outL = (T*)a.vL;
    T* __restrict__ outR = (T*)a.vR;
    T(*tl)[F][33] = tile[warp];
    const long long nwarps = (long long)gridDim.x * (blockDim.x >> 5);
    for (long long item = (long long)blockIdx.x * (blockDim.x >> 5) + warp; item < a.n_items; item += nwarps) {
        // item -> (segment, u tile, w, v)
        const int sg = (int)(item % a.n_seg);
        long long t = item / a.n_seg;
        const int ut = (int)(t % a.n_ut);
        t /= a.n_ut;
        const int wv = (int)(t % a.Nw);
        const int vv = (int)(t / a.Nw);
        const int u = ut * 32 + lane;
        const bool col_ok = u < a.Nu;
        const int uc = col_ok ? u : a.Nu - 1;  // idle lanes shadow a valid column
        const T* __restrict__ col = in + a.in_off + uc * a.sU + wv * a.sW + vv * a.sV;
        const long long o_begin = 3 + (long long)sg * a.seg;   // first face of the segment
        long long o_end = o_begin + a.seg;
        if (o_end > a.ns - 3) o_end = a.ns - 3;
        // face o has centre cell J = o + 3: cells o+1 .. o+5
        MarchWin<T> w;
        {
            const T* p = col + (o_begin + 1) * a.sJ;
            w.init(__ldg(p), __ldg(p + a.sJ), __ldg(p + 2 * a.sJ), __ldg(p + 3 * a.sJ), __ldg(p + 4 * a.sJ));
        }
        const long long obase_u = (long long)ut * 32;
        const long long obase = wv * a.oW + vv * a.oV;
        // cells are loaded CH at a time, one chunk ahead of their use (cell
        // J+3 of face o is o+6)
        constexpr int CH = MarchFlush<T>::CH;
        T cur[CH], nxt[CH];
        long long J_next = o_begin + 6;
        auto load_chunk = [&](T* dst) {
#pragma unroll
            for (int i = 0; i < CH; ++i) {
                const long long J = J_next + i;
                dst[i] = (J < a.ns + 6) ? __ldg(col + J * a.sJ) : T(0);
            }
            J_next += CH;
        };
        load_chunk(cur);
        for (long long f0 = o_begin; f0 < o_end; f0 += F) {
            const int nF = (int)min((long long)F, o_end - f0);
            for (int c0 = 0; c0 < nF; c0 += CH) {
                load_chunk(nxt);
#pragma unroll
                for (int i = 0; i < CH; ++i) {
                    if (c0 + i < nF) {
                        T L, R;
                        march_face<MPF, T>(w, cf, a.ucf32, a.wp.eps, L, R);
                        tl[0][c0 + i][lane] = L;
                        tl[1][c0 + i][lane] = R;
                        w.push(cur[i]);
                    }
                }
#pragma unroll
                for (int i = 0; i < CH; ++i) cur[i] = nxt[i];
            }
            __syncwarp();
            // write out: lanes take faces, the warp walks the columns
            constexpr int CPI = 32 / F;  // columns per store instruction
            const int fi = lane % F, cj = lane / F;
            for (int c = cj; c < 32; c += CPI) {
                const long long uu = obase_u + c;
                if (uu < a.Nu && fi < nF) {
                    const long long oi = obase + uu * a.oU + f0 + fi;
                    outL[oi] = tl[0][fi][c];
                    outR[oi] = tl[1][fi][c];
                }
            }
            __syncwarp();
        }
    }
}

// Launch for face-independent WENO5-JS coefficients.  Returns 1003 when
// the sweep has too few faces for the window.
template <typename T>
int launch_march_sweep(const SweepGeom& g, bool mp, const T* in, T* vL, T* vR, const WenoParams& wp,
                       const double* ucf, cudaStream_t st, int sms) {
    if (g.nc < 1 || !ucf) return 1003;
    MarchArgs a{};
    a.in = in; a.vL = vL; a.vR = vR; a.wp = wp;
    a.ns = g.ns; a.nc = g.nc;
    a.sJ = g.sJ; a.sV = g.sV; a.in_off = g.in_off;
    // lanes along the cross axis with unit stride when there is one
    if (g.sB == 1 && g.sA != 1) {
        a.sU = g.sB; a.sW = g.sA; a.Nu = (int)g.c2; a.Nw = (int)g.c1;
        a.oU = g.ns * g.c1; a.oW = g.ns;
    } else {
        a.sU = g.sA; a.sW = g.sB; a.Nu = (int)g.c1; a.Nw = (int)g.c2;
        a.oU = g.ns; a.oW = g.ns * g.c1;
    }
    a.oV = g.ns * g.c1 * g.c2;
    a.NV = (int)g.nv;
    a.n_ut = (a.Nu + 31) / 32;
    for (int q = 0; q < 56; ++q) a.ucf[q] = ucf[q];
    for (int q = 0; q < 6; ++q) {
        a.ucf32[q] = (float)ucf[q];          // polyL (Coef<5>::pL)
        a.ucf32[6 + q] = (float)ucf[6 + q];  // polyR
    }
    // segments: enough warps to fill the GPU about four times over
    constexpr int F = MarchFlush<T>::F;
    const long long cols = (long long)a.n_ut * a.Nw * a.NV;
    const long long want = (long long)sms * 16 * 4;
    long long nseg = (want + cols - 1) / cols;
    const long long max_seg = (g.nc + F - 1) / F;
    if (nseg > max_seg) nseg = max_seg;
    if (nseg < 1) nseg = 1;
    long long seg = (g.nc + nseg - 1) / nseg;
    seg = ((seg + F - 1) / F) * F;
    a.seg = (int)seg;
    a.n_seg = (int)((g.nc + seg - 1) / seg);
    a.n_items = cols * a.n_seg;
    const long long warps_per_block = 4;
    long long blocks = (a.n_items + warps_per_block - 1) / warps_per_block;
    const long long cap = (long long)sms * 64;
    if (blocks > cap) blocks = cap;
    if (blocks < 1) blocks = 1;
    if (mp) sweep_march_kernel<true, T><<<(unsigned)blocks, 128, 0, st>>>(a);
    else sweep_march_kernel<false, T><<<(unsigned)blocks, 128, 0, st>>>(a);
    return 0;
}

}  // namespace wsb
