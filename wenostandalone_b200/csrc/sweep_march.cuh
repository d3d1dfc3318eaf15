// sweep_march.cuh -- marching WENO engines: WENO3 / WENO5 / WENO7 (+MP)
// along the sweep axis, and the WENO5 marching kernel with per-lane loads.
//
// The face-parallel kernels (sweep_pipe.cuh, sweep_tma.cuh) give every
// thread one face and recompute, for each face, everything its stencil
// shares with the neighbouring faces: 4 differences, the products in the 3
// smoothness indicators, 3 second differences and 2 minmods of the MP
// limiter (and, for FP32-bulk storage, 5 widenings to FP64).  Consecutive
// faces overlap in all but one of their stencil cells, so here a thread owns
// one column of the sweep and walks along it: per face it loads one new
// cell, forms one new difference (FP64, plus its FP32 twin for FP32-bulk),
// the new products of the smoothness indicators it enters, one new second
// difference and one new minmod, and slides the rest along in registers.
//
// Engines (init / push / face, and face_teno for TENO weights):
//   March64, March32       WENO5, FP64 / FP32-bulk
//   March64_7, March32_7   WENO7
//   March64_3, March32_3   WENO3 (every face written; MP on core faces)
// The TMA kernel that drives them is sweep_march_tma.cuh; batched.cuh runs
// them one column per thread.  Coefficients are face-independent and come
// from the kernel-parameter bank (MarchArgs), except for the FP64 WENO5
// kernel with a per-face table (march_face_table_kernel, FaceRow, BetaRow).
// Arithmetic per face follows weno_math.cuh: FP64 differences, beta and the
// one-reciprocal weights (the reference sequence redoes a face whose sums
// leave the reciprocal form's range); FP64 or FP32 (FP32-bulk) candidate
// polynomials; the MP limiter in the storage precision, one-sided on the
// sign of the state's offset from v0.
#pragma once

#include <cuda_runtime.h>

#include <type_traits>

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
    // FP64 kernel: candidate-polynomial coefficients scaled by the ideal
    // weights, kL[2r+s] = dL[r] * polyL[s][r] (and kR likewise)
    double kL[6], kR[6];
    // FP32-bulk engine: (polyL, polyR) float pairs, Coef<5>::pL index order
    float2 pf2[6];
    // WENO7 engine (ucf in the Coef<7> layout): kL7[3s+t] = dL[s] polyL[3(3-s)+t]
    // for stencil s, term t (and kR7 likewise)
    double kL7[12], kR7[12];
    // FP32-bulk WENO7 engine: float polyL[0..11], polyR[0..11] (Coef<7> order)
    float pf7[24];
    // mapped WENO5 engine: per stencil k, (d + d^2, 3 d, 1 - 2 d, d^2) of the
    // left / right ideal weights at 4k .. 4k + 3
    double mcL[12], mcR[12];
    // face-dependent coefficients (FP64 kernels): the per-face table built by
    // march_face_table_kernel, and the arrays it was built from (for faces
    // that are redone); ftab is null for face-independent coefficients
    const double* ftab;
    CoefPtrs cp;
};

// Row of the per-face table (doubles per face; 224 bytes, a multiple of 16).
constexpr int kFaceRow = 28;

// Coefficient sources of the FP64 marching engine.  ParamCoefs reads the
// face-independent coefficients from the kernel-parameter bank; FaceRow and
// BetaRow hold one face's row of the per-face table (FaceRow: the candidate
// coefficients and ideal weights of face f; BetaRow: the beta coefficients
// that the difference pair (d[f], d[f+1]) enters, b(f + r, r, s) at 3r + s).
struct ParamCoefs {
    const MarchArgs& a;
    __device__ __forceinline__ double kL(int q) const { return a.kL[q]; }
    __device__ __forceinline__ double kR(int q) const { return a.kR[q]; }
    __device__ __forceinline__ double dL(int r) const { return a.ucf[12 + r]; }
    __device__ __forceinline__ double dR(int r) const { return a.ucf[15 + r]; }
    __device__ __forceinline__ double b(int q) const { return a.ucf[18 + q]; }
};

// (rows are read from the per-face table in global memory or from a copy
// staged in shared memory)
struct FaceRow {
    double2 k[9];  // kL[0..5], kR[0..5], dL[0..2], dR[0..2]
    __device__ __forceinline__ explicit FaceRow(const double* row) {
        const double2* p = reinterpret_cast<const double2*>(row);
#pragma unroll
        for (int q = 0; q < 9; ++q) k[q] = p[q];
    }
    __device__ __forceinline__ double g(int q) const { return (q & 1) ? k[q >> 1].y : k[q >> 1].x; }
    __device__ __forceinline__ double kL(int q) const { return g(q); }
    __device__ __forceinline__ double kR(int q) const { return g(6 + q); }
    __device__ __forceinline__ double dL(int r) const { return g(12 + r); }
    __device__ __forceinline__ double dR(int r) const { return g(15 + r); }
};

struct BetaRow {
    double2 k[5];  // b[0..8] (row entries 18 .. 26) and the pad at 27
    __device__ __forceinline__ explicit BetaRow(const double* row) {
        const double2* p = reinterpret_cast<const double2*>(row) + 9;
#pragma unroll
        for (int q = 0; q < 5; ++q) k[q] = p[q];
    }
    __device__ __forceinline__ double b(int q) const { return (q & 1) ? k[q >> 1].y : k[q >> 1].x; }
};

// Builds the per-face table: row f (f = 0 .. rows-1, face f of the sweep)
// from core face c(f) = clamp(f - 3, 0, nc - 1) of the coefficient arrays
// (f90:541-550, 552-555, 623-625 read polyL/R(j, r, s), d(r, j) and
// beta_coef(j, r, s) at the core index of the face):
//   [0..5]    kL[2r+s] = dL(r) polyL(c, r, s) (the ideal weight folded in)
//   [6..11]   kR[2r+s] = dR(r) polyR(c, r, s)
//   [12..14]  dL(r), [15..17] dR(r)
//   [18+3r+s] beta_coef(c(f + r), r, s); [27] zero
// A face with a negative ideal weight gets a NaN in dL(0): its normalisation
// test fails and the kernels redo it from the arrays, as the one-sided MP
// median needs sign(v_L - v_0) = sign(E_L), which non-negative weights give.
__global__ void march_face_table_kernel(CoefPtrs cp, long long nc, int rows, double* __restrict__ tab) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= rows) return;
    auto core = [&](long long x) { x -= 3; return x < 0 ? 0 : (x > nc - 1 ? nc - 1 : x); };
    const long long c = core(f);
    double* row = tab + (long long)f * kFaceRow;
    bool neg = false;
    for (int r = 0; r < 3; ++r) {
        const double dl = cp.dL[r + 5 * c], dr = cp.dR[r + 5 * c];
        neg |= !(dl >= 0.0) || !(dr >= 0.0);
        for (int s = 0; s < 2; ++s) {
            row[2 * r + s] = dl * cp.polyL[c + nc * (r + 5 * s)];
            row[6 + 2 * r + s] = dr * cp.polyR[c + nc * (r + 5 * s)];
        }
        row[12 + r] = dl;
        row[15 + r] = dr;
        const long long cr = core(f + r);
        for (int s = 0; s < 3; ++s) row[18 + 3 * r + s] = cp.beta[cr + nc * (r + 5 * s)];
    }
    if (neg) row[12] = __longlong_as_double(0x7ff8000000000000LL);
    row[27] = 0.0;
}

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

// ---------------------------------------------------------------------
// FP64 marching sweep with a branch-free face body.
//
// Per face the FP64 issue slots are the bound (a B200 SM retires 64 FP64
// lanes per clock against 128 for FP32 and integer work), so the body is
// arranged to spend as few as the arithmetic allows while keeping FP64
// throughout:
//  * each new difference pair (d[k], d[k+1]) enters beta_0 of face k,
//    beta_1 of face k+1 and beta_2 of face k+2 (three FMA chains of the
//    reference's form, so the beta are the ones the per-face kernels
//    compute) and the pending beta_1 / beta_2 ride along with the window;
//  * the ideal weights are folded into the candidate polynomials on the
//    host, kL[2r+s] = dL[r] polyL[s][r], so with P_k = prod_{m!=k} beta_m^2
//    the state is v0 + E_L / S_L, E_L = sum_k P_k (kL . differences),
//    S_L = sum_k dL[k] P_k: the weights' rounding multiplies only the
//    offset from v0, and one Newton step on the hardware reciprocal seed
//    of S_L S_R leaves a relative error near 2^-46 in that offset;
//  * the MP limiter takes the curvature minmod of the newest pair only
//    (the other one slides along), the half-sums (v[j-1]+v[j])/2 slide
//    too, and since lo <= v0 <= hi, median(L, lo, hi) is min(L, hi) when
//    L >= v0 and max(L, lo) otherwise: one bound per state, with min or
//    max picked by the sign of the offset.  Values and roundings are those
//    of mp_core.
// A face whose normalisation sums leave the range of the one-reciprocal
// form is flagged and redone after its chunk with the reference sequence
// (weno5_face, then mp_limit), so the common path has no branch.
// ---------------------------------------------------------------------
// min (up = false) or max (up = true) of two doubles: one comparison and a
// select, no NaN special-casing (the CUDA fmin/fmax handle NaN operands and
// cost several more instructions each).
__device__ __forceinline__ double mm_sel(double a, double b, bool up) { return ((a < b) != up) ? a : b; }

// minmod of the MP limiter: the value of mp_minmod (up to the sign of a
// zero result), with the "signs differ or 4m - M < 0" test on sign bits.
__device__ __forceinline__ double mm64(double dl, double dr) {
    const double a = fabs(dl), b = fabs(dr);
    const bool al = a < b;
    const double m = al ? a : b, M = al ? b : a;
    const double t = fma(4.0, m, -M);
    const double u = (t < m) ? t : m;
    const int hl = __double2hiint(dl), hu = __double2hiint(u);
    const int kill = ((hl ^ __double2hiint(dr)) | hu) >> 31;
    const int hi = (hu & ~kill) | (hl & (int)0x80000000);
    const int lo = __double2loint(u) & ~kill;
    return __hiloint2double(hi, lo);
}

// Reciprocal of a positive normal double: hardware seed and one Newton step.
__device__ __forceinline__ double rcp1(double s) {
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(s));
    return fma(r, fma(-s, r, 1.0), r);
}

// One-sided MP median of an FP64 engine's face (see March64::face), with the
// side of each state given by the sign of its offset from v0.
__device__ __forceinline__ void mp64_sided(double vm1, double v0, double vp1, double dm1, double d0, double mA,
                                           double mB, bool posL, bool posR, double& L, double& R) {
    const double kBetaMP = 4.0 / 3.0;
    const bool up_l = sign_clear(dm1), up_r = sign_clear(d0);
    {
        const bool pos = posL;
        const double UL = fma(-2.0, d0, v0);
        const double MD = fma(-0.5, dm1 + mA, v0);
        const double LC = fma(kBetaMP, mB, fma(-0.5, d0, v0));
        const double Q1 = (pos == up_l) ? v0 : vm1;
        const double Q2 = (pos == up_r) ? v0 : UL;
        const double A = mm_sel(Q1, MD, pos), B = mm_sel(Q2, LC, pos);
        L = mm_sel(mm_sel(L, A, !pos), B, !pos);
    }
    {
        const bool pos = posR;
        const double UL = fma(2.0, dm1, v0);
        const double MD = fma(0.5, d0 - mB, v0);
        const double LC = fma(kBetaMP, mA, fma(0.5, dm1, v0));
        const double Q1 = (pos == up_r) ? vp1 : v0;
        const double Q2 = (pos == up_l) ? UL : v0;
        const double A = mm_sel(Q1, MD, pos), B = mm_sel(Q2, LC, pos);
        R = mm_sel(mm_sel(R, A, !pos), B, !pos);
    }
}

// The same in FP32 offset space (see March32::face): x = state - v0, with
// b = v0 - vm1 = fm1 and c = vp1 - v0 = f0.
__device__ __forceinline__ void mp32_sided(float fm1, float f0, float mA, float mB, float& xL, float& xR) {
    const float kB = 4.0f / 3.0f;
    {
        const bool pos = xL >= 0.0f;
        const float md = -0.5f * (fm1 + mA), ul = -2.0f * f0, lc = fmaf(kB, mB, -0.5f * f0), nb = -fm1;
        const float A = pos ? fmaxf(fmaxf(0.0f, nb), md) : fminf(fminf(0.0f, nb), md);
        const float B = pos ? fmaxf(fmaxf(0.0f, ul), lc) : fminf(fminf(0.0f, ul), lc);
        xL = pos ? fminf(fminf(xL, A), B) : fmaxf(fmaxf(xL, A), B);
    }
    {
        const bool pos = xR >= 0.0f;
        const float md = -0.5f * (mB - f0), ul = 2.0f * fm1, lc = fmaf(kB, mA, 0.5f * fm1), nb = f0;
        const float A = pos ? fmaxf(fmaxf(0.0f, nb), md) : fminf(fminf(0.0f, nb), md);
        const float B = pos ? fmaxf(fmaxf(0.0f, ul), lc) : fminf(fminf(0.0f, ul), lc);
        xR = pos ? fminf(fminf(xR, A), B) : fmaxf(fmaxf(xR, A), B);
    }
}

// TENO weights of WENO5 (f90:578-606) for betas b0..b2: the cutoff flags
// (alpha_k / sum alpha >= CT, alpha_k = (1 + tau / beta_k)^6,
// tau = |beta_2 - beta_0|); false when the alpha sum leaves [1, 2^996)
// (a zero beta, or ratios past 10^50).
__device__ __forceinline__ bool teno5_keep(double b0, double b1, double b2, double ct, bool& k0, bool& k1, bool& k2) {
    const double tau = fabs(b2 - b0);
    const double t0 = fma(tau, rcp1(b0), 1.0), t1 = fma(tau, rcp1(b1), 1.0), t2 = fma(tau, rcp1(b2), 1.0);
    const double x0 = t0 * t0, x1 = t1 * t1, x2 = t2 * t2;
    const double al0 = x0 * x0 * x0, al1 = x1 * x1 * x1, al2 = x2 * x2 * x2;
    const double s = (al0 + al1) + al2;
    const double rs = rcp1(s);
    k0 = !(al0 * rs < ct); k1 = !(al1 * rs < ct); k2 = !(al2 * rs < ct);
    return mid_range_prod(s);
}

// TENO weights of WENO7 as the reference writes them (f90:1491-1506):
// beta(4) = eps, tau = |beta(4) - beta(3)|, alpha_q = (1 + tau / beta_q)^6 for
// q = 0..4, cutoff flags for q = 0..3, and alpha(4) kept in the final sums
// (returned in a4).  False when the sums leave the reciprocal form's range.
__device__ __forceinline__ bool teno7_keep(double b0, double b1, double b2, double b3, double eps, double ct, bool& k0,
                                           bool& k1, bool& k2, bool& k3, double& a4) {
    const double tau = fabs(eps - b3);
    const double t0 = fma(tau, rcp1(b0), 1.0), t1 = fma(tau, rcp1(b1), 1.0), t2 = fma(tau, rcp1(b2), 1.0),
                 t3 = fma(tau, rcp1(b3), 1.0), t4 = fma(tau, rcp1(eps), 1.0);
    const double x0 = t0 * t0, x1 = t1 * t1, x2 = t2 * t2, x3 = t3 * t3, x4 = t4 * t4;
    const double al0 = x0 * x0 * x0, al1 = x1 * x1 * x1, al2 = x2 * x2 * x2, al3 = x3 * x3 * x3;
    a4 = x4 * x4 * x4;
    const double s = ((al0 + al1) + (al2 + al3)) + a4;
    const double rs = rcp1(s);
    k0 = !(al0 * rs < ct); k1 = !(al1 * rs < ct); k2 = !(al2 * rs < ct); k3 = !(al3 * rs < ct);
    // a4 >= 1; (S + a4)^2 must stay below 2^996 for the final reciprocal
    return mid_range_prod(s) && mid_range(a4);
}

struct March64 {
    double vm1, v0, vp1, vp2;   // cells J-1 .. J+2
    double dm2, dm1, d0, dp1;   // d[k] = v[k+1] - v[k], k = J-2 .. J+1
    double s1;                  // d[J+1]^2
    double b0, b1, b2;          // beta_0, beta_1, beta_2 of face J
    double b1n, b2n, b2nn;      // beta_1(J+1), beta_2(J+1), beta_2(J+2)
    double e2;                  // curvature d[J+1] - d[J]
    double mA, mB;              // minmod(e2[J-1], e2[J]), minmod(e2[J], e2[J+1])
    // MP bounds shared by the two states of an interface (f90:1573-1599):
    // the left state of face J and the right state of face J-1 sit on the
    // same interface, whose MD bound is one value, and the LC bound of the
    // right state of face J is that of the left state of face J-1 plus
    // 2 (v[J] - v[J-1]); both are carried from face J-1.
    double mdc;                 // MD of face J's left state
    double lcc;                 // LC of face J-1's left state

    // beta of the three stencils that pair (x, y) = (d[k], d[k+1]) enters:
    // stencil 0 of face k, 1 of face k+1, 2 of face k+2 (coefficients of
    // those faces from the source c)
    template <class C>
    __device__ __forceinline__ static void betas(const MarchArgs& a, const C& c, double sx, double cxy, double sy,
                                                 double& g0, double& g1, double& g2) {
        const double eps = a.wp.eps;
        g0 = fma(c.b(0), sy, fma(c.b(1), cxy, fma(c.b(2), sx, eps)));
        g1 = fma(c.b(3), sy, fma(c.b(4), cxy, fma(c.b(5), sx, eps)));
        g2 = fma(c.b(6), sy, fma(c.b(7), cxy, fma(c.b(8), sx, eps)));
    }
    __device__ __forceinline__ static void betas(const MarchArgs& a, double sx, double cxy, double sy, double& g0,
                                                 double& g1, double& g2) {
        betas(a, ParamCoefs{a}, sx, cxy, sy, g0, g1, g2);
    }

    // Window of face J from cells J-2 .. J+2; cm2, cm1, cz are the beta
    // sources of the pairs starting at d[J-2], d[J-1], d[J].
    template <class C2, class C1, class C0>
    __device__ __forceinline__ void init(const MarchArgs& a, const C2& cm2, const C1& cm1, const C0& cz, double c0,
                                         double c1, double c2, double c3, double c4) {
        vm1 = c1; v0 = c2; vp1 = c3; vp2 = c4;
        dm2 = c1 - c0; dm1 = c2 - c1; d0 = c3 - c2; dp1 = c4 - c3;
        const double sm2 = dm2 * dm2, sm1 = dm1 * dm1, s0 = d0 * d0;
        s1 = dp1 * dp1;
        double g0, g1, g2, u;
        betas(a, cm2, sm2, dm2 * dm1, sm1, u, u, b2);      // pair (d[J-2], d[J-1])
        betas(a, cm1, sm1, dm1 * d0, s0, u, b1, b2n);      // pair (d[J-1], d[J])
        betas(a, cz, s0, d0 * dp1, s1, g0, g1, g2);        // pair (d[J], d[J+1])
        b0 = g0; b1n = g1; b2nn = g2;
        const double em = dm1 - dm2, ez = d0 - dm1;
        e2 = dp1 - d0;
        mA = mm64(em, ez);
        mB = mm64(ez, e2);
        // the bounds face J-1 would have carried, by the same expressions, so
        // a face's result does not depend on where its segment starts
        mdc = fma(0.5, dm1 - mA, vm1);
        lcc = fma(4.0 / 3.0, mA, fma(-0.5, dm1, vm1));
    }

    __device__ __forceinline__ void init(const MarchArgs& a, double c0, double c1, double c2, double c3,
                                         double c4) {
        const ParamCoefs u{a};
        init(a, u, u, u, c0, c1, c2, c3, c4);
    }

    // Advance to face J+1; n is cell J+3; c is the beta source of the new
    // pair (d[J+1], d[J+2]).
    template <class C>
    __device__ __forceinline__ void push(const MarchArgs& a, const C& c, double n) {
        const double dn = n - vp2;
        const double sn = dn * dn;
        double g0, g1, g2;
        betas(a, c, s1, dp1 * dn, sn, g0, g1, g2);
        const double ne2 = dn - dp1;
        const double nmB = mm64(e2, ne2);
        vm1 = v0; v0 = vp1; vp1 = vp2; vp2 = n;
        dm2 = dm1; dm1 = d0; d0 = dp1; dp1 = dn;
        s1 = sn;
        b0 = g0; b1 = b1n; b2 = b2n;
        b1n = g1; b2n = b2nn; b2nn = g2;
        e2 = ne2; mA = mB; mB = nmB;
    }
    __device__ __forceinline__ void push(const MarchArgs& a, double n) { push(a, ParamCoefs{a}, n); }

    // WENO5-JS (+ MP) state of face J; false when the one-reciprocal form
    // is out of range (the caller redoes the face).
    template <bool MPF>
    __device__ __forceinline__ bool face(const MarchArgs& a, double& L, double& R) {
        return face<MPF, ParamCoefs>(a, ParamCoefs{a}, L, R);
    }
    template <bool MPF, class C>
    __device__ __forceinline__ bool face(const MarchArgs& a, const C& c, double& L, double& R) {
        const double q0 = b0 * b0, q1 = b1 * b1, q2 = b2 * b2;
        const double P0 = q1 * q2, P1 = q0 * q2, P2 = q0 * q1;
        return fold<MPF>(c, P0, P1, P2, L, R);
    }
    // WENO5-Z (+ MP) state of face J (f90:586-590): tau = |beta_2 - beta_0|,
    // alpha_k = d_k (1 + tau / beta_k).  Times beta_0 beta_1 beta_2 the
    // weights are d_k P_k / sum d P with P_k = (beta_k + tau) prod_{j != k}
    // beta_j: the folded form of JS with these P_k.
    template <bool MPF>
    __device__ __forceinline__ bool face_z(const MarchArgs& a, double& L, double& R) {
        return face_z<MPF, ParamCoefs>(a, ParamCoefs{a}, L, R);
    }
    template <bool MPF, class C>
    __device__ __forceinline__ bool face_z(const MarchArgs& a, const C& c, double& L, double& R) {
        const double tau = fabs(b2 - b0);
        const double P0 = (b0 + tau) * (b1 * b2), P1 = (b1 + tau) * (b0 * b2), P2 = (b2 + tau) * (b0 * b1);
        return fold<MPF>(c, P0, P1, P2, L, R);
    }
    // Mapped WENO5 (+ MP) state of face J (f90:557-568; Henrick, Aslam and
    // Powers, J. Comput. Phys. 207 (2005)): per side, with its own ideal
    // weights d_k, omega_k = d_k P_k / sum d P (the JS weights, P_k =
    // prod_{j != k} beta_j^2), N_k = d_k (1 + d_k - 3 omega_k) + omega_k^2,
    // D_k = d_k^2 + omega_k (1 - 2 d_k), mapped weights omega_k N_k / D_k
    // normalised.  Folded over the denominators, G_k = omega_k N_k prod_{j !=
    // k} D_j and the state is v0 + sum G_k e_k / sum G_k, e_k the candidate
    // offsets with the raw coefficients.  Face-independent coefficients
    // (the per-side constants d + d^2, 3 d, 1 - 2 d, d^2 in MarchArgs::mcL /
    // mcR); the ideal weights must lie in (0, 0.8), where every G_k >= 0, so
    // the offset's sign is that of E (the one-sided MP median needs it).
    // False when a sum leaves the reciprocal forms' range.
    template <bool MPF>
    __device__ __forceinline__ bool face_mapped(const MarchArgs& a, double& L, double& R) {
        const double q0 = b0 * b0, q1 = b1 * b1, q2 = b2 * b2;
        const double P0 = q1 * q2, P1 = q0 * q2, P2 = q0 * q1;
        bool ok = true;
        double EL, GL, ER, GR;
        mapped_side(a.ucf + 12, a.mcL, a.ucf, P0, P1, P2, EL, GL, ok);
        mapped_side(a.ucf + 15, a.mcR, a.ucf + 6, P0, P1, P2, ER, GR, ok);
        const double p = GL * GR;
        ok = ok && mid_range_prod(p);
        const double r = rcp1(p);
        L = fma(EL * GR, r, v0);
        R = fma(ER * GL, r, v0);
        if constexpr (MPF) mp_sided(sign_clear(EL), sign_clear(ER), L, R);
        return ok;
    }
    // One side of face_mapped: ideal weights d[0..2], their constants
    // mc[4k + 0..3] = (d + d^2, 3 d, 1 - 2 d, d^2), raw candidate
    // coefficients pc[2r + s] (Coef<5> order).
    __device__ __forceinline__ void mapped_side(const double* d, const double* mc, const double* pc, double P0,
                                                double P1, double P2, double& E, double& G, bool& ok) const {
        const double S = fma(d[0], P0, fma(d[1], P1, d[2] * P2));
        ok = ok && mid_range(S);
        const double rS = nr_rcp(S);
        const double w0 = (d[0] * P0) * rS, w1 = (d[1] * P1) * rS, w2 = (d[2] * P2) * rS;
        const double N0 = fma(w0, w0 - mc[1], mc[0]), N1 = fma(w1, w1 - mc[5], mc[4]),
                     N2 = fma(w2, w2 - mc[9], mc[8]);
        const double D0 = fma(w0, mc[2], mc[3]), D1 = fma(w1, mc[6], mc[7]), D2 = fma(w2, mc[10], mc[11]);
        const double G0 = (w0 * N0) * (D1 * D2), G1 = (w1 * N1) * (D0 * D2), G2 = (w2 * N2) * (D0 * D1);
        G = (G0 + G1) + G2;
        const double e0 = fma(pc[1], d0, pc[0] * dp1), e1 = fma(pc[3], dm1, pc[2] * d0),
                     e2 = fma(pc[5], dm2, pc[4] * dm1);
        E = fma(G0, e0, fma(G1, e1, G2 * e2));
    }
    // The folded state of face J from the stencils' factors P_k (weights
    // d_k P_k / sum d P; JS and Z weights).
    template <bool MPF, class C>
    __device__ __forceinline__ bool fold(const C& c, double P0, double P1, double P2, double& L, double& R) {
        const double SL = fma(c.dL(0), P0, fma(c.dL(1), P1, c.dL(2) * P2));
        const double SR = fma(c.dR(0), P0, fma(c.dR(1), P1, c.dR(2) * P2));
        const double eL0 = fma(c.kL(1), d0, c.kL(0) * dp1), eL1 = fma(c.kL(3), dm1, c.kL(2) * d0),
                     eL2 = fma(c.kL(5), dm2, c.kL(4) * dm1);
        const double eR0 = fma(c.kR(1), d0, c.kR(0) * dp1), eR1 = fma(c.kR(3), dm1, c.kR(2) * d0),
                     eR2 = fma(c.kR(5), dm2, c.kR(4) * dm1);
        const double EL = fma(P0, eL0, fma(P1, eL1, P2 * eL2));
        const double ER = fma(P0, eR0, fma(P1, eR1, P2 * eR2));
        // one range test on S_L S_R: the two sums share the P_k, so they are
        // within the ratio of the ideal weights of each other
        const double p = SL * SR;
        const bool ok = mid_range_prod(p);
        const double r = rcp1(p);
        L = fma(EL * SR, r, v0);
        R = fma(ER * SL, r, v0);
        if constexpr (MPF) mp_sided(sign_clear(EL), sign_clear(ER), L, R);
        return ok;
    }

    // MP limiter (f90:1564-1608) of face J's states, one-sided: since
    // lo <= v0 <= hi, median(L, lo, hi) is min(L, hi) for L >= v0 (pos) and
    // max(L, lo) otherwise, so only one bound is formed, with min or max
    // picked by that sign.  The left state's MD and the right state's LC
    // come from the carried values; the right state's MD and the left
    // state's LC are carried on to face J+1.
    __device__ __forceinline__ void mp_sided(bool posL, bool posR, double& L, double& R) {
        const double kBetaMP = 4.0 / 3.0;
        const bool up_l = sign_clear(dm1), up_r = sign_clear(d0);
        const double mdR = fma(0.5, d0 - mB, v0);       // ((v0 + vp1) - mB) / 2
        const double lcL = fma(kBetaMP, mB, fma(-0.5, d0, v0));
        {
            const bool pos = posL;
            const double UL = fma(-2.0, d0, v0);
            const double P1 = (pos == up_l) ? v0 : vm1;  // max / min of (v0, vm1)
            const double P2 = (pos == up_r) ? v0 : UL;   // max / min of (v0, UL)
            const double A = mm_sel(P1, mdc, pos), B = mm_sel(P2, lcL, pos);
            L = mm_sel(mm_sel(L, A, !pos), B, !pos);
        }
        {
            const bool pos = posR;
            const double UL = fma(2.0, dm1, v0);
            const double lcR = fma(2.0, dm1, lcc);       // v0 + (v0 - vm1) / 2 + beta_mp mA
            const double P1 = (pos == up_r) ? vp1 : v0;  // max / min of (v0, vp1)
            const double P2 = (pos == up_l) ? UL : v0;   // max / min of (v0, UL)
            const double A = mm_sel(P1, mdR, pos), B = mm_sel(P2, lcR, pos);
            R = mm_sel(mm_sel(R, A, !pos), B, !pos);
        }
        mdc = mdR;
        lcc = lcL;
    }
    // WENO5-TENO (+ MP) state of face J (f90:578-606): tau = |beta_2 - beta_0|,
    // alpha_k = (1 + tau / beta_k)^6, delta_k = [alpha_k / sum alpha >= CT],
    // weights d_k delta_k / sum d delta; the offsets v - v0 in the folded form
    // E = sum delta_k (kL_k . differences), S = sum delta_k d_k.  False when a
    // sum leaves the range of the reciprocal form (the caller redoes the face).
    template <bool MPF>
    __device__ __forceinline__ bool face_teno(const MarchArgs& a, double& L, double& R) {
        return face_teno<MPF, ParamCoefs>(a, ParamCoefs{a}, L, R);
    }
    template <bool MPF, class C>
    __device__ __forceinline__ bool face_teno(const MarchArgs& a, const C& c, double& L, double& R) {
        const double tau = fabs(b2 - b0);
        const double t0 = fma(tau, rcp1(b0), 1.0), t1 = fma(tau, rcp1(b1), 1.0), t2 = fma(tau, rcp1(b2), 1.0);
        const double x0 = t0 * t0, x1 = t1 * t1, x2 = t2 * t2;
        const double al0 = x0 * x0 * x0, al1 = x1 * x1 * x1, al2 = x2 * x2 * x2;
        const double s = (al0 + al1) + al2;
        // s >= 1 (every alpha is); below 2^996 its reciprocal and the
        // products with it stay normal (NaN and inf fail the test too)
        const bool s_ok = mid_range_prod(s);
        const double rs = rcp1(s), ct = a.wp.teno_ct;
        const bool k0 = !(al0 * rs < ct), k1 = !(al1 * rs < ct), k2 = !(al2 * rs < ct);
        const double eL0 = fma(c.kL(1), d0, c.kL(0) * dp1), eL1 = fma(c.kL(3), dm1, c.kL(2) * d0),
                     eL2 = fma(c.kL(5), dm2, c.kL(4) * dm1);
        const double eR0 = fma(c.kR(1), d0, c.kR(0) * dp1), eR1 = fma(c.kR(3), dm1, c.kR(2) * d0),
                     eR2 = fma(c.kR(5), dm2, c.kR(4) * dm1);
        const double EL = ((k0 ? eL0 : 0.0) + (k1 ? eL1 : 0.0)) + (k2 ? eL2 : 0.0);
        const double ER = ((k0 ? eR0 : 0.0) + (k1 ? eR1 : 0.0)) + (k2 ? eR2 : 0.0);
        const double SL = ((k0 ? c.dL(0) : 0.0) + (k1 ? c.dL(1) : 0.0)) + (k2 ? c.dL(2) : 0.0);
        const double SR = ((k0 ? c.dR(0) : 0.0) + (k1 ? c.dR(1) : 0.0)) + (k2 ? c.dR(2) : 0.0);
        const double p = SL * SR;
        bool ok = s_ok && mid_range_prod(p);
        // a per-face row marks a face with a negative ideal weight by a NaN in
        // dL(0), which the cutoff may leave out of the sums: test it here
        if constexpr (!std::is_same_v<C, ParamCoefs>) ok = ok && (c.dL(0) == c.dL(0));
        const double r = rcp1(p);
        L = fma(EL * SR, r, v0);
        R = fma(ER * SL, r, v0);
        if constexpr (MPF) mp_sided(sign_clear(EL), sign_clear(ER), L, R);
        return ok;
    }
};

// The reference sequence for one face (cells o+1 .. o+5 of the column).
template <bool MPF>
__device__ __noinline__ void march64_redo(const MarchArgs& a, const double* __restrict__ col, long long o,
                                          double& L, double& R) {
    Coef<5> c;
#pragma unroll
    for (int q = 0; q < 6; ++q) {
        c.pL[q] = a.ucf[q];
        c.pR[q] = a.ucf[6 + q];
    }
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        c.dL[q] = a.ucf[12 + q];
        c.dR[q] = a.ucf[15 + q];
    }
#pragma unroll
    for (int q = 0; q < 9; ++q) c.b[q] = a.ucf[18 + q];
    const double* p = col + (o + 1) * a.sJ;
    const double vm2 = __ldg(p), vm1 = __ldg(p + a.sJ), v0 = __ldg(p + 2 * a.sJ), vp1 = __ldg(p + 3 * a.sJ),
                 vp2 = __ldg(p + 4 * a.sJ);
    weno5_face<double>(vm2, vm1, v0, vp1, vp2, c, a.wp.scheme, a.wp.eps, a.wp.teno_ct, L, R);
    if (MPF) mp_limit(vm2, vm1, v0, vp1, vp2, L, R);
}

// ---------------------------------------------------------------------
// WENO7-JS (+ MP) marching engine, FP64, face-independent coefficients
// (Coef<7> layout in MarchArgs::ucf: polyL 0..11, polyR 12..23, dL 24..27,
// dR 28..31, beta 32..55).  Stencil s (0..3) of face J reads the triple
// (a, b, e) = (d[J+s-1], d[J+s-2], d[J+s-3]) with coefficient row r = 3 - s
// (f90:1462-1473 and 1480-1488: beta(3-r) and poly(3-r) from dvd(2-r),
// dvd(1-r), dvd(-r)).  The newest triple T_m = (d[m], d[m+1], d[m+2]) is
// stencil 3 of face m, 2 of m+1, 1 of m+2 and 0 of m+3: each pushed cell
// gives one beta to each of four faces (its six products: three new, three
// carried from the previous triple), kept in registers until its face.
// Weights as March64: ideal weights folded into the candidate coefficients
// (MarchArgs::kL7 / kR7), one reciprocal of S_L S_R, the one-sided MP median.
// ---------------------------------------------------------------------
// Coefficient sources of the WENO7 engine: ParamCoefs7 (kernel-parameter
// bank) and Row7, one row of the per-face table read at each use (the rows
// of a chunk sit in shared memory; reading them where they are used keeps
// WENO7's already large register state from growing).  Row layout
// (kFaceRow7 doubles): [0..11] kL7, [12..23] kR7, [24..27] dL, [28..31] dR,
// [32 + 6r + q] the beta coefficients of row r that the triple pushed into
// face f enters (stencil 3 - r of face f + r).
constexpr int kFaceRow7 = 56;

struct ParamCoefs7 {
    const MarchArgs& a;
    __device__ __forceinline__ double kL(int q) const { return a.kL7[q]; }
    __device__ __forceinline__ double kR(int q) const { return a.kR7[q]; }
    __device__ __forceinline__ double dL(int s) const { return a.ucf[24 + s]; }
    __device__ __forceinline__ double dR(int s) const { return a.ucf[28 + s]; }
    __device__ __forceinline__ double b(int r, int q) const { return a.ucf[32 + 6 * r + q]; }
};

struct Row7 {
    const double* p;
    __device__ __forceinline__ double kL(int q) const { return p[q]; }
    __device__ __forceinline__ double kR(int q) const { return p[12 + q]; }
    __device__ __forceinline__ double dL(int s) const { return p[24 + s]; }
    __device__ __forceinline__ double dR(int s) const { return p[28 + s]; }
    __device__ __forceinline__ double b(int r, int q) const { return p[32 + 6 * r + q]; }
};

// The WENO7 per-face table (rows f = 0 .. rows-1, core face c(f) =
// clamp(f - 3, 0, nc - 1); f90:1462-1488 read polyL/R(j, r, s), d(r, j) and
// beta_coef(j, r, s) at the core index): kL7[3s+t] = dL(s) polyL(c, 3-s, t),
// kR7 likewise, dL, dR, and beta_coef(c(f + r), r, q).  A negative ideal
// weight puts a NaN in dL(0), as march_face_table_kernel.
__global__ void march_face_table7_kernel(CoefPtrs cp, long long nc, int rows, double* __restrict__ tab) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= rows) return;
    auto core = [&](long long x) { x -= 3; return x < 0 ? 0 : (x > nc - 1 ? nc - 1 : x); };
    const long long c = core(f);
    double* row = tab + (long long)f * kFaceRow7;
    bool neg = false;
    for (int s = 0; s < 4; ++s) {
        const double dl = cp.dL[s + 5 * c], dr = cp.dR[s + 5 * c];
        neg |= !(dl >= 0.0) || !(dr >= 0.0);
        for (int t = 0; t < 3; ++t) {
            row[3 * s + t] = dl * cp.polyL[c + nc * ((3 - s) + 5 * t)];
            row[12 + 3 * s + t] = dr * cp.polyR[c + nc * ((3 - s) + 5 * t)];
        }
        row[24 + s] = dl;
        row[28 + s] = dr;
    }
    for (int r = 0; r < 4; ++r) {
        const long long cr = core(f + r);
        for (int q = 0; q < 6; ++q) row[32 + 6 * r + q] = cp.beta[cr + nc * (r + 5 * q)];
    }
    if (neg) row[24] = __longlong_as_double(0x7ff8000000000000LL);
}

struct March64_7 {
    double vm1, v0, vp1, vp2, vp3;        // cells J-1 .. J+3
    double dm3, dm2, dm1, d0, dp1, dp2;    // d[k] = v[k+1] - v[k], k = J-3 .. J+2
    double s1, s2, c12;                    // d[J+1]^2, d[J+2]^2, d[J+1] d[J+2]
    double B0, B1, B2, B3;                 // beta_s(J)
    double n0a, n0b, n0c, n1a, n1b, n2a;   // beta_0(J+1 .. J+3), beta_1(J+1 .. J+2), beta_2(J+1)
    double e2, mA, mB;                     // d[J+1] - d[J]; minmods of the MP limiter

    // beta of coefficient row r from the products of a triple (a newest, e oldest)
    template <class C>
    __device__ __forceinline__ static double beta_row(const MarchArgs& a, const C& c, int r, double aa, double ab,
                                                      double ae, double bb, double be, double ee) {
        return fma(c.b(r, 0), aa, fma(c.b(r, 1), ab, fma(c.b(r, 2), ae,
                   fma(c.b(r, 3), bb, fma(c.b(r, 4), be, fma(c.b(r, 5), ee, a.wp.eps))))));
    }
    template <class C>
    __device__ __forceinline__ static double beta_row(const MarchArgs& a, const C& c, int r, double x, double y,
                                                      double z) {
        // triple (e, b, a) = (x, y, z)
        return beta_row(a, c, r, z * z, z * y, z * x, y * y, y * x, x * x);
    }
    __device__ __forceinline__ static double beta_row(const MarchArgs& a, int r, double aa, double ab, double ae,
                                                      double bb, double be, double ee) {
        return beta_row(a, ParamCoefs7{a}, r, aa, ab, ae, bb, be, ee);
    }
    __device__ __forceinline__ static double beta_row(const MarchArgs& a, int r, double x, double y, double z) {
        return beta_row(a, ParamCoefs7{a}, r, x, y, z);
    }

    // Window of face J from cells J-3 .. J+3; cm3 .. cz are the beta sources
    // of the triples starting at d[J-3] .. d[J].
    __device__ __forceinline__ void init(const MarchArgs& a, double c0, double c1, double c2, double c3, double c4,
                                         double c5, double c6) {
        const ParamCoefs7 u{a};
        init(a, u, u, u, u, c0, c1, c2, c3, c4, c5, c6);
    }
    template <class C3, class C2, class C1, class C0>
    __device__ __forceinline__ void init(const MarchArgs& a, const C3& cm3, const C2& cm2, const C1& cm1,
                                         const C0& cz, double c0, double c1, double c2, double c3, double c4,
                                         double c5, double c6) {
        vm1 = c2; v0 = c3; vp1 = c4; vp2 = c5; vp3 = c6;
        dm3 = c1 - c0; dm2 = c2 - c1; dm1 = c3 - c2; d0 = c4 - c3; dp1 = c5 - c4; dp2 = c6 - c5;
        s1 = dp1 * dp1; s2 = dp2 * dp2; c12 = dp1 * dp2;
        const double b0 = beta_row(a, cm3, 3, dm3, dm2, dm1);          // T_{J-3}
        const double b1 = beta_row(a, cm2, 2, dm2, dm1, d0);           // T_{J-2}
        n0a = beta_row(a, cm2, 3, dm2, dm1, d0);
        const double b2 = beta_row(a, cm1, 1, dm1, d0, dp1);           // T_{J-1}
        n1a = beta_row(a, cm1, 2, dm1, d0, dp1);
        n0b = beta_row(a, cm1, 3, dm1, d0, dp1);
        const double b3 = beta_row(a, cz, 0, d0, dp1, dp2);            // T_J
        n2a = beta_row(a, cz, 1, d0, dp1, dp2);
        n1b = beta_row(a, cz, 2, d0, dp1, dp2);
        n0c = beta_row(a, cz, 3, d0, dp1, dp2);
        B0 = b0; B1 = b1; B2 = b2; B3 = b3;
        const double em = dm1 - dm2, ez = d0 - dm1;
        e2 = dp1 - d0;
        mA = mm64(em, ez);
        mB = mm64(ez, e2);
    }

    // Advance to face J+1; n is cell J+4; c is the beta source of the new
    // triple (d[J+1], d[J+2], d[J+3]).
    __device__ __forceinline__ void push(const MarchArgs& a, double n) { push(a, ParamCoefs7{a}, n); }
    template <class C>
    __device__ __forceinline__ void push(const MarchArgs& a, const C& c, double n) {
        const double dn = n - vp3;
        const double aa = dn * dn, ab = dn * dp2, ae = dn * dp1;       // T_{J+1}: a = dn, b = dp2, e = dp1
        const double g0 = beta_row(a, c, 0, aa, ab, ae, s2, c12, s1);
        const double g1 = beta_row(a, c, 1, aa, ab, ae, s2, c12, s1);
        const double g2 = beta_row(a, c, 2, aa, ab, ae, s2, c12, s1);
        const double g3 = beta_row(a, c, 3, aa, ab, ae, s2, c12, s1);
        B0 = n0a; B1 = n1a; B2 = n2a; B3 = g0;
        n0a = n0b; n0b = n0c; n0c = g3;
        n1a = n1b; n1b = g2;
        n2a = g1;
        const double ne2 = dp2 - dp1;
        const double nmB = mm64(e2, ne2);
        vm1 = v0; v0 = vp1; vp1 = vp2; vp2 = vp3; vp3 = n;
        dm3 = dm2; dm2 = dm1; dm1 = d0; d0 = dp1; dp1 = dp2; dp2 = dn;
        s1 = s2; s2 = aa; c12 = ab;
        e2 = ne2; mA = mB; mB = nmB;
    }

    // WENO7-JS (+ MP) state of face J; false when the one-reciprocal form is
    // out of range (the caller redoes the face).
    template <bool MPF>
    __device__ __forceinline__ bool face(const MarchArgs& a, double& L, double& R) const {
        return face<MPF, ParamCoefs7>(a, ParamCoefs7{a}, L, R);
    }
    template <bool MPF, class C>
    __device__ __forceinline__ bool face(const MarchArgs& a, const C& c, double& L, double& R) const {
        const double q0 = B0 * B0, q1 = B1 * B1, q2 = B2 * B2, q3 = B3 * B3;
        const double q01 = q0 * q1, q23 = q2 * q3;
        const double P0 = q1 * q23, P1 = q0 * q23, P2 = q01 * q3, P3 = q01 * q2;
        const double SL = fma(c.dL(0), P0, fma(c.dL(1), P1, fma(c.dL(2), P2, c.dL(3) * P3)));
        const double SR = fma(c.dR(0), P0, fma(c.dR(1), P1, fma(c.dR(2), P2, c.dR(3) * P3)));
        // stencil s: (a, b, e) = (d[J+s-1], d[J+s-2], d[J+s-3])
        const double eL0 = fma(c.kL(0), dm1, fma(c.kL(1), dm2, c.kL(2) * dm3));
        const double eL1 = fma(c.kL(3), d0, fma(c.kL(4), dm1, c.kL(5) * dm2));
        const double eL2 = fma(c.kL(6), dp1, fma(c.kL(7), d0, c.kL(8) * dm1));
        const double eL3 = fma(c.kL(9), dp2, fma(c.kL(10), dp1, c.kL(11) * d0));
        const double eR0 = fma(c.kR(0), dm1, fma(c.kR(1), dm2, c.kR(2) * dm3));
        const double eR1 = fma(c.kR(3), d0, fma(c.kR(4), dm1, c.kR(5) * dm2));
        const double eR2 = fma(c.kR(6), dp1, fma(c.kR(7), d0, c.kR(8) * dm1));
        const double eR3 = fma(c.kR(9), dp2, fma(c.kR(10), dp1, c.kR(11) * d0));
        const double EL = fma(P0, eL0, fma(P1, eL1, fma(P2, eL2, P3 * eL3)));
        const double ER = fma(P0, eR0, fma(P1, eR1, fma(P2, eR2, P3 * eR3)));
        const double p = SL * SR;
        const bool ok = mid_range_prod(p);
        const double r = rcp1(p);
        L = fma(EL * SR, r, v0);
        R = fma(ER * SL, r, v0);
        if constexpr (MPF) {
            // the one-sided MP median of March64::face (the limiter reads
            // cells J-2 .. J+2 for every order)
            const double kBetaMP = 4.0 / 3.0;
            const bool up_l = sign_clear(dm1), up_r = sign_clear(d0);
            {
                const bool pos = sign_clear(EL);
                const double UL = fma(-2.0, d0, v0);
                const double MD = fma(-0.5, dm1 + mA, v0);
                const double LC = fma(kBetaMP, mB, fma(-0.5, d0, v0));
                const double Q1 = (pos == up_l) ? v0 : vm1;
                const double Q2 = (pos == up_r) ? v0 : UL;
                const double A = mm_sel(Q1, MD, pos), B = mm_sel(Q2, LC, pos);
                L = mm_sel(mm_sel(L, A, !pos), B, !pos);
            }
            {
                const bool pos = sign_clear(ER);
                const double UL = fma(2.0, dm1, v0);
                const double MD = fma(0.5, d0 - mB, v0);
                const double LC = fma(kBetaMP, mA, fma(0.5, dm1, v0));
                const double Q1 = (pos == up_r) ? vp1 : v0;
                const double Q2 = (pos == up_l) ? UL : v0;
                const double A = mm_sel(Q1, MD, pos), B = mm_sel(Q2, LC, pos);
                R = mm_sel(mm_sel(R, A, !pos), B, !pos);
            }
        }
        return ok;
    }
    // WENO7-TENO (+ MP) state of face J, with the reference's alpha(4) in the
    // sums (teno7_keep): L = (S_L v0 + E_L) / (S_L + alpha4), S_L = sum delta d,
    // E_L = sum delta (kL . differences).
    template <bool MPF>
    __device__ __forceinline__ bool face_teno(const MarchArgs& a, double& L, double& R) const {
        return face_teno<MPF, ParamCoefs7>(a, ParamCoefs7{a}, L, R);
    }
    template <bool MPF, class C>
    __device__ __forceinline__ bool face_teno(const MarchArgs& a, const C& c, double& L, double& R) const {
        bool k0, k1, k2, k3;
        double a4;
        const bool ok0 = teno7_keep(B0, B1, B2, B3, a.wp.eps, a.wp.teno_ct, k0, k1, k2, k3, a4);
        const double eL0 = fma(c.kL(0), dm1, fma(c.kL(1), dm2, c.kL(2) * dm3));
        const double eL1 = fma(c.kL(3), d0, fma(c.kL(4), dm1, c.kL(5) * dm2));
        const double eL2 = fma(c.kL(6), dp1, fma(c.kL(7), d0, c.kL(8) * dm1));
        const double eL3 = fma(c.kL(9), dp2, fma(c.kL(10), dp1, c.kL(11) * d0));
        const double eR0 = fma(c.kR(0), dm1, fma(c.kR(1), dm2, c.kR(2) * dm3));
        const double eR1 = fma(c.kR(3), d0, fma(c.kR(4), dm1, c.kR(5) * dm2));
        const double eR2 = fma(c.kR(6), dp1, fma(c.kR(7), d0, c.kR(8) * dm1));
        const double eR3 = fma(c.kR(9), dp2, fma(c.kR(10), dp1, c.kR(11) * d0));
        const double EL = ((k0 ? eL0 : 0.0) + (k1 ? eL1 : 0.0)) + ((k2 ? eL2 : 0.0) + (k3 ? eL3 : 0.0));
        const double ER = ((k0 ? eR0 : 0.0) + (k1 ? eR1 : 0.0)) + ((k2 ? eR2 : 0.0) + (k3 ? eR3 : 0.0));
        const double SL = ((k0 ? c.dL(0) : 0.0) + (k1 ? c.dL(1) : 0.0)) + ((k2 ? c.dL(2) : 0.0) + (k3 ? c.dL(3) : 0.0));
        const double SR = ((k0 ? c.dR(0) : 0.0) + (k1 ? c.dR(1) : 0.0)) + ((k2 ? c.dR(2) : 0.0) + (k3 ? c.dR(3) : 0.0));
        const double DL = SL + a4, DR = SR + a4;
        const double p = DL * DR;
        bool ok = ok0 && mid_range_prod(p);
        // a per-face row's NaN mark (negative ideal weight) may be cut from the sums
        if constexpr (!std::is_same_v<C, ParamCoefs7>) ok = ok && (c.dL(0) == c.dL(0));
        const double r = rcp1(p);
        L = fma(SL, v0, EL) * (DR * r);
        R = fma(SR, v0, ER) * (DL * r);
        if constexpr (MPF) mp64_sided(vm1, v0, vp1, dm1, d0, mA, mB, sign_clear(L - v0), sign_clear(R - v0), L, R);
        return ok;
    }
};
// The reference sequence for one WENO7 face with face-dependent
// coefficients: core face o - 3 of the arrays.
template <bool MPF>
__device__ __noinline__ void march64_7_redo_faces(const MarchArgs& a, const double* __restrict__ col, long long o,
                                                  double& L, double& R) {
    Coef<7> c;
    long long ci = o - 3;
    ci = ci < 0 ? 0 : (ci > a.nc - 1 ? a.nc - 1 : ci);
    c.load(a.cp.polyL, a.cp.polyR, a.cp.dL, a.cp.dR, a.cp.beta, a.nc, ci);
    double v[7];
#pragma unroll
    for (int q = 0; q < 7; ++q) v[q] = __ldg(col + (o + q) * a.sJ);
    weno7_face<double>(v + 3, c, a.wp.scheme, a.wp.eps, a.wp.teno_ct, L, R);
    if (MPF) mp_limit(v[1], v[2], v[3], v[4], v[5], L, R);
}

// The reference sequence for one WENO7 face (cells o .. o+6 of the column).
template <bool MPF>
__device__ __noinline__ void march64_7_redo(const MarchArgs& a, const double* __restrict__ col, long long o,
                                            double& L, double& R) {
    const Coef<7>& c = *reinterpret_cast<const Coef<7>*>(a.ucf);
    double v[7];
#pragma unroll
    for (int q = 0; q < 7; ++q) v[q] = __ldg(col + (o + q) * a.sJ);
    weno7_face<double>(v + 3, c, a.wp.scheme, a.wp.eps, a.wp.teno_ct, L, R);
    if (MPF) mp_limit(v[1], v[2], v[3], v[4], v[5], L, R);
}

// The same for face-dependent coefficients: core face o - 3 of the arrays.
template <bool MPF>
__device__ __noinline__ void march64_redo_faces(const MarchArgs& a, const double* __restrict__ col, long long o,
                                                double& L, double& R) {
    Coef<5> c;
    long long ci = o - 3;
    ci = ci < 0 ? 0 : (ci > a.nc - 1 ? a.nc - 1 : ci);
    c.load(a.cp.polyL, a.cp.polyR, a.cp.dL, a.cp.dR, a.cp.beta, a.nc, ci);
    const double* p = col + (o + 1) * a.sJ;
    const double vm2 = __ldg(p), vm1 = __ldg(p + a.sJ), v0 = __ldg(p + 2 * a.sJ), vp1 = __ldg(p + 3 * a.sJ),
                 vp2 = __ldg(p + 4 * a.sJ);
    weno5_face<double>(vm2, vm1, v0, vp1, vp2, c, a.wp.scheme, a.wp.eps, a.wp.teno_ct, L, R);
    if (MPF) mp_limit(vm2, vm1, v0, vp1, vp2, L, R);
}

// ---------------------------------------------------------------------
// FP32-bulk marching engine: FP32 cells and face states; FP64 differences,
// beta and weight normalisation (the parts that cancel or need eps = 1e-16),
// as weno5_js_mixed; FP32 candidate offsets and MP limiter.  (Written with
// scalar FP32 arithmetic: the sm_100 paired FP32 instructions need both
// halves in a register pair, and broadcasting the shared differences into
// pairs cost more moves than the pairing saved.)
// ---------------------------------------------------------------------
// FP32 minmod of the MP limiter (the value of mp_minmod_f up to the sign of
// a zero result).
__device__ __forceinline__ float mm32(float dl, float dr) {
    const float m = fminf(fabsf(dl), fabsf(dr)), M = fmaxf(fabsf(dl), fabsf(dr));
    const float u = fminf(fmaf(4.0f, m, -M), m);
    const int hl = __float_as_int(dl), hu = __float_as_int(u);
    const int kill = ((hl ^ __float_as_int(dr)) | hu) >> 31;
    return __int_as_float((hu & ~kill) | (hl & (int)0x80000000));
}


struct March32 {
    float vm1, v0, vp1, vp2;    // cells J-1 .. J+2
    float fm2, fm1, f0, fp1;    // FP32 differences v[k+1] - v[k], k = J-2 .. J+1
    double Dp2;                 // vp2, widened
    double dp1;                 // FP64 d[J+1]
    double s1;                  // d[J+1]^2
    double b0, b1, b2;          // beta_0, beta_1, beta_2 of face J
    double b1n, b2n, b2nn;      // beta_1(J+1), beta_2(J+1), beta_2(J+2)
    float e2;                   // curvature fp1 - f0
    float mA, mB;               // minmod(e2[J-1], e2[J]), minmod(e2[J], e2[J+1])

    __device__ __forceinline__ void init(const MarchArgs& a, float c0, float c1, float c2, float c3, float c4) {
        vm1 = c1; v0 = c2; vp1 = c3; vp2 = c4;
        fm2 = c1 - c0; fm1 = c2 - c1; f0 = c3 - c2; fp1 = c4 - c3;
        const double D0 = c0, D1 = c1, D2 = c2, D3 = c3;
        Dp2 = c4;
        const double dm2 = D1 - D0, dm1 = D2 - D1, d0 = D3 - D2;
        dp1 = Dp2 - D3;
        const double sm2 = dm2 * dm2, sm1 = dm1 * dm1, s0 = d0 * d0;
        s1 = dp1 * dp1;
        double g0, g1, g2, u;
        March64::betas(a, sm2, dm2 * dm1, sm1, u, u, b2);
        March64::betas(a, sm1, dm1 * d0, s0, u, b1, b2n);
        March64::betas(a, s0, d0 * dp1, s1, g0, g1, g2);
        b0 = g0; b1n = g1; b2nn = g2;
        const float em = fm1 - fm2, ez = f0 - fm1;
        e2 = fp1 - f0;
        mA = mm32(em, ez);
        mB = mm32(ez, e2);
    }

    __device__ __forceinline__ void push(const MarchArgs& a, float n) {
        const double Dn = n;
        const double dn = Dn - Dp2;
        const double sn = dn * dn;
        double g0, g1, g2;
        March64::betas(a, s1, dp1 * dn, sn, g0, g1, g2);
        const float fn = n - vp2;
        const float ne2 = fn - fp1;
        const float nmB = mm32(e2, ne2);
        vm1 = v0; v0 = vp1; vp1 = vp2; vp2 = n;
        fm2 = fm1; fm1 = f0; f0 = fp1; fp1 = fn;
        Dp2 = Dn; dp1 = dn; s1 = sn;
        b0 = g0; b1 = b1n; b2 = b2n;
        b1n = g1; b2n = b2nn; b2nn = g2;
        e2 = ne2; mA = mB; mB = nmB;
    }

    template <bool MPF>
    __device__ __forceinline__ bool face(const MarchArgs& a, float& L, float& R) const {
        const double q0 = b0 * b0, q1 = b1 * b1, q2 = b2 * b2;
        const double P0 = q1 * q2, P1 = q0 * q2, P2 = q0 * q1;
        const double aL0 = a.ucf[12] * P0, aL2 = a.ucf[14] * P2, aR0 = a.ucf[15] * P0, aR2 = a.ucf[17] * P2;
        const double SL = fma(a.ucf[13], P1, aL0 + aL2), SR = fma(a.ucf[16], P1, aR0 + aR2);
        const double p = SL * SR;
        const bool ok = mid_range_prod(p);
        const double r = rcp1(p), gL = SR * r, gR = SL * r;
        const float wL0 = __double2float_rn(aL0 * gL), wL2 = __double2float_rn(aL2 * gL),
                    wR0 = __double2float_rn(aR0 * gR), wR2 = __double2float_rn(aR2 * gR);
        // candidate offsets e_k = p_k - v0; pf2[q] = (polyL, polyR) of Coef<5> index q
        const float eL0 = fmaf(a.pf2[0].x, fp1, a.pf2[1].x * f0), eR0 = fmaf(a.pf2[0].y, fp1, a.pf2[1].y * f0);
        const float eL1 = fmaf(a.pf2[2].x, f0, a.pf2[3].x * fm1), eR1 = fmaf(a.pf2[2].y, f0, a.pf2[3].y * fm1);
        const float eL2 = fmaf(a.pf2[4].x, fm1, a.pf2[5].x * fm2), eR2 = fmaf(a.pf2[4].y, fm1, a.pf2[5].y * fm2);
        // x = e1 + w0 (e0 - e1) + w2 (e2 - e1)
        float xL = fmaf(wL0, eL0 - eL1, fmaf(wL2, eL2 - eL1, eL1));
        float xR = fmaf(wR0, eR0 - eR1, fmaf(wR2, eR2 - eR1, eR1));
        if constexpr (MPF) {
            // one-sided median in offset space (see March64::face): the
            // bounds relative to v0 are lo = max(min(0, -b, md), min(0, ul, lc))
            // and hi = min(max(0, -b, md), max(0, ul, lc)) with b = v0 - vm1,
            // c = vp1 - v0, md = -(b + mA)/2, ul = -2c, lc = 4/3 mB - c/2;
            // for x >= 0 the result is min(x, hi), else max(x, lo), so each
            // min/max below is chosen by the sign of x.  The right state is the
            // same formula with (b, c, mA, mB) -> (-c, -b, mB, mA).
            const float kB = 4.0f / 3.0f;
            {
                const bool pos = xL >= 0.0f;
                const float md = -0.5f * (fm1 + mA), ul = -2.0f * f0, lc = fmaf(kB, mB, -0.5f * f0), nb = -fm1;
                const float A = pos ? fmaxf(fmaxf(0.0f, nb), md) : fminf(fminf(0.0f, nb), md);
                const float B = pos ? fmaxf(fmaxf(0.0f, ul), lc) : fminf(fminf(0.0f, ul), lc);
                xL = pos ? fminf(fminf(xL, A), B) : fmaxf(fmaxf(xL, A), B);
            }
            {
                const bool pos = xR >= 0.0f;
                const float md = -0.5f * (mB - f0), ul = 2.0f * fm1, lc = fmaf(kB, mA, 0.5f * fm1), nb = f0;
                const float A = pos ? fmaxf(fmaxf(0.0f, nb), md) : fminf(fminf(0.0f, nb), md);
                const float B = pos ? fmaxf(fmaxf(0.0f, ul), lc) : fminf(fminf(0.0f, ul), lc);
                xR = pos ? fminf(fminf(xR, A), B) : fmaxf(fmaxf(xR, A), B);
            }
        }
        L = v0 + xL;
        R = v0 + xR;
        return ok;
    }
    // FP32-bulk WENO5-TENO: flags and weights d_k delta_k / S from the FP64
    // betas (teno5_keep), candidates and MP in FP32 (pivot on stencil 1).
    template <bool MPF>
    __device__ __forceinline__ bool face_teno(const MarchArgs& a, float& L, float& R) const {
        bool k0, k1, k2;
        const bool ok0 = teno5_keep(b0, b1, b2, a.wp.teno_ct, k0, k1, k2);
        const double aL0 = k0 ? a.ucf[12] : 0.0, aL1 = k1 ? a.ucf[13] : 0.0, aL2 = k2 ? a.ucf[14] : 0.0;
        const double aR0 = k0 ? a.ucf[15] : 0.0, aR1 = k1 ? a.ucf[16] : 0.0, aR2 = k2 ? a.ucf[17] : 0.0;
        const double SL = (aL0 + aL1) + aL2, SR = (aR0 + aR1) + aR2;
        const double p = SL * SR;
        const bool ok = ok0 && mid_range_prod(p);
        const double r = rcp1(p), gL = SR * r, gR = SL * r;
        const float wL0 = __double2float_rn(aL0 * gL), wL2 = __double2float_rn(aL2 * gL),
                    wR0 = __double2float_rn(aR0 * gR), wR2 = __double2float_rn(aR2 * gR);
        const float eL0 = fmaf(a.pf2[0].x, fp1, a.pf2[1].x * f0), eR0 = fmaf(a.pf2[0].y, fp1, a.pf2[1].y * f0);
        const float eL1 = fmaf(a.pf2[2].x, f0, a.pf2[3].x * fm1), eR1 = fmaf(a.pf2[2].y, f0, a.pf2[3].y * fm1);
        const float eL2 = fmaf(a.pf2[4].x, fm1, a.pf2[5].x * fm2), eR2 = fmaf(a.pf2[4].y, fm1, a.pf2[5].y * fm2);
        float xL = fmaf(wL0, eL0 - eL1, fmaf(wL2, eL2 - eL1, eL1));
        float xR = fmaf(wR0, eR0 - eR1, fmaf(wR2, eR2 - eR1, eR1));
        if constexpr (MPF) mp32_sided(fm1, f0, mA, mB, xL, xR);
        L = v0 + xL;
        R = v0 + xR;
        return ok;
    }
};
// The reference sequence for one FP32-bulk face (cells o+1 .. o+5).
template <bool MPF>
__device__ __noinline__ void march32_redo(const MarchArgs& a, const float* __restrict__ col, long long o, float& L,
                                          float& R) {
    Coef<5> c;
#pragma unroll
    for (int q = 0; q < 6; ++q) {
        c.pL[q] = a.ucf[q];
        c.pR[q] = a.ucf[6 + q];
    }
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        c.dL[q] = a.ucf[12 + q];
        c.dR[q] = a.ucf[15 + q];
    }
#pragma unroll
    for (int q = 0; q < 9; ++q) c.b[q] = a.ucf[18 + q];
    const float* p = col + (o + 1) * a.sJ;
    const float vm2 = __ldg(p), vm1 = __ldg(p + a.sJ), v0 = __ldg(p + 2 * a.sJ), vp1 = __ldg(p + 3 * a.sJ),
                vp2 = __ldg(p + 4 * a.sJ);
    double Ld, Rd;
    weno5_face<float>(f2d_bits(vm2), f2d_bits(vm1), f2d_bits(v0), f2d_bits(vp1), f2d_bits(vp2), c, a.wp.scheme,
                      a.wp.eps, a.wp.teno_ct, Ld, Rd);
    L = (float)Ld;
    R = (float)Rd;
    if (MPF) MP<float>::apply(vm2, vm1, v0, vp1, vp2, L, R);
}

// ---------------------------------------------------------------------
// FP32-bulk WENO7-JS (+ MP) marching engine: FP32 cells, candidates, MP and
// face states; FP64 differences, beta and weight normalisation (the split of
// weno7_js_mixed), with March64_7's carrying of betas from difference
// triples.  Weights pivot on stencil 1: x = e1 + sum_{s != 1} w_s (e_s - e1).
// ---------------------------------------------------------------------
struct March32_7 {
    float vm1, v0, vp1, vp2, vp3;          // cells J-1 .. J+3
    float fm3, fm2, fm1, f0, fp1, fp2;      // FP32 differences, k = J-3 .. J+2
    double Dp3;                             // vp3, widened
    double dp1, dp2, s1, s2, c12;           // FP64 d[J+1], d[J+2], their squares and product
    double B0, B1, B2, B3;                  // beta_s(J)
    double n0a, n0b, n0c, n1a, n1b, n2a;    // as March64_7
    float e2, mA, mB;

    __device__ __forceinline__ void init(const MarchArgs& a, float c0, float c1, float c2, float c3, float c4,
                                         float c5, float c6) {
        vm1 = c2; v0 = c3; vp1 = c4; vp2 = c5; vp3 = c6;
        fm3 = c1 - c0; fm2 = c2 - c1; fm1 = c3 - c2; f0 = c4 - c3; fp1 = c5 - c4; fp2 = c6 - c5;
        const double D0 = c0, D1 = c1, D2 = c2, D3 = c3, D4 = c4, D5 = c5;
        Dp3 = c6;
        const double dm3 = D1 - D0, dm2 = D2 - D1, dm1 = D3 - D2, d0 = D4 - D3;
        dp1 = D5 - D4; dp2 = Dp3 - D5;
        s1 = dp1 * dp1; s2 = dp2 * dp2; c12 = dp1 * dp2;
        const double b0 = March64_7::beta_row(a, 3, dm3, dm2, dm1);
        const double b1 = March64_7::beta_row(a, 2, dm2, dm1, d0);
        n0a = March64_7::beta_row(a, 3, dm2, dm1, d0);
        const double b2 = March64_7::beta_row(a, 1, dm1, d0, dp1);
        n1a = March64_7::beta_row(a, 2, dm1, d0, dp1);
        n0b = March64_7::beta_row(a, 3, dm1, d0, dp1);
        const double b3 = March64_7::beta_row(a, 0, d0, dp1, dp2);
        n2a = March64_7::beta_row(a, 1, d0, dp1, dp2);
        n1b = March64_7::beta_row(a, 2, d0, dp1, dp2);
        n0c = March64_7::beta_row(a, 3, d0, dp1, dp2);
        B0 = b0; B1 = b1; B2 = b2; B3 = b3;
        const float em = fm1 - fm2, ez = f0 - fm1;
        e2 = fp1 - f0;
        mA = mm32(em, ez);
        mB = mm32(ez, e2);
    }

    __device__ __forceinline__ void push(const MarchArgs& a, float n) {
        const double Dn = n;
        const double dn = Dn - Dp3;
        const double aa = dn * dn, ab = dn * dp2, ae = dn * dp1;
        const double g0 = March64_7::beta_row(a, 0, aa, ab, ae, s2, c12, s1);
        const double g1 = March64_7::beta_row(a, 1, aa, ab, ae, s2, c12, s1);
        const double g2 = March64_7::beta_row(a, 2, aa, ab, ae, s2, c12, s1);
        const double g3 = March64_7::beta_row(a, 3, aa, ab, ae, s2, c12, s1);
        B0 = n0a; B1 = n1a; B2 = n2a; B3 = g0;
        n0a = n0b; n0b = n0c; n0c = g3;
        n1a = n1b; n1b = g2;
        n2a = g1;
        const float fn = n - vp3;
        const float ne2 = fp2 - fp1;
        const float nmB = mm32(e2, ne2);
        vm1 = v0; v0 = vp1; vp1 = vp2; vp2 = vp3; vp3 = n;
        fm3 = fm2; fm2 = fm1; fm1 = f0; f0 = fp1; fp1 = fp2; fp2 = fn;
        Dp3 = Dn; dp1 = dp2; dp2 = dn;
        s1 = s2; s2 = aa; c12 = ab;
        e2 = ne2; mA = mB; mB = nmB;
    }

    template <bool MPF>
    __device__ __forceinline__ bool face(const MarchArgs& a, float& L, float& R) const {
        const double q0 = B0 * B0, q1 = B1 * B1, q2 = B2 * B2, q3 = B3 * B3;
        const double q01 = q0 * q1, q23 = q2 * q3;
        const double P0 = q1 * q23, P1 = q0 * q23, P2 = q01 * q3, P3 = q01 * q2;
        const double aL0 = a.ucf[24] * P0, aL2 = a.ucf[26] * P2, aL3 = a.ucf[27] * P3;
        const double aR0 = a.ucf[28] * P0, aR2 = a.ucf[30] * P2, aR3 = a.ucf[31] * P3;
        const double SL = fma(a.ucf[25], P1, (aL0 + aL2) + aL3), SR = fma(a.ucf[29], P1, (aR0 + aR2) + aR3);
        const double p = SL * SR;
        const bool ok = mid_range_prod(p);
        const double r = rcp1(p), gL = SR * r, gR = SL * r;
        const float wL0 = __double2float_rn(aL0 * gL), wL2 = __double2float_rn(aL2 * gL),
                    wL3 = __double2float_rn(aL3 * gL);
        const float wR0 = __double2float_rn(aR0 * gR), wR2 = __double2float_rn(aR2 * gR),
                    wR3 = __double2float_rn(aR3 * gR);
        // candidate offsets of stencil s (row 3 - s), (a, b, e) = (f[J+s-1], f[J+s-2], f[J+s-3])
        const float eL0 = fmaf(a.pf7[9], fm1, fmaf(a.pf7[10], fm2, a.pf7[11] * fm3));
        const float eL1 = fmaf(a.pf7[6], f0, fmaf(a.pf7[7], fm1, a.pf7[8] * fm2));
        const float eL2 = fmaf(a.pf7[3], fp1, fmaf(a.pf7[4], f0, a.pf7[5] * fm1));
        const float eL3 = fmaf(a.pf7[0], fp2, fmaf(a.pf7[1], fp1, a.pf7[2] * f0));
        const float eR0 = fmaf(a.pf7[21], fm1, fmaf(a.pf7[22], fm2, a.pf7[23] * fm3));
        const float eR1 = fmaf(a.pf7[18], f0, fmaf(a.pf7[19], fm1, a.pf7[20] * fm2));
        const float eR2 = fmaf(a.pf7[15], fp1, fmaf(a.pf7[16], f0, a.pf7[17] * fm1));
        const float eR3 = fmaf(a.pf7[12], fp2, fmaf(a.pf7[13], fp1, a.pf7[14] * f0));
        float xL = fmaf(wL0, eL0 - eL1, fmaf(wL2, eL2 - eL1, fmaf(wL3, eL3 - eL1, eL1)));
        float xR = fmaf(wR0, eR0 - eR1, fmaf(wR2, eR2 - eR1, fmaf(wR3, eR3 - eR1, eR1)));
        if constexpr (MPF) {
            // the one-sided median of March32::face
            const float kB = 4.0f / 3.0f;
            {
                const bool pos = xL >= 0.0f;
                const float md = -0.5f * (fm1 + mA), ul = -2.0f * f0, lc = fmaf(kB, mB, -0.5f * f0), nb = -fm1;
                const float A = pos ? fmaxf(fmaxf(0.0f, nb), md) : fminf(fminf(0.0f, nb), md);
                const float B = pos ? fmaxf(fmaxf(0.0f, ul), lc) : fminf(fminf(0.0f, ul), lc);
                xL = pos ? fminf(fminf(xL, A), B) : fmaxf(fmaxf(xL, A), B);
            }
            {
                const bool pos = xR >= 0.0f;
                const float md = -0.5f * (mB - f0), ul = 2.0f * fm1, lc = fmaf(kB, mA, 0.5f * fm1), nb = f0;
                const float A = pos ? fmaxf(fmaxf(0.0f, nb), md) : fminf(fminf(0.0f, nb), md);
                const float B = pos ? fmaxf(fmaxf(0.0f, ul), lc) : fminf(fminf(0.0f, ul), lc);
                xR = pos ? fminf(fminf(xR, A), B) : fmaxf(fmaxf(xR, A), B);
            }
        }
        L = v0 + xL;
        R = v0 + xR;
        return ok;
    }
    // FP32-bulk WENO7-TENO with the reference's alpha(4) (teno7_keep): the
    // state is W v0 + sum w_s e_s with W = S / (S + alpha4), w_s = delta_s d_s /
    // (S + alpha4) from FP64, candidates and MP in FP32.
    template <bool MPF>
    __device__ __forceinline__ bool face_teno(const MarchArgs& a, float& L, float& R) const {
        bool k0, k1, k2, k3;
        double a4;
        const bool ok0 = teno7_keep(B0, B1, B2, B3, a.wp.eps, a.wp.teno_ct, k0, k1, k2, k3, a4);
        const double aL0 = k0 ? a.ucf[24] : 0.0, aL1 = k1 ? a.ucf[25] : 0.0, aL2 = k2 ? a.ucf[26] : 0.0,
                     aL3 = k3 ? a.ucf[27] : 0.0;
        const double aR0 = k0 ? a.ucf[28] : 0.0, aR1 = k1 ? a.ucf[29] : 0.0, aR2 = k2 ? a.ucf[30] : 0.0,
                     aR3 = k3 ? a.ucf[31] : 0.0;
        const double SL = (aL0 + aL1) + (aL2 + aL3), SR = (aR0 + aR1) + (aR2 + aR3);
        const double DL = SL + a4, DR = SR + a4;
        const double p = DL * DR;
        const bool ok = ok0 && mid_range_prod(p);
        const double r = rcp1(p), gL = DR * r, gR = DL * r;
        const float wL0 = __double2float_rn(aL0 * gL), wL1 = __double2float_rn(aL1 * gL),
                    wL2 = __double2float_rn(aL2 * gL), wL3 = __double2float_rn(aL3 * gL),
                    WL = __double2float_rn(SL * gL);
        const float wR0 = __double2float_rn(aR0 * gR), wR1 = __double2float_rn(aR1 * gR),
                    wR2 = __double2float_rn(aR2 * gR), wR3 = __double2float_rn(aR3 * gR),
                    WR = __double2float_rn(SR * gR);
        const float eL0 = fmaf(a.pf7[9], fm1, fmaf(a.pf7[10], fm2, a.pf7[11] * fm3));
        const float eL1 = fmaf(a.pf7[6], f0, fmaf(a.pf7[7], fm1, a.pf7[8] * fm2));
        const float eL2 = fmaf(a.pf7[3], fp1, fmaf(a.pf7[4], f0, a.pf7[5] * fm1));
        const float eL3 = fmaf(a.pf7[0], fp2, fmaf(a.pf7[1], fp1, a.pf7[2] * f0));
        const float eR0 = fmaf(a.pf7[21], fm1, fmaf(a.pf7[22], fm2, a.pf7[23] * fm3));
        const float eR1 = fmaf(a.pf7[18], f0, fmaf(a.pf7[19], fm1, a.pf7[20] * fm2));
        const float eR2 = fmaf(a.pf7[15], fp1, fmaf(a.pf7[16], f0, a.pf7[17] * fm1));
        const float eR3 = fmaf(a.pf7[12], fp2, fmaf(a.pf7[13], fp1, a.pf7[14] * f0));
        L = fmaf(WL, v0, fmaf(wL0, eL0, fmaf(wL1, eL1, fmaf(wL2, eL2, wL3 * eL3))));
        R = fmaf(WR, v0, fmaf(wR0, eR0, fmaf(wR1, eR1, fmaf(wR2, eR2, wR3 * eR3))));
        if constexpr (MPF) {
            float xL = L - v0, xR = R - v0;
            mp32_sided(fm1, f0, mA, mB, xL, xR);
            L = v0 + xL;
            R = v0 + xR;
        }
        return ok;
    }
};
// The reference sequence for one WENO7 face, FP32 storage (FP64 arithmetic).
template <bool MPF>
__device__ __noinline__ void march32_7_redo(const MarchArgs& a, const float* __restrict__ col, long long o, float& L,
                                            float& R) {
    const Coef<7>& c = *reinterpret_cast<const Coef<7>*>(a.ucf);
    float f[7];
    double v[7];
#pragma unroll
    for (int q = 0; q < 7; ++q) {
        f[q] = __ldg(col + (o + q) * a.sJ);
        v[q] = f[q];
    }
    double Ld, Rd;
    weno7_face<double>(v + 3, c, a.wp.scheme, a.wp.eps, a.wp.teno_ct, Ld, Rd);
    L = (float)Ld;
    R = (float)Rd;
    if (MPF) MP<float>::apply(f[1], f[2], f[3], f[4], f[5], L, R);
}

// ---------------------------------------------------------------------
// WENO3-JS (+ MP) marching engines, face-independent coefficients (Coef<3>
// layout in MarchArgs::ucf: polyL 0..1, polyR 2..3, dL 4..5, dR 6..7,
// beta 8..9; f90:416-468).  beta_0(J) = b0 d[J]^2 + eps, beta_1(J) =
// b1 d[J-1]^2 + eps.  WENO3 writes every face of the sweep (the reference's
// is1 range) and the fused MP limiter applies on the core faces only, so
// face() takes that as an argument; the window is still cells J-2 .. J+2
// for the limiter's minmods.
// ---------------------------------------------------------------------
// Coefficient sources of the FP64 WENO3 engine: ParamCoefs3 (kernel
// parameters) and Row3, one row of the WENO3 per-face table (kFaceRow3
// doubles: [0..1] kL, [2..3] kR, [4..5] dL, [6..7] dR, [8..9] beta_coef of
// the face; a push into face f reads row f).
constexpr int kFaceRow3 = 12;

struct ParamCoefs3 {
    const MarchArgs& a;
    __device__ __forceinline__ double kL(int q) const { return a.kL[q]; }
    __device__ __forceinline__ double kR(int q) const { return a.kR[q]; }
    __device__ __forceinline__ double dL(int r) const { return a.ucf[4 + r]; }
    __device__ __forceinline__ double dR(int r) const { return a.ucf[6 + r]; }
    __device__ __forceinline__ double b(int r) const { return a.ucf[8 + r]; }
};

struct Row3 {
    const double* p;
    __device__ __forceinline__ double kL(int q) const { return p[q]; }
    __device__ __forceinline__ double kR(int q) const { return p[2 + q]; }
    __device__ __forceinline__ double dL(int r) const { return p[4 + r]; }
    __device__ __forceinline__ double dR(int r) const { return p[6 + r]; }
    __device__ __forceinline__ double b(int r) const { return p[8 + r]; }
};

// The WENO3 per-face table (f90:416-468: polyL/R(j, r, 0), d(r, j),
// beta_coef(j, r, 0) at the core index c(f) = clamp(f - 3, 0, nc - 1), the
// convention of every kernel here for the faces outside the core): kL[r] =
// dL(r) polyL(c, r, 0), kR likewise, dL, dR, beta_coef(c, r, 0).  A negative
// ideal weight puts a NaN in dL(0).
__global__ void march_face_table3_kernel(CoefPtrs cp, long long nc, int rows, double* __restrict__ tab) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= rows) return;
    long long c = f - 3;
    c = c < 0 ? 0 : (c > nc - 1 ? nc - 1 : c);
    double* row = tab + (long long)f * kFaceRow3;
    bool neg = false;
    for (int r = 0; r < 2; ++r) {
        const double dl = cp.dL[r + 5 * c], dr = cp.dR[r + 5 * c];
        neg |= !(dl >= 0.0) || !(dr >= 0.0);
        row[r] = dl * cp.polyL[c + nc * r];
        row[2 + r] = dr * cp.polyR[c + nc * r];
        row[4 + r] = dl;
        row[6 + r] = dr;
        row[8 + r] = cp.beta[c + nc * r];
    }
    row[10] = row[11] = 0.0;
    if (neg) row[4] = __longlong_as_double(0x7ff8000000000000LL);
}

struct March64_3 {
    double vm1, v0, vp1, vp2;   // cells J-1 .. J+2
    double dm1, d0, dp1;        // d[J-1], d[J], d[J+1]
    double B0, B1;              // beta_0(J), beta_1(J)
    double e2, mA, mB;

    __device__ __forceinline__ void init(const MarchArgs& a, double c0, double c1, double c2, double c3, double c4) {
        init(a, ParamCoefs3{a}, c0, c1, c2, c3, c4);
    }
    // c: the coefficients of face J
    template <class C>
    __device__ __forceinline__ void init(const MarchArgs& a, const C& c, double c0, double c1, double c2, double c3,
                                         double c4) {
        vm1 = c1; v0 = c2; vp1 = c3; vp2 = c4;
        const double dm2 = c1 - c0;
        dm1 = c2 - c1; d0 = c3 - c2; dp1 = c4 - c3;
        B0 = fma(c.b(0), d0 * d0, a.wp.eps);
        B1 = fma(c.b(1), dm1 * dm1, a.wp.eps);
        const double em = dm1 - dm2, ez = d0 - dm1;
        e2 = dp1 - d0;
        mA = mm64(em, ez);
        mB = mm64(ez, e2);
    }
    __device__ __forceinline__ void push(const MarchArgs& a, double n) { push(a, ParamCoefs3{a}, n); }
    // c: the coefficients of face J+1
    template <class C>
    __device__ __forceinline__ void push(const MarchArgs& a, const C& c, double n) {
        const double dn = n - vp2;
        const double nB0 = fma(c.b(0), dp1 * dp1, a.wp.eps), nB1 = fma(c.b(1), d0 * d0, a.wp.eps);
        const double ne2 = dn - dp1;
        const double nmB = mm64(e2, ne2);
        vm1 = v0; v0 = vp1; vp1 = vp2; vp2 = n;
        dm1 = d0; d0 = dp1; dp1 = dn;
        B0 = nB0; B1 = nB1;
        e2 = ne2; mA = mB; mB = nmB;
    }
    template <bool MPF>
    __device__ __forceinline__ bool face(const MarchArgs& a, double& L, double& R) const {
        return face<MPF>(a, L, R, true);
    }
    template <bool MPF>
    __device__ __forceinline__ bool face(const MarchArgs& a, double& L, double& R, bool core) const {
        return face<MPF, ParamCoefs3>(a, ParamCoefs3{a}, L, R, core);
    }
    template <bool MPF, class C>
    __device__ __forceinline__ bool face(const MarchArgs& a, const C& c, double& L, double& R, bool core) const {
        const double P0 = B1 * B1, P1 = B0 * B0;
        const double SL = fma(c.dL(0), P0, c.dL(1) * P1), SR = fma(c.dR(0), P0, c.dR(1) * P1);
        const double EL = fma(P0, c.kL(0) * d0, P1 * (c.kL(1) * dm1));
        const double ER = fma(P0, c.kR(0) * d0, P1 * (c.kR(1) * dm1));
        const double p = SL * SR;
        const bool ok = mid_range_prod(p);
        const double r = rcp1(p);
        L = fma(EL * SR, r, v0);
        R = fma(ER * SL, r, v0);
        if (MPF && core) mp64_sided(vm1, v0, vp1, dm1, d0, mA, mB, sign_clear(EL), sign_clear(ER), L, R);
        return ok;
    }
};

struct March32_3 {
    float vm1, v0, vp1, vp2;    // cells J-1 .. J+2
    float fm1, f0, fp1;         // FP32 differences
    double Dp2, Dd0, Ddp1;      // vp2 widened; FP64 d[J], d[J+1]
    double B0, B1;
    float e2, mA, mB;

    __device__ __forceinline__ void init(const MarchArgs& a, float c0, float c1, float c2, float c3, float c4) {
        vm1 = c1; v0 = c2; vp1 = c3; vp2 = c4;
        const float fm2 = c1 - c0;
        fm1 = c2 - c1; f0 = c3 - c2; fp1 = c4 - c3;
        const double D1 = c1, D2 = c2, D3 = c3;
        Dp2 = c4;
        const double ddm1 = D2 - D1;
        Dd0 = D3 - D2; Ddp1 = Dp2 - D3;
        B0 = fma(a.ucf[8], Dd0 * Dd0, a.wp.eps);
        B1 = fma(a.ucf[9], ddm1 * ddm1, a.wp.eps);
        const float em = fm1 - fm2, ez = f0 - fm1;
        e2 = fp1 - f0;
        mA = mm32(em, ez);
        mB = mm32(ez, e2);
    }
    __device__ __forceinline__ void push(const MarchArgs& a, float n) {
        const double Dn = n;
        const double dn = Dn - Dp2;
        const double nB0 = fma(a.ucf[8], Ddp1 * Ddp1, a.wp.eps), nB1 = fma(a.ucf[9], Dd0 * Dd0, a.wp.eps);
        const float fn = n - vp2;
        const float ne2 = fn - fp1;
        const float nmB = mm32(e2, ne2);
        vm1 = v0; v0 = vp1; vp1 = vp2; vp2 = n;
        fm1 = f0; f0 = fp1; fp1 = fn;
        Dp2 = Dn; Dd0 = Ddp1; Ddp1 = dn;
        B0 = nB0; B1 = nB1;
        e2 = ne2; mA = mB; mB = nmB;
    }
    template <bool MPF>
    __device__ __forceinline__ bool face(const MarchArgs& a, float& L, float& R) const {
        return face<MPF>(a, L, R, true);
    }
    template <bool MPF>
    __device__ __forceinline__ bool face(const MarchArgs& a, float& L, float& R, bool core) const {
        const double P0 = B1 * B1, P1 = B0 * B0;
        const double aL0 = a.ucf[4] * P0, aR0 = a.ucf[6] * P0;
        const double SL = fma(a.ucf[5], P1, aL0), SR = fma(a.ucf[7], P1, aR0);
        const double p = SL * SR;
        const bool ok = mid_range_prod(p);
        const double r = rcp1(p);
        const float wL0 = __double2float_rn(aL0 * (SR * r)), wR0 = __double2float_rn(aR0 * (SL * r));
        const float eL0 = a.pf2[0].x * f0, eL1 = a.pf2[1].x * fm1;
        const float eR0 = a.pf2[0].y * f0, eR1 = a.pf2[1].y * fm1;
        float xL = fmaf(wL0, eL0 - eL1, eL1), xR = fmaf(wR0, eR0 - eR1, eR1);
        if (MPF && core) mp32_sided(fm1, f0, mA, mB, xL, xR);
        L = v0 + xL;
        R = v0 + xR;
        return ok;
    }
};

// The same with face-dependent coefficient arrays (core face clamp(o - 3)).
template <bool MPF>
__device__ __noinline__ void march3_redo_faces(const MarchArgs& a, const double* __restrict__ col, long long o,
                                               double& L, double& R) {
    Coef<3> c;
    long long ci = o - 3;
    ci = ci < 0 ? 0 : (ci > a.nc - 1 ? a.nc - 1 : ci);
    c.load(a.cp.polyL, a.cp.polyR, a.cp.dL, a.cp.dR, a.cp.beta, a.nc, ci);
    const double* p = col + (o + 1) * a.sJ;
    const double vm2 = __ldg(p), vm1 = __ldg(p + a.sJ), v0 = __ldg(p + 2 * a.sJ), vp1 = __ldg(p + 3 * a.sJ),
                 vp2 = __ldg(p + 4 * a.sJ);
    weno3_face(vm1, v0, vp1, c, a.wp.scheme, a.wp.eps, L, R);
    if (MPF && o >= 3 && o <= a.ns - 4) mp_limit(vm2, vm1, v0, vp1, vp2, L, R);
}

// The reference sequence for one WENO3 face (cells o+1 .. o+5; MP on the
// core faces).
template <bool MPF, typename T>
__device__ __noinline__ void march3_redo(const MarchArgs& a, const T* __restrict__ col, long long o, T& L, T& R) {
    const Coef<3>& c = *reinterpret_cast<const Coef<3>*>(a.ucf);
    const T* p = col + (o + 1) * a.sJ;
    const T vm2 = __ldg(p), vm1 = __ldg(p + a.sJ), v0 = __ldg(p + 2 * a.sJ), vp1 = __ldg(p + 3 * a.sJ),
            vp2 = __ldg(p + 4 * a.sJ);
    double Ld, Rd;
    weno3_face((double)vm1, (double)v0, (double)vp1, c, a.wp.scheme, a.wp.eps, Ld, Rd);
    L = (T)Ld;
    R = (T)Rd;
    if (MPF && o >= 3 && o <= a.ns - 4) MP<T>::apply(vm2, vm1, v0, vp1, vp2, L, R);
}

#ifndef WSB_MARCH64_MIN_BLOCKS
#define WSB_MARCH64_MIN_BLOCKS 3
#endif
#ifndef WSB_MARCH64_GROUP
#define WSB_MARCH64_GROUP 8
#endif
constexpr int kMarch64F = 16;                  // faces per chunk (and per shared-memory flush)
constexpr int kMarch64H = WSB_MARCH64_GROUP;   // cells per prefetch group
static_assert(kMarch64F % (2 * kMarch64H) == 0, "an even number of prefetch groups per chunk");

template <bool MPF>
__global__ void __launch_bounds__(128, WSB_MARCH64_MIN_BLOCKS)
    sweep_march64_kernel(const __grid_constant__ MarchArgs a) {
    constexpr int F = kMarch64F, H = kMarch64H;
    __shared__ double tile[4][2][F][33];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const double* __restrict__ in = (const double*)a.in;
    double* __restrict__ outL = (double*)a.vL;
    double* __restrict__ outR = (double*)a.vR;
    double(*tl)[F][33] = tile[warp];
    const long long nwarps = (long long)gridDim.x * (blockDim.x >> 5);
    const long long ncell = a.ns + 6;
    for (long long item = (long long)blockIdx.x * (blockDim.x >> 5) + warp; item < a.n_items; item += nwarps) {
        const int sg = (int)(item % a.n_seg);
        long long t = item / a.n_seg;
        const int ut = (int)(t % a.n_ut);
        t /= a.n_ut;
        const int wv = (int)(t % a.Nw);
        const int vv = (int)(t / a.Nw);
        const int u = ut * 32 + lane;
        const int uc = u < a.Nu ? u : a.Nu - 1;  // idle lanes shadow a valid column
        const double* __restrict__ col = in + a.in_off + uc * a.sU + wv * a.sW + vv * a.sV;
        const long long o_begin = 3 + (long long)sg * a.seg;
        long long o_end = o_begin + a.seg;
        if (o_end > a.ns - 3) o_end = a.ns - 3;
        // face o: centre cell o + 3, cells o+1 .. o+5; after face o the
        // window takes cell o + 6
        March64 w;
        {
            const double* p = col + (o_begin + 1) * a.sJ;
            w.init(a, __ldg(p), __ldg(p + a.sJ), __ldg(p + 2 * a.sJ), __ldg(p + 3 * a.sJ), __ldg(p + 4 * a.sJ));
        }
        const long long obase = (long long)ut * 32 * a.oU + wv * a.oW + vv * a.oV;
        // cells arrive H at a time, one group ahead of their use
        double buf[2][H];
        auto load = [&](double* dst, long long J0) {
#pragma unroll
            for (int i = 0; i < H; ++i) {
                const long long J = J0 + i;
                dst[i] = (J < ncell) ? __ldg(col + J * a.sJ) : 0.0;
            }
        };
        load(buf[0], o_begin + 6);
        for (long long f0 = o_begin; f0 < o_end; f0 += F) {
            const int nF = (int)min((long long)F, o_end - f0);
            unsigned bad = 0;
#pragma unroll
            for (int gi = 0; gi < F / H; ++gi) {
                load(buf[(gi + 1) & 1], f0 + 6 + (gi + 1) * H);
#pragma unroll
                for (int i = 0; i < H; ++i) {
                    double L, R;
                    if (!w.face<MPF>(a, L, R)) bad |= 1u << (gi * H + i);
                    tl[0][gi * H + i][lane] = L;
                    tl[1][gi * H + i][lane] = R;
                    w.push(a, buf[gi & 1][i]);
                }
            }
            bad &= (nF >= 32) ? ~0u : ((1u << nF) - 1u);
            while (bad) {
                const int i = __ffs(bad) - 1;
                bad &= bad - 1;
                double L, R;
                march64_redo<MPF>(a, col, f0 + i, L, R);
                tl[0][i][lane] = L;
                tl[1][i][lane] = R;
            }
            __syncwarp();
            // lanes take faces, the warp walks the columns (two per store)
            const int fi = lane & (F - 1), cj = lane / F;
#pragma unroll 4
            for (int c = cj; c < 32; c += 32 / F) {
                if (ut * 32 + c < a.Nu && fi < nF) {
                    const long long oi = obase + c * a.oU + f0 + fi;
                    outL[oi] = tl[0][fi][c];
                    outR[oi] = tl[1][fi][c];
                }
            }
            __syncwarp();
        }
    }
}

// Arguments of a marching sweep for face-independent WENO5-JS coefficients
// (everything but the segmentation).
inline MarchArgs make_march_args(const SweepGeom& g, const void* in, void* vL, void* vR, const WenoParams& wp,
                                 const double* ucf, int order = 5) {
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
    if (!ucf) return a;  // face-dependent coefficients: the caller sets ftab and cp
    for (int q = 0; q < 56; ++q) a.ucf[q] = ucf[q];
    if (order == 3) {
        // Coef<3>: polyL 0..1, polyR 2..3, dL 4..5, dR 6..7
        for (int r = 0; r < 2; ++r) {
            a.kL[r] = ucf[4 + r] * ucf[r];
            a.kR[r] = ucf[6 + r] * ucf[2 + r];
            a.pf2[r] = make_float2((float)ucf[r], (float)ucf[2 + r]);
        }
        return a;
    }
    if (order == 7) {
        for (int s = 0; s < 4; ++s)
            for (int t = 0; t < 3; ++t) {
                a.kL7[3 * s + t] = ucf[24 + s] * ucf[3 * (3 - s) + t];
                a.kR7[3 * s + t] = ucf[28 + s] * ucf[12 + 3 * (3 - s) + t];
            }
        for (int q = 0; q < 24; ++q) a.pf7[q] = (float)ucf[q];
        return a;
    }
    for (int q = 0; q < 6; ++q) {
        a.ucf32[q] = (float)ucf[q];          // polyL (Coef<5>::pL)
        a.ucf32[6 + q] = (float)ucf[6 + q];  // polyR
    }
    for (int r = 0; r < 3; ++r)
        for (int s = 0; s < 2; ++s) {
            a.kL[2 * r + s] = ucf[12 + r] * ucf[2 * r + s];
            a.kR[2 * r + s] = ucf[15 + r] * ucf[6 + 2 * r + s];
        }
    for (int q = 0; q < 6; ++q) a.pf2[q] = make_float2((float)ucf[q], (float)ucf[6 + q]);
    for (int k = 0; k < 3; ++k) {
        const double dl = ucf[12 + k], dr = ucf[15 + k];
        a.mcL[4 * k] = dl + dl * dl; a.mcL[4 * k + 1] = 3.0 * dl; a.mcL[4 * k + 2] = 1.0 - 2.0 * dl;
        a.mcL[4 * k + 3] = dl * dl;
        a.mcR[4 * k] = dr + dr * dr; a.mcR[4 * k + 1] = 3.0 * dr; a.mcR[4 * k + 2] = 1.0 - 2.0 * dr;
        a.mcR[4 * k + 3] = dr * dr;
    }
    return a;
}

// Launch for face-independent WENO5-JS coefficients.  Returns 1003 when
// the sweep has too few faces for the window.
template <typename T>
int launch_march_sweep(const SweepGeom& g, bool mp, const T* in, T* vL, T* vR, const WenoParams& wp,
                       const double* ucf, cudaStream_t st, int sms) {
    if (g.nc < 1 || !ucf) return 1003;
    MarchArgs a = make_march_args(g, in, vL, vR, wp, ucf);
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
    if constexpr (sizeof(T) == 8) {
        static_assert(MarchFlush<double>::F == kMarch64F, "FP64 segment rounding");
        if (mp) sweep_march64_kernel<true><<<(unsigned)blocks, 128, 0, st>>>(a);
        else sweep_march64_kernel<false><<<(unsigned)blocks, 128, 0, st>>>(a);
    } else {
        if (mp) sweep_march_kernel<true, T><<<(unsigned)blocks, 128, 0, st>>>(a);
        else sweep_march_kernel<false, T><<<(unsigned)blocks, 128, 0, st>>>(a);
    }
    return 0;
}

}  // namespace wsb
