// vjp_march.cuh -- adjoint (VJP) of the FP64 WENO5 (+MP) sweep with JS or
// TENO weights and face-independent coefficients, marching along the sweep
// like the forward kernel of sweep_march_tma.cuh.
//
// A warp owns 32 adjacent columns of one (w, v) and walks the whole column.
// At face J it recomputes the forward state from the carried window
// (March64: the beta of the new difference pair, P_k, S_L, S_R, one
// reciprocal) with the weights made explicit, then pulls the face's
// cotangents gL, gR back:
//   * MP (f90:1564-1608): the one-sided median of the forward kernel picks
//     one expression (the WENO value, v0, a neighbour, MD, UL or LC); the
//     cotangent goes to that expression's cells (and, for MD and LC, through
//     the minmod to the curvature it picked).  Faces whose median passes the
//     WENO value through -- the common case -- skip this part as a warp.
//   * weights: d out/d p_k = w_k, d out/d beta_k = -2 w_k (p_k - out)/beta_k
//     (JS); TENO weights d_k delta_k / sum d delta are constant between
//     cutoff flips, so they pull nothing back to beta; sum_k w_k = 1, so
//     d out/d v0 through the candidates is the cotangent itself;
//   * candidates and beta are linear / quadratic in the differences
//     d[k] = v[k+1] - v[k]; their gradients are summed per difference and a
//     difference is turned into its two cells once its last face is done.
// Face o (output index) is centred on cell o + 3 and reads cells o+1 .. o+5,
// so cell o + 1 is final after face o; the sums keep it one face longer
// and emit cell o after face o, so the 8 faces of a chunk starting at an
// even face emit 8 cells starting at an even index (16-byte aligned for the
// TMA unit): row tiles by a bulk tensor store from a swizzled shared tile,
// column tiles (folded y/z, lanes along x) by coalesced stores.  With
// accumulation the previous gradient arrives in the same input stage.
//
// Staging: a ring of 3 stages per warp; stage k carries the cells
// [4 + 8k, 12 + 8k) of v, the cotangents of faces [4 + 8k, 12 + 8k) and
// (accumulating) the old gradient of cells [4 + 8k, 12 + 8k), all completed
// on one mbarrier.  Waits are bounded as in the forward kernel.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include "sweep_march_tma.cuh"
#include "weno_adjoint.cuh"

namespace wsb {

constexpr int kVjpStages = 3;
constexpr int kVjpWarps = 8;  // one CTA per SM: 8 warps x 28 KB of shared memory, 255 registers

struct VjpMarchArgs {
    int kind;           // 0 row tiles, 1 column tiles (as MarchTmaArgs)
    int dimJ, dimU, dimW, uoff, woff;
    int odimU;          // cotangent map dimension of the lane axis (1 or 2)
    int acc;            // add to the gradient already in gv
    int vbytes;         // one v (or old-gradient) tile
    int stage_bytes;    // v (and old gradient) tiles of one stage
    int warp_bytes;     // multiple of 1024
    int ring_off;       // unused (0)
    unsigned tx_bytes;  // bytes one stage receives
    const double* gLp;  // cotangents (ns, c1, c2, V), for the first core face
    const double* gRp;
};

// beta in [2^-100, 2^100): then the one-reciprocal weights, 1/beta and
// their products stay normal (an integer test on the exponent field).
__device__ __forceinline__ bool beta_ok(double b) {
    const unsigned hi = (unsigned)__double2hiint(b);
    return (hi - (923u << 20)) < (200u << 20);
}

// Gradient of one minmod (mm64) with respect to its two arguments:
// c1 = d/d(dl), c2 = d/d(dr).
__device__ __forceinline__ void mm64_grad(double dl, double dr, double& c1, double& c2) {
    const double a = fabs(dl), b = fabs(dr);
    const bool al = a < b;  // dl is the smaller
    const double m = al ? a : b, M = al ? b : a;
    const double t = fma(4.0, m, -M);
    const bool same = ((__double2hiint(dl) ^ __double2hiint(dr)) >= 0) && (t > 0.0);
    const bool pick_t = t < m;  // 4 x_small - x_large, else x_small
    const double cs = same ? (pick_t ? 4.0 : 1.0) : 0.0;
    const double cl = (same && pick_t) ? -1.0 : 0.0;
    c1 = al ? cs : cl;
    c2 = al ? cl : cs;
}

// Expression codes of the one-sided median.
enum : int { kPickW = 0, kPickV0 = 1, kPickNb = 2, kPickMD = 3, kPickUL = 4, kPickLC = 5 };

// Median of one side with the picked expression's code (same values as
// March64::face).  nb: the neighbour (vm1 left, vp1 right).
__device__ __forceinline__ double mp_pick(double x, double v0, double nb, double UL, double MD, double LC, bool pos,
                                          bool nb_first, bool ul_first, int& code) {
    // pos: P1 = max(v0, nb) else min; nb_first: P1 is nb
    const double P1 = nb_first ? nb : v0, P2 = ul_first ? UL : v0;
    const int c1 = nb_first ? kPickNb : kPickV0, c2 = ul_first ? kPickUL : kPickV0;
    const bool sA = (P1 < MD) != pos, sB = (P2 < LC) != pos;
    const double A = sA ? P1 : MD, B = sB ? P2 : LC;
    const int cA = sA ? c1 : kPickMD, cB = sB ? c2 : kPickLC;
    const bool s1 = (x < A) != !pos;
    const double T1 = s1 ? x : A;
    const int cT1 = s1 ? kPickW : cA;
    const bool s2 = (T1 < B) != !pos;
    code = s2 ? cT1 : cB;
    return s2 ? T1 : B;
}

struct MarchVjp {
    March64 f;                          // forward window at face J
    double cA1, cA2, cB1, cB2;          // minmod gradients of mA (e2[J-1], e2[J]) and mB (e2[J], e2[J+1])
    double gdm2, gdm1, gd0, gdp1;       // pending gradients of d[J-2] .. d[J+1]
    double gcm3, gcm2, gcm1, gc0, gcp1; // pending gradients of cells J-3 .. J+1

    __device__ __forceinline__ void init(const MarchArgs& a, double c0, double c1, double c2, double c3,
                                         double c4) {
        f.init(a, c0, c1, c2, c3, c4);
        const double em = (c2 - c1) - (c1 - c0), ez = (c3 - c2) - (c2 - c1);
        mm64_grad(em, ez, cA1, cA2);
        mm64_grad(ez, f.e2, cB1, cB2);
        gdm2 = gdm1 = gd0 = gdp1 = 0.0;
        gcm3 = gcm2 = gcm1 = gc0 = gcp1 = 0.0;
    }

    // Face o (centre J = o + 3): accumulate the pull-back of (gL, gR)
    // through the weights and candidates.  Straight-line code (consecutive
    // faces overlap): the limiter's choice is only recorded -- `pick` gets
    // the codes of the left and right state (0: the WENO value passed
    // through) -- and a state whose limiter returned a bound gets its
    // cotangent routed after the chunk (route_side).  `ok` is false when a
    // beta is outside [2^-100, 2^100): the face then contributes nothing
    // here and is redone after the chunk with the generic pull-back.
    // TENOW: TENO weights (f90:578-606), d_k delta_k / sum d delta with the
    // cutoff flags delta_k of the forward sequence; the flags are constant
    // between cutoff flips, so the weights pull nothing back to beta.
    template <bool MPF, bool TENOW = false>
    __device__ __forceinline__ void face(const MarchArgs& a, double gLin, double gRin, int& pick, bool& ok) {
        const March64& w = f;
        ok = beta_ok(w.b0) && beta_ok(w.b1) && beta_ok(w.b2);
        const double B0 = ok ? w.b0 : 1.0, B1 = ok ? w.b1 : 1.0, B2 = ok ? w.b2 : 1.0;
        double P0, P1, P2;
        if constexpr (TENOW) {
            bool k0, k1, k2;
            ok = teno5_keep(B0, B1, B2, a.wp.teno_ct, k0, k1, k2) && ok;
            P0 = k0 ? 1.0 : 0.0;
            P1 = k1 ? 1.0 : 0.0;
            P2 = k2 ? 1.0 : 0.0;
        } else {
            const double q0 = B0 * B0, q1 = B1 * B1, q2 = B2 * B2;
            P0 = q1 * q2; P1 = q0 * q2; P2 = q0 * q1;
        }
        const double gL = ok ? gLin : 0.0, gR = ok ? gRin : 0.0;
        const double aL0 = a.ucf[12] * P0, aL1 = a.ucf[13] * P1, aL2 = a.ucf[14] * P2;
        const double aR0 = a.ucf[15] * P0, aR1 = a.ucf[16] * P1, aR2 = a.ucf[17] * P2;
        const double SL = (aL0 + aL1) + aL2, SR = (aR0 + aR1) + aR2;
        const double r = rcp1(SL * SR), gSL = SR * r, gSR = SL * r;
        const double wL0 = aL0 * gSL, wL1 = aL1 * gSL, wL2 = aL2 * gSL;
        const double wR0 = aR0 * gSR, wR1 = aR1 * gSR, wR2 = aR2 * gSR;
        // candidate offsets e_k = p_k - v0
        const double eL0 = fma(a.ucf[1], w.d0, a.ucf[0] * w.dp1), eL1 = fma(a.ucf[3], w.dm1, a.ucf[2] * w.d0),
                     eL2 = fma(a.ucf[5], w.dm2, a.ucf[4] * w.dm1);
        const double eR0 = fma(a.ucf[7], w.d0, a.ucf[6] * w.dp1), eR1 = fma(a.ucf[9], w.dm1, a.ucf[8] * w.d0),
                     eR2 = fma(a.ucf[11], w.dm2, a.ucf[10] * w.dm1);
        const double xL = fma(wL0, eL0, fma(wL1, eL1, wL2 * eL2));
        const double xR = fma(wR0, eR0, fma(wR1, eR1, wR2 * eR2));
        double gLw = gL, gRw = gR;
        pick = 0;
        if constexpr (MPF) {
            const double kBetaMP = 4.0 / 3.0;
            const bool up_l = sign_clear(w.dm1), up_r = sign_clear(w.d0);
            const double v0 = w.v0;
            int cl, cr;
            {
                const bool pos = sign_clear(xL);
                const double UL = fma(-2.0, w.d0, v0);
                const double MD = fma(-0.5, w.dm1 + w.mA, v0);
                const double LC = fma(kBetaMP, w.mB, fma(-0.5, w.d0, v0));
                mp_pick(v0 + xL, v0, w.vm1, UL, MD, LC, pos, pos != up_l, pos != up_r, cl);
            }
            {
                const bool pos = sign_clear(xR);
                const double UL = fma(2.0, w.dm1, v0);
                const double MD = fma(0.5, w.d0 - w.mB, v0);
                const double LC = fma(kBetaMP, w.mA, fma(0.5, w.dm1, v0));
                mp_pick(v0 + xR, v0, w.vp1, UL, MD, LC, pos, pos == up_r, pos == up_l, cr);
            }
            gLw = cl == kPickW ? gL : 0.0;
            gRw = cr == kPickW ? gR : 0.0;
            pick = ok ? (cl | (cr << 3)) : 0;
        }
        // weights and candidates
        const double gpL0 = gLw * wL0, gpL1 = gLw * wL1, gpL2 = gLw * wL2;
        const double gpR0 = gRw * wR0, gpR1 = gRw * wR1, gpR2 = gRw * wR2;
        gc0 += gLw + gRw;
        gdp1 = fma(a.ucf[0], gpL0, fma(a.ucf[6], gpR0, gdp1));
        gd0 = fma(a.ucf[1], gpL0, fma(a.ucf[7], gpR0, fma(a.ucf[2], gpL1, fma(a.ucf[8], gpR1, gd0))));
        gdm1 = fma(a.ucf[3], gpL1, fma(a.ucf[9], gpR1, fma(a.ucf[4], gpL2, fma(a.ucf[10], gpR2, gdm1))));
        gdm2 = fma(a.ucf[5], gpL2, fma(a.ucf[11], gpR2, gdm2));
        if constexpr (TENOW) return;
        // d out / d beta_k = -2 w_k (e_k - x) / beta_k
        const double t0 = fma(gpL0, eL0 - xL, gpR0 * (eR0 - xR));
        const double t1 = fma(gpL1, eL1 - xL, gpR1 * (eR1 - xR));
        const double t2 = fma(gpL2, eL2 - xL, gpR2 * (eR2 - xR));
        const double b12 = B1 * B2, b02 = B0 * B2, b01 = B0 * B1;
        const double rB = -2.0 * rcp1(B0 * b12);
        const double gb0 = t0 * (rB * b12), gb1 = t1 * (rB * b02), gb2 = t2 * (rB * b01);
        // beta_0 (d0, dp1): b0 dp1^2 + b1 d0 dp1 + b2 d0^2; beta_1 (dm1, d0); beta_2 (dm2, dm1)
        gdp1 = fma(gb0, fma(2.0 * a.ucf[18], w.dp1, a.ucf[19] * w.d0), gdp1);
        gd0 = fma(gb0, fma(a.ucf[19], w.dp1, 2.0 * a.ucf[20] * w.d0), gd0);
        gd0 = fma(gb1, fma(2.0 * a.ucf[21], w.d0, a.ucf[22] * w.dm1), gd0);
        gdm1 = fma(gb1, fma(a.ucf[22], w.d0, 2.0 * a.ucf[23] * w.dm1), gdm1);
        gdm1 = fma(gb2, fma(2.0 * a.ucf[24], w.dm1, a.ucf[25] * w.dm2), gdm1);
        gdm2 = fma(gb2, fma(a.ucf[25], w.dm1, 2.0 * a.ucf[26] * w.dm2), gdm2);
    }

    // After face o (centre J): d[J-2] is complete, so is cell J-2; returns
    // cell J-3 (= o) and advances to face o+1 with cell J+3 = n.
    __device__ __forceinline__ double advance(const MarchArgs& a, double n) {
        gcm1 += gdm2;
        gcm2 -= gdm2;
        const double out = gcm3;
        const double ne2 = (n - f.vp2) - f.dp1;
        double c1, c2;
        mm64_grad(f.e2, ne2, c1, c2);
        f.push(a, n);
        cA1 = cB1; cA2 = cB2; cB1 = c1; cB2 = c2;
        gdm2 = gdm1; gdm1 = gd0; gd0 = gdp1; gdp1 = 0.0;
        gcm3 = gcm2; gcm2 = gcm1; gcm1 = gc0; gc0 = gcp1; gcp1 = 0.0;
        return out;
    }
};

// Cotangent of one limited state routed to the picked bound expression,
// on cells c[0..4] = J-2 .. J+2 of the face (centre J), added to the
// per-cell sums acc[0..4].  left: nb = J-1, far = J+1; right mirrored.
// MD = (v0 + nb - m)/2, UL = 3 v0 - 2 far, LC = 1.5 v0 - 0.5 far + 4/3 m'
// with m, m' the two minmods; their gradients go through the curvatures
// e2[k] = (v[k+1] - v[k]) - (v[k] - v[k-1]) they picked.
__device__ __forceinline__ void route_side(bool left, int code, double g, const double* c, double* acc) {
    const double kBetaMP = 4.0 / 3.0;
    const int nb = left ? 1 : 3, far = left ? 3 : 1;
    double gmMD = 0.0, gmLC = 0.0;  // cotangents of the minmod in MD and in LC
    switch (code) {
        case kPickV0: acc[2] += g; break;
        case kPickNb: acc[nb] += g; break;
        case kPickMD:
            acc[2] += 0.5 * g;
            acc[nb] += 0.5 * g;
            gmMD = -0.5 * g;
            break;
        case kPickUL:
            acc[2] += 3.0 * g;
            acc[far] -= 2.0 * g;
            break;
        case kPickLC:
            acc[2] += 1.5 * g;
            acc[far] -= 0.5 * g;
            gmLC = kBetaMP * g;
            break;
        default: break;
    }
    // mA = minmod(e2[J-1], e2[J]), mB = minmod(e2[J], e2[J+1]); MD uses mA
    // on the left and mB on the right, LC the other one
    const double gmA = left ? gmMD : gmLC, gmB = left ? gmLC : gmMD;
    if (gmA != 0.0 || gmB != 0.0) {
        const double d0 = c[1] - c[0], d1 = c[2] - c[1], d2 = c[3] - c[2], d3 = c[4] - c[3];
        const double em = d1 - d0, ez = d2 - d1, ep = d3 - d2;
        double a1, a2, b1, b2;
        mm64_grad(em, ez, a1, a2);
        mm64_grad(ez, ep, b1, b2);
        const double ge[3] = {gmA * a1, fma(gmA, a2, gmB * b1), gmB * b2};  // e2[J-1], e2[J], e2[J+1]
        // e2[J+q] = c[q+3] - 2 c[q+2] + c[q+1]
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            acc[q + 2] += ge[q];
            acc[q + 1] -= 2.0 * ge[q];
            acc[q] += ge[q];
        }
    }
}

template <bool MPF, int KIND, bool TENOW = false>
__global__ void __launch_bounds__(kVjpWarps * 32, 1)
    vjp_march_kernel(const __grid_constant__ CUtensorMap tv, const __grid_constant__ CUtensorMap tgL,
                     const __grid_constant__ CUtensorMap tgR, const __grid_constant__ CUtensorMap tgo,
                     const __grid_constant__ CUtensorMap tgs, const __grid_constant__ MarchArgs a,
                     const VjpMarchArgs t, double* __restrict__ gv) {
    constexpr int F = kTmaF, S = kVjpStages;
    constexpr int XW = 34, XS = 1;  // column tiles: 34 cells from one left of column 0
    extern __shared__ __align__(1024) unsigned char smem_vj[];
    unsigned char* base = smem_vj + ((1024u - (smem_u32(smem_vj) & 1023u)) & 1023u);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned char* wbase = base + (size_t)warp * t.warp_bytes;
    // per warp: the cotangent tiles of the S stages (gL, gR: 2048 bytes each,
    // 512-aligned for the swizzle), the field (and old-gradient) tiles of
    // the S stages, then one area that holds the per-lane corrections of a
    // chunk and afterwards (row tiles) the outgoing [32 u][8 cells] tile
    unsigned char* gring = wbase;
    unsigned char* vring = wbase + S * 4096;
    unsigned char* obuf = wbase + S * 4096 + S * t.stage_bytes;   // t.stage_bytes: v (+ old) per stage
    double* slot = (double*)obuf;  // 13 cells f0 .. f0+12 x 32 lanes
    unsigned long long* bars = (unsigned long long*)(base + (size_t)kVjpWarps * t.warp_bytes) + warp * S;
    if (lane == 0) {
        for (int s = 0; s < S; ++s) mbar_init(&bars[s], 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    __syncwarp();
    const long long nwarps = (long long)gridDim.x * kVjpWarps;
    const int ns = (int)a.ns;
    const int o_last = ns - 3;                // one past the last core face
    const long long ncell = a.ns + 6;
    unsigned n_issued = 0, n_waited = 0, n_out = 0;
    bool failed = false;

    auto gstage = [&](unsigned k) { return gring + (size_t)(k % S) * 4096; };
    auto vstage = [&](unsigned k) { return vring + (size_t)(k % S) * t.stage_bytes; };
    auto issue = [&](unsigned k, int c, int u0, int w, int v) {
        if (lane == 0) {
            unsigned long long* bar = &bars[k % S];
            unsigned char* sp = gstage(k);
            unsigned char* vp = vstage(k);
            const int J0 = 4 + F * c;
            const int cU = t.uoff + u0, cW = t.woff + w;
            mbar_arrive_expect_tx(bar, t.tx_bytes);
            const int o1 = t.odimU == 1 ? u0 : w, o2 = t.odimU == 2 ? u0 : w;
            tma_load_4d(sp, &tgL, bar, J0, o1, o2, v);
            tma_load_4d(sp + 2048, &tgR, bar, J0, o1, o2, v);
            const int c0 = t.dimJ == 0 ? J0 : (t.dimU == 0 ? cU : cW);
            const int c1 = t.dimJ == 1 ? J0 : (t.dimU == 1 ? cU : cW);
            const int c2 = t.dimJ == 2 ? J0 : (t.dimU == 2 ? cU : cW);
            tma_load_4d(vp, &tv, bar, c0, c1, c2, v);
            if (t.acc) tma_load_4d(vp + t.vbytes, &tgo, bar, c0, c1, c2, v);
        }
    };
    auto wait_stage = [&](unsigned k) -> bool {
        if (!mbar_wait(&bars[k % S], (k / S) & 1u)) return false;
        n_waited = k + 1;
        return true;
    };
    auto voff = [&](int p) -> unsigned {  // position p of this lane's column in a v / old-gradient tile
        if constexpr (KIND == 0) return swz<double>((unsigned)lane, (unsigned)p);
        else return (unsigned)((p * XW + lane + XS) * 8);
    };
    auto cell = [&](unsigned k, int p) -> double { return *(const double*)(vstage(k) + voff(p)); };
    auto oldg = [&](unsigned k, int p) -> double {
        return t.acc ? *(const double*)(vstage(k) + t.vbytes + voff(p)) : 0.0;
    };
    auto cot = [&](unsigned k, int arr, int i) -> double {
        return *(const double*)(gstage(k) + arr * 2048 + swz<double>((unsigned)lane, (unsigned)i));
    };

    for (long long item = (long long)blockIdx.x * kVjpWarps + warp; item < a.n_items && !failed; item += nwarps) {
        long long tt = item;
        const int ut = (int)(tt % a.n_ut);
        tt /= a.n_ut;
        const int wv = (int)(tt % a.Nw);
        const int vv = (int)(tt / a.Nw);
        const int u0 = ut * 32;
        const bool live = u0 + lane < a.Nu;
        const int uc = live ? u0 + lane : a.Nu - 1;
        const double* col = (const double*)a.in + a.in_off + uc * a.sU + wv * a.sW + vv * a.sV;
        double* gcol = gv + a.in_off + uc * a.sU + wv * a.sW + vv * a.sV;
        const int nch = (ns + 1) / F + 1;       // chunks until cell ns+5 is out
        const int ntiles = nch + 1;
        const unsigned k0 = n_issued;
        for (int k = 0; k < ntiles && k < S; ++k) issue(k0 + k, k, u0, wv, vv);
        n_issued += (ntiles < S ? ntiles : S);
        if (!wait_stage(k0)) { failed = true; break; }

        // cells 0..3 receive nothing; face 3 (cells 4..8 = stage 0 positions
        // 0..4) starts the window
        if (live && !t.acc)
            for (int q = 0; q < 4; ++q) gcol[q * a.sJ] = 0.0;
        MarchVjp m;
        m.init(a, cell(k0, 0), cell(k0, 1), cell(k0, 2), cell(k0, 3), cell(k0, 4));
        {
            const long long oi = 3 + (long long)uc * a.oU + wv * a.oW + vv * a.oV;
            const double gL = live ? __ldg(t.gLp + oi) : 0.0, gR = live ? __ldg(t.gRp + oi) : 0.0;
            int pk;
            bool ok;
            m.face<MPF, TENOW>(a, gL, gR, pk, ok);
            if (pk || (!ok && live)) {
                // cells 3..9 of the column = J-3 .. J+3 of face 3 (J = 6)
                double c7[7], acc7[7] = {0, 0, 0, 0, 0, 0, 0};
                for (int q = 0; q < 7; ++q) c7[q] = __ldg(col + (3 + q) * a.sJ);
                if (!ok) {
                    Coef<5> cf;
                    for (int q = 0; q < 6; ++q) { cf.pL[q] = a.ucf[q]; cf.pR[q] = a.ucf[6 + q]; }
                    for (int q = 0; q < 3; ++q) { cf.dL[q] = a.ucf[12 + q]; cf.dR[q] = a.ucf[15 + q]; }
                    for (int q = 0; q < 9; ++q) cf.b[q] = a.ucf[18 + q];
                    face_vjp<5>(c7 + 3, cf, JS, a.wp.eps, 0.0, MPF, gL, gR, acc7);
                } else {
                    route_side(true, pk & 7, gL, c7 + 1, acc7 + 1);
                    route_side(false, pk >> 3, gR, c7 + 1, acc7 + 1);
                }
                // acc7[q] is cell J-3+q; pending: J-3 .. J+1, and J+2 through d[J+1]
                m.gcm3 += acc7[0];
                m.gcm2 += acc7[1];
                m.gcm1 += acc7[2];
                m.gc0 += acc7[3];
                m.gcp1 += acc7[4] + acc7[5];
                m.gdp1 += acc7[5];
            }
            (void)m.advance(a, cell(k0, 5));  // cell 3: nothing
        }
        // chunk c: faces f0 .. f0+7 (f0 = 4 + 8c); face f0+i pushes cell
        // f0+i+6 = stage c position 6+i (i < 2) or stage c+1 position i-2,
        // and emits cell f0+i = position i of stage c's tiles
        for (int c = 0; c < nch; ++c) {
            const unsigned kc = k0 + c;
            if (!wait_stage(kc + 1)) { failed = true; break; }
            const int f0 = 4 + F * c;
            if constexpr (KIND == 0) {
                if (n_out >= 1) {
                    if (lane == 0) bulk_wait_read0();
                    __syncwarp();
                }
            }
            double outv[F];
            unsigned long long picks = 0;
            unsigned bad = 0;
#pragma unroll
            for (int i = 0; i < F; ++i) {
                const int o = f0 + i;
                const bool valid = live && o < o_last;
                const double gL = valid ? cot(kc, 0, i) : 0.0;
                const double gR = valid ? cot(kc, 1, i) : 0.0;
                int pk;
                bool ok;
                m.face<MPF, TENOW>(a, gL, gR, pk, ok);
                picks |= (unsigned long long)(valid ? pk : 0) << (6 * i);
                bad |= (ok || !valid) ? 0u : (1u << i);
                outv[i] = m.advance(a, (i < 2) ? cell(kc, 6 + i) : cell(kc + 1, i - 2)) + oldg(kc, i);
            }
            if (__any_sync(0xffffffffu, picks != 0ull || bad != 0u)) {
                // (the area is the row tiles' outgoing tile too; its last store
                // has been read: waited at the start of the chunk)
                // limited states and faces outside the one-reciprocal range:
                // their pull-backs go to per-lane slots of cells f0 .. f0+12
#pragma unroll
                for (int k = 0; k < 13; ++k) slot[k * 32 + lane] = 0.0;
                for (int i = 0; i < F; ++i) {
                    const int pk = (int)((picks >> (6 * i)) & 63ull);
                    const bool redo = (bad >> i) & 1u;
                    if (!pk && !redo) continue;
                    // cells f0+i .. f0+i+6 = J-3 .. J+3 (J = f0+i+3)
                    double c7[7], acc7[7] = {0, 0, 0, 0, 0, 0, 0};
                    for (int q = 0; q < 7; ++q) {
                        const int k = i + q;  // cell f0 + k: tile c below 8, tile c+1 from 8
                        c7[q] = k < 8 ? cell(kc, k) : cell(kc + 1, k - 8);
                    }
                    const double gL = cot(kc, 0, i), gR = cot(kc, 1, i);
                    if (redo) {
                        Coef<5> cf;
                        for (int q = 0; q < 6; ++q) { cf.pL[q] = a.ucf[q]; cf.pR[q] = a.ucf[6 + q]; }
                        for (int q = 0; q < 3; ++q) { cf.dL[q] = a.ucf[12 + q]; cf.dR[q] = a.ucf[15 + q]; }
                        for (int q = 0; q < 9; ++q) cf.b[q] = a.ucf[18 + q];
                        face_vjp<5>(c7 + 3, cf, TENOW ? TENO : JS, a.wp.eps, a.wp.teno_ct, MPF, gL, gR, acc7);
                    } else {
                        route_side(true, pk & 7, gL, c7 + 1, acc7 + 1);
                        route_side(false, pk >> 3, gR, c7 + 1, acc7 + 1);
                    }
                    for (int q = 0; q < 7; ++q)
                        if (i + q < 13) slot[(i + q) * 32 + lane] += acc7[q];
                }
                // slots 0..7 are this chunk's emitted cells, 8..12 the pending
                // cells J-3 .. J+1 of the next face
#pragma unroll
                for (int k = 0; k < F; ++k) outv[k] += slot[k * 32 + lane];
                m.gcm3 += slot[8 * 32 + lane];
                m.gcm2 += slot[9 * 32 + lane];
                m.gcm1 += slot[10 * 32 + lane];
                m.gc0 += slot[11 * 32 + lane];
                m.gcp1 += slot[12 * 32 + lane];
            }
            if constexpr (KIND == 0) {
                unsigned char* ob = obuf;
#pragma unroll
                for (int i = 0; i < F; ++i) *(double*)(ob + swz<double>((unsigned)lane, (unsigned)i)) = outv[i];
                fence_async_shared();
                __syncwarp();
                if (lane == 0) {
                    const int cU = t.uoff + u0, cW = t.woff + wv;
                    const int c0 = t.dimJ == 0 ? f0 : (t.dimU == 0 ? cU : cW);
                    const int c1 = t.dimJ == 1 ? f0 : (t.dimU == 1 ? cU : cW);
                    const int c2 = t.dimJ == 2 ? f0 : (t.dimU == 2 ? cU : cW);
                    tma_store_4d(&tgs, ob, c0, c1, c2, vv);
                    bulk_commit();
                }
                ++n_out;
            } else {
#pragma unroll
                for (int i = 0; i < F; ++i) {
                    const long long J = (long long)f0 + i;
                    if (live && J < ncell) gcol[J * a.sJ] = outv[i];
                }
            }
            __syncwarp();
            if (c + S < ntiles) {
                issue(kc + S, c + S, u0, wv, vv);
                ++n_issued;
            }
        }
        if (failed) break;
    }
    if (failed) {
        for (unsigned k = n_waited; k < n_issued; ++k) mbar_wait(&bars[k % S], (k / S) & 1u);
    }
    if (lane == 0) bulk_wait_all();
    __syncwarp();
}

// Host side: the marching adjoint for FP64 WENO5-JS with face-independent
// coefficients.  Returns 1003 (unsupported) when a tensor map cannot be
// made (16-byte alignment of bases and strides, an even face count); the
// caller then runs vjp_kernel.  gv must already hold what is to be added to
// when acc is set.
inline int launch_vjp_march(const long long E[3], const SweepGeom& g, int dir, bool folded, bool mp, bool acc,
                            const double* v, const double* ucf, const WenoParams& wp, const double* gL,
                            const double* gR, double* gv, cudaStream_t st, int sms) {
    EncodeTiledFn enc = encode_tiled_fn();
    if (!enc) return 1003;
    if ((((uintptr_t)v) | ((uintptr_t)gL) | ((uintptr_t)gR) | ((uintptr_t)gv)) & 15) return 1003;
    if (g.ns < 8 || (g.ns & 1) || g.nc < 1) return 1003;
    MarchArgs a = make_march_args(g, v, nullptr, nullptr, wp, ucf);
    VjpMarchArgs t{};
    const bool kind1 = folded && dir != 0;
    t.kind = kind1 ? 1 : 0;
    t.acc = acc ? 1 : 0;
    t.gLp = gL;
    t.gRp = gR;
    cuuint64_t dims[4], strides[3];
    cuuint32_t box[4], estr[4] = {1, 1, 1, 1};
    if (!folded) {
        dims[0] = g.ns + 6; dims[1] = g.c1; dims[2] = g.c2; dims[3] = g.nv;
        t.dimJ = 0; t.dimU = 1; t.dimW = 2; t.uoff = 0; t.woff = 0;
    } else {
        dims[0] = E[0]; dims[1] = E[1]; dims[2] = E[2]; dims[3] = g.nv;
        if (dir == 0) { t.dimJ = 0; t.dimU = 1; t.dimW = 2; t.uoff = 3; t.woff = 3; }
        else if (dir == 1) { t.dimJ = 1; t.dimU = 0; t.dimW = 2; t.uoff = 2; t.woff = 3; }
        else { t.dimJ = 2; t.dimU = 0; t.dimW = 1; t.uoff = 2; t.woff = 3; }
    }
    CUtensorMapSwizzle swz;
    if (!kind1) {
        box[0] = kTmaF; box[1] = 32; box[2] = 1; box[3] = 1;
        swz = CU_TENSOR_MAP_SWIZZLE_64B;
        t.vbytes = 2048;
    } else {
        box[0] = 34; box[1] = 1; box[2] = 1; box[3] = 1;
        box[t.dimJ] = kTmaF;
        swz = CU_TENSOR_MAP_SWIZZLE_NONE;
        t.vbytes = kTmaF * 34 * 8;
    }
    strides[0] = dims[0] * 8;
    strides[1] = dims[0] * dims[1] * 8;
    strides[2] = dims[0] * dims[1] * dims[2] * 8;
    if (strides[0] % 16) return 1003;
    if ((t.kind == 1) != (a.sU == 1)) return 1003;
    const CUtensorMapDataType dt = CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
    CUtensorMap mv, mL, mR, mo, ms;
    std::memset(&mo, 0, sizeof(mo));
    std::memset(&ms, 0, sizeof(ms));
    auto make = [&](CUtensorMap* m, const void* p, const cuuint64_t* d, const cuuint64_t* s2, const cuuint32_t* b,
                    CUtensorMapSwizzle z) {
        return enc(m, dt, 4, (void*)p, d, s2, b, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, z,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
    };
    if (!make(&mv, v, dims, strides, box, swz)) return 1003;
    if (acc && !make(&mo, gv, dims, strides, box, swz)) return 1003;
    if (!kind1) {
        // the store map ends at the last column of the sweep, so the lanes
        // past it (the last 32-column tile) write nothing
        cuuint64_t sd[4] = {dims[0], dims[1], dims[2], dims[3]};
        sd[t.dimU] = (cuuint64_t)(t.uoff + a.Nu);
        if (!make(&ms, gv, sd, strides, box, swz)) return 1003;
    }
    cuuint64_t od[4] = {(cuuint64_t)g.ns, (cuuint64_t)g.c1, (cuuint64_t)g.c2, (cuuint64_t)g.nv};
    cuuint64_t os[3] = {(cuuint64_t)g.ns * 8, (cuuint64_t)(g.ns * g.c1) * 8, (cuuint64_t)(g.ns * g.c1 * g.c2) * 8};
    cuuint32_t ob[4] = {kTmaF, 1, 1, 1};
    t.odimU = (a.oU == g.ns) ? 1 : 2;
    ob[t.odimU] = 32;
    if (!make(&mL, gL, od, os, ob, CU_TENSOR_MAP_SWIZZLE_64B) || !make(&mR, gR, od, os, ob, CU_TENSOR_MAP_SWIZZLE_64B))
        return 1003;
    // one item per 32-column tile of a whole column
    a.seg = (int)g.ns;
    a.n_seg = 1;
    a.n_items = (long long)a.n_ut * a.Nw * a.NV;
    t.stage_bytes = t.vbytes * (acc ? 2 : 1);   // field (+ old gradient) tiles of one stage
    t.ring_off = 0;
    t.warp_bytes = ((kVjpStages * 4096 + kVjpStages * t.stage_bytes + 13 * 32 * 8 + 1023) / 1024) * 1024;
    t.tx_bytes = (unsigned)(2 * 2048 + t.vbytes * (acc ? 2 : 1));
    const size_t smem = 1024 + (size_t)kVjpWarps * t.warp_bytes + (size_t)kVjpWarps * kVjpStages * 8;
    using KFn = void (*)(CUtensorMap, CUtensorMap, CUtensorMap, CUtensorMap, CUtensorMap, MarchArgs, VjpMarchArgs,
                         double*);
    const bool teno = wp.scheme == TENO;
    static const KFn table[2][2][2] = {
        {{vjp_march_kernel<false, 0, false>, vjp_march_kernel<false, 1, false>},
         {vjp_march_kernel<true, 0, false>, vjp_march_kernel<true, 1, false>}},
        {{vjp_march_kernel<false, 0, true>, vjp_march_kernel<false, 1, true>},
         {vjp_march_kernel<true, 0, true>, vjp_march_kernel<true, 1, true>}}};
    const KFn kfn = table[teno ? 1 : 0][mp ? 1 : 0][kind1 ? 1 : 0];
    cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int occ = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kfn, kVjpWarps * 32, smem);
    if (occ < 1) return 1003;
    long long blocks = (a.n_items + kVjpWarps - 1) / kVjpWarps;
    const long long cap = (long long)sms * occ;
    if (blocks > cap) blocks = cap;
    kfn<<<(unsigned)blocks, kVjpWarps * 32, smem, st>>>(mv, mL, mR, mo, ms, a, t, gv);
    return 0;
}

}  // namespace wsb
