// sweep_tma.cuh -- pipelined reconstruction sweep (the hot path).
//
// Work decomposition.  A sweep reconstructs vL/vR at `nf` faces along the
// sweep axis for every cross-section column (a, b, v).  A CTA owns a tile of
// TJ consecutive faces (one thread per face) and walks over groups of
// columns.  Each thread loads its face's coefficients (poly, d, beta:
// indexed by the face only, f90:535-555) into registers once and reuses
// them for every column, so the coefficient arrays cost nothing per point.
//
// Staging.  The stencil window of a column group (TJ + 2H values along the
// sweep per column, H = stencil half width) is copied global -> shared by a
// STAGES-deep asynchronous pipeline, so HBM reads stay in flight while the
// FP64 arithmetic of the previous group runs.  Two tile shapes:
//   KIND 0  sweep axis contiguous in memory (v_rs_ws in any direction, or
//           v_vf in x): the tile is R rows of the window, thread f reads
//           row[f .. f+2H] -- consecutive threads, consecutive words.
//   KIND 1  sweep axis strided (the folded y/z sweeps read v_vf directly):
//           the tile is the window x XW consecutive x-columns, row pitch
//           XW+1 so a warp reading one column at 32 consecutive faces hits
//           32 distinct banks; the y/z reshape is thereby folded away.
// Stores go straight from registers to vL/vR, whose face index is the
// fastest one, so every warp store is one contiguous segment.
#pragma once

#include <cuda_runtime.h>

#include "weno_math.cuh"
#include "sweep_generic.cuh"

namespace wsb {

struct FastArgs {
    const void* in;
    void* vL;
    void* vR;
    CoefPtrs cp;
    WenoParams wp;
    long long ns, nc;
    int o_first;      // first face handled (0 for WENO3, 3 otherwise)
    int nf;           // faces handled
    int TJ;           // faces per tile
    int n_jt;         // number of face tiles
    int SW;           // window length along the sweep (TJ + 2H)
    int pitch;        // KIND 0: smem row pitch (elements); KIND 1: XW + 1
    int U;            // columns per group (R for KIND 0, XW for KIND 1)
    // Column groups: U consecutive values of cross axis u, at fixed (w, v).
    int Nu, Nw, NV, n_ut;
    long long n_groups;
    long long sJ;          // input stride along the sweep
    long long sU, sWw, sV; // input strides of u, w, v
    long long in_off;      // input offset of (J=0, u=0, w=0, v=0)
    long long o_sU, o_sW, o_sV;  // output strides of u, w, v
    // Face-independent coefficients (laid out as Coef<ORDER>), used by the
    // UNI kernel instances straight from the kernel-parameter (constant)
    // bank instead of 27-56 registers per thread.
    double ucf[56];
};

template <typename T>
__device__ __forceinline__ void cp_async_elem(T* smem, const T* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    if constexpr (sizeof(T) == 8) {
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem));
    } else {
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem));
    }
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

template <int ORDER, bool MPF>
struct Halo {
    static constexpr int H0 = (ORDER - 1) / 2;
    static constexpr int H = (MPF && H0 < 2) ? 2 : H0;
};

struct GroupInfo {
    long long in0;   // input offset of (J = 0, first column)
    long long out0;  // output offset of (face 0, first column)
    int ucnt;        // valid columns in the group
};

__device__ __forceinline__ GroupInfo group_info(const FastArgs& a, long long grp) {
    const unsigned g = (unsigned)grp;
    const unsigned ut = g % (unsigned)a.n_ut;
    const unsigned t = g / (unsigned)a.n_ut;
    const unsigned w = t % (unsigned)a.Nw;
    const unsigned v = t / (unsigned)a.Nw;
    const int u0 = (int)ut * a.U;
    GroupInfo gi;
    gi.ucnt = min(a.U, a.Nu - u0);
    gi.in0 = a.in_off + (long long)u0 * a.sU + (long long)w * a.sWw + (long long)v * a.sV;
    gi.out0 = (long long)u0 * a.o_sU + (long long)w * a.o_sW + (long long)v * a.o_sV;
    return gi;
}

template <typename T, int KIND, int XW>
__device__ __forceinline__ void issue_stage(const FastArgs& a, T* buf, long long grp, int J0, int Jcnt) {
    const T* __restrict__ in = (const T*)a.in;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const GroupInfo gi = group_info(a, grp);
    if constexpr (KIND == 0) {
        for (int r = warp; r < gi.ucnt; r += nw) {
            const T* src = in + gi.in0 + (long long)r * a.sU + J0;
            T* dst = buf + r * a.pitch;
            for (int j = lane; j < Jcnt; j += 32) cp_async_elem(dst + j, src + j);
        }
    } else {
        // rows of XW consecutive u values; 32/XW rows per warp instruction
        constexpr int RPW = 32 / XW;
        const int k = lane % XW;
        if (k < gi.ucnt) {
            const T* src = in + gi.in0 + k;
            for (int j = warp * RPW + lane / XW; j < Jcnt; j += nw * RPW)
                cp_async_elem(buf + j * a.pitch + k, src + (long long)(J0 + j) * a.sJ);
        }
    }
}

// Views of a staged column group seen from one face: element q (stencil
// offset from the face's centre cell) of column k.
template <typename T>
struct LinearTile {  // plain row-major staging (cp.async, or TMA without swizzle)
    const T* p;      // centre element of column 0
    int js, ks;      // strides along the sweep and between columns
    __device__ __forceinline__ T operator()(int q, int k) const { return p[k * ks + q * js]; }
    __device__ __forceinline__ void pair(int q, int k, T& x, T& y) const {
        x = p[k * ks + q * js];
        y = p[(k + 1) * ks + q * js];
    }
};

template <typename T>
struct Swz128Tile {  // TMA box of 128-byte rows in the 128B swizzle pattern
    const unsigned char* base;  // stage base (1024-byte aligned)
    int row0;                   // window row of the face's centre cell
    __device__ __forceinline__ T operator()(int q, int k) const {
        const int row = row0 + q;
        const int byte = k * (int)sizeof(T);
        return *reinterpret_cast<const T*>(base + row * 128 + ((((byte >> 4) ^ (row & 7))) << 4) + (byte & 15));
    }
    // columns k and k+1 (k even, doubles): one 16-byte chunk, one LDS.128
    __device__ __forceinline__ void pair(int q, int k, T& x, T& y) const {
        const int row = row0 + q;
        const double2 v = *reinterpret_cast<const double2*>(base + row * 128 + ((((k >> 1) ^ (row & 7))) << 4));
        x = v.x;
        y = v.y;
    }
};

// Reconstruct columns [kb, ke) of one staged group for this thread's face
// (index o); the output of column k goes to oidx0 + k*o_sU.
// SCH >= 0 fixes the weight family at compile time (0 = JS, the common
// case, so the other families' code is not carried); -1 reads it at run time.
template <int ORDER, bool MPF, typename T, int SCH, typename Tile>
__device__ __forceinline__ void compute_columns(const FastArgs& a, const Coef<ORDER>& cf, const Tile& t, int kb,
                                                int ke, long long oidx0, long long o,
                                                const PolyF<ORDER>* pf = nullptr) {
    const int scheme = (SCH >= 0) ? SCH : a.wp.scheme;
    // FP32-bulk with JS weights: the conversion-free mixed form
    constexpr bool MIXED = (sizeof(T) == 4) && SCH == 0 && (ORDER == 5 || ORDER == 7);
    T* __restrict__ vL = (T*)a.vL;
    T* __restrict__ vR = (T*)a.vR;
    long long oidx = oidx0 + (long long)kb * a.o_sU;
    for (int k = kb; k < ke; ++k, oidx += a.o_sU) {
        T Lt, Rt;
        if constexpr (ORDER == 3) {
            double L, R;
            weno3_face((double)t(-1, k), (double)t(0, k), (double)t(1, k), cf, scheme, a.wp.eps, L, R);
            Lt = (T)L;
            Rt = (T)R;
            if (MPF && o >= 3 && o <= a.ns - 4) MP<T>::apply(t(-2, k), t(-1, k), t(0, k), t(1, k), t(2, k), Lt, Rt);
        } else if constexpr (ORDER == 5) {
            const T m2 = t(-2, k), m1 = t(-1, k), z0 = t(0, k), p1 = t(1, k), p2 = t(2, k);
            bool done = false;
            if constexpr (MIXED) done = weno5_js_mixed(m2, m1, z0, p1, p2, cf, *pf, a.wp.eps, Lt, Rt);
            if (!done) {
                double L, R;
                weno5_face<T>((double)m2, (double)m1, (double)z0, (double)p1, (double)p2, cf, scheme, a.wp.eps,
                              a.wp.teno_ct, L, R);
                Lt = (T)L;
                Rt = (T)R;
            }
            if (MPF) MP<T>::apply(m2, m1, z0, p1, p2, Lt, Rt);
        } else {
            bool done = false;
            if constexpr (MIXED) {
                float s7[7];
#pragma unroll
                for (int q = 0; q < 7; ++q) s7[q] = t(q - 3, k);
                done = weno7_js_mixed(s7 + 3, cf, *pf, a.wp.eps, Lt, Rt);
            }
            if (!done) {
                double s7[7];
#pragma unroll
                for (int q = 0; q < 7; ++q) s7[q] = (double)t(q - 3, k);
                double L, R;
                weno7_face<T>(s7 + 3, cf, scheme, a.wp.eps, a.wp.teno_ct, L, R);
                Lt = (T)L;
                Rt = (T)R;
            }
            if (MPF) MP<T>::apply(t(-2, k), t(-1, k), t(0, k), t(1, k), t(2, k), Lt, Rt);
        }
        vL[oidx] = Lt;
        vR[oidx] = Rt;
    }
}

// WENO5-JS (+MP) on columns [kb, ke), two columns per iteration: both
// columns' straight-line fast paths are issued before either fallback
// check, so the compiler interleaves two independent dependency chains.
// Pairs start at an even column (the swizzled tile serves a pair with one
// 16-byte load); a pair member outside [kb, ke) is computed but not stored.
template <bool MPF, typename Tile>
__device__ __forceinline__ void compute_js5_pairs(const FastArgs& a, const Coef<5>& cf, const Tile& t, int kb,
                                                  int ke, long long oidx0) {
    double* __restrict__ vL = (double*)a.vL;
    double* __restrict__ vR = (double*)a.vR;
    const double eps = a.wp.eps;
    for (int k = kb & ~1; k < ke; k += 2) {
        double A[5], B[5];
#pragma unroll
        for (int q = 0; q < 5; ++q) t.pair(q - 2, k, A[q], B[q]);
        double LA, RA, LB, RB;
        const bool okA = weno5_js_fast<double>(A[0], A[1], A[2], A[3], A[4], cf, eps, LA, RA);
        const bool okB = weno5_js_fast<double>(B[0], B[1], B[2], B[3], B[4], cf, eps, LB, RB);
        if (!okA) weno5_face<double>(A[0], A[1], A[2], A[3], A[4], cf, JS, eps, a.wp.teno_ct, LA, RA);
        if (!okB) weno5_face<double>(B[0], B[1], B[2], B[3], B[4], cf, JS, eps, a.wp.teno_ct, LB, RB);
        if (MPF) {
            mp_limit(A[0], A[1], A[2], A[3], A[4], LA, RA);
            mp_limit(B[0], B[1], B[2], B[3], B[4], LB, RB);
        }
        const long long oa = oidx0 + (long long)k * a.o_sU;
        if (k >= kb) {
            vL[oa] = LA;
            vR[oa] = RA;
        }
        if (k + 1 < ke) {
            vL[oa + a.o_sU] = LB;
            vR[oa + a.o_sU] = RB;
        }
    }
}

template <int ORDER, bool MPF, typename T, int KIND, int XW, int STAGES, int SCH>
__global__ void __launch_bounds__(256, (ORDER == 7 ? 1 : 2)) sweep_fast_kernel(const FastArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* smem = reinterpret_cast<T*>(smem_raw);
    constexpr int H = Halo<ORDER, MPF>::H;
    const int stage_elems = (KIND == 0) ? a.U * a.pitch : a.SW * a.pitch;

    const int jt = blockIdx.x % a.n_jt;
    const long long g0 = blockIdx.x / a.n_jt;
    const long long gstep = gridDim.x / a.n_jt;
    const int f_first = jt * a.TJ;                 // first face (0-based among the nf handled)
    const int f_cnt = min(a.TJ, a.nf - f_first);   // faces in this tile
    const int o_begin = a.o_first + f_first;       // face index o of the tile's first face
    const int J0 = o_begin + 3 - H;                // first input index of the window
    const int Jcnt = f_cnt + 2 * H;                // window length (always inside [0, ns+6))

    const int f = threadIdx.x;                     // tile-local face
    const bool active = f < f_cnt;
    const long long o = o_begin + f;
    long long cidx = o - 3;
    cidx = cidx < 0 ? 0 : (cidx > a.nc - 1 ? a.nc - 1 : cidx);
    Coef<ORDER> cf;
    if (active) {
        if (a.cp.polyL) cf.load(a.cp.polyL, a.cp.polyR, a.cp.dL, a.cp.dR, a.cp.beta, a.nc, cidx);
        else cf = *reinterpret_cast<const Coef<ORDER>*>(a.ucf);  // face-independent coefficients
    }
    PolyF<ORDER> pf;  // float polynomial coefficients of the FP32-bulk form
    if constexpr (sizeof(T) == 4) pf.from(cf);

    const int js = (KIND == 0) ? 1 : a.pitch;     // smem stride along the sweep
    const int ks = (KIND == 0) ? a.pitch : 1;     // smem stride between columns

#pragma unroll
    for (int s = 0; s < STAGES - 1; ++s) {
        const long long gg = g0 + s * gstep;
        if (gg < a.n_groups) issue_stage<T, KIND, XW>(a, smem + s * stage_elems, gg, J0, Jcnt);
        cp_async_commit();
    }
    long long grp = g0;
    for (int it = 0; grp < a.n_groups; ++it, grp += gstep) {
        cp_async_wait<STAGES - 2>();
        __syncthreads();
        {
            const long long gg = grp + (long long)(STAGES - 1) * gstep;
            if (gg < a.n_groups)
                issue_stage<T, KIND, XW>(a, smem + ((it + STAGES - 1) % STAGES) * stage_elems, gg, J0, Jcnt);
            cp_async_commit();
        }
        if (!active) continue;
        const GroupInfo gi = group_info(a, grp);
        const LinearTile<T> tile{smem + (it % STAGES) * stage_elems + (f + H) * js, js, ks};
        compute_columns<ORDER, MPF, T, SCH>(a, cf, tile, 0, gi.ucnt, gi.out0 + o, o, &pf);
    }
    cp_async_wait<0>();
}

template <int ORDER, bool MPF, typename T, int KIND, int XW, int STAGES, int SCH>
int launch_fast_s(FastArgs a, cudaStream_t st, int sms) {
    const int threads = ((a.TJ + 31) / 32) * 32;
    size_t smem;
    if (KIND == 0) {
        a.pitch = a.SW;
        smem = (size_t)STAGES * a.U * a.pitch * sizeof(T);
    } else {
        a.U = XW;
        a.pitch = XW + 1;
        smem = (size_t)STAGES * a.SW * a.pitch * sizeof(T);
    }
    a.n_ut = (a.Nu + a.U - 1) / a.U;
    a.n_groups = (long long)a.n_ut * a.Nw * a.NV;
    auto kfn = sweep_fast_kernel<ORDER, MPF, T, KIND, XW, STAGES, SCH>;
    static bool attr_set = false;
    if (!attr_set) {
        cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        attr_set = true;
    }
    int occ = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kfn, threads, smem);
    if (occ < 1) occ = 1;
    long long per_jt = ((long long)sms * occ) / a.n_jt;
    if (per_jt < 1) per_jt = 1;
    if (per_jt > a.n_groups) per_jt = a.n_groups;
    const long long grid = per_jt * a.n_jt;
    kfn<<<(unsigned)grid, threads, smem, st>>>(a);
    return 0;
}

template <int ORDER, bool MPF, typename T, int KIND, int XW, int STAGES>
int launch_fast_t(FastArgs a, cudaStream_t st, int sms) {
    if (a.wp.scheme == JS) return launch_fast_s<ORDER, MPF, T, KIND, XW, STAGES, 0>(a, st, sms);
    return launch_fast_s<ORDER, MPF, T, KIND, XW, STAGES, -1>(a, st, sms);
}

// Returns WENO_SB_ERR_UNSUPPORTED (1003) when the layout does not fit this
// kernel, so the caller can fall back to the general-stride one.
template <typename T>
int launch_tma_sweep(const long long E[3], const SweepGeom& g, int dir, bool folded, int order, bool mp,
                     const T* in, T* vL, T* vR, const CoefPtrs& cp, const WenoParams& wp, cudaStream_t st,
                     const double* ucf = nullptr) {
    (void)E;
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 148;
    }
    if (g.c1 > (1LL << 30) || g.c2 > (1LL << 30) || g.cols > (1LL << 31)) return 1003;
    FastArgs a{};
    a.in = in;
    a.vL = vL;
    a.vR = vR;
    a.cp = cp;
    a.wp = wp;
    if (ucf) {
        for (int q = 0; q < 56; ++q) a.ucf[q] = ucf[q];
        a.cp = CoefPtrs{nullptr, nullptr, nullptr, nullptr, nullptr};
    }
    a.ns = g.ns;
    a.nc = g.nc;
    a.o_first = (order == 3) ? 0 : 3;
    a.nf = (int)((order == 3) ? g.ns : g.nc);
    const int Hh = ((order - 1) / 2 < 2 && mp) ? 2 : (order - 1) / 2;
    const int maxTJ = 224;
    a.n_jt = (a.nf + maxTJ - 1) / maxTJ;
    a.TJ = (a.nf + a.n_jt - 1) / a.n_jt;
    a.SW = a.TJ + 2 * Hh;
    a.sJ = g.sJ;
    a.sV = g.sV;
    a.in_off = g.in_off;
    a.o_sV = g.ns * g.c1 * g.c2;
    const bool kind1 = folded && dir != 0;
    if (!kind1 || dir == 1) {
        // u = a (first cross axis), w = b
        a.Nu = (int)g.c1; a.Nw = (int)g.c2; a.sU = g.sA; a.sWw = g.sB;
        a.o_sU = g.ns; a.o_sW = g.ns * g.c1;
    } else {
        // folded z: u = b (x, unit stride), w = a (y)
        a.Nu = (int)g.c2; a.Nw = (int)g.c1; a.sU = g.sB; a.sWw = g.sA;
        a.o_sU = g.ns * g.c1; a.o_sW = g.ns;
    }
    a.U = 8;
    a.NV = (int)g.nv;
    constexpr int S0 = 4, S1 = 3;
    const int key = order * 4 + (mp ? 2 : 0) + (kind1 ? 1 : 0);
    switch (key) {
        case 12: return launch_fast_t<3, false, T, 0, 16, S0>(a, st, sms);
        case 13: return launch_fast_t<3, false, T, 1, 16, S1>(a, st, sms);
        case 14: return launch_fast_t<3, true, T, 0, 16, S0>(a, st, sms);
        case 15: return launch_fast_t<3, true, T, 1, 16, S1>(a, st, sms);
        case 20: return launch_fast_t<5, false, T, 0, 16, S0>(a, st, sms);
        case 21: return launch_fast_t<5, false, T, 1, 16, S1>(a, st, sms);
        case 22: return launch_fast_t<5, true, T, 0, 16, S0>(a, st, sms);
        case 23: return launch_fast_t<5, true, T, 1, 16, S1>(a, st, sms);
        case 28: return launch_fast_t<7, false, T, 0, 16, S0>(a, st, sms);
        case 29: return launch_fast_t<7, false, T, 1, 16, S1>(a, st, sms);
        case 30: return launch_fast_t<7, true, T, 0, 16, S0>(a, st, sms);
        case 31: return launch_fast_t<7, true, T, 1, 16, S1>(a, st, sms);
        default: return 1003;
    }
}

}  // namespace wsb
