// batched.cuh -- many uneven blocks in one persistent launch.
//
// Each batch entry is one sweep of one block (its own extents, v_size,
// order 3/5/7, JS or TENO weights, MP on/off, FP64 or FP32-bulk storage,
// drop-in or folded input).  The entries are cut into work items
// (entry, face tile, group of U columns); a persistent grid of CTAs takes
// items from a global atomic counter until the list is exhausted, so large
// and small blocks share the GPU without one launch per block and without
// a tail of idle SMs.  Nothing waits on another CTA: a CTA that finds the
// counter past the end simply exits.
//
// Inside an item, thread f owns face f of the tile, loads that face's
// coefficients once for the item and reads its stencil straight from
// global memory (the tile's columns are contiguous along the sweep for the
// drop-in layout and for x; L1 serves the overlap of neighbouring faces).
//
// Entries whose coefficient arrays are the same on every face (checked when
// the batch is built) and that a marching engine covers (WENO3 with JS
// weights, WENO5 / WENO7 with JS or TENO weights; FP64 or FP32-bulk) take
// marching items instead: an item
// is one CTA-width group of columns, each thread marches its own column over
// the core faces (sweep_march.cuh engines) with the entry's MarchArgs copied
// to shared memory, so each face costs one new cell and one new difference
// instead of a full stencil.
#pragma once

#include <type_traits>

#include "weno_math.cuh"
#include "sweep_generic.cuh"
#include "sweep_march.cuh"

namespace wsb {

struct BatchEntry {
    SweepGeom g;        // extents and input strides (drop-in or folded)
    const void* in;
    void* vL;
    void* vR;
    CoefPtrs cp;
    WenoParams wp;
    int order;          // 3, 5, 7
    int mp;             // fused MP limiter
    int fp32;           // FP32-bulk storage (input and face states are float)
    int o_first, nf;    // faces handled
    int n_jt;           // face tiles
    int TJ;             // faces per tile (<= blockDim.x)
    long long n_groups; // column groups of U columns (marching: of blockDim.x columns)
    long long item0;    // first work item of this entry
    int march;          // 0: per-face items; 1 + k: marching items with MarchArgs k of the batch
};

// One marching item: thread t marches column cg * blockDim.x + t over the
// core faces 3 .. ns-4 (cells o+1 .. o+5 for WENO5, o .. o+6 for WENO7).
// Faces per output chunk of a marching item: each warp stages kBatchF faces
// x 32 columns of vL and vR in shared memory and writes them back as
// kBatchF-face segments of each column (64 bytes in FP64), so a store
// instruction covers 4 columns instead of 32 (the face-fastest layout puts
// neighbouring columns ns elements apart).
constexpr int kBatchF = 8;

template <typename T, int ORDER, bool TENOW, bool MPF>
__device__ __forceinline__ void batch_march(const MarchArgs& a, const BatchEntry& e, long long cg,
                                            T (*tl)[kBatchF][33]) {
    using Engine = std::conditional_t<
        ORDER == 7, std::conditional_t<sizeof(T) == 8, March64_7, March32_7>,
        std::conditional_t<ORDER == 3, std::conditional_t<sizeof(T) == 8, March64_3, March32_3>,
                           std::conditional_t<sizeof(T) == 8, March64, March32>>>;
    const int lane = threadIdx.x & 31;
    const long long wcol0 = cg * blockDim.x + (threadIdx.x & ~31);  // this warp's first column
    if (wcol0 >= e.g.cols) return;                                   // (whole warp)
    // lanes past the last column shadow it (loads stay in bounds, nothing is stored)
    const long long col = min(wcol0 + lane, e.g.cols - 1);
    const long long ca = col % e.g.c1, t = col / e.g.c1;
    const long long cb = t % e.g.c2, cv = t / e.g.c2;
    const T* __restrict__ cp = (const T*)e.in + e.g.in_off + ca * e.g.sA + cb * e.g.sB + cv * e.g.sV;
    const long long sJ = e.g.sJ, ns = e.g.ns, ncell = e.g.ns + 6;
    T* __restrict__ outL = (T*)e.vL;
    T* __restrict__ outR = (T*)e.vR;
    auto ld = [&](long long J) { return J < ncell ? __ldg(cp + J * sJ) : T(0); };
    // WENO3 writes every face (MP on the core faces), the others the core faces
    const long long o0 = ORDER == 3 ? 0 : 3, o1 = ORDER == 3 ? ns : ns - 3;
    constexpr int PUSH = ORDER == 7 ? 7 : 6;  // cell pushed after face o: o + PUSH
    Engine w;
    if constexpr (ORDER == 7) w.init(a, ld(o0), ld(o0 + 1), ld(o0 + 2), ld(o0 + 3), ld(o0 + 4), ld(o0 + 5), ld(o0 + 6));
    else w.init(a, ld(o0 + 1), ld(o0 + 2), ld(o0 + 3), ld(o0 + 4), ld(o0 + 5));
    const int fi = lane & (kBatchF - 1), cj = lane / kBatchF;
    for (long long f0 = o0; f0 < o1; f0 += kBatchF) {
        const int nF = (int)min((long long)kBatchF, o1 - f0);
#pragma unroll 1
        for (int i = 0; i < kBatchF; ++i) {
            const long long o = f0 + i;  // faces past o1 (i >= nF) are computed and dropped
            const T n = ld(o + PUSH);
            T L, R;
            bool ok;
            if constexpr (TENOW) ok = w.template face_teno<MPF>(a, L, R);
            else if constexpr (ORDER == 3) ok = w.template face<MPF>(a, L, R, o >= 3 && o <= ns - 4);
            else ok = w.template face<MPF>(a, L, R);
            if (!ok && i < nF) {
                if constexpr (ORDER == 3) {
                    march3_redo<MPF, T>(a, cp, o, L, R);
                } else if constexpr (ORDER == 7) {
                    if constexpr (sizeof(T) == 8) march64_7_redo<MPF>(a, cp, o, L, R);
                    else march32_7_redo<MPF>(a, cp, o, L, R);
                } else if constexpr (sizeof(T) == 8) {
                    march64_redo<MPF>(a, cp, o, L, R);
                } else {
                    march32_redo<MPF>(a, cp, o, L, R);
                }
            }
            tl[0][i][lane] = L;
            tl[1][i][lane] = R;
            w.push(a, n);
        }
        __syncwarp();
#pragma unroll
        for (int c = cj; c < 32; c += 32 / kBatchF) {
            const long long cc = wcol0 + c;
            if (cc < e.g.cols && fi < nF) {
                outL[cc * ns + f0 + fi] = tl[0][fi][c];
                outR[cc * ns + f0 + fi] = tl[1][fi][c];
            }
        }
        __syncwarp();
    }
}

template <bool MPF>
__device__ __forceinline__ void batch_march_dispatch(const MarchArgs& a, const BatchEntry& e, long long cg,
                                                     double (*tile)[kBatchF][33]) {
    float (*tile32)[kBatchF][33] = reinterpret_cast<float (*)[kBatchF][33]>(tile);
    // (the redo sequences take the weights from the arguments)
    const bool teno = e.wp.scheme == TENO;
    if (e.order == 3) {
        if (e.fp32) batch_march<float, 3, false, MPF>(a, e, cg, tile32);
        else batch_march<double, 3, false, MPF>(a, e, cg, tile);
        return;
    }
    if (e.fp32) {
        if (e.order == 7) {
            if (teno) batch_march<float, 7, true, MPF>(a, e, cg, tile32);
            else batch_march<float, 7, false, MPF>(a, e, cg, tile32);
        } else {
            if (teno) batch_march<float, 5, true, MPF>(a, e, cg, tile32);
            else batch_march<float, 5, false, MPF>(a, e, cg, tile32);
        }
    } else if (e.order == 7) {
        if (teno) batch_march<double, 7, true, MPF>(a, e, cg, tile);
        else batch_march<double, 7, false, MPF>(a, e, cg, tile);
    } else {
        if (teno) batch_march<double, 5, true, MPF>(a, e, cg, tile);
        else batch_march<double, 5, false, MPF>(a, e, cg, tile);
    }
}

template <int ORDER, typename T>
__device__ __forceinline__ void batch_item(const BatchEntry& e, long long grp, int jt, int U) {
    const int f = threadIdx.x;
    if (f >= e.TJ) return;
    const int fi = jt * e.TJ + f;
    if (fi >= e.nf) return;
    const long long o = e.o_first + fi;
    long long c = o - 3;
    c = c < 0 ? 0 : (c > e.g.nc - 1 ? e.g.nc - 1 : c);
    Coef<ORDER> cf;
    cf.load(e.cp.polyL, e.cp.polyR, e.cp.dL, e.cp.dR, e.cp.beta, e.g.nc, c);
    const T* __restrict__ in = (const T*)e.in;
    T* __restrict__ vL = (T*)e.vL;
    T* __restrict__ vR = (T*)e.vR;
    const long long col0 = grp * U;
    const long long col1 = min(col0 + U, e.g.cols);
    for (long long col = col0; col < col1; ++col) {
        const long long a = col % e.g.c1;
        const long long t = col / e.g.c1;
        const long long b = t % e.g.c2;
        const long long v = t / e.g.c2;
        const T* __restrict__ p = in + e.g.in_off + (o + 3) * e.g.sJ + a * e.g.sA + b * e.g.sB + v * e.g.sV;
        const long long oi = o + e.g.ns * col;
        const long long sJ = e.g.sJ;
        T Lt, Rt;
        if constexpr (ORDER == 3) {
            double L, R;
            weno3_face((double)__ldg(p - sJ), (double)__ldg(p), (double)__ldg(p + sJ), cf, e.wp.scheme, e.wp.eps, L,
                       R);
            Lt = (T)L;
            Rt = (T)R;
            if (e.mp && o >= 3 && o <= e.g.ns - 4)
                MP<T>::apply(__ldg(p - 2 * sJ), __ldg(p - sJ), __ldg(p), __ldg(p + sJ), __ldg(p + 2 * sJ), Lt, Rt);
        } else if constexpr (ORDER == 5) {
            const T m2 = __ldg(p - 2 * sJ), m1 = __ldg(p - sJ), z0 = __ldg(p), p1 = __ldg(p + sJ), p2 = __ldg(p + 2 * sJ);
            double L, R;
            weno5_face<T>((double)m2, (double)m1, (double)z0, (double)p1, (double)p2, cf, e.wp.scheme, e.wp.eps,
                          e.wp.teno_ct, L, R);
            Lt = (T)L;
            Rt = (T)R;
            if (e.mp) MP<T>::apply(m2, m1, z0, p1, p2, Lt, Rt);
        } else {
            double s7[7];
#pragma unroll
            for (int q = 0; q < 7; ++q) s7[q] = (double)__ldg(p + (q - 3) * sJ);
            double L, R;
            weno7_face<T>(s7 + 3, cf, e.wp.scheme, e.wp.eps, e.wp.teno_ct, L, R);
            Lt = (T)L;
            Rt = (T)R;
            if (e.mp) MP<T>::apply(__ldg(p - 2 * sJ), __ldg(p - sJ), __ldg(p), __ldg(p + sJ), __ldg(p + 2 * sJ), Lt, Rt);
        }
        vL[oi] = Lt;
        vR[oi] = Rt;
    }
}

// Persistent kernel: CTAs take items from *counter until n_items.
#ifndef WSB_BATCH_MIN_BLOCKS
#define WSB_BATCH_MIN_BLOCKS 2  // 2 CTAs of 256 per SM (128 registers; the marching paths spill a little, still faster than 168-255)
#endif
__global__ void __launch_bounds__(256, WSB_BATCH_MIN_BLOCKS)
    batch_kernel(const BatchEntry* __restrict__ entries, int n_entries, long long n_items,
                 unsigned long long* __restrict__ counter, int U, const MarchArgs* __restrict__ margs) {
    __shared__ long long s_item;
    __shared__ int s_entry;
    __shared__ MarchArgs s_ma;   // marching items: the entry's arguments
    // marching items: per warp, vL / vR of kBatchF faces x 32 columns (8 warps of 256 threads)
    __shared__ double s_tile[8][2][kBatchF][33];
    int ma_loaded = -1;          // index of the MarchArgs in s_ma (same on every thread)
    while (true) {
        if (threadIdx.x == 0) {
            const long long it = (long long)atomicAdd(counter, 1ull);
            s_item = it;
            // entry of this item: entries are sorted by item0 (binary search)
            int lo = 0, hi = n_entries - 1;
            if (it < n_items) {
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (entries[mid].item0 <= it) lo = mid;
                    else hi = mid - 1;
                }
            }
            s_entry = lo;
        }
        __syncthreads();
        const long long it = s_item;
        const int ei = s_entry;
        __syncthreads();
        if (it >= n_items) break;
        const BatchEntry& e = entries[ei];
        const long long local = it - e.item0;
        if (e.march) {
            const int k = e.march - 1;
            if (k != ma_loaded) {
                // every thread reaches this branch (the entry is the CTA's)
                const unsigned* src = reinterpret_cast<const unsigned*>(margs + k);
                unsigned* dst = reinterpret_cast<unsigned*>(&s_ma);
                for (int q = threadIdx.x; q < (int)(sizeof(MarchArgs) / 4); q += blockDim.x) dst[q] = __ldg(src + q);
                ma_loaded = k;
                __syncthreads();
            }
            double(*tile)[kBatchF][33] = s_tile[threadIdx.x >> 5];
            if (e.mp) batch_march_dispatch<true>(s_ma, e, local, tile);
            else batch_march_dispatch<false>(s_ma, e, local, tile);
            continue;
        }
        const int jt = (int)(local % e.n_jt);
        const long long grp = local / e.n_jt;
        if (e.fp32) {
            switch (e.order) {
                case 3: batch_item<3, float>(e, grp, jt, U); break;
                case 5: batch_item<5, float>(e, grp, jt, U); break;
                default: batch_item<7, float>(e, grp, jt, U); break;
            }
        } else {
            switch (e.order) {
                case 3: batch_item<3, double>(e, grp, jt, U); break;
                case 5: batch_item<5, double>(e, grp, jt, U); break;
                default: batch_item<7, double>(e, grp, jt, U); break;
            }
        }
    }
}

}  // namespace wsb
