// sweep_march_tma.cuh -- FP64 WENO5-JS (+MP) marching sweep with TMA
// staging of its input cells and output face states.
//
// The marching kernel of sweep_march.cuh spends, at 200^3 x 8, about as
// much time waiting on its per-lane global loads (a few cells ahead in
// registers) and on its shared-memory transpose + scattered stores as on
// the arithmetic.  Here each warp owns its own little pipeline instead:
//  * input: a ring of kTmaStages shared-memory tiles of 8 consecutive cells
//    (along the sweep) by 32 columns, each one cp.async.bulk.tensor issued
//    by lane 0 and completed on the stage's mbarrier; tiles are requested
//    kTmaStages - 1 chunks ahead, so several KB per warp are in flight and
//    the registers hold no prefetch buffers;
//  * output: the 8 faces x 32 columns of vL and of vR go to a 64-byte
//    swizzled shared tile (double-buffered) and leave as one bulk tensor
//    store each, so the face-fastest layout is written by the TMA engine
//    and the warp issues no global stores.
// No CTA-wide barrier: the four warps of a CTA are independent.
//
// Alignment (the innermost TMA coordinate must be a multiple of 16 bytes):
// chunks start at even faces (4, 12, 20, ...), whose push cells (face + 6)
// and output coordinate are then even; the first core face, 3, is done
// before the first chunk and stored with plain stores.  Column tiles whose
// innermost axis is the cross axis (folded y / z sweeps) start one cell
// left of the first column (x + 3 pad cells is odd) and are 34 cells wide.
// The output map's face extent is ns - 4 (the store unit clips the
// innermost axis in 16-byte steps, so the extent is kept even and the last
// core face, ns - 4, is stored by the lanes), so a chunk reaching past the
// core faces is clipped by the TMA unit; loads past the end of a column
// read the zero fill.
//
// Every mbarrier wait is bounded; on expiry the warp records
// WENO_SB_ERR_TIMEOUT, waits (bounded again) for the tiles it still has in
// flight, and stops.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include "sweep_march.cuh"
#include "sweep_pipe.cuh"

namespace wsb {

constexpr int kTmaF = 8;        // faces per chunk = cells per input tile
constexpr int kTmaStages = 4;   // input tiles per warp
constexpr int kTmaWarps = 4;    // warps per CTA

struct MarchTmaArgs {
    int kind;          // 0: sweep axis innermost (row tiles), 1: cross axis innermost
    int dimJ, dimU, dimW;  // input map dimension of the sweep, lane and outer cross axes
    int uoff, woff;    // coordinate offsets of column 0 on the lane / outer cross axis
    int odimU, odimW;  // output map dimension of the lane / outer cross axis
    int stage_bytes;   // one input tile (KIND 0: 2048, KIND 1: 8 rows x 34 cells)
    int warp_bytes;    // shared memory per warp, a multiple of 1024
    unsigned box_bytes;
};

__device__ __forceinline__ void tma_store_4d(const CUtensorMap* map, const void* src, int c0, int c1, int c2, int c3) {
    asm volatile(
        "cp.async.bulk.tensor.4d.global.shared::cta.bulk_group [%0, {%2, %3, %4, %5}], [%1];\n" ::"l"(map),
        "r"(smem_u32(src)), "r"(c0), "r"(c1), "r"(c2), "r"(c3)
        : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read1() { asm volatile("cp.async.bulk.wait_group.read 1;\n" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory"); }
__device__ __forceinline__ void fence_async_shared() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

// Byte offset of element (row, i) of a tile of 64-byte rows under the
// 64-byte swizzle (16-byte chunk index XOR row bits 1..2).
__device__ __forceinline__ unsigned sw64(unsigned row, unsigned i) {
    const unsigned off = row * 64u + i * 8u;
    return off ^ ((off >> 3) & 0x30u);
}

template <bool MPF, int KIND>
__global__ void __launch_bounds__(kTmaWarps * 32, 3)
    sweep_march_tma_kernel(const __grid_constant__ CUtensorMap tin, const __grid_constant__ CUtensorMap toutL,
                           const __grid_constant__ CUtensorMap toutR, const __grid_constant__ MarchArgs a,
                           const MarchTmaArgs t) {
    constexpr int F = kTmaF, S = kTmaStages;
    extern __shared__ __align__(1024) unsigned char smem_mt[];
    unsigned char* base = smem_mt + ((1024u - (smem_u32(smem_mt) & 1023u)) & 1023u);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // per warp: 2 output buffers x (vL, vR) x 2048 bytes, then S input tiles
    const int warp_bytes = t.warp_bytes;
    unsigned char* wbase = base + (size_t)warp * warp_bytes;
    unsigned char* obuf = wbase;
    unsigned char* ring = wbase + 4 * 2048;
    unsigned long long* bars = (unsigned long long*)(base + (size_t)kTmaWarps * warp_bytes) + warp * S;
    if (lane == 0) {
        for (int s = 0; s < S; ++s) mbar_init(&bars[s], 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    __syncwarp();

    double* __restrict__ outL = (double*)a.vL;
    double* __restrict__ outR = (double*)a.vR;
    const long long nwarps = (long long)gridDim.x * kTmaWarps;
    const int o_last = (int)a.ns - 3;         // one past the last core face
    unsigned long long n_issued = 0, n_waited = 0;  // tiles requested / completed (waited on) by this warp
    unsigned n_chunks = 0;                    // output chunks stored by this warp
    bool failed = false;

    auto tile_ptr = [&](unsigned long long k) { return ring + (size_t)(k % S) * t.stage_bytes; };
    // request tile k (cells J0 .. J0+7) of the column group (u0, w, v)
    auto issue = [&](unsigned long long k, int J0, int u0, int w, int v) {
        if (lane == 0) {
            unsigned long long* bar = &bars[k % S];
            const int cU = t.uoff + u0, cW = t.woff + w;
            const int c0 = t.dimJ == 0 ? J0 : (t.dimU == 0 ? cU : cW);
            const int c1 = t.dimJ == 1 ? J0 : (t.dimU == 1 ? cU : cW);
            const int c2 = t.dimJ == 2 ? J0 : (t.dimU == 2 ? cU : cW);
            mbar_arrive_expect_tx(bar, t.box_bytes);
            tma_load_4d(tile_ptr(k), &tin, bar, c0, c1, c2, v);
        }
    };
    auto wait_tile = [&](unsigned long long k) -> bool {
        if (!mbar_wait(&bars[k % S], (unsigned)((k / S) & 1ull))) return false;
        n_waited = k + 1;
        return true;
    };
    // cell at position p (0..7) of tile k for this lane's column
    auto cell = [&](unsigned long long k, int p) -> double {
        const unsigned char* tp = tile_ptr(k);
        if constexpr (KIND == 0) return *(const double*)(tp + sw64((unsigned)lane, (unsigned)p));
        else return *(const double*)(tp + p * (34 * 8) + (lane + 1) * 8);
    };

    for (long long item = (long long)blockIdx.x * kTmaWarps + warp; item < a.n_items && !failed; item += nwarps) {
        const int sg = (int)(item % a.n_seg);
        long long tt = item / a.n_seg;
        const int ut = (int)(tt % a.n_ut);
        tt /= a.n_ut;
        const int wv = (int)(tt % a.Nw);
        const int vv = (int)(tt / a.Nw);
        const int u0 = ut * 32;
        const int f_start = 4 + sg * a.seg;                       // even
        int f_end = f_start + a.seg;
        if (f_end > o_last) f_end = o_last;
        const int nch = f_end > f_start ? (f_end - f_start + F - 1) / F : 0;
        const int ntiles = nch + 1;                               // tiles 0 .. nch
        const unsigned long long k0 = n_issued;                   // first tile of this item
        for (int k = 0; k < ntiles && k < S; ++k) issue(k0 + k, f_start + F * k, u0, wv, vv);
        n_issued += (ntiles < S ? ntiles : S);
        if (!wait_tile(k0)) { failed = true; break; }

        March64 w;
        if (sg == 0) {
            // face 3 (cells 4..8 = tile positions 0..4), plain stores
            w.init(a, cell(k0, 0), cell(k0, 1), cell(k0, 2), cell(k0, 3), cell(k0, 4));
            double L, R;
            if (!w.face<MPF>(a, L, R)) {
                const int uc = u0 + lane < a.Nu ? u0 + lane : a.Nu - 1;
                const double* col = (const double*)a.in + a.in_off + uc * a.sU + wv * a.sW + vv * a.sV;
                march64_redo<MPF>(a, col, 3, L, R);
            }
            if (u0 + lane < a.Nu) {
                const long long oi = 3 + (long long)(u0 + lane) * a.oU + wv * a.oW + vv * a.oV;
                outL[oi] = L;
                outR[oi] = R;
            }
            w.push(a, cell(k0, 5));
        } else {
            w.init(a, cell(k0, 1), cell(k0, 2), cell(k0, 3), cell(k0, 4), cell(k0, 5));
        }
        // chunk c: faces f0 .. f0+7 (f0 = f_start + 8c), pushes cells
        // f0+6 .. f0+13 = positions 6, 7 of tile c and 0 .. 5 of tile c+1
        for (int c = 0; c < nch; ++c) {
            const unsigned long long kc = k0 + c;
            if (!wait_tile(kc + 1)) { failed = true; break; }
            const int f0 = f_start + F * c;
            unsigned char* ob = obuf + (size_t)(n_chunks & 1u) * 4096;
            if (n_chunks >= 2) {
                if (lane == 0) bulk_wait_read1();  // the store issued from this buffer two chunks ago has read it
                __syncwarp();
            }
            unsigned bad = 0;
#pragma unroll
            for (int i = 0; i < F; ++i) {
                double L, R;
                if (!w.face<MPF>(a, L, R)) bad |= 1u << i;
                *(double*)(ob + sw64((unsigned)lane, (unsigned)i)) = L;
                *(double*)(ob + 2048 + sw64((unsigned)lane, (unsigned)i)) = R;
                w.push(a, (i < 2) ? cell(kc, 6 + i) : cell(kc + 1, i - 2));
            }
            const int nF = f_end - f0 < F ? f_end - f0 : F;
            bad &= (1u << nF) - 1u;
            const int i_last = o_last - 1 - f0;  // the last core face, when in this chunk
            if (bad) {
                const int uc = u0 + lane < a.Nu ? u0 + lane : a.Nu - 1;
                const double* col = (const double*)a.in + a.in_off + uc * a.sU + wv * a.sW + vv * a.sV;
                while (bad) {
                    const int i = __ffs(bad) - 1;
                    bad &= bad - 1;
                    double L, R;
                    march64_redo<MPF>(a, col, f0 + i, L, R);
                    *(double*)(ob + sw64((unsigned)lane, (unsigned)i)) = L;
                    *(double*)(ob + 2048 + sw64((unsigned)lane, (unsigned)i)) = R;
                }
            }
            if (i_last >= 0 && i_last < F && u0 + lane < a.Nu) {
                // outside the store map's extent (see launch_march_tma)
                const long long oi = (o_last - 1) + (long long)(u0 + lane) * a.oU + wv * a.oW + vv * a.oV;
                outL[oi] = *(const double*)(ob + sw64((unsigned)lane, (unsigned)i_last));
                outR[oi] = *(const double*)(ob + 2048 + sw64((unsigned)lane, (unsigned)i_last));
            }
            fence_async_shared();
            __syncwarp();
            if (lane == 0) {
                const int c1 = t.odimU == 1 ? u0 : wv, c2 = t.odimU == 2 ? u0 : wv;
                tma_store_4d(&toutL, ob, f0, c1, c2, vv);
                tma_store_4d(&toutR, ob + 2048, f0, c1, c2, vv);
                bulk_commit();
            }
            ++n_chunks;
            // tile c is consumed: refill its stage with tile c + S
            __syncwarp();
            if (c + S < ntiles) {
                issue(kc + S, f_start + F * (c + S), u0, wv, vv);
                ++n_issued;
            }
        }
        if (failed) break;
    }
    if (failed) {
        // let the tiles still in flight land before the CTA's shared memory
        // is released (bounded, as every wait here); tiles are waited in
        // order, so those past the last completed one are the ones in flight
        for (unsigned long long k = n_waited; k < n_issued; ++k)
            mbar_wait(&bars[k % S], (unsigned)((k / S) & 1ull));
    }
    if (lane == 0) bulk_wait_all();
    __syncwarp();
}

// Host side.  Returns 1003 (unsupported) when the layout does not meet the
// TMA rules (16-byte aligned bases, strides that are multiples of 16 bytes)
// or the driver entry point is missing; the caller then uses sweep_march64.
inline int launch_march_tma(const long long E[3], const SweepGeom& g, int dir, bool folded, bool mp, const double* in,
                     double* vL, double* vR, const MarchArgs& a0, cudaStream_t st, int sms) {
    EncodeTiledFn enc = encode_tiled_fn();
    if (!enc) return 1003;
    if ((((uintptr_t)in) | ((uintptr_t)vL) | ((uintptr_t)vR)) & 15) return 1003;
    if (g.ns < 7 || (g.ns & 1)) return 1003;
    MarchArgs a = a0;
    MarchTmaArgs t{};
    const bool kind1 = folded && dir != 0;
    t.kind = kind1 ? 1 : 0;
    cuuint64_t dims[4], strides[3];
    cuuint32_t box[4], estr[4] = {1, 1, 1, 1};
    CUtensorMapSwizzle swz;
    if (!folded) {
        // v_rs_ws (ns+6, c1, c2, V): lanes along c1
        dims[0] = g.ns + 6; dims[1] = g.c1; dims[2] = g.c2; dims[3] = g.nv;
        t.dimJ = 0; t.dimU = 1; t.dimW = 2; t.uoff = 0; t.woff = 0;
    } else {
        dims[0] = E[0]; dims[1] = E[1]; dims[2] = E[2]; dims[3] = g.nv;
        if (dir == 0) { t.dimJ = 0; t.dimU = 1; t.dimW = 2; t.uoff = 3; t.woff = 3; }
        else if (dir == 1) { t.dimJ = 1; t.dimU = 0; t.dimW = 2; t.uoff = 2; t.woff = 3; }
        else { t.dimJ = 2; t.dimU = 0; t.dimW = 1; t.uoff = 2; t.woff = 3; }
    }
    if (!kind1) {
        box[0] = kTmaF; box[1] = 32; box[2] = 1; box[3] = 1;
        swz = CU_TENSOR_MAP_SWIZZLE_64B;
        t.stage_bytes = 2048;
    } else {
        box[0] = 34; box[1] = 1; box[2] = 1; box[3] = 1;
        box[t.dimJ] = kTmaF;
        swz = CU_TENSOR_MAP_SWIZZLE_NONE;
        t.stage_bytes = kTmaF * 34 * 8;  // 2176, a multiple of 128
    }
    t.box_bytes = (unsigned)(box[0] * box[1] * box[2] * box[3] * 8);
    strides[0] = dims[0] * 8;
    strides[1] = dims[0] * dims[1] * 8;
    strides[2] = dims[0] * dims[1] * dims[2] * 8;
    if (strides[0] % 16) return 1003;
    CUtensorMap mi, mL, mR;
    if (enc(&mi, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, (void*)in, dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, swz, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return 1003;
    // outputs (ns, c1, c2, V).  The store unit clips the innermost axis in
    // 16-byte steps, so the face extent is ns - 4 (even): faces up to ns-5
    // are stored by the TMA unit, the last core face ns-4 with plain stores,
    // and the non-core faces ns-3 .. ns-1 are never written.
    cuuint64_t od[4] = {(cuuint64_t)(g.ns - 4), (cuuint64_t)g.c1, (cuuint64_t)g.c2, (cuuint64_t)g.nv};
    cuuint64_t os[3] = {(cuuint64_t)g.ns * 8, (cuuint64_t)(g.ns * g.c1) * 8, (cuuint64_t)(g.ns * g.c1 * g.c2) * 8};
    cuuint32_t ob[4] = {kTmaF, 1, 1, 1};
    // lanes run along the output axis with the smaller stride of the two
    // cross axes the march launcher picked (a.oU == ns: c1, else c2)
    if (a.oU == g.ns) { t.odimU = 1; t.odimW = 2; }
    else { t.odimU = 2; t.odimW = 1; }
    ob[t.odimU] = 32;
    if (enc(&mL, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, (void*)vL, od, os, ob, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) !=
            CUDA_SUCCESS ||
        enc(&mR, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, (void*)vR, od, os, ob, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) !=
            CUDA_SUCCESS)
        return 1003;
    // lane axis must be the one the march launcher chose
    if ((t.kind == 1) != (a.sU == 1)) return 1003;
    // segments over faces [4, ns-3), a multiple of 8 faces each
    const long long nf4 = g.ns - 3 - 4 > 0 ? g.ns - 3 - 4 : 0;
    const long long cols = (long long)a.n_ut * a.Nw * a.NV;
    const long long want = (long long)sms * kTmaWarps * 3 * 2;
    long long nseg = (want + cols - 1) / cols;
    const long long max_seg = nf4 > 0 ? (nf4 + kTmaF - 1) / kTmaF : 1;
    if (nseg > max_seg) nseg = max_seg;
    if (nseg < 1) nseg = 1;
    long long seg = nf4 > 0 ? (nf4 + nseg - 1) / nseg : kTmaF;
    seg = ((seg + kTmaF - 1) / kTmaF) * kTmaF;
    a.seg = (int)seg;
    a.n_seg = nf4 > 0 ? (int)((nf4 + seg - 1) / seg) : 1;
    a.n_items = cols * a.n_seg;
    t.warp_bytes = ((4 * 2048 + kTmaStages * t.stage_bytes + 1023) / 1024) * 1024;
    const size_t smem = 1024 + (size_t)kTmaWarps * t.warp_bytes + (size_t)kTmaWarps * kTmaStages * 8;
    auto kfn = mp ? (kind1 ? sweep_march_tma_kernel<true, 1> : sweep_march_tma_kernel<true, 0>)
                  : (kind1 ? sweep_march_tma_kernel<false, 1> : sweep_march_tma_kernel<false, 0>);
    cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int occ = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kfn, kTmaWarps * 32, smem);
    if (occ < 1) return 1003;
    long long blocks = (a.n_items + kTmaWarps - 1) / kTmaWarps;
    const long long cap = (long long)sms * occ;
    if (blocks > cap) blocks = cap;
    kfn<<<(unsigned)blocks, kTmaWarps * 32, smem, st>>>(mi, mL, mR, a, t);
    return 0;
}

}  // namespace wsb
