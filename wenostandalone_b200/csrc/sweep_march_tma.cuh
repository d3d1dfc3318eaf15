// sweep_march_tma.cuh -- the marching sweep (sweep_march.cuh engines: WENO3
// / WENO5 / WENO7, JS or TENO weights, FP64 or FP32-bulk, face-independent
// coefficients or, FP64 WENO5-JS, a per-face table) with TMA staging of its
// input cells and output face states.
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

#include <cstring>
#include <type_traits>

#include "sweep_march.cuh"
#include "sweep_pipe.cuh"

namespace wsb {

#ifndef WSB_MTMA_MIN_BLOCKS
#define WSB_MTMA_MIN_BLOCKS 3   // CTAs per SM the kernel is register-capped for
#endif
#ifndef WSB_MTMA_STAGES
#define WSB_MTMA_STAGES 4       // input tiles per warp
#endif
#ifndef WSB_MTMA_OUTBUF
#define WSB_MTMA_OUTBUF 2       // output tiles per warp (1: each store is waited before the next chunk)
#endif
constexpr int kTmaF = 8;        // faces per chunk = cells per input tile
constexpr int kTmaStages = WSB_MTMA_STAGES;
constexpr int kTmaOut = WSB_MTMA_OUTBUF;
// Face-dependent coefficients: each input stage also holds the chunk's
// kTmaF + 1 rows of the per-face table (one bulk copy on the tile's
// mbarrier), so the kernels run fewer stages and output buffers to keep
// three CTAs per SM.
#ifndef WSB_MTMA_PF_STAGES
#define WSB_MTMA_PF_STAGES 3
#endif
#ifndef WSB_MTMA_PF_OUTBUF
#define WSB_MTMA_PF_OUTBUF 1
#endif
constexpr int kPfStages = WSB_MTMA_PF_STAGES;
constexpr int kPfOut = WSB_MTMA_PF_OUTBUF;
// rows f0 .. f0 + 8 of a chunk (WENO5 / WENO7 table rows)
__host__ __device__ constexpr int pf_row_doubles(int order) {
    return order == 7 ? kFaceRow7 : (order == 3 ? kFaceRow3 : kFaceRow);
}
__host__ __device__ constexpr int pf_chunk_bytes(int order) { return (kTmaF + 1) * pf_row_doubles(order) * 8; }
static_assert(pf_chunk_bytes(3) % 16 == 0 && pf_chunk_bytes(5) % 16 == 0 && pf_chunk_bytes(7) % 16 == 0,
              "bulk copies move 16-byte multiples");
static_assert(WSB_MTMA_PF_STAGES <= 4 && WSB_MTMA_PF_STAGES >= 2, "stages of the per-face kernels");
#ifndef WSB_MTMA_WARPS
#define WSB_MTMA_WARPS 4        // warps per CTA (each with its own pipeline)
#endif
constexpr int kTmaWarps = WSB_MTMA_WARPS;
static_assert(WSB_MTMA_STAGES <= 4, "the per-lane copy loader waits with at most 3 groups in flight");

struct MarchTmaArgs {
    int kind;          // 0: sweep axis innermost (row tiles), 1: cross axis innermost
    int dimJ, dimU, dimW;  // input map dimension of the sweep, lane and outer cross axes
    int uoff, woff;    // coordinate offsets of column 0 on the lane / outer cross axis
    int odimU, odimW;  // output map dimension of the lane / outer cross axis
    int stage_bytes;   // one input tile (KIND 0: 2048, KIND 1: 8 rows x 34 cells)
    int warp_bytes;    // shared memory per warp, a multiple of 1024
    int ring_off;      // byte offset of the input ring within a warp's area
    int rows_off;      // face-dependent coefficients: byte offset of the table-row ring
    int ldr8;          // per-lane loader, row tiles of floats: cells copied in 8-byte pairs
    int ldr;           // 1: per-lane loader (the field's rows or base do not suit TMA)
    int pst;           // 1: plain stores of the face states (face rows not 16-byte multiples)
    unsigned box_bytes;
};

__device__ __forceinline__ void tma_store_4d(const CUtensorMap* map, const void* src, int c0, int c1, int c2, int c3) {
    asm volatile(
        "cp.async.bulk.tensor.4d.global.shared::cta.bulk_group [%0, {%2, %3, %4, %5}], [%1];\n" ::"l"(map),
        "r"(smem_u32(src)), "r"(c0), "r"(c1), "r"(c2), "r"(c3)
        : "memory");
}
// 1-D bulk copy global -> shared (16-byte aligned addresses, size a multiple
// of 16), completed on the mbarrier like a tensor tile.
__device__ __forceinline__ void bulk_load_1d(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read1() { asm volatile("cp.async.bulk.wait_group.read 1;\n" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read0() { asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory"); }
__device__ __forceinline__ void fence_async_shared() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

// Byte offset of element (row, i) of a tile with rows of 8 elements of T
// under the TMA swizzle of that row width: 64-byte rows (double) swap
// 16-byte chunks by row bits 1..2, 32-byte rows (float) by row bit 2.
template <typename T>
__device__ __forceinline__ unsigned swz(unsigned row, unsigned i) {
    if constexpr (sizeof(T) == 8) {
        const unsigned off = row * 64u + i * 8u;
        return off ^ ((off >> 3) & 0x30u);
    } else {
        const unsigned off = row * 32u + i * 4u;
        return off ^ ((off >> 3) & 0x10u);
    }
}

template <typename T> struct MarchEngine;
template <> struct MarchEngine<double> { using type = March64; };
template <> struct MarchEngine<float> { using type = March32; };

template <bool MPF, bool PF>
__device__ __forceinline__ void march_redo(const MarchArgs& a, const double* col, long long o, double& L, double& R) {
    if constexpr (PF) march64_redo_faces<MPF>(a, col, o, L, R);
    else march64_redo<MPF>(a, col, o, L, R);
}
template <bool MPF>
__device__ __forceinline__ void march7_redo(const MarchArgs& a, const double* col, long long o, double& L, double& R) {
    march64_7_redo<MPF>(a, col, o, L, R);
}
template <bool MPF>
__device__ __forceinline__ void march7_redo(const MarchArgs& a, const float* col, long long o, float& L, float& R) {
    march32_7_redo<MPF>(a, col, o, L, R);
}
template <bool MPF, bool PF>
__device__ __forceinline__ void march_redo(const MarchArgs& a, const float* col, long long o, float& L, float& R) {
    static_assert(!PF, "face-dependent coefficients: FP64 kernels only");
    march32_redo<MPF>(a, col, o, L, R);
}

// One sweep of a grouped launch (sweep_march_tma_multi_kernel): its maps,
// its arguments, and its first work item within the launch.  The sweeps of
// a group share the kernel instance (order, weights, storage, tile kind,
// MP), the coefficients (the kernel's MarchArgs) and the shared-memory
// layout (the kernel's MarchTmaArgs); extents, strides, pointers, map axes,
// loader and store kind are the entry's.
// The part of a sweep's arguments a grouped work item reads outside the
// face body; each item copies it (with the sweep's MarchTmaArgs) into its
// warp's slot of shared memory, so the chunk loop reads it from there
// rather than from the entry table (the table stays in global memory, and
// every asynchronous copy or wait in the loop would reload it).
struct MtmaGeo {
    const void* in;
    void* vL;
    void* vR;
    long long ns, sJ, sU, sW, sV, in_off, oU, oW, oV;
    int Nu, Nw, n_ut, seg, n_seg, pad_;
};
struct MtmaItemArgs {
    MtmaGeo geo;
    MarchTmaArgs t;
};
struct MtmaEntry;
// A warp's slot: the item's arguments and its entry (read where the maps or
// the full arguments are needed, so no register holds it across the face
// body).
struct MtmaSlot {
    MtmaItemArgs ia;
    const MtmaEntry* e;
};
static_assert(sizeof(MtmaItemArgs) % 8 == 0 && sizeof(MtmaSlot) <= 256, "per-warp argument slot");
constexpr int kMtmaSlot = 256;  // bytes of shared memory per warp for the item's arguments
inline MtmaGeo mtma_geo(const MarchArgs& a) {
    MtmaGeo g{};
    g.in = a.in; g.vL = a.vL; g.vR = a.vR;
    g.ns = a.ns; g.sJ = a.sJ; g.sU = a.sU; g.sW = a.sW; g.sV = a.sV; g.in_off = a.in_off;
    g.oU = a.oU; g.oW = a.oW; g.oV = a.oV;
    g.Nu = a.Nu; g.Nw = a.Nw; g.n_ut = a.n_ut; g.seg = a.seg; g.n_seg = a.n_seg;
    return g;
}
struct MtmaEntry {
    CUtensorMap tin, toutL, toutR;
    MtmaItemArgs ia;
    MarchArgs a;  // for the faces redone by the reference sequence
};

// The geometry of an item: the kernel's parameters (one sweep) or the
// warp's shared-memory copy (grouped sweeps).
template <bool MULTI>
__device__ __forceinline__ const auto& mtma_geo_of(const MarchArgs& a, const MtmaSlot* slot) {
    if constexpr (MULTI) return slot->ia.geo;
    else return a;
}

// PF: face-dependent coefficients from the per-face table a.ftab (FP64).
// ORDER 7: the WENO7 engine (face-independent coefficients); face f reads
// cells f .. f+6 and pushes cell f+7.  WS: the nonlinear weights, numbered
// as the reference's schemes: 0 JS (the engines' face), 1 mapped
// (face_mapped; FP64 WENO5, face-independent coefficients), 2 Z (face_z;
// FP64 WENO5), 3 TENO (face_teno).  MULTI: the work items of
// several sweeps (entries ents[0 .. n_ents), items numbered entry after
// entry); each item finds its entry, whose geometry, maps, loader (TMA or
// per lane) and store kind (TMA or plain) it uses, with the coefficients of
// the kernel's MarchArgs.
template <bool MPF, int KIND, typename T, int LDR, bool PF, int ORDER, int WS, bool MULTI>
__device__ __forceinline__ void march_tma_body(const CUtensorMap* tin0, const CUtensorMap* toutL0,
                                               const CUtensorMap* toutR0, const MarchArgs& a, const MarchTmaArgs& t,
                                               const MtmaEntry* __restrict__ ents,
                                               const long long* __restrict__ item0s, int n_ents, long long n_items) {
    constexpr bool TENOW = WS == 3;                       // TENO weights
    static_assert(WS == 0 || WS == 3 || (ORDER == 5 && sizeof(T) == 8),
                  "mapped / Z weights: the FP64 WENO5 engine");
    static_assert(WS != 1 || !PF, "mapped weights: face-independent coefficients");
    constexpr int F = kTmaF, S = PF ? kPfStages : kTmaStages;
    constexpr int NOUT = PF ? kPfOut : kTmaOut;             // output tiles per warp
    constexpr unsigned OB = 32u * F * sizeof(T);          // one output array tile
    constexpr int XW = sizeof(T) == 8 ? 34 : 36;          // KIND 1 tile width
    constexpr int XS = sizeof(T) == 8 ? 1 : 3;            // KIND 1 column of lane 0
    static_assert(ORDER != 3 || !PF || (sizeof(T) == 8 && !TENOW), "WENO3 per-face table: FP64, JS");
    static_assert(ORDER != 7 || !PF || sizeof(T) == 8, "WENO7 per-face table: FP64");
    static_assert(!MULTI || !PF, "grouped sweeps: face-independent coefficients");
    constexpr int RW = pf_row_doubles(ORDER), RB = pf_chunk_bytes(ORDER);  // per-face table rows
    static_assert(!TENOW || !PF || ORDER != 3, "TENO with a per-face table: WENO5 / WENO7");
    using Engine = std::conditional_t<
        ORDER == 7, std::conditional_t<sizeof(T) == 8, March64_7, March32_7>,
        std::conditional_t<ORDER == 3, std::conditional_t<sizeof(T) == 8, March64_3, March32_3>,
                           typename MarchEngine<T>::type>>;
    constexpr int PUSH0 = ORDER == 7 ? 7 : 6;             // tile position of the cell pushed after face f0
    extern __shared__ __align__(1024) unsigned char smem_mt[];
    unsigned char* base = smem_mt + ((1024u - (smem_u32(smem_mt) & 1023u)) & 1023u);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // per warp: NOUT output buffers x (vL, vR), then S input tiles (and, PF,
    // S chunks of table rows)
    const int warp_bytes = t.warp_bytes;
    unsigned char* wbase = base + (size_t)warp * warp_bytes;
    unsigned char* obuf = wbase;
    unsigned char* ring = wbase + t.ring_off;
    unsigned long long* bars = (unsigned long long*)(base + (size_t)kTmaWarps * warp_bytes) + warp * S;
    // grouped sweeps: the warp's argument slot, after the mbarriers
    MtmaSlot* slot = (MtmaSlot*)(base + (size_t)kTmaWarps * warp_bytes + (size_t)kTmaWarps * S * 8 +
                                 (size_t)warp * kMtmaSlot);
    if (lane == 0) {
        for (int s = 0; s < S; ++s) mbar_init(&bars[s], 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    __syncwarp();

    const long long nwarps = (long long)gridDim.x * kTmaWarps;
    unsigned n_issued = 0, n_waited = 0;      // tiles requested / completed (waited on) by this warp
    unsigned n_chunks = 0;                    // output chunks stored by this warp
    // grouped sweeps mix tiles loaded by TMA (completed on the stage's
    // mbarrier) with tiles copied per lane (no mbarrier phase): bit s is the
    // parity of the next phase of stage s's mbarrier
    unsigned ph = 0;
    bool failed = false;

    auto tile_ptr = [&](unsigned k) { return ring + (size_t)(k % S) * t.stage_bytes; };
    auto parity = [&](unsigned k) -> unsigned {
        if constexpr (MULTI) return (ph >> (k % S)) & 1u;
        else return (k / S) & 1u;
    };
    auto phase_done = [&](unsigned k) {
        if constexpr (MULTI) ph ^= 1u << (k % S);
    };
    // per-face table rows (PF): in global memory, and the chunk's rows
    // staged with input tile k
    auto row = [&](int f) { return a.ftab + (long long)f * RW; };
    auto srow = [&](unsigned k, int i) {
        return (const double*)(wbase + t.rows_off + (size_t)(k % S) * RB) + i * RW;
    };
    // byte offset in a tile of position p (0..7) of this lane's column
    auto cell_off = [&](int p) -> unsigned {
        if constexpr (KIND == 0) return swz<T>((unsigned)lane, (unsigned)p);
        else return (unsigned)((p * XW + lane + XS) * sizeof(T));
    };
    // cell at position p (0..7) of tile k for this lane's column
    auto cell = [&](unsigned k, int p) -> T { return *(const T*)(tile_ptr(k) + cell_off(p)); };

    for (long long item = (long long)blockIdx.x * kTmaWarps + warp; item < n_items && !failed; item += nwarps) {
        long long li = item;
        const MtmaEntry* E = nullptr;
        if constexpr (MULTI) {
            // the entry holding this item: entries in item order, their first
            // items in the dense array item0s (a few hundred bytes, L1-resident)
            int lo = 0, hi = n_ents - 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (__ldg(item0s + mid) <= item) lo = mid;
                else hi = mid - 1;
            }
            E = ents + lo;
            li = item - __ldg(item0s + lo);
            // the item's arguments into the warp's slot (the previous item's
            // reads of it are done at the first sync)
            constexpr int NW = (int)(sizeof(MtmaItemArgs) / 8);
            __syncwarp();
            if (lane < NW)
                reinterpret_cast<unsigned long long*>(&slot->ia)[lane] =
                    __ldg(reinterpret_cast<const unsigned long long*>(&E->ia) + lane);
            if (lane == 0) {
                slot->e = E;
                // the entry's maps are read by the TMA unit from global
                // memory, where a table freed and allocated again may hold
                // other maps at the same address: drop any copy cached for
                // it (lane 0 issues the item's bulk copies)
                asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;\n" ::"l"(&E->tin) : "memory");
                asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;\n" ::"l"(&E->toutL) : "memory");
                asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;\n" ::"l"(&E->toutR) : "memory");
            }
            __syncwarp();
        }
        // geometry, maps, loader and store kind of this item's sweep; the
        // sweep's full arguments for the faces redone by the reference sequence
        const auto& g = mtma_geo_of<MULTI>(a, slot);
        const MarchTmaArgs& te = MULTI ? slot->ia.t : t;
        // (grouped: read from the slot where used)
        auto ga = [&]() -> const MarchArgs& {
            if constexpr (MULTI) return slot->e->a;
            else return a;
        };
        auto mapI = [&]() { return MULTI ? &slot->e->tin : tin0; };
        auto mapL = [&]() { return MULTI ? &slot->e->toutL : toutL0; };
        auto mapR = [&]() { return MULTI ? &slot->e->toutR : toutR0; };
        const bool ldr = MULTI ? te.ldr != 0 : LDR == 1;
        // plain stores (face rows not 16-byte multiples): grouped sweeps only
        // (the single-sweep kernels keep their registers for the face body)
        const bool pst = MULTI && te.pst != 0;
        T* __restrict__ outL = (T*)g.vL;
        T* __restrict__ outR = (T*)g.vR;
        // faces written: the core faces 3 .. ns-4 (chunks from face 4, face 3 by
        // the prologue), or every face 0 .. ns-1 for WENO3 (chunks from face 0)
        const int o_last = ORDER == 3 ? (int)g.ns : (int)g.ns - 3;  // one past the last face
        auto column = [&](int u0, int wv, int vv) {
            const int uc = u0 + lane < g.Nu ? u0 + lane : g.Nu - 1;
            return (const T*)g.in + g.in_off + uc * g.sU + wv * g.sW + vv * g.sV;
        };
        // request tile k (cells J0 .. J0+7) of the column group (u0, w, v)
        auto issue = [&](unsigned k, int J0, int u0, int w, int v) {
            if (!ldr) {
                if (lane == 0) {
                    unsigned long long* bar = &bars[k % S];
                    const int cU = te.uoff + u0, cW = te.woff + w;
                    const int c0 = te.dimJ == 0 ? J0 : (te.dimU == 0 ? cU : cW);
                    const int c1 = te.dimJ == 1 ? J0 : (te.dimU == 1 ? cU : cW);
                    const int c2 = te.dimJ == 2 ? J0 : (te.dimU == 2 ? cU : cW);
                    mbar_arrive_expect_tx(bar, te.box_bytes + (PF ? (unsigned)RB : 0u));
                    tma_load_4d(tile_ptr(k), mapI(), bar, c0, c1, c2, v);
                    // rows J0 .. J0 + 8: the faces of the chunk starting at face J0
                    if constexpr (PF) bulk_load_1d((void*)srow(k, 0), row(J0), RB, bar);
                }
            } else {
                // each lane copies its own column's cells; cells past the end of
                // the column are zero-filled without being read
                unsigned char* tp = tile_ptr(k);
                const long long ncell = g.ns + 6;
                const T* col = column(u0, w, v);
                if (ORDER == 3 && KIND == 0 && sizeof(T) == 4 && te.ldr8) {
                    // WENO3 (latency-bound, few registers): the warp copies
                    // the tile together in 8-byte pairs.  In copy k, lane l
                    // takes pair l % 4 of column l / 4 + 8k, so one
                    // instruction reads 8 columns' 32 contiguous bytes (8
                    // sectors) rather than one pair of each of 32 columns;
                    // wait_tile then syncs the warp.  (WENO5 / WENO7 run
                    // 2-3% faster with the per-lane pairs below.)
                    const int pp = 2 * (lane & 3);
                    const long long J = (long long)J0 + pp;
                    const bool inb = J < ncell;
#pragma unroll
                    for (int kk = 0; kk < 4; ++kk) {
                        const int r = (lane >> 2) + 8 * kk;
                        const int uc = u0 + r < g.Nu ? u0 + r : g.Nu - 1;
                        const T* colr = (const T*)g.in + g.in_off + uc * g.sU + w * g.sW + v * g.sV;
                        const T* src = colr + (inb ? J : 0);
                        const unsigned dst = smem_u32(tp + swz<T>((unsigned)r, (unsigned)pp));
                        asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(dst), "l"(src),
                                     "r"(inb ? 8u : 0u)
                                     : "memory");
                    }
                } else if (KIND == 0 && sizeof(T) == 4 && te.ldr8) {
                    // contiguous, 8-byte aligned cell pairs (even J0, even column
                    // offsets, even ncell: a pair is wholly inside or outside the
                    // column); the 32-byte swizzle keeps pairs adjacent
#pragma unroll
                    for (int p = 0; p < F; p += 2) {
                        const long long J = (long long)J0 + p;
                        const bool inb = J < ncell;
                        const T* src = col + (inb ? J : 0);
                        const unsigned dst = smem_u32(tp + cell_off(p));
                        asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(dst), "l"(src),
                                     "r"(inb ? 8u : 0u)
                                     : "memory");
                    }
                } else {
#pragma unroll
                    for (int p = 0; p < F; ++p) {
                        const long long J = (long long)J0 + p;
                        const bool inb = J < ncell;
                        const T* src = col + (inb ? J : 0) * g.sJ;
                        const unsigned dst = smem_u32(tp + cell_off(p));
                        asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;\n" ::"r"(dst), "l"(src),
                                     "n"(sizeof(T)), "r"(inb ? (unsigned)sizeof(T) : 0u)
                                     : "memory");
                    }
                }
                asm volatile("cp.async.commit_group;\n" ::: "memory");
            }
        };
        auto wait_tile = [&](unsigned k) -> bool {
            if (!ldr) {
                if (!mbar_wait(&bars[k % S], parity(k))) return false;
                phase_done(k);
            } else {
                // copy groups issued after tile k may stay in flight (every
                // tile of earlier items has been waited on)
                const unsigned after = n_issued - (k + 1);
                if (after >= 3) asm volatile("cp.async.wait_group 3;\n" ::: "memory");
                else if (after == 2) asm volatile("cp.async.wait_group 2;\n" ::: "memory");
                else if (after == 1) asm volatile("cp.async.wait_group 1;\n" ::: "memory");
                else asm volatile("cp.async.wait_group 0;\n" ::: "memory");
                // the cooperative WENO3 loader fills rows that other lanes read
                if (ORDER == 3 && KIND == 0 && sizeof(T) == 4 && te.ldr8) __syncwarp();
            }
            n_waited = k + 1;
            return true;
        };

        const int sg = (int)(li % g.n_seg);
        long long tt = li / g.n_seg;
        const int ut = (int)(tt % g.n_ut);
        tt /= g.n_ut;
        const int wv = (int)(tt % g.Nw);
        const int vv = (int)(tt / g.Nw);
        const int u0 = ut * 32;
        const int f_start = (ORDER == 3 ? 0 : 4) + sg * g.seg;    // 4 mod 8 (WENO3: 0 mod 8)
        int f_end = f_start + g.seg;
        if (f_end > o_last) f_end = o_last;
        const int nch = f_end > f_start ? (f_end - f_start + F - 1) / F : 0;
        const int ntiles = nch + 1;                               // tiles 0 .. nch
        const unsigned k0 = n_issued;                             // first tile of this item
        if (MULTI && !ldr) {
            // the ring's stages may last have been written by per-lane copies
            fence_async_shared();
            __syncwarp();
        }
        for (int k = 0; k < ntiles && k < S; ++k) issue(k0 + k, f_start + F * k, u0, wv, vv);
        n_issued += (ntiles < S ? ntiles : S);
        if (!wait_tile(k0)) { failed = true; break; }

        Engine w;
        if (sg == 0 && ORDER != 3) {
            // face 3 (cells 4..8 = tile positions 0..4), plain stores
            T L, R;
            bool ok;
            if constexpr (ORDER == 7) {
                // face 3 reads cells 3 .. 9: cell 3 lies before tile 0 (cells 4 .. 11)
                const T c3 = __ldg(column(u0, wv, vv) + 3 * g.sJ);
                if constexpr (PF) {
                    w.init(a, Row7{row(0)}, Row7{row(1)}, Row7{row(2)}, Row7{row(3)}, c3, cell(k0, 0), cell(k0, 1),
                           cell(k0, 2), cell(k0, 3), cell(k0, 4), cell(k0, 5));
                    if constexpr (TENOW) ok = w.template face_teno<MPF>(a, Row7{row(3)}, L, R);
                    else ok = w.template face<MPF>(a, Row7{row(3)}, L, R);
                } else {
                    w.init(a, c3, cell(k0, 0), cell(k0, 1), cell(k0, 2), cell(k0, 3), cell(k0, 4), cell(k0, 5));
                    if constexpr (TENOW) ok = w.template face_teno<MPF>(a, L, R);
                    else ok = w.template face<MPF>(a, L, R);
                }
            } else if constexpr (PF && ORDER == 5) {
                w.init(a, BetaRow(row(1)), BetaRow(row(2)), BetaRow(row(3)), cell(k0, 0), cell(k0, 1), cell(k0, 2),
                       cell(k0, 3), cell(k0, 4));
                if constexpr (TENOW) ok = w.template face_teno<MPF>(a, FaceRow(row(3)), L, R);
                else if constexpr (WS == 2) ok = w.template face_z<MPF>(a, FaceRow(row(3)), L, R);
                else ok = w.template face<MPF>(a, FaceRow(row(3)), L, R);
            } else if constexpr (TENOW) {
                w.init(a, cell(k0, 0), cell(k0, 1), cell(k0, 2), cell(k0, 3), cell(k0, 4));
                ok = w.template face_teno<MPF>(a, L, R);
            } else if constexpr (WS == 1 || WS == 2) {
                w.init(a, cell(k0, 0), cell(k0, 1), cell(k0, 2), cell(k0, 3), cell(k0, 4));
                if constexpr (WS == 1) ok = w.template face_mapped<MPF>(a, L, R);
                else ok = w.template face_z<MPF>(a, L, R);
            } else {
                w.init(a, cell(k0, 0), cell(k0, 1), cell(k0, 2), cell(k0, 3), cell(k0, 4));
                ok = w.template face<MPF>(a, L, R);
            }
            if (!ok) {
                // (the redo sequences take the weights and strides from the
                // sweep's arguments)
                if constexpr (ORDER == 7 && PF) march64_7_redo_faces<MPF>(ga(), column(u0, wv, vv), 3, L, R);
                else if constexpr (ORDER == 7) march7_redo<MPF>(ga(), column(u0, wv, vv), 3, L, R);
                else march_redo<MPF, PF>(ga(), column(u0, wv, vv), 3, L, R);
            }
            if (u0 + lane < g.Nu) {
                const long long oi = 3 + (long long)(u0 + lane) * g.oU + wv * g.oW + vv * g.oV;
                outL[oi] = L;
                outR[oi] = R;
            }
            if constexpr (ORDER == 7 && PF) w.push(a, Row7{row(4)}, cell(k0, 6));
            else if constexpr (ORDER == 7) w.push(a, cell(k0, 6));
            else if constexpr (PF) w.push(a, BetaRow(row(4)), cell(k0, 5));
            else w.push(a, cell(k0, 5));
        } else {
            if constexpr (ORDER == 3 && PF)
                w.init(a, Row3{row(f_start)}, cell(k0, 1), cell(k0, 2), cell(k0, 3), cell(k0, 4), cell(k0, 5));
            else if constexpr (ORDER == 7 && PF)
                w.init(a, Row7{row(f_start - 3)}, Row7{row(f_start - 2)}, Row7{row(f_start - 1)}, Row7{row(f_start)},
                       cell(k0, 0), cell(k0, 1), cell(k0, 2), cell(k0, 3), cell(k0, 4), cell(k0, 5), cell(k0, 6));
            else if constexpr (ORDER == 7)
                w.init(a, cell(k0, 0), cell(k0, 1), cell(k0, 2), cell(k0, 3), cell(k0, 4), cell(k0, 5), cell(k0, 6));
            else if constexpr (PF)
                w.init(a, BetaRow(row(f_start - 2)), BetaRow(row(f_start - 1)), BetaRow(row(f_start)), cell(k0, 1),
                       cell(k0, 2), cell(k0, 3), cell(k0, 4), cell(k0, 5));
            else
                w.init(a, cell(k0, 1), cell(k0, 2), cell(k0, 3), cell(k0, 4), cell(k0, 5));
        }
        // chunk c: faces f0 .. f0+7 (f0 = f_start + 8c), pushes cells
        // f0+6 .. f0+13 = positions 6, 7 of tile c and 0 .. 5 of tile c+1
        for (int c = 0; c < nch; ++c) {
            const unsigned kc = k0 + c;
            if (!wait_tile(kc + 1)) { failed = true; break; }
            const int f0 = f_start + F * c;
            unsigned char* ob = obuf + (size_t)(n_chunks % NOUT) * (2 * OB);
            // the store issued from this buffer NOUT chunks ago must have read
            // it before the chunk's face states are written: waited here, or
            // (one output buffer) just before the first write, so the first
            // faces' arithmetic overlaps it.  A chunk of plain stores waits
            // for every store in flight (grouped sweeps: the last bulk store
            // may be the one from this buffer)
            const bool wait_out = n_chunks >= (unsigned)NOUT;
            if (NOUT > 1 && wait_out) {
                if (lane == 0) {
                    if (MULTI && pst) bulk_wait_read0();
                    else bulk_wait_read1();
                }
                __syncwarp();
            }
            unsigned bad = 0;
            // face states leave as 16-byte groups (G faces) of the lane's
            // row; row-tile cells arrive as 16-byte groups too (the swizzle
            // moves whole 16-byte chunks), column-tile cells one by one
            constexpr int G = 16 / (int)sizeof(T);
            T Lg[G], Rg[G], cg[G];
#pragma unroll
            for (int i = 0; i < F; ++i) {
                const int q = PUSH0 + i;                  // position of the pushed cell, tiles c / c+1
                const unsigned kq = q < 8 ? kc : kc + 1;
                const int pq = q & 7;
                if constexpr (KIND == 0) {
                    if (i == 0 || pq % G == 0) {
                        const int p0 = pq - pq % G;
                        const unsigned char* src = tile_ptr(kq) + swz<T>((unsigned)lane, (unsigned)p0);
                        if constexpr (sizeof(T) == 8) {
                            const double2 v2 = *(const double2*)src;
                            cg[0] = v2.x; cg[1] = v2.y;
                        } else {
                            const float4 v4 = *(const float4*)src;
                            cg[0] = v4.x; cg[1] = v4.y; cg[2] = v4.z; cg[3] = v4.w;
                        }
                    }
                }
                T L, R;
                bool ok;
                if constexpr (ORDER == 3 && PF)
                    ok = w.template face<MPF>(a, Row3{srow(kc, i)}, L, R, f0 + i >= 3 && f0 + i <= o_last - 4);
                else if constexpr (ORDER == 3) ok = w.template face<MPF>(a, L, R, f0 + i >= 3 && f0 + i <= o_last - 4);
                else if constexpr (PF && ORDER == 7 && TENOW) ok = w.template face_teno<MPF>(a, Row7{srow(kc, i)}, L, R);
                else if constexpr (PF && ORDER == 7) ok = w.template face<MPF>(a, Row7{srow(kc, i)}, L, R);
                else if constexpr (PF && TENOW) ok = w.template face_teno<MPF>(a, FaceRow(srow(kc, i)), L, R);
                else if constexpr (PF && WS == 2) ok = w.template face_z<MPF>(a, FaceRow(srow(kc, i)), L, R);
                else if constexpr (PF) ok = w.template face<MPF>(a, FaceRow(srow(kc, i)), L, R);
                else if constexpr (TENOW) ok = w.template face_teno<MPF>(a, L, R);
                else if constexpr (WS == 2) ok = w.template face_z<MPF>(a, L, R);
                else if constexpr (WS == 1) ok = w.template face_mapped<MPF>(a, L, R);
                else ok = w.template face<MPF>(a, L, R);
                if (!ok) bad |= 1u << i;
                Lg[i % G] = L;
                Rg[i % G] = R;
                if (NOUT == 1 && i == G - 1 && wait_out) {
                    if (lane == 0) bulk_wait_read0();
                    __syncwarp();
                }
                if (i % G == G - 1) {
                    unsigned char* dL = ob + swz<T>((unsigned)lane, (unsigned)(i - G + 1));
                    if constexpr (sizeof(T) == 8) {
                        *(double2*)dL = make_double2(Lg[0], Lg[1]);
                        *(double2*)(dL + OB) = make_double2(Rg[0], Rg[1]);
                    } else {
                        *(float4*)dL = make_float4(Lg[0], Lg[1], Lg[2], Lg[3]);
                        *(float4*)(dL + OB) = make_float4(Rg[0], Rg[1], Rg[2], Rg[3]);
                    }
                }
                T n;
                if constexpr (KIND == 0) n = cg[pq % G];
                else n = cell(kq, pq);
                if constexpr (PF && ORDER == 7) w.push(a, Row7{srow(kc, i + 1)}, n);
                else if constexpr (PF && ORDER == 3) w.push(a, Row3{srow(kc, i + 1)}, n);
                else if constexpr (PF) w.push(a, BetaRow(srow(kc, i + 1)), n);
                else w.push(a, n);
            }
            const int nF = f_end - f0 < F ? f_end - f0 : F;
            bad &= (1u << nF) - 1u;
            if (bad) {
                const T* col = column(u0, wv, vv);
                while (bad) {
                    const int i = __ffs(bad) - 1;
                    bad &= bad - 1;
                    T L, R;
                    if constexpr (ORDER == 7 && PF) march64_7_redo_faces<MPF>(ga(), col, f0 + i, L, R);
                    else if constexpr (ORDER == 7) march7_redo<MPF>(ga(), col, f0 + i, L, R);
                    else if constexpr (ORDER == 3 && PF) march3_redo_faces<MPF>(ga(), col, f0 + i, L, R);
                    else if constexpr (ORDER == 3) march3_redo<MPF, T>(ga(), col, f0 + i, L, R);
                    else march_redo<MPF, PF>(ga(), col, f0 + i, L, R);
                    *(T*)(ob + swz<T>((unsigned)lane, (unsigned)i)) = L;
                    *(T*)(ob + OB + swz<T>((unsigned)lane, (unsigned)i)) = R;
                }
            }
            if (pst) {
                // plain stores: lane l writes face f0 + l % 8 of columns
                // l / 8, l / 8 + 4, ..., so one instruction writes four
                // columns' runs of 8 consecutive faces
                __syncwarp();
                const int fi = lane & (F - 1);
                if (fi < nF) {
                    // (a rolled loop with one running index: unrolled, its
                    // addresses took 24 registers of the face body)
                    const int c_end = g.Nu - u0 < 32 ? g.Nu - u0 : 32;
                    const long long step = (long long)(32 / F) * g.oU;
                    long long oi = (long long)(f0 + fi) + (long long)(u0 + lane / F) * g.oU + wv * g.oW + vv * g.oV;
#pragma unroll 1
                    for (int cc = lane / F; cc < c_end; cc += 32 / F, oi += step) {
                        outL[oi] = *(const T*)(ob + swz<T>((unsigned)cc, (unsigned)fi));
                        outR[oi] = *(const T*)(ob + OB + swz<T>((unsigned)cc, (unsigned)fi));
                    }
                }
            } else {
                const int i_last = ORDER == 3 ? -1 : o_last - 1 - f0;  // the last core face, when in this chunk
                if (i_last >= 0 && i_last < F && u0 + lane < g.Nu) {
                    // outside the store map's extent (see plan_march_tma)
                    const long long oi = (o_last - 1) + (long long)(u0 + lane) * g.oU + wv * g.oW + vv * g.oV;
                    outL[oi] = *(const T*)(ob + swz<T>((unsigned)lane, (unsigned)i_last));
                    outR[oi] = *(const T*)(ob + OB + swz<T>((unsigned)lane, (unsigned)i_last));
                }
                fence_async_shared();
                __syncwarp();
                if (lane == 0) {
                    const int c1 = te.odimU == 1 ? u0 : wv, c2 = te.odimU == 2 ? u0 : wv;
                    tma_store_4d(mapL(), ob, f0, c1, c2, vv);
                    tma_store_4d(mapR(), ob + OB, f0, c1, c2, vv);
                    bulk_commit();
                }
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
        // (only TMA tiles fail, and an item's tiles are all of one kind)
        for (unsigned k = n_waited; k < n_issued; ++k) {
            mbar_wait(&bars[k % S], parity(k));
            phase_done(k);
        }
    }
    if (LDR == 1 || MULTI) asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    if (lane == 0) bulk_wait_all();
    __syncwarp();
}

#ifndef WSB_MTMA_MIN_BLOCKS_F32
#define WSB_MTMA_MIN_BLOCKS_F32 3
#endif
#ifndef WSB_MTMA_MIN_BLOCKS_W7
#define WSB_MTMA_MIN_BLOCKS_W7 2  // WENO7 carries ~27 doubles of state: 3 CTAs per SM would spill
#endif
#define WSB_MTMA_BOUNDS(ORDER, T)                                                      \
    __launch_bounds__(kTmaWarps * 32, (ORDER) == 7 ? WSB_MTMA_MIN_BLOCKS_W7            \
                                                   : (sizeof(T) == 8 ? WSB_MTMA_MIN_BLOCKS : WSB_MTMA_MIN_BLOCKS_F32))

// One sweep: maps and arguments in the parameter bank.
template <bool MPF, int KIND, typename T, int LDR, bool PF, int ORDER = 5, int WS = 0>
__global__ void WSB_MTMA_BOUNDS(ORDER, T)
    sweep_march_tma_kernel(const __grid_constant__ CUtensorMap tin, const __grid_constant__ CUtensorMap toutL,
                           const __grid_constant__ CUtensorMap toutR, const __grid_constant__ MarchArgs a,
                           const MarchTmaArgs t) {
    march_tma_body<MPF, KIND, T, LDR, PF, ORDER, WS, false>(&tin, &toutL, &toutR, a, t, nullptr, nullptr, 0,
                                                              a.n_items);
}

// A group of sweeps in one launch: entries (64-byte aligned, in global
// memory, written before the launch) in item order, n_items in all;
// coefficients and shared-memory layout of the group in a and t.
// CTAs per SM the FP64 grouped kernels are bounded for: column tiles 3
// (WENO5's body fits 168 registers there), row tiles 2 (at 3 their WENO5
// body spills 36-44 bytes and runs 2-3% slower); FP32 3.
#ifndef WSB_MTMA_MULTI_MIN_BLOCKS
#define WSB_MTMA_MULTI_MIN_BLOCKS 2     // FP64 row tiles
#endif
#ifndef WSB_MTMA_MULTI_MIN_BLOCKS_K1
#define WSB_MTMA_MULTI_MIN_BLOCKS_K1 3  // FP64 column tiles
#endif
template <bool MPF, int KIND, typename T, int ORDER, int WS>
__global__ void __launch_bounds__(kTmaWarps * 32,
                                  ORDER == 7 ? WSB_MTMA_MIN_BLOCKS_W7
                                             : (sizeof(T) == 8 ? (KIND == 1 ? WSB_MTMA_MULTI_MIN_BLOCKS_K1
                                                                            : WSB_MTMA_MULTI_MIN_BLOCKS)
                                                               : WSB_MTMA_MIN_BLOCKS_F32))
    sweep_march_tma_multi_kernel(const MtmaEntry* __restrict__ ents, const long long* __restrict__ item0s,
                                 int n_ents, long long n_items, const __grid_constant__ MarchArgs a,
                                 const MarchTmaArgs t) {
    march_tma_body<MPF, KIND, T, 0, false, ORDER, WS, true>(nullptr, nullptr, nullptr, a, t, ents, item0s, n_ents,
                                                              n_items);
}

// Host side.  A sweep's plan: its maps, arguments and shared-memory layout.
// Inputs come by TMA when the field's rows are 16-byte multiples from a
// 16-byte aligned base, else by per-lane copies into the same tiles; face
// states leave by TMA stores when the face rows (ns elements) are 16-byte
// multiples from 16-byte aligned bases, else by plain stores from the same
// staging tiles.  seg_faces > 0 cuts every column into segments of about
// that many faces; 0 sizes the segments to fill `sms` SMs about eight
// work items per resident warp.  Returns 1003 (unsupported) for sweeps of
// fewer than 8 faces, a lane axis the march arguments did not choose, or a
// missing driver entry point.
struct MtmaPlan {
    CUtensorMap mi, mL, mR;
    MarchArgs a;
    MarchTmaArgs t;
    size_t smem;
};

template <typename T>
int plan_march_tma(const long long E[3], const SweepGeom& g, int dir, bool folded, const T* in, T* vL, T* vR,
                   const MarchArgs& a0, int sms, int order, long long seg_faces, MtmaPlan& P) {
    constexpr int ES = (int)sizeof(T);
    EncodeTiledFn enc = encode_tiled_fn();
    if (!enc) return 1003;
    if (((uintptr_t)in) & (ES - 1)) return 1003;
    if ((((uintptr_t)vL) | ((uintptr_t)vR)) & (ES - 1)) return 1003;
    if (g.ns < 8) return 1003;
    std::memset(&P, 0, sizeof(P));
    MarchArgs& a = P.a;
    MarchTmaArgs& t = P.t;
    a = a0;
    const bool kind1 = folded && dir != 0;
    t.kind = kind1 ? 1 : 0;
    cuuint64_t dims[4], strides[3];
    cuuint32_t box[4], estr[4] = {1, 1, 1, 1};
    CUtensorMapSwizzle swz;
    const int xw = ES == 8 ? 34 : 36;  // column-tile width: starts 16-byte aligned, left of column 0
    if (!folded) {
        // v_rs_ws (ns+6, c1, c2, V): lanes along c1
        dims[0] = g.ns + 6; dims[1] = g.c1; dims[2] = g.c2; dims[3] = g.nv;
        t.dimJ = 0; t.dimU = 1; t.dimW = 2; t.uoff = 0; t.woff = 0;
    } else {
        // v_vf: column u, w sit at pad + 3; the column tile starts xw - 32 - 1 cells left of column 0
        dims[0] = E[0]; dims[1] = E[1]; dims[2] = E[2]; dims[3] = g.nv;
        const int xo = 3 - (xw - 32 - 1);
        if (dir == 0) { t.dimJ = 0; t.dimU = 1; t.dimW = 2; t.uoff = 3; t.woff = 3; }
        else if (dir == 1) { t.dimJ = 1; t.dimU = 0; t.dimW = 2; t.uoff = xo; t.woff = 3; }
        else { t.dimJ = 2; t.dimU = 0; t.dimW = 1; t.uoff = xo; t.woff = 3; }
    }
    if (!kind1) {
        box[0] = kTmaF; box[1] = 32; box[2] = 1; box[3] = 1;
        swz = ES == 8 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_32B;
        t.stage_bytes = kTmaF * 32 * ES;
    } else {
        box[0] = xw; box[1] = 1; box[2] = 1; box[3] = 1;
        box[t.dimJ] = kTmaF;
        swz = CU_TENSOR_MAP_SWIZZLE_NONE;
        t.stage_bytes = ((kTmaF * xw * ES + 127) / 128) * 128;
    }
    t.box_bytes = (unsigned)(box[0] * box[1] * box[2] * box[3] * ES);
    strides[0] = dims[0] * ES;
    strides[1] = dims[0] * dims[1] * ES;
    strides[2] = dims[0] * dims[1] * dims[2] * ES;
    const CUtensorMapDataType dt = ES == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    // input tiles by TMA when the field's rows are 16-byte multiples and its
    // base is 16-byte aligned; otherwise (e.g. FP32 rows of 218 cells) each
    // lane stages its own cells with cp.async into the same tile layout
    t.ldr = 1;
    if (strides[0] % 16 == 0 && (((uintptr_t)in) & 15) == 0 &&
        enc(&P.mi, dt, 4, (void*)in, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, swz,
            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS)
        t.ldr = 0;
    // per-lane loader in 8-byte pairs: float row tiles whose column starts
    // are all even cells from an 8-byte aligned base (chunks start at even
    // cells, and an even column length keeps every pair inside or outside)
    t.ldr8 = (ES == 4 && !kind1 && a.sJ == 1 && ((uintptr_t)in & 7) == 0 && (a.in_off & 1) == 0 &&
              (a.sU & 1) == 0 && (a.sW & 1) == 0 && (a.sV & 1) == 0 && ((g.ns + 6) & 1) == 0)
                 ? 1
                 : 0;
    // outputs (ns, c1, c2, V).  The store unit clips the innermost axis in
    // 16-byte steps, so the face extent is ns - 4 (a 16-byte multiple):
    // faces up to ns-5 are stored by the TMA unit, the last core face ns-4
    // with plain stores, and the non-core faces ns-3 .. ns-1 are never written.
    // (WENO3 writes every face: extent ns)
    cuuint64_t od[4] = {(cuuint64_t)(order == 3 ? g.ns : g.ns - 4), (cuuint64_t)g.c1, (cuuint64_t)g.c2,
                        (cuuint64_t)g.nv};
    cuuint64_t os[3] = {(cuuint64_t)g.ns * ES, (cuuint64_t)(g.ns * g.c1) * ES, (cuuint64_t)(g.ns * g.c1 * g.c2) * ES};
    cuuint32_t ob[4] = {kTmaF, 1, 1, 1};
    // lanes run along the output axis the march arguments chose (oU == ns: c1, else c2)
    if (a.oU == g.ns) { t.odimU = 1; t.odimW = 2; }
    else { t.odimU = 2; t.odimW = 1; }
    ob[t.odimU] = 32;
    const CUtensorMapSwizzle oswz = ES == 8 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_32B;
    t.pst = 1;
    if (((g.ns * ES) & 15) == 0 && ((((uintptr_t)vL) | ((uintptr_t)vR)) & 15) == 0 &&
        enc(&P.mL, dt, 4, (void*)vL, od, os, ob, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, oswz,
            CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS &&
        enc(&P.mR, dt, 4, (void*)vR, od, os, ob, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, oswz,
            CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS)
        t.pst = 0;
    // the lane axis must be the one the march arguments chose
    if ((t.kind == 1) != (a.sU == 1)) return 1003;
    // segments over faces [4, ns-3), a multiple of 8 faces each
    const long long nf4 = order == 3 ? g.ns : g.ns - 7;  // faces in the chunked range
    const long long cols = (long long)a.n_ut * a.Nw * a.NV;
#ifndef WSB_MTMA_ITEMS_PER_WARP
#define WSB_MTMA_ITEMS_PER_WARP 8  // target work items per resident warp (200^3: two segments per column)
#endif
    long long nseg;
    if (seg_faces > 0) {
        nseg = (nf4 + seg_faces - 1) / seg_faces;
    } else {
        const long long want = (long long)sms * kTmaWarps * 3 * WSB_MTMA_ITEMS_PER_WARP;
        nseg = (want + cols - 1) / cols;
    }
    const long long max_seg = (nf4 + kTmaF - 1) / kTmaF;
    if (nseg > max_seg) nseg = max_seg;
    if (nseg < 1) nseg = 1;
    long long seg = (nf4 + nseg - 1) / nseg;
    seg = ((seg + kTmaF - 1) / kTmaF) * kTmaF;
    a.seg = (int)seg;
    a.n_seg = (int)((nf4 + seg - 1) / seg);
    a.n_items = cols * a.n_seg;
    const bool pf = a.ftab != nullptr;
    const int nst = pf ? kPfStages : kTmaStages;
    const int out_bytes = (pf ? kPfOut : kTmaOut) * 2 * 32 * kTmaF * ES;
    t.ring_off = out_bytes;
    t.rows_off = out_bytes + nst * t.stage_bytes;
    t.warp_bytes = ((t.rows_off + (pf ? nst * pf_chunk_bytes(order) : 0) + 1023) / 1024) * 1024;
    P.smem = 1024 + (size_t)kTmaWarps * t.warp_bytes + (size_t)kTmaWarps * nst * 8;
    return 0;
}

// One sweep.  Returns 1003 (unsupported) as plan_march_tma, for face rows
// that are not 16-byte multiples, or for a per-face table whose field does
// not suit TMA; the caller then uses another kernel.
template <typename T>
int launch_march_tma(const long long E[3], const SweepGeom& g, int dir, bool folded, bool mp, const T* in, T* vL,
                     T* vR, const MarchArgs& a0, cudaStream_t st, int sms, int order = 5, int ws = 0) {
    MtmaPlan P;
    const int prc = plan_march_tma<T>(E, g, dir, folded, in, vL, vR, a0, sms, order, 0, P);
    if (prc) return prc;
    // face rows that are not 16-byte multiples: the grouped kernel's plain
    // stores (batches), other kernels here
    if (P.t.pst) return 1003;
    const MarchArgs& a = P.a;
    const MarchTmaArgs& t = P.t;
    const bool kind1 = t.kind == 1;
    const int ldr = t.ldr;
    const size_t smem = P.smem;
    using KFn = void (*)(CUtensorMap, CUtensorMap, CUtensorMap, MarchArgs, MarchTmaArgs);
    static const KFn table[2][2][2] = {
        {{sweep_march_tma_kernel<false, 0, T, 0, false>, sweep_march_tma_kernel<false, 0, T, 1, false>},
         {sweep_march_tma_kernel<false, 1, T, 0, false>, sweep_march_tma_kernel<false, 1, T, 1, false>}},
        {{sweep_march_tma_kernel<true, 0, T, 0, false>, sweep_march_tma_kernel<true, 0, T, 1, false>},
         {sweep_march_tma_kernel<true, 1, T, 0, false>, sweep_march_tma_kernel<true, 1, T, 1, false>}}};
    KFn kfn = table[mp ? 1 : 0][kind1 ? 1 : 0][ldr];
    const bool teno = ws == 3;
    if ((ws == 1 || ws == 2) && (order != 5 || sizeof(T) != 8 || (ws == 1 && a.ftab))) return 1003;
    if (ws == 2 && a.ftab) {
        // WENO5-Z with the per-face table: FP64 with TMA input tiles
        if constexpr (sizeof(T) == 8) {
            if (ldr) return 1003;
            static const KFn ptablez[2][2] = {
                {sweep_march_tma_kernel<false, 0, T, 0, true, 5, 2>, sweep_march_tma_kernel<false, 1, T, 0, true, 5, 2>},
                {sweep_march_tma_kernel<true, 0, T, 0, true, 5, 2>, sweep_march_tma_kernel<true, 1, T, 0, true, 5, 2>}};
            kfn = ptablez[mp ? 1 : 0][kind1 ? 1 : 0];
        }
    } else if (ws == 1 || ws == 2) {
        // mapped / Z weights of WENO5, FP64, face-independent coefficients
        if constexpr (sizeof(T) == 8) {
            static const KFn tablemz[2][2][2][2] = {
                {{{sweep_march_tma_kernel<false, 0, T, 0, false, 5, 1>, sweep_march_tma_kernel<false, 0, T, 1, false, 5, 1>},
                  {sweep_march_tma_kernel<false, 1, T, 0, false, 5, 1>, sweep_march_tma_kernel<false, 1, T, 1, false, 5, 1>}},
                 {{sweep_march_tma_kernel<true, 0, T, 0, false, 5, 1>, sweep_march_tma_kernel<true, 0, T, 1, false, 5, 1>},
                  {sweep_march_tma_kernel<true, 1, T, 0, false, 5, 1>, sweep_march_tma_kernel<true, 1, T, 1, false, 5, 1>}}},
                {{{sweep_march_tma_kernel<false, 0, T, 0, false, 5, 2>, sweep_march_tma_kernel<false, 0, T, 1, false, 5, 2>},
                  {sweep_march_tma_kernel<false, 1, T, 0, false, 5, 2>, sweep_march_tma_kernel<false, 1, T, 1, false, 5, 2>}},
                 {{sweep_march_tma_kernel<true, 0, T, 0, false, 5, 2>, sweep_march_tma_kernel<true, 0, T, 1, false, 5, 2>},
                  {sweep_march_tma_kernel<true, 1, T, 0, false, 5, 2>, sweep_march_tma_kernel<true, 1, T, 1, false, 5, 2>}}}};
            kfn = tablemz[ws == 2 ? 1 : 0][mp ? 1 : 0][kind1 ? 1 : 0][ldr];
        }
    } else if (teno && a.ftab) {
        // TENO with the per-face table (WENO5, WENO7): FP64 with TMA input tiles
        if constexpr (sizeof(T) == 8) {
            if (ldr) return 1003;
            static const KFn ptablet[2][2][2] = {
                {{sweep_march_tma_kernel<false, 0, T, 0, true, 5, 3>, sweep_march_tma_kernel<false, 1, T, 0, true, 5, 3>},
                 {sweep_march_tma_kernel<true, 0, T, 0, true, 5, 3>, sweep_march_tma_kernel<true, 1, T, 0, true, 5, 3>}},
                {{sweep_march_tma_kernel<false, 0, T, 0, true, 7, 3>, sweep_march_tma_kernel<false, 1, T, 0, true, 7, 3>},
                 {sweep_march_tma_kernel<true, 0, T, 0, true, 7, 3>, sweep_march_tma_kernel<true, 1, T, 0, true, 7, 3>}}};
            kfn = ptablet[order == 7 ? 1 : 0][mp ? 1 : 0][kind1 ? 1 : 0];
        } else {
            return 1003;
        }
    } else if (teno) {
        // TENO weights, WENO5 or WENO7: face-independent coefficients
        static const KFn tablet[2][2][2][2] = {
            {{{sweep_march_tma_kernel<false, 0, T, 0, false, 5, 3>,
               sweep_march_tma_kernel<false, 0, T, 1, false, 5, 3>},
              {sweep_march_tma_kernel<false, 1, T, 0, false, 5, 3>,
               sweep_march_tma_kernel<false, 1, T, 1, false, 5, 3>}},
             {{sweep_march_tma_kernel<true, 0, T, 0, false, 5, 3>,
               sweep_march_tma_kernel<true, 0, T, 1, false, 5, 3>},
              {sweep_march_tma_kernel<true, 1, T, 0, false, 5, 3>,
               sweep_march_tma_kernel<true, 1, T, 1, false, 5, 3>}}},
            {{{sweep_march_tma_kernel<false, 0, T, 0, false, 7, 3>,
               sweep_march_tma_kernel<false, 0, T, 1, false, 7, 3>},
              {sweep_march_tma_kernel<false, 1, T, 0, false, 7, 3>,
               sweep_march_tma_kernel<false, 1, T, 1, false, 7, 3>}},
             {{sweep_march_tma_kernel<true, 0, T, 0, false, 7, 3>,
               sweep_march_tma_kernel<true, 0, T, 1, false, 7, 3>},
              {sweep_march_tma_kernel<true, 1, T, 0, false, 7, 3>,
               sweep_march_tma_kernel<true, 1, T, 1, false, 7, 3>}}}};
        kfn = tablet[order == 7 ? 1 : 0][mp ? 1 : 0][kind1 ? 1 : 0][ldr];
    } else if (order == 3 && a.ftab) {
        // WENO3-JS with the per-face table: FP64 with TMA input tiles
        if constexpr (sizeof(T) == 8) {
            if (ldr) return 1003;
            static const KFn ptable3[2][2] = {
                {sweep_march_tma_kernel<false, 0, T, 0, true, 3>, sweep_march_tma_kernel<false, 1, T, 0, true, 3>},
                {sweep_march_tma_kernel<true, 0, T, 0, true, 3>, sweep_march_tma_kernel<true, 1, T, 0, true, 3>}};
            kfn = ptable3[mp ? 1 : 0][kind1 ? 1 : 0];
        } else {
            return 1003;
        }
    } else if (order == 3) {
        // WENO3: JS, face-independent coefficients
        static const KFn table3[2][2][2] = {
            {{sweep_march_tma_kernel<false, 0, T, 0, false, 3>, sweep_march_tma_kernel<false, 0, T, 1, false, 3>},
             {sweep_march_tma_kernel<false, 1, T, 0, false, 3>, sweep_march_tma_kernel<false, 1, T, 1, false, 3>}},
            {{sweep_march_tma_kernel<true, 0, T, 0, false, 3>, sweep_march_tma_kernel<true, 0, T, 1, false, 3>},
             {sweep_march_tma_kernel<true, 1, T, 0, false, 3>, sweep_march_tma_kernel<true, 1, T, 1, false, 3>}}};
        kfn = table3[mp ? 1 : 0][kind1 ? 1 : 0][ldr];
    } else if (order == 7 && a.ftab) {
        // WENO7-JS with the per-face table: FP64 with TMA input tiles
        if constexpr (sizeof(T) == 8) {
            if (ldr) return 1003;
            static const KFn ptable7[2][2] = {
                {sweep_march_tma_kernel<false, 0, T, 0, true, 7>, sweep_march_tma_kernel<false, 1, T, 0, true, 7>},
                {sweep_march_tma_kernel<true, 0, T, 0, true, 7>, sweep_march_tma_kernel<true, 1, T, 0, true, 7>}};
            kfn = ptable7[mp ? 1 : 0][kind1 ? 1 : 0];
        } else {
            return 1003;
        }
    } else if (order == 7) {
        // WENO7: face-independent coefficients
        static const KFn table7[2][2][2] = {
            {{sweep_march_tma_kernel<false, 0, T, 0, false, 7>, sweep_march_tma_kernel<false, 0, T, 1, false, 7>},
             {sweep_march_tma_kernel<false, 1, T, 0, false, 7>, sweep_march_tma_kernel<false, 1, T, 1, false, 7>}},
            {{sweep_march_tma_kernel<true, 0, T, 0, false, 7>, sweep_march_tma_kernel<true, 0, T, 1, false, 7>},
             {sweep_march_tma_kernel<true, 1, T, 0, false, 7>, sweep_march_tma_kernel<true, 1, T, 1, false, 7>}}};
        kfn = table7[mp ? 1 : 0][kind1 ? 1 : 0][ldr];
    } else if (a.ftab) {
        // face-dependent coefficients: FP64 with TMA input tiles
        if constexpr (sizeof(T) == 8) {
            if (ldr) return 1003;
            static const KFn ptable[2][2] = {
                {sweep_march_tma_kernel<false, 0, T, 0, true>, sweep_march_tma_kernel<false, 1, T, 0, true>},
                {sweep_march_tma_kernel<true, 0, T, 0, true>, sweep_march_tma_kernel<true, 1, T, 0, true>}};
            kfn = ptable[mp ? 1 : 0][kind1 ? 1 : 0];
        } else {
            return 1003;
        }
    }
    cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int occ = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kfn, kTmaWarps * 32, smem);
    if (occ < 1) return 1003;
    long long blocks = (a.n_items + kTmaWarps - 1) / kTmaWarps;
    const long long cap = (long long)sms * occ;
    if (blocks > cap) blocks = cap;
    kfn<<<(unsigned)blocks, kTmaWarps * 32, smem, st>>>(P.mi, P.mL, P.mR, a, t);
    return 0;
}

// Kernel of a group of sweeps, by storage T, order, weights, MP and tile
// kind (null for WENO3 with TENO weights, which no engine covers).
using MtmaMultiFn = void (*)(const MtmaEntry*, const long long*, int, long long, MarchArgs, MarchTmaArgs);
template <typename T, int ORDER, int WS>
MtmaMultiFn mtma_multi_pick(bool mp, bool kind1) {
    static const MtmaMultiFn tab[2][2] = {
        {sweep_march_tma_multi_kernel<false, 0, T, ORDER, WS>, sweep_march_tma_multi_kernel<false, 1, T, ORDER, WS>},
        {sweep_march_tma_multi_kernel<true, 0, T, ORDER, WS>, sweep_march_tma_multi_kernel<true, 1, T, ORDER, WS>}};
    return tab[mp ? 1 : 0][kind1 ? 1 : 0];
}
template <typename T>
MtmaMultiFn mtma_multi_kernel(int order, bool teno, bool mp, bool kind1) {
    if (order == 3) return teno ? nullptr : mtma_multi_pick<T, 3, 0>(mp, kind1);
    if (order == 7) return teno ? mtma_multi_pick<T, 7, 3>(mp, kind1) : mtma_multi_pick<T, 7, 0>(mp, kind1);
    return teno ? mtma_multi_pick<T, 5, 3>(mp, kind1) : mtma_multi_pick<T, 5, 0>(mp, kind1);
}

}  // namespace wsb
