// sweep_pipe.cuh -- TMA + mbarrier pipelined reconstruction sweep (FP64).
//
// Same work decomposition as the cp.async kernel (a CTA owns TJ faces, one
// consumer thread per face with its coefficients in registers, and walks
// column groups), but the staging is warp-specialised:
//   * one producer warp (lane 0) issues one cp.async.bulk.tensor per column
//     group into a ring of STAGES shared-memory buffers, arming the stage's
//     "full" mbarrier with the box's byte count;
//   * the consumer warps wait on "full", compute, and each warp arrives once
//     on the stage's "empty" mbarrier; the producer refills a stage only
//     after all consumer warps released it.
// No CTA-wide barrier sits in the loop, so a slow warp only delays the
// refill of the stage it still reads.
//
// Tiles.  KIND 0 (sweep axis innermost): box {SWp, U, 1, 1} over a rank-4
// map, plain row-major in shared memory.  KIND 1 (folded y/z, sweep axis
// strided): box of 16 x-values (128 bytes) by SWp rows along the sweep with
// the 128-byte swizzle, so a warp reading one x-column at 32 consecutive
// faces touches 8 distinct 16-byte bank groups per 8 rows.  The x-tiles
// start one cell left of a 16-cell boundary so that the TMA's innermost
// coordinate (x + 3 pad cells) is even, i.e. 16-byte aligned.
//
// Every wait is bounded (about one second of SM clock); on expiry the thread
// records WENO_SB_ERR_TIMEOUT in a device flag and leaves its loop, so a
// stuck copy turns into an error status instead of a hung GPU.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include "sweep_tma.cuh"

namespace wsb {

__device__ int g_wsb_device_error = 0;

// Tuning: CTAs per SM the FP64 WENO3/5 pipeline kernels are compiled for
// (register cap 65536 / (256 * this)), and whether WENO5-JS with
// face-independent coefficients processes two columns per iteration.
#ifndef WSB_PIPE_MIN_BLOCKS
#define WSB_PIPE_MIN_BLOCKS 2
#endif
#ifndef WSB_PIPE_PAIRS
#define WSB_PIPE_PAIRS 1
#endif
// Stage-ring depths of the row-tile (KIND 0) and swizzled column-tile
// (KIND 1) instances of WENO3/5; WENO7 keeps 6 / 3 (one CTA per SM).
#ifndef WSB_PIPE_STAGES0
#define WSB_PIPE_STAGES0 6
#endif
#ifndef WSB_PIPE_STAGES1
#define WSB_PIPE_STAGES1 3
#endif

constexpr long long kWaitLimitCycles = 2000000000LL;  // ~1 s at 2 GHz

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive(unsigned long long* bar) {
    asm volatile("{\n .reg .b64 st;\n mbarrier.arrive.shared::cta.b64 st, [%0];\n}\n" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long* bar, unsigned bytes) {
    asm volatile("{\n .reg .b64 st;\n mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n}\n" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try(unsigned addr, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(addr), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait for the phase with parity `parity` to complete.  The clock
// is read once every 16 polls; `backoff_ns` > 0 sleeps between polls (the
// producer uses it, since it has STAGES-1 stages of slack and would
// otherwise take issue slots from the consumer warps).
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity,
                                          long long limit = kWaitLimitCycles, unsigned backoff_ns = 0) {
    const unsigned addr = smem_u32(bar);
    if (mbar_try(addr, parity)) return true;
    const long long t0 = clock64();
    for (unsigned it = 1;; ++it) {
        if (backoff_ns) __nanosleep(backoff_ns);
        if (mbar_try(addr, parity)) return true;
        if ((it & 15u) == 0 && clock64() - t0 > limit) {
            atomicExch(&g_wsb_device_error, 1005 /* WENO_SB_ERR_TIMEOUT */);
            return false;
        }
    }
}

__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, unsigned long long* bar, int c0, int c1,
                                            int c2, int c3) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];\n" ::"r"(
            smem_u32(dst)),
        "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
        : "memory");
}

struct PipeArgs {
    FastArgs a;
    int KIND;
    int SWp;          // box extent along the sweep
    int off;          // KIND 0: window start J0 minus the box start (0 or 1)
    int stage_bytes;  // bytes of one stage buffer (multiple of 1024)
    unsigned box_bytes;
    int folded;       // 1: coordinates address v_vf (pad cells of 3 on cross axes)
    int dir;
};

template <int ORDER, bool MPF, int KIND, int STAGES, int SCH, bool UNI>
__global__ void __launch_bounds__(256, (ORDER == 7 ? 1 : WSB_PIPE_MIN_BLOCKS))
    sweep_pipe_kernel(const __grid_constant__ CUtensorMap tmap, const PipeArgs P) {
    using T = double;
    const FastArgs& a = P.a;
    extern __shared__ __align__(1024) unsigned char smem_pipe[];
    // 1024-byte aligned stage ring, then the barriers.  The ring pointer is
    // formed by indexing the shared array (not through an integer cast) so
    // the compiler keeps it in the shared window and emits LDS, not generic
    // loads.
    unsigned char* ring = smem_pipe + ((1024u - (smem_u32(smem_pipe) & 1023u)) & 1023u);
    unsigned long long* full = (unsigned long long*)(ring + (size_t)STAGES * P.stage_bytes);
    unsigned long long* empty = full + STAGES;
    constexpr int H = Halo<ORDER, MPF>::H;

    const int nwarps = blockDim.x >> 5;
    const int ncons = nwarps - 1;  // the last warp produces
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    const int jt = blockIdx.x % a.n_jt;
    const long long g0 = blockIdx.x / a.n_jt;
    const long long gstep = gridDim.x / a.n_jt;
    const int f_first = jt * a.TJ;
    const int f_cnt = min(a.TJ, a.nf - f_first);
    const int o_begin = a.o_first + f_first;
    const int J0 = o_begin + 3 - H;  // first window element (sweep index)

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], (unsigned)ncons);
        }
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    __syncthreads();

    if (warp == ncons) {
        // ---------------- producer ----------------
        if (lane != 0) return;
        int i = 0;
        for (long long g = g0; g < a.n_groups; g += gstep, ++i) {
            const int s = i % STAGES;
            if (i >= STAGES && !mbar_wait(&empty[s], ((i / STAGES) & 1) ^ 1, kWaitLimitCycles, 256)) return;
            // group -> (u tile, w, v)
            const unsigned gg = (unsigned)g;
            const unsigned ut = gg % (unsigned)a.n_ut;
            const unsigned t = gg / (unsigned)a.n_ut;
            const int w = (int)(t % (unsigned)a.Nw);
            const int v = (int)(t / (unsigned)a.Nw);
            int c0, c1, c2, c3;
            if (KIND == 0) {
                const int u0 = (int)ut * a.U;
                c0 = J0 - P.off;
                c1 = u0 + (P.folded ? 3 : 0);
                c2 = w + (P.folded ? 3 : 0);
                c3 = v;
            } else {
                const int x0 = (int)ut * 16 - 1 + 3;  // v_vf x coordinate of tile column 0
                c0 = x0;
                if (P.dir == 1) { c1 = J0; c2 = w + 3; }   // (x, y=sweep, z)
                else { c1 = w + 3; c2 = J0; }              // (x, y, z=sweep)
                c3 = v;
            }
            mbar_arrive_expect_tx(&full[s], P.box_bytes);
            tma_load_4d(ring + (size_t)s * P.stage_bytes, &tmap, &full[s], c0, c1, c2, c3);
        }
        return;
    }

    // ---------------- consumers ----------------
    const int f = threadIdx.x;
    const bool active = f < f_cnt;
    const long long o = o_begin + f;
    long long cidx = o - 3;
    cidx = cidx < 0 ? 0 : (cidx > a.nc - 1 ? a.nc - 1 : cidx);
    Coef<ORDER> cfr;
    if constexpr (!UNI) {
        if (active) cfr.load(a.cp.polyL, a.cp.polyR, a.cp.dL, a.cp.dR, a.cp.beta, a.nc, cidx);
    }
    const Coef<ORDER>& cf = UNI ? *reinterpret_cast<const Coef<ORDER>*>(a.ucf) : cfr;
    constexpr bool PAIRS = WSB_PIPE_PAIRS && (ORDER == 5 && SCH == 0 && UNI);  // needs the registers UNI frees

    int i = 0;
    for (long long g = g0; g < a.n_groups; g += gstep, ++i) {
        const int s = i % STAGES;
        if (!mbar_wait(&full[s], (i / STAGES) & 1)) return;
        const unsigned char* st = ring + (size_t)s * P.stage_bytes;
        if (active) {
            const unsigned gg = (unsigned)g;
            const unsigned ut = gg % (unsigned)a.n_ut;
            const unsigned t = gg / (unsigned)a.n_ut;
            const long long w = (long long)(t % (unsigned)a.Nw);
            const long long v = (long long)(t / (unsigned)a.Nw);
            if (KIND == 0) {
                const int u0 = (int)ut * a.U;
                const int ucnt = min(a.U, a.Nu - u0);
                const LinearTile<T> tile{(const T*)st + (f + H + P.off), 1, P.SWp};
                const long long oidx0 = (long long)u0 * a.o_sU + w * a.o_sW + v * a.o_sV + o;
                if constexpr (PAIRS)
                    compute_js5_pairs<MPF>(a, *reinterpret_cast<const Coef<5>*>(&cf), tile, 0, ucnt, oidx0);
                else
                    compute_columns<ORDER, MPF, T, SCH>(a, cf, tile, 0, ucnt, oidx0, o);
            } else {
                const int u0 = (int)ut * 16 - 1;  // u of tile column 0
                const int kb = (u0 < 0) ? 1 : 0;
                const int ke = min(16, a.Nu - u0);
                const Swz128Tile<T> tile{st, f + H};
                const long long oidx0 = (long long)u0 * a.o_sU + w * a.o_sW + v * a.o_sV + o;
                if constexpr (PAIRS)
                    compute_js5_pairs<MPF>(a, *reinterpret_cast<const Coef<5>*>(&cf), tile, kb, ke, oidx0);
                else
                    compute_columns<ORDER, MPF, T, SCH>(a, cf, tile, kb, ke, oidx0, o);
            }
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[s]);
    }
}

// ---------------------------------------------------------------------
// Host side: tensor maps through the driver entry point (no -lcuda).
// ---------------------------------------------------------------------
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

inline EncodeTiledFn encode_tiled_fn() {
    static EncodeTiledFn fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (EncodeTiledFn)p;
    }
    return fn;
}

// Which staging a sweep uses (WENO_SB_KERNEL=tma|cpasync|generic|auto).
inline int sweep_path_override() {
    const char* e = getenv("WENO_SB_KERNEL");
    if (!e) return 0;
    if (!strcmp(e, "tma")) return 1;
    if (!strcmp(e, "cpasync")) return 2;
    return 0;
}

template <int ORDER, bool MPF, int KIND, int STAGES, int SCH, bool UNI>
int launch_pipe_s(const CUtensorMap& map, PipeArgs P, cudaStream_t st, int sms) {
    const int cons = (P.a.TJ + 31) / 32;
    const int threads = (cons + 1) * 32;
    const size_t smem = 1024 + (size_t)STAGES * P.stage_bytes + 2 * STAGES * sizeof(unsigned long long);
    auto kfn = sweep_pipe_kernel<ORDER, MPF, KIND, STAGES, SCH, UNI>;
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024);
        attr = true;
    }
    int occ = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kfn, threads, smem);
    if (occ < 1) return 1003;
    long long per_jt = ((long long)sms * occ) / P.a.n_jt;
    if (per_jt < 1) per_jt = 1;
    if (per_jt > P.a.n_groups) per_jt = P.a.n_groups;
    kfn<<<(unsigned)(per_jt * P.a.n_jt), threads, smem, st>>>(map, P);
    return 0;
}

template <int ORDER, bool MPF, int KIND, int STAGES>
int launch_pipe_t(const CUtensorMap& map, PipeArgs P, cudaStream_t st, int sms) {
    const bool uni = P.a.cp.polyL == nullptr;  // face-independent coefficients in P.a.ucf
    if (P.a.wp.scheme == JS)
        return uni ? launch_pipe_s<ORDER, MPF, KIND, STAGES, 0, true>(map, P, st, sms)
                   : launch_pipe_s<ORDER, MPF, KIND, STAGES, 0, false>(map, P, st, sms);
    return uni ? launch_pipe_s<ORDER, MPF, KIND, STAGES, -1, true>(map, P, st, sms)
               : launch_pipe_s<ORDER, MPF, KIND, STAGES, -1, false>(map, P, st, sms);
}

// FP64 TMA sweep when the layout allows it; 1003 (unsupported) otherwise.
inline int launch_pipe_sweep(const long long E[3], const SweepGeom& g, int dir, bool folded, int order, bool mp,
                             const double* in, double* vL, double* vR, const CoefPtrs& cp, const WenoParams& wp,
                             cudaStream_t st, int sms, const double* ucf = nullptr) {
    EncodeTiledFn enc = encode_tiled_fn();
    if (!enc) return 1003;
    if (((uintptr_t)in & 15) != 0) return 1003;
    const bool kind1 = folded && dir != 0;
    const int Hh = ((order - 1) / 2 < 2 && mp) ? 2 : (order - 1) / 2;
    PipeArgs P{};
    FastArgs& a = P.a;
    a.in = in; a.vL = vL; a.vR = vR; a.cp = cp; a.wp = wp;
    if (ucf) {
        for (int q = 0; q < 56; ++q) a.ucf[q] = ucf[q];
        a.cp = CoefPtrs{nullptr, nullptr, nullptr, nullptr, nullptr};
    }
    a.ns = g.ns; a.nc = g.nc;
    a.o_first = (order == 3) ? 0 : 3;
    a.nf = (int)((order == 3) ? g.ns : g.nc);
    const int maxTJ = 224;
    a.n_jt = (a.nf + maxTJ - 1) / maxTJ;
    a.TJ = (a.nf + a.n_jt - 1) / a.n_jt;
    a.TJ += a.TJ & 1;  // even, so every tile's window start has the same parity
    a.SW = a.TJ + 2 * Hh;
    a.o_sV = g.ns * g.c1 * g.c2;
    a.NV = (int)g.nv;
    P.dir = dir;
    P.folded = folded ? 1 : 0;
    cuuint64_t dims[4], strides[3];
    cuuint32_t box[4], estr[4] = {1, 1, 1, 1};
    CUtensorMapSwizzle swz = CU_TENSOR_MAP_SWIZZLE_NONE;
    if (!kind1) {
        a.Nu = (int)g.c1; a.Nw = (int)g.c2;
        a.o_sU = g.ns; a.o_sW = g.ns * g.c1;
        a.U = 8;
        a.n_ut = (a.Nu + a.U - 1) / a.U;
        const int J0first = a.o_first + 3 - Hh;
        P.off = J0first & 1;
        P.SWp = a.SW + P.off;
        P.SWp += P.SWp & 1;
        if (P.SWp > 256) return 1003;
        if (!folded) {
            dims[0] = g.ns + 6; dims[1] = g.c1; dims[2] = g.c2; dims[3] = g.nv;
        } else {
            dims[0] = E[0]; dims[1] = E[1]; dims[2] = E[2]; dims[3] = g.nv;
        }
        box[0] = P.SWp; box[1] = a.U; box[2] = 1; box[3] = 1;
        P.stage_bytes = ((P.SWp * a.U * 8 + 1023) / 1024) * 1024;
    } else {
        if (dir == 1) { a.Nu = (int)g.c1; a.Nw = (int)g.c2; a.o_sU = g.ns; a.o_sW = g.ns * g.c1; }
        else { a.Nu = (int)g.c2; a.Nw = (int)g.c1; a.o_sU = g.ns * g.c1; a.o_sW = g.ns; }
        a.U = 16;
        a.n_ut = (a.Nu + 1 + 15) / 16;  // tiles cover u in [-1, 16*n_ut - 1)
        P.off = 0;
        P.SWp = a.SW;
        if (P.SWp > 256) return 1003;
        dims[0] = E[0]; dims[1] = E[1]; dims[2] = E[2]; dims[3] = g.nv;
        if (dir == 1) { box[0] = 16; box[1] = P.SWp; box[2] = 1; box[3] = 1; }
        else { box[0] = 16; box[1] = 1; box[2] = P.SWp; box[3] = 1; }
        swz = CU_TENSOR_MAP_SWIZZLE_128B;
        P.stage_bytes = ((P.SWp * 128 + 1023) / 1024) * 1024;
    }
    strides[0] = dims[0] * 8;
    strides[1] = dims[0] * dims[1] * 8;
    strides[2] = dims[0] * dims[1] * dims[2] * 8;
    if (strides[0] % 16 != 0) return 1003;
    P.box_bytes = box[0] * box[1] * box[2] * box[3] * 8;
    a.n_groups = (long long)a.n_ut * a.Nw * a.NV;
    P.KIND = kind1 ? 1 : 0;
    CUtensorMap map;
    CUresult r = enc(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, (void*)in, dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, swz, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return 1003;
    const int key = order * 4 + (mp ? 2 : 0) + (kind1 ? 1 : 0);
    switch (key) {
        case 12: return launch_pipe_t<3, false, 0, WSB_PIPE_STAGES0>(map, P, st, sms);
        case 13: return launch_pipe_t<3, false, 1, WSB_PIPE_STAGES1>(map, P, st, sms);
        case 14: return launch_pipe_t<3, true, 0, WSB_PIPE_STAGES0>(map, P, st, sms);
        case 15: return launch_pipe_t<3, true, 1, WSB_PIPE_STAGES1>(map, P, st, sms);
        case 20: return launch_pipe_t<5, false, 0, WSB_PIPE_STAGES0>(map, P, st, sms);
        case 21: return launch_pipe_t<5, false, 1, WSB_PIPE_STAGES1>(map, P, st, sms);
        case 22: return launch_pipe_t<5, true, 0, WSB_PIPE_STAGES0>(map, P, st, sms);
        case 23: return launch_pipe_t<5, true, 1, WSB_PIPE_STAGES1>(map, P, st, sms);
        case 28: return launch_pipe_t<7, false, 0, 6>(map, P, st, sms);
        case 29: return launch_pipe_t<7, false, 1, 3>(map, P, st, sms);
        case 30: return launch_pipe_t<7, true, 0, 6>(map, P, st, sms);
        case 31: return launch_pipe_t<7, true, 1, 3>(map, P, st, sms);
        default: return 1003;
    }
}

// ---------------------------------------------------------------------
// Diagnostics used by the tests.
// ---------------------------------------------------------------------
// Newton reciprocal next to IEEE division, elementwise.
__global__ void selftest_rcp_kernel(const double* __restrict__ x, double* __restrict__ fast,
                                    double* __restrict__ ieee, long long n) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        fast[i] = nr_rcp(x[i]);
        ieee[i] = 1.0 / x[i];
    }
}

// A bounded wait on an mbarrier that nothing ever completes: it must expire
// after `limit` cycles and raise the timeout flag (no fault, no hang).
__global__ void selftest_timeout_kernel(long long limit) {
    __shared__ unsigned long long bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x == 0) mbar_wait(&bar, 0, limit);
}

// Read and clear the device error flag (after synchronising `st`).
inline int pipe_check_device_error(cudaStream_t st) {
    cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return (int)e;
    int v = 0;
    e = cudaMemcpyFromSymbol(&v, g_wsb_device_error, sizeof(int));
    if (e != cudaSuccess) return (int)e;
    if (v) {
        const int zero = 0;
        cudaMemcpyToSymbol(g_wsb_device_error, &zero, sizeof(int));
    }
    return v;
}

}  // namespace wsb
