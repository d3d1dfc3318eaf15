// weno_sb.cu -- C ABI of the B200 WENO library (declared in include/weno_sb.h).
//
// Host side: argument checks, handle bookkeeping (the harness's module
// arrays, f90:87-100, as device allocations), launch geometry, and the
// dispatch from (order, scheme, flags, precision) to kernel instances.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <algorithm>
#include <fstream>
#include <sstream>
#include <vector>

#include "weno_sb.h"
#include "layout.cuh"
#include "sweep_generic.cuh"
#include "sweep_tma.cuh"
#include "sweep_pipe.cuh"
#include "sweep_march.cuh"
#include "sweep_march_tma.cuh"
#include "vjp_march.cuh"
#include "weno_coefficients.h"
#include "weno_adjoint.cuh"
#include "batched.cuh"

using namespace wsb;

// ----------------------------------------------------------------------
// Errors
// ----------------------------------------------------------------------
namespace {

thread_local std::string g_last_error = "no error";

int set_err(int code, const char* fmt, ...) __attribute__((format(printf, 2, 3)));
int set_err(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

int cuda_err(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return WENO_SB_OK;
    return set_err((int)e, "%s: %s (%s)", what, cudaGetErrorName(e), cudaGetErrorString(e));
}

#define WSB_CUDA(call)                                   \
    do {                                                 \
        cudaError_t e__ = (call);                        \
        if (e__ != cudaSuccess) return cuda_err(e__, #call); \
    } while (0)

// Host-side fault injection for error-path tests: WENO_SB_FAULT is a comma
// separated list of operation names ("init", "upload", "download",
// "launch", "sync"); a listed operation fails with WENO_SB_ERR_INJECTED
// before it touches the GPU.
bool fault_injected(const char* op) {
    const char* env = getenv("WENO_SB_FAULT");
    if (!env || !*env) return false;
    const size_t n = strlen(op);
    for (const char* s = env; *s;) {
        const char* e = strchr(s, ',');
        const size_t len = e ? (size_t)(e - s) : strlen(s);
        if (len == n && strncmp(s, op, n) == 0) return true;
        if (!e) break;
        s = e + 1;
    }
    return false;
}

#define WSB_FAULT(op)                                                                      \
    do {                                                                                   \
        if (fault_injected(op))                                                            \
            return set_err(WENO_SB_ERR_INJECTED, "injected failure in '%s' (WENO_SB_FAULT)", op); \
    } while (0)

// ----------------------------------------------------------------------
// Grid geometry
// ----------------------------------------------------------------------
struct Dims {
    long long N[3];  // Nd = cells + 2*buff
    long long E[3];  // Nd + 6 (v_vf extents)
    long long nv;
};

int check_grid(const weno_sb_grid* g, Dims* d) {
    if (!g) return set_err(WENO_SB_ERR_ARG, "grid pointer is NULL");
    if (g->m_cells < 0 || g->n_cells < 0 || g->p_cells < 0)
        return set_err(WENO_SB_ERR_ARG, "negative cell count (m=%d n=%d p=%d)", g->m_cells,
                       g->n_cells, g->p_cells);
    if (g->v_size < 1) return set_err(WENO_SB_ERR_ARG, "v_size must be >= 1 (got %d)", g->v_size);
    if (g->buff_size < 3)
        return set_err(WENO_SB_ERR_ARG, "buff_size must be >= 3 (got %d)", g->buff_size);
    if (g->scheme < WENO_SB_JS || g->scheme > WENO_SB_NONE)
        return set_err(WENO_SB_ERR_ARG, "unknown scheme %d", g->scheme);
    const int cells[3] = {g->m_cells, g->n_cells, g->p_cells};
    for (int k = 0; k < 3; ++k) {
        d->N[k] = (long long)cells[k] + 2LL * g->buff_size + 1;
        d->E[k] = d->N[k] + 6;
    }
    d->nv = g->v_size;
    // 32-bit grid limits on cross-section counts are not a concern; keep
    // element counts within int64.
    const long long tot = d->E[0] * d->E[1] * d->E[2] * d->nv;
    if (tot <= 0 || tot > (1LL << 40)) return set_err(WENO_SB_ERR_ARG, "grid too large");
    return WENO_SB_OK;
}

void sweep_ext(const Dims& d, int dir, long long* ns, long long* c1, long long* c2) {
    if (dir == 0) { *ns = d.N[0]; *c1 = d.N[1]; *c2 = d.N[2]; }
    else if (dir == 1) { *ns = d.N[1]; *c1 = d.N[0]; *c2 = d.N[2]; }
    else { *ns = d.N[2]; *c1 = d.N[1]; *c2 = d.N[0]; }
}

int check_dir(int dir) {
    if (dir < 0 || dir > 2) return set_err(WENO_SB_ERR_ARG, "dir must be 0 (x), 1 (y) or 2 (z), got %d", dir);
    return WENO_SB_OK;
}

int check_dtype(int dt) {
    if (dt != WENO_SB_FP64 && dt != WENO_SB_FP32)
        return set_err(WENO_SB_ERR_ARG, "dtype must be WENO_SB_FP64 or WENO_SB_FP32, got %d", dt);
    return WENO_SB_OK;
}

// Sweep geometry for the drop-in layout (v_rs_ws) or the folded one (v_vf).
SweepGeom make_geom(const Dims& d, int dir, bool folded) {
    SweepGeom g;
    sweep_ext(d, dir, &g.ns, &g.c1, &g.c2);
    g.nc = g.ns - 6;
    g.nv = d.nv;
    g.cols = g.c1 * g.c2 * g.nv;
    if (!folded) {
        g.sJ = 1;
        g.sA = g.ns + 6;
        g.sB = (g.ns + 6) * g.c1;
        g.sV = (g.ns + 6) * g.c1 * g.c2;
        g.in_off = 0;
    } else {
        const long long E1 = d.E[0], E2 = d.E[1], E3 = d.E[2];
        g.sV = E1 * E2 * E3;
        if (dir == 0) {        // J=x, a=y, b=z
            g.sJ = 1; g.sA = E1; g.sB = E1 * E2; g.in_off = 3 * E1 + 3 * E1 * E2;
        } else if (dir == 1) { // J=y, a=x, b=z
            g.sJ = E1; g.sA = 1; g.sB = E1 * E2; g.in_off = 3 + 3 * E1 * E2;
        } else {               // J=z, a=y, b=x
            g.sJ = E1 * E2; g.sA = E1; g.sB = 1; g.in_off = 3 * E1 + 3;
        }
    }
    return g;
}

// SMs a sweep launch sizes its grid and work items for: the whole GPU, or,
// while a batch captures its graph branches, the branch's share of it
// (the branches' kernels run side by side).
thread_local int t_sm_share = 0;

int num_sms() {
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 148;
    }
    return t_sm_share > 0 ? std::min(t_sm_share, sms) : sms;
}

// ----------------------------------------------------------------------
// Launchers
// ----------------------------------------------------------------------
template <typename T>
int launch_reshape(const Dims& d, int dir, const double* v_vf, T* rs, cudaStream_t st) {
    long long ns, c1, c2;
    sweep_ext(d, dir, &ns, &c1, &c2);
    const long long E1 = d.E[0], E2 = d.E[1], E3 = d.E[2];
    if (dir == 0) {
        // rows (l=y, q=z, var): in row at y=l+3, z=q+3
        RowCopyArgs a{v_vf + 3 * E1 + 3 * E1 * E2, E1, c1, c2, d.nv, E1, E1 * E2, E1 * E2 * E3};
        const long long rows = c1 * c2 * d.nv;
        dim3 blk(32, 8);
        const unsigned grid = (unsigned)std::min<long long>((rows + 7) / 8, 65535LL * 8);
        row_copy_kernel<T, 1><<<grid, blk, 0, st>>>(a, rs, nullptr);
    } else {
        TransposeArgs a;
        if (dir == 1) {
            // out(k=y, l=x, q=z, v) = v_vf(x=l+3, y=k, z=q+3): A=k (E2), B=l (N1), P=q (N3)
            a = TransposeArgs{v_vf + 3 + 3 * E1 * E2, ns + 6, c1, c2, d.nv, E1, E1 * E2, E1 * E2 * E3,
                              ns + 6, (ns + 6) * c1, (ns + 6) * c1 * c2};
        } else {
            // out(k=z, l=y, q=x, v) = v_vf(x=q+3, y=l+3, z=k): A=k (E3), B=q (N1), P=l (N2)
            a = TransposeArgs{v_vf + 3 + 3 * E1, ns + 6, c2, c1, d.nv, E1 * E2, E1, E1 * E2 * E3,
                              (ns + 6) * c1, ns + 6, (ns + 6) * c1 * c2};
        }
        dim3 blk(32, 8);
        const long long planes = a.P * a.V;
        dim3 grid((unsigned)((a.A + 31) / 32), (unsigned)((a.B + 31) / 32),
                  (unsigned)std::min<long long>(planes, 65535));
        transpose_kernel<T, 1><<<grid, blk, 0, st>>>(a, rs, nullptr);
    }
    return cuda_err(cudaGetLastError(), "reshape launch");
}

template <typename T>
int launch_order1(const Dims& d, int dir, const double* v_vf, T* vL, T* vR, cudaStream_t st) {
    long long ns, c1, c2;
    sweep_ext(d, dir, &ns, &c1, &c2);
    const long long E1 = d.E[0], E2 = d.E[1], E3 = d.E[2];
    const double* base = v_vf + 3 + 3 * E1 + 3 * E1 * E2;
    if (dir == 0) {
        RowCopyArgs a{base, ns, c1, c2, d.nv, E1, E1 * E2, E1 * E2 * E3};
        const long long rows = c1 * c2 * d.nv;
        dim3 blk(32, 8);
        const unsigned grid = (unsigned)std::min<long long>((rows + 7) / 8, 65535LL * 8);
        row_copy_kernel<T, 2><<<grid, blk, 0, st>>>(a, vL, vR);
    } else {
        TransposeArgs a;
        if (dir == 1) {
            // vL(j=y, k=x, l=z) = v_vf(x=k+3, y=j+3, z=l+3): A=j, B=k, P=l
            a = TransposeArgs{base, ns, c1, c2, d.nv, E1, E1 * E2, E1 * E2 * E3, ns, ns * c1, ns * c1 * c2};
        } else {
            // vL(j=z, k=y, l=x) = v_vf(x=l+3, y=k+3, z=j+3): A=j, B=l, P=k
            a = TransposeArgs{base, ns, c2, c1, d.nv, E1 * E2, E1, E1 * E2 * E3, ns * c1, ns, ns * c1 * c2};
        }
        dim3 blk(32, 8);
        const long long planes = a.P * a.V;
        dim3 grid((unsigned)((a.A + 31) / 32), (unsigned)((a.B + 31) / 32),
                  (unsigned)std::min<long long>(planes, 65535));
        transpose_kernel<T, 2><<<grid, blk, 0, st>>>(a, vL, vR);
    }
    return cuda_err(cudaGetLastError(), "order-1 copy launch");
}

template <int ORDER, bool MPF, typename T>
void launch_generic_t(const SweepGeom& g, const T* in, T* vL, T* vR, const CoefPtrs& cp,
                      const WenoParams& wp, cudaStream_t st, const UniCoefs& uc) {
    const long long nf = (ORDER == 3) ? g.ns : g.nc;
    dim3 blk(128);
    const long long tiles = (nf + 127) / 128;
    const long long want = (long long)num_sms() * 16 / tiles + 1;
    dim3 grid((unsigned)tiles, (unsigned)std::min<long long>(std::min<long long>(g.cols, want * 8), 65535));
    sweep_generic_kernel<ORDER, MPF, T><<<grid, blk, 0, st>>>(g, in, vL, vR, cp, wp, uc);
}

template <typename T>
int launch_generic(const SweepGeom& g, int order, bool mp, const T* in, T* vL, T* vR,
                   const CoefPtrs& cp, const WenoParams& wp, cudaStream_t st, const double* ucf = nullptr) {
    UniCoefs uc{};
    if (ucf)
        for (int q = 0; q < 56; ++q) uc.v[q] = ucf[q];
    switch (order * 2 + (mp ? 1 : 0)) {
        case 0: launch_generic_t<0, false, T>(g, in, vL, vR, cp, wp, st, uc); break;
        case 1: launch_generic_t<0, true, T>(g, in, vL, vR, cp, wp, st, uc); break;
        case 6: launch_generic_t<3, false, T>(g, in, vL, vR, cp, wp, st, uc); break;
        case 7: launch_generic_t<3, true, T>(g, in, vL, vR, cp, wp, st, uc); break;
        case 10: launch_generic_t<5, false, T>(g, in, vL, vR, cp, wp, st, uc); break;
        case 11: launch_generic_t<5, true, T>(g, in, vL, vR, cp, wp, st, uc); break;
        case 14: launch_generic_t<7, false, T>(g, in, vL, vR, cp, wp, st, uc); break;
        case 15: launch_generic_t<7, true, T>(g, in, vL, vR, cp, wp, st, uc); break;
        default: return set_err(WENO_SB_ERR_ARG, "order must be 3, 5 or 7 (got %d)", order);
    }
    return cuda_err(cudaGetLastError(), "reconstruction launch");
}

// Which implementation serves reconstruction sweeps, from WENO_SB_KERNEL
// (read per call): "auto" (default: TMA pipeline for FP64 when the layout
// allows it, else the cp.async pipeline, else the general-stride kernel),
// "tma", "cpasync" or "generic" to pin one for testing.
// WENO_SB_KERNEL: auto (0), generic (1), cpasync (2), march (3), tma (4),
// march_ldg (5: the marching kernel with per-lane loads, no TMA staging).
// A forced kernel that does not cover the case falls through to the next
// one in the auto order (march, tma, cp.async, generic).
int kernel_choice() {
    const char* e = getenv("WENO_SB_KERNEL");
    if (e && strcmp(e, "generic") == 0) return 1;
    if (e && strcmp(e, "cpasync") == 0) return 2;
    if (e && strcmp(e, "march") == 0) return 3;
    if (e && strcmp(e, "tma") == 0) return 4;
    if (e && strcmp(e, "march_ldg") == 0) return 5;
    return 0;
}

// The marching kernels' one-sided MP median takes sign(v_L - v_0) from the
// sign of the weighted candidate sum, which holds for non-negative ideal
// weights (Coef<5> layout: dL, dR at 12..17; Coef<7>: at 24..31).
bool march_weights_ok(const double* ucf, int order = 5) {
    const int q0 = order == 7 ? 24 : (order == 3 ? 4 : 12), q1 = order == 7 ? 32 : (order == 3 ? 8 : 18);
    for (int q = q0; q < q1; ++q)
        if (!(ucf[q] >= 0.0)) return false;
    return true;
}

// The mapped-WENO5 engine needs every ideal weight in (0, 0.8): there each
// mapped weight is positive (numerator and denominator of the map), so a
// state's offset from v0 has the sign of its folded sum.
bool march_mapped_ok(const double* ucf) {
    for (int q = 12; q < 18; ++q)
        if (!(ucf[q] > 0.0 && ucf[q] < 0.8)) return false;
    return true;
}

// FP64 marching sweep with face-dependent coefficient arrays (WENO5 and
// WENO7 with JS or TENO weights, WENO3-JS): the per-face table (one row per
// face, 224 bytes for WENO5, 448 for WENO7, 96 for WENO3; ns + 16 rows: the kernel stages rows f0 .. f0 + 8
// with every input tile, and its last tile starts below ns + 5) is built on
// the stream, used by the TMA marching kernel and freed stream-ordered.
// Returns WENO_SB_ERR_UNSUPPORTED when the layout does not suit the kernel
// or the table cannot be allocated.
int launch_march_faces(const long long E[3], const SweepGeom& g, int dir, bool folded, bool mp, const double* in,
                       double* vL, double* vR, const CoefPtrs& cp, const WenoParams& wp, cudaStream_t st,
                       int ws = 0, int order = 5) {
    if (!cp.polyL || !cp.polyR || !cp.dL || !cp.dR || !cp.beta) return WENO_SB_ERR_UNSUPPORTED;
    if (g.ns < 8 || ((uintptr_t)in & 15)) return WENO_SB_ERR_UNSUPPORTED;
    const int rows = (int)g.ns + 16;
    double* tab = nullptr;
    // an error left by an earlier call is reported, not cleared by the
    // allocation's own error handling below
    const cudaError_t pending = cudaPeekAtLastError();
    if (pending != cudaSuccess) return cuda_err(cudaGetLastError(), "error pending before the per-face table");
    // no stream-ordered allocation available (or no memory): the caller
    // falls back to the one-thread-per-face kernels, which need no table;
    // during a stream capture the failed allocation has invalidated the
    // capture, so its error is returned instead
    const cudaError_t ae = cudaMallocAsync((void**)&tab, sizeof(double) * pf_row_doubles(order) * (size_t)rows, st);
    if (ae != cudaSuccess) {
        cudaGetLastError();
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        if (cudaStreamIsCapturing(st, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone)
            return cuda_err(ae, "per-face table allocation during stream capture");
        return WENO_SB_ERR_UNSUPPORTED;
    }
    if (order == 7) march_face_table7_kernel<<<(rows + 127) / 128, 128, 0, st>>>(cp, g.nc, rows, tab);
    else if (order == 3) march_face_table3_kernel<<<(rows + 127) / 128, 128, 0, st>>>(cp, g.nc, rows, tab);
    else march_face_table_kernel<<<(rows + 127) / 128, 128, 0, st>>>(cp, g.nc, rows, tab);
    MarchArgs a0 = make_march_args(g, in, vL, vR, wp, nullptr);
    a0.ftab = tab;
    a0.cp = cp;
    const int rc = launch_march_tma<double>(E, g, dir, folded, mp, in, vL, vR, a0, st, num_sms(), order, ws);
    const cudaError_t le = cudaGetLastError();
    WSB_CUDA(cudaFreeAsync(tab, st));
    if (rc) return rc;
    return cuda_err(le, "march sweep launch (per-face coefficients)");
}

// Status of a marching launch helper as the library's: 0 -> the launch's
// own error, a CUDA error (< 1000) with its message, else as is.
int march_rc(int rc, const char* what) {
    if (rc == 0) return cuda_err(cudaGetLastError(), what);
    if (rc < 1000) return cuda_err((cudaError_t)rc, what);
    return rc;
}

// Coefficients come either per face (cf, device arrays) or, when ucf is
// non-null, as one face-independent set laid out like Coef<order>.
template <typename T>
int run_weno(const Dims& d, const weno_sb_grid* gr, int dir, int order, unsigned flags,
             const T* in, const weno_sb_coefs* cf, T* vL, T* vR, cudaStream_t st,
             const double* ucf = nullptr) {
    const bool folded = (flags & WENO_SB_F_FOLDED) != 0;
    const bool mp = (flags & WENO_SB_F_MP) != 0;
    SweepGeom g = make_geom(d, dir, folded);
    if (g.nc < 1) return set_err(WENO_SB_ERR_ARG, "sweep has no core faces (Ns=%lld)", g.ns);
    CoefPtrs cp{nullptr, nullptr, nullptr, nullptr, nullptr};
    if (!ucf) cp = CoefPtrs{cf->polyL, cf->polyR, cf->dL, cf->dR, cf->beta_coef};
    WenoParams wp{gr->scheme, gr->weno_eps, gr->teno_CT};
    const int choice = kernel_choice();
    if ((choice == 0 || choice == 3) && ucf && (order == 5 || order == 7) && gr->scheme == WENO_SB_TENO &&
        march_weights_ok(ucf, order)) {
        const MarchArgs a0 = make_march_args(g, in, vL, vR, wp, ucf, order);
        int rc = launch_march_tma<T>(d.E, g, dir, folded, mp, in, vL, vR, a0, st, num_sms(), order, WENO_SB_TENO);
        if (rc != WENO_SB_ERR_UNSUPPORTED)
            return march_rc(rc, "march tma sweep launch (TENO)");
    }
    if ((choice == 0 || choice == 3) && ucf && order == 5 && sizeof(T) == 8 &&
        ((gr->scheme == WENO_SB_Z && march_weights_ok(ucf)) || (gr->scheme == WENO_SB_MAPPED && march_mapped_ok(ucf)))) {
        const MarchArgs a0 = make_march_args(g, in, vL, vR, wp, ucf, 5);
        int rc = launch_march_tma<T>(d.E, g, dir, folded, mp, in, vL, vR, a0, st, num_sms(), 5, gr->scheme);
        if (rc != WENO_SB_ERR_UNSUPPORTED)
            return march_rc(rc, "march tma sweep launch (mapped / Z)");
    }
    if ((choice == 0 || choice == 3) && ucf && order == 3 && gr->scheme == WENO_SB_JS && march_weights_ok(ucf, 3)) {
        const MarchArgs a0 = make_march_args(g, in, vL, vR, wp, ucf, 3);
        int rc = launch_march_tma<T>(d.E, g, dir, folded, mp, in, vL, vR, a0, st, num_sms(), 3);
        if (rc != WENO_SB_ERR_UNSUPPORTED)
            return march_rc(rc, "march tma sweep launch (WENO3)");
    }
    if ((choice == 0 || choice == 3) && ucf && order == 7 && gr->scheme == WENO_SB_JS && march_weights_ok(ucf, 7)) {
        const MarchArgs a0 = make_march_args(g, in, vL, vR, wp, ucf, 7);
        int rc = launch_march_tma<T>(d.E, g, dir, folded, mp, in, vL, vR, a0, st, num_sms(), 7);
        if (rc != WENO_SB_ERR_UNSUPPORTED)
            return march_rc(rc, "march tma sweep launch (WENO7)");
    }
    if ((choice == 0 || choice == 3 || choice == 5) && ucf && order == 5 && gr->scheme == WENO_SB_JS &&
        march_weights_ok(ucf)) {
        if (choice != 5 && g.nc >= 1) {
            const MarchArgs a0 = make_march_args(g, in, vL, vR, wp, ucf);
            int rc = launch_march_tma<T>(d.E, g, dir, folded, mp, in, vL, vR, a0, st, num_sms());
            if (rc != WENO_SB_ERR_UNSUPPORTED)
                return march_rc(rc, "march tma sweep launch");
        }
        int rc = launch_march_sweep<T>(g, mp, in, vL, vR, wp, ucf, st, num_sms());
        if (rc != WENO_SB_ERR_UNSUPPORTED) return rc == 0 ? cuda_err(cudaGetLastError(), "march sweep launch") : rc;
    }
    if constexpr (sizeof(T) == 8) {
        if ((choice == 0 || choice == 3) && !ucf &&
            (((order == 5 || order == 7) && (gr->scheme == WENO_SB_JS || gr->scheme == WENO_SB_TENO)) ||
             (order == 5 && gr->scheme == WENO_SB_Z) || (order == 3 && gr->scheme == WENO_SB_JS))) {
            int rc = launch_march_faces(d.E, g, dir, folded, mp, in, vL, vR, cp, wp, st, gr->scheme,
                                        order);
            if (rc != WENO_SB_ERR_UNSUPPORTED) return rc;
        }
    }
    if constexpr (sizeof(T) == 8) {
        if (choice == 0 || choice == 3 || choice == 4) {
            int rc = launch_pipe_sweep(d.E, g, dir, folded, order, mp, in, vL, vR, cp, wp, st, num_sms(), ucf);
            if (rc != WENO_SB_ERR_UNSUPPORTED) return rc == 0 ? cuda_err(cudaGetLastError(), "tma sweep launch") : rc;
        }
    }
    if (choice != 1) {
        int rc = launch_tma_sweep<T>(d.E, g, dir, folded, order, mp, in, vL, vR, cp, wp, st, ucf);
        if (rc != WENO_SB_ERR_UNSUPPORTED) return rc == 0 ? cuda_err(cudaGetLastError(), "cp.async sweep launch") : rc;
    }
    return launch_generic<T>(g, order, mp, in, vL, vR, cp, wp, st, ucf);
}

// One face's coefficients (weno_sb_face_coefs, index order [s][r]) laid out
// as the kernels' Coef<order> register block.
void build_ucf(int order, const weno_sb_face_coefs* f, double* out) {
    for (int q = 0; q < 56; ++q) out[q] = 0.0;
    const int R = (order + 1) / 2;    // stencils
    const int S = R - 1;              // poly terms per stencil
    const int B = (order == 7) ? 6 : (order == 5 ? 3 : 1);  // beta terms per stencil
    int k = 0;
    for (int r = 0; r < R; ++r)
        for (int s = 0; s < S; ++s) out[k++] = f->polyL[s][r];
    for (int r = 0; r < R; ++r)
        for (int s = 0; s < S; ++s) out[k++] = f->polyR[s][r];
    for (int r = 0; r < R; ++r) out[k++] = f->dL[r];
    for (int r = 0; r < R; ++r) out[k++] = f->dR[r];
    for (int r = 0; r < R; ++r)
        for (int s = 0; s < B; ++s) out[k++] = f->beta_coef[s][r];
}

// Adjoint of one sweep (weno_adjoint.cuh).  gv has the layout of v_in.
int launch_vjp(const Dims& d, const weno_sb_grid* gr, int dir, int order, unsigned flags, const double* v,
               const CoefPtrs& cp, const double* ucf, const double* gL, const double* gR, double* gv,
               cudaStream_t st) {
    const bool folded = (flags & WENO_SB_F_FOLDED) != 0;
    const bool acc_flag = (flags & WENO_SB_F_ACCUMULATE) != 0;
    VjpArgs a{};
    a.g = make_geom(d, dir, folded);
    if (a.g.nc < 1) return set_err(WENO_SB_ERR_ARG, "sweep has no core faces");
    a.v = v;
    a.gL = gL;
    a.gR = gR;
    a.gv = gv;
    a.cp = cp;
    if (ucf)
        for (int q = 0; q < 56; ++q) a.uc.v[q] = ucf[q];
    a.wp = WenoParams{gr->scheme, gr->weno_eps, gr->teno_CT};
    a.mp = (flags & WENO_SB_F_MP) ? 1 : 0;
    // the folded layout has cells no sweep touches: clear them once and add
    a.accumulate = (acc_flag || folded) ? 1 : 0;
    if (folded && !acc_flag)
        WSB_CUDA(cudaMemsetAsync(gv, 0, sizeof(double) * d.E[0] * d.E[1] * d.E[2] * d.nv, st));
    const bool uni = ucf != nullptr;
    if (uni && order == 5 && (gr->scheme == WENO_SB_JS || gr->scheme == WENO_SB_TENO) && kernel_choice() != 1 &&
        march_weights_ok(ucf)) {
        int rc = launch_vjp_march(d.E, a.g, dir, folded, a.mp != 0, a.accumulate != 0, v, ucf, a.wp, gL, gR, gv, st,
                                  num_sms());
        if (rc != WENO_SB_ERR_UNSUPPORTED) return rc == 0 ? cuda_err(cudaGetLastError(), "vjp march launch") : rc;
    }
    const int threads = 128;
    long long blocks = (a.g.cols + threads - 1) / threads;
    if (blocks < 1) blocks = 1;
    if (blocks > (1LL << 30)) blocks = 1LL << 30;
    const unsigned grid = (unsigned)blocks;
    switch (order * 2 + (uni ? 1 : 0)) {
        case 6: vjp_kernel<3, false><<<grid, threads, 0, st>>>(a); break;
        case 7: vjp_kernel<3, true><<<grid, threads, 0, st>>>(a); break;
        case 10: vjp_kernel<5, false><<<grid, threads, 0, st>>>(a); break;
        case 11: vjp_kernel<5, true><<<grid, threads, 0, st>>>(a); break;
        case 14: vjp_kernel<7, false><<<grid, threads, 0, st>>>(a); break;
        case 15: vjp_kernel<7, true><<<grid, threads, 0, st>>>(a); break;
        default: return set_err(WENO_SB_ERR_ARG, "order must be 3, 5 or 7 (got %d)", order);
    }
    return cuda_err(cudaGetLastError(), "vjp launch");
}

// ----------------------------------------------------------------------
// Batches of uneven blocks (batched.cuh)
// ----------------------------------------------------------------------
// Two ways to run a batch, chosen by the autotuner (or weno_sb_batch_configure):
//  mode 0: one persistent kernel (batch_kernel) takes work items of every
//          entry from a global counter;
//  mode 1: every entry's sweep is the single-block sweep kernel specialised
//          for its order, weights, precision and layout (TMA marching sweeps
//          where one covers it), and the launches are spread over `branches`
//          parallel branches of the graph, balanced by longest-processing-
//          time-first on the entries' estimated cost, so small blocks run
//          beside each other and beside the tails of large ones.
//  mode 2: the entries that a marching engine covers are grouped by kernel
//          instance (storage, order, weights, MP, tile kind) and
//          coefficients; each group is one launch of the grouped TMA
//          marching kernel over the work items of all its sweeps (columns
//          cut into segments of about `seg_faces` faces), the groups spread
//          over `branches` graph branches by longest-processing-time-first;
//          the other entries run as in mode 1.
// Every way a launch is one cudaGraphLaunch of the captured work.
constexpr int kBatchMaxBranches = 16;

// Mode 2: the sweeps of one grouped launch.
struct MtmaGroup {
    int fp32 = 0, order = 5, teno = 0, mp = 0, kind = 0;
    MarchArgs a{};            // coefficients of the group (its first entry's arguments)
    MarchTmaArgs t{};         // shared-memory layout (the same for every entry)
    size_t smem = 0;
    std::vector<MtmaEntry> ents;
    std::vector<long long> item0s;  // first work item of each entry
    MtmaEntry* d_ents = nullptr;
    long long* d_item0s = nullptr;
    long long n_items = 0;
    double cost = 0;
};

struct Batch {
    std::vector<weno_sb_block> blocks;
    std::vector<BatchEntry> entries;
    BatchEntry* d_entries = nullptr;
    std::vector<MarchArgs> margs;     // marching entries' arguments (BatchEntry::march - 1)
    MarchArgs* d_margs = nullptr;
    unsigned long long* d_counter = nullptr;
    long long n_items = 0;
    int threads = 128;  // face-tile width = CTA size
    int U = 8;          // columns per work item
    int grid = 0;
    int mode = 2;       // 0: persistent kernel, 1: graph of specialised sweeps, 2: grouped sweeps
    int branches = 8;   // modes 1, 2: parallel branches of the graph
    int seg_faces = 64; // mode 2: faces per work item (segment of a column)
    std::vector<MtmaGroup> groups;   // mode 2: grouped launches
    std::vector<size_t> rest;        // mode 2: entries outside the groups
    // mode 1: each entry's face-independent coefficients (Coef<order>
    // layout), when its arrays hold the same values on every face
    std::vector<std::vector<double>> ucf;
    cudaStream_t br[kBatchMaxBranches] = {};
    cudaEvent_t fork = nullptr;
    cudaEvent_t join[kBatchMaxBranches] = {};
    cudaStream_t cap = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int device = 0;
};

std::mutex g_batch_mu;
std::vector<Batch*> g_batches;

Batch* get_batch(int b) {
    std::lock_guard<std::mutex> lk(g_batch_mu);
    if (b < 1 || b > (int)g_batches.size()) return nullptr;
    return g_batches[b - 1];
}

void batch_release_graph(Batch* B) {
    if (B->exec) cudaGraphExecDestroy(B->exec);
    if (B->graph) cudaGraphDestroy(B->graph);
    B->exec = nullptr;
    B->graph = nullptr;
}

// Cut the entries into work items for tile width `threads` and `U` columns
// per item, upload the table and size the persistent grid.
int batch_layout(Batch* B, int threads, int U) {
    B->threads = threads;
    B->U = U;
    long long item = 0;
    for (auto& e : B->entries) {
        e.TJ = threads;
        e.n_jt = e.march ? 1 : (e.nf + threads - 1) / threads;
        e.n_groups = e.march ? (e.g.cols + threads - 1) / threads : (e.g.cols + U - 1) / U;
        e.item0 = item;
        item += (long long)e.n_jt * e.n_groups;
    }
    B->n_items = item;
    WSB_CUDA(cudaMemcpy(B->d_entries, B->entries.data(), sizeof(BatchEntry) * B->entries.size(),
                        cudaMemcpyHostToDevice));
    int occ = 0;
    WSB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, batch_kernel, threads, 0));
    if (occ < 1) occ = 1;
    B->grid = num_sms() * occ;
    batch_release_graph(B);
    return WENO_SB_OK;
}

int batch_enqueue(Batch* B, cudaStream_t st) {
    WSB_CUDA(cudaMemsetAsync(B->d_counter, 0, sizeof(unsigned long long), st));
    batch_kernel<<<B->grid, B->threads, 0, st>>>(B->d_entries, (int)B->entries.size(), B->n_items, B->d_counter,
                                                 B->U, B->d_margs);
    return cuda_err(cudaGetLastError(), "batch launch");
}

// Estimated cost of one entry's sweep, for balancing the graph branches:
// its face states, weighted by the measured cost of its engine relative to
// FP64 WENO5-JS with face-independent coefficients.
double batch_entry_cost(const Batch* B, size_t i) {
    const BatchEntry& e = B->entries[i];
    double c = 2.0 * (double)e.nf * (double)e.g.cols;
    c *= e.order == 7 ? 1.5 : (e.order == 3 ? 0.85 : 1.0);
    if (e.wp.scheme == WENO_SB_TENO) c *= 1.3;
    if (B->ucf[i].empty()) c *= 1.25;
    if (e.fp32) c *= 0.8;
    return c;
}

// Mode 1: every entry's sweep on one of B->branches parallel streams forked
// from (and joined back into) the capturing stream.
int batch_enqueue_sweeps(Batch* B, cudaStream_t st) {
    const int nb = std::max(1, std::min(B->branches, kBatchMaxBranches));
    WSB_CUDA(cudaEventRecord(B->fork, st));
    for (int k = 0; k < nb; ++k) WSB_CUDA(cudaStreamWaitEvent(B->br[k], B->fork, 0));
    std::vector<size_t> order(B->entries.size());
    for (size_t i = 0; i < order.size(); ++i) order[i] = i;
    std::vector<double> cost(order.size());
    for (size_t i = 0; i < order.size(); ++i) cost[i] = batch_entry_cost(B, i);
    std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return cost[a] > cost[b]; });
    std::vector<double> load(nb, 0.0);
    int rc = 0;
    const int all_sms = num_sms();
    t_sm_share = nb > 1 ? (all_sms + nb - 1) / nb : 0;
    for (size_t i : order) {
        const int k = (int)(std::min_element(load.begin(), load.end()) - load.begin());
        load[k] += cost[i];
        const weno_sb_block& b = B->blocks[i];
        Dims d;
        rc = check_grid(&b.grid, &d);
        if (rc) break;
        const double* u = B->ucf[i].empty() ? nullptr : B->ucf[i].data();
        if (b.dtype == WENO_SB_FP64)
            rc = run_weno<double>(d, &b.grid, b.dir, b.order, b.flags, (const double*)b.v_in, &b.coefs,
                                  (double*)b.vL, (double*)b.vR, B->br[k], u);
        else
            rc = run_weno<float>(d, &b.grid, b.dir, b.order, b.flags, (const float*)b.v_in, &b.coefs, (float*)b.vL,
                                 (float*)b.vR, B->br[k], u);
        if (rc) break;
    }
    t_sm_share = 0;
    // join every branch, also after a failed launch, so a capture ends cleanly
    for (int k = 0; k < nb; ++k) {
        cudaEventRecord(B->join[k], B->br[k]);
        cudaStreamWaitEvent(st, B->join[k], 0);
    }
    return rc;
}

void batch_free_groups(Batch* B) {
    for (auto& G : B->groups) {
        if (G.d_ents) cudaFree(G.d_ents);
        if (G.d_item0s) cudaFree(G.d_item0s);
    }
    B->groups.clear();
    B->rest.clear();
}

// The coefficient part of two entries' march arguments is the same (the
// values a grouped launch takes from its kernel parameters).
bool march_coefs_equal(const MarchArgs& x, const MarchArgs& y) {
    return x.wp.scheme == y.wp.scheme && std::memcmp(&x.wp.eps, &y.wp.eps, sizeof(double)) == 0 &&
           std::memcmp(&x.wp.teno_ct, &y.wp.teno_ct, sizeof(double)) == 0 &&
           std::memcmp(x.ucf, y.ucf, sizeof(x.ucf)) == 0 && std::memcmp(x.ucf32, y.ucf32, sizeof(x.ucf32)) == 0 &&
           std::memcmp(x.kL, y.kL, sizeof(x.kL)) == 0 && std::memcmp(x.kR, y.kR, sizeof(x.kR)) == 0 &&
           std::memcmp(x.pf2, y.pf2, sizeof(x.pf2)) == 0 && std::memcmp(x.kL7, y.kL7, sizeof(x.kL7)) == 0 &&
           std::memcmp(x.kR7, y.kR7, sizeof(x.kR7)) == 0 && std::memcmp(x.pf7, y.pf7, sizeof(x.pf7)) == 0;
}

// Mode 2: plan every marching entry's sweep (segments of about seg_faces
// faces), group the sweeps by kernel instance and coefficients, and upload
// each group's entry table.  Entries that no group takes go to B->rest.
int batch_plan_groups(Batch* B, int seg_faces) {
    batch_free_groups(B);
    B->seg_faces = seg_faces;
    for (size_t i = 0; i < B->entries.size(); ++i) {
        const BatchEntry& e = B->entries[i];
        const weno_sb_block& b = B->blocks[i];
        bool placed = false;
        if (e.march && kernel_choice() != 1) {
            Dims d;
            if (check_grid(&b.grid, &d) == 0) {
                const bool folded = (b.flags & WENO_SB_F_FOLDED) != 0;
                const MarchArgs& a0 = B->margs[e.march - 1];
                MtmaPlan P;
                const int prc =
                    e.fp32 ? plan_march_tma<float>(d.E, e.g, b.dir, folded, (const float*)e.in, (float*)e.vL,
                                                   (float*)e.vR, a0, num_sms(), e.order, seg_faces, P)
                           : plan_march_tma<double>(d.E, e.g, b.dir, folded, (const double*)e.in, (double*)e.vL,
                                                    (double*)e.vR, a0, num_sms(), e.order, seg_faces, P);
                const bool teno = e.wp.scheme == WENO_SB_TENO;
                if (prc == 0 && !(e.order == 3 && teno)) {
                    MtmaGroup* G = nullptr;
                    for (auto& q : B->groups)
                        if (q.fp32 == e.fp32 && q.order == e.order && q.teno == (int)teno && q.mp == e.mp &&
                            q.kind == P.t.kind && march_coefs_equal(q.a, P.a)) {
                            G = &q;
                            break;
                        }
                    if (!G) {
                        B->groups.emplace_back();
                        G = &B->groups.back();
                        G->fp32 = e.fp32;
                        G->order = e.order;
                        G->teno = teno ? 1 : 0;
                        G->mp = e.mp;
                        G->kind = P.t.kind;
                        G->a = P.a;
                        G->t = P.t;
                        // plus the warps' argument slots
                        G->smem = P.smem + (size_t)kTmaWarps * kMtmaSlot;
                    }
                    MtmaEntry me;
                    std::memset(&me, 0, sizeof(me));
                    me.tin = P.mi;
                    me.toutL = P.mL;
                    me.toutR = P.mR;
                    me.ia.geo = mtma_geo(P.a);
                    me.ia.t = P.t;
                    me.a = P.a;
                    G->ents.push_back(me);
                    G->item0s.push_back(G->n_items);
                    G->n_items += P.a.n_items;
                    G->cost += batch_entry_cost(B, i);
                    placed = true;
                }
            }
        }
        if (!placed) B->rest.push_back(i);
    }
    for (auto& G : B->groups) {
        WSB_CUDA(cudaMalloc((void**)&G.d_ents, sizeof(MtmaEntry) * G.ents.size()));
        WSB_CUDA(cudaMemcpy(G.d_ents, G.ents.data(), sizeof(MtmaEntry) * G.ents.size(), cudaMemcpyHostToDevice));
        WSB_CUDA(cudaMalloc((void**)&G.d_item0s, sizeof(long long) * G.item0s.size()));
        WSB_CUDA(cudaMemcpy(G.d_item0s, G.item0s.data(), sizeof(long long) * G.item0s.size(),
                            cudaMemcpyHostToDevice));
    }
    batch_release_graph(B);
    return WENO_SB_OK;
}

// Mode 2: the grouped launches and the remaining entries' sweeps on
// B->branches parallel streams forked from (and joined back into) the
// capturing stream, longest first onto the least loaded branch.
int batch_enqueue_groups(Batch* B, cudaStream_t st) {
    const int nb = std::max(1, std::min(B->branches, kBatchMaxBranches));
    WSB_CUDA(cudaEventRecord(B->fork, st));
    for (int k = 0; k < nb; ++k) WSB_CUDA(cudaStreamWaitEvent(B->br[k], B->fork, 0));
    // work units: groups (index >= 0) and remaining entries (~index)
    std::vector<std::pair<double, long long>> units;
    for (size_t q = 0; q < B->groups.size(); ++q) units.push_back({B->groups[q].cost, (long long)q});
    for (size_t i : B->rest) units.push_back({batch_entry_cost(B, i), ~(long long)i});
    std::stable_sort(units.begin(), units.end(), [](const auto& x, const auto& y) { return x.first > y.first; });
    std::vector<double> load(nb, 0.0);
    int rc = 0;
    const int sms = num_sms();
    for (const auto& u : units) {
        const int k = (int)(std::min_element(load.begin(), load.end()) - load.begin());
        load[k] += u.first;
        if (u.second >= 0) {
            const MtmaGroup& G = B->groups[(size_t)u.second];
            const MtmaMultiFn kfn = G.fp32 ? mtma_multi_kernel<float>(G.order, G.teno != 0, G.mp != 0, G.kind == 1)
                                           : mtma_multi_kernel<double>(G.order, G.teno != 0, G.mp != 0, G.kind == 1);
            if (!kfn) { rc = set_err(WENO_SB_ERR_UNSUPPORTED, "no grouped kernel for a batch group"); break; }
            rc = cuda_err(cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)G.smem),
                          "cudaFuncSetAttribute");
            if (rc) break;
            int occ = 0;
            rc = cuda_err(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kfn, kTmaWarps * 32, G.smem),
                          "occupancy");
            if (rc) break;
            if (occ < 1) occ = 1;
            long long blocks = (G.n_items + kTmaWarps - 1) / kTmaWarps;
            blocks = std::min(blocks, (long long)sms * occ);
            if (blocks < 1) continue;
            kfn<<<(unsigned)blocks, kTmaWarps * 32, G.smem, B->br[k]>>>(G.d_ents, G.d_item0s, (int)G.ents.size(),
                                                                          G.n_items, G.a, G.t);
            rc = cuda_err(cudaGetLastError(), "grouped sweep launch");
        } else {
            const size_t i = (size_t)(~u.second);
            const weno_sb_block& b = B->blocks[i];
            Dims d;
            rc = check_grid(&b.grid, &d);
            if (rc) break;
            const double* uc = B->ucf[i].empty() ? nullptr : B->ucf[i].data();
            if (b.dtype == WENO_SB_FP64)
                rc = run_weno<double>(d, &b.grid, b.dir, b.order, b.flags, (const double*)b.v_in, &b.coefs,
                                      (double*)b.vL, (double*)b.vR, B->br[k], uc);
            else
                rc = run_weno<float>(d, &b.grid, b.dir, b.order, b.flags, (const float*)b.v_in, &b.coefs,
                                     (float*)b.vL, (float*)b.vR, B->br[k], uc);
        }
        if (rc) break;
    }
    // join every branch, also after a failed launch, so a capture ends cleanly
    for (int k = 0; k < nb; ++k) {
        cudaEventRecord(B->join[k], B->br[k]);
        cudaStreamWaitEvent(st, B->join[k], 0);
    }
    return rc;
}

// Capture the batch into a CUDA graph: mode 0 the counter reset and the
// persistent kernel, mode 1 the branches of specialised sweeps, mode 2 the
// branches of grouped sweeps.
int batch_build_graph(Batch* B) {
    batch_release_graph(B);
    WSB_CUDA(cudaStreamBeginCapture(B->cap, cudaStreamCaptureModeThreadLocal));
    const int rc = B->mode == 2 ? batch_enqueue_groups(B, B->cap)
                                : (B->mode == 1 ? batch_enqueue_sweeps(B, B->cap) : batch_enqueue(B, B->cap));
    cudaGraph_t gph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(B->cap, &gph);
    if (rc) {
        if (gph) cudaGraphDestroy(gph);
        return rc;
    }
    if (e != cudaSuccess) return cuda_err(e, "cudaStreamEndCapture");
    B->graph = gph;
    WSB_CUDA(cudaGraphInstantiate(&B->exec, B->graph, 0));
    return WENO_SB_OK;
}

// FNV-1a signature of what the tile choice depends on: per entry the order,
// v_size, storage, direction, layout and extents in 16-cell buckets.
unsigned long long batch_signature(const Batch* B) {
    unsigned long long h = 1469598103934665603ull;
    auto mix = [&](long long x) {
        for (int i = 0; i < 8; ++i) {
            h ^= (unsigned long long)((x >> (8 * i)) & 0xff);
            h *= 1099511628211ull;
        }
    };
    for (size_t i = 0; i < B->entries.size(); ++i) {
        const BatchEntry& e = B->entries[i];
        mix(e.wp.scheme);
        mix(B->ucf[i].empty() ? 0 : 1);
        mix(e.order);
        mix(e.g.nv);
        mix(e.fp32);
        mix(e.mp);
        mix(e.g.sJ == 1 ? 0 : 1);
        mix(e.g.ns / 16);
        mix(e.g.c1 / 16);
        mix(e.g.c2 / 16);
    }
    return h;
}

// ----------------------------------------------------------------------
// Handles
// ----------------------------------------------------------------------
struct Handle {
    weno_sb_grid grid;
    Dims dims;
    int precision = WENO_SB_FP64;
    cudaStream_t stream = nullptr;
    void* arr[WENO_SB_A_COUNT] = {};
    long long n[WENO_SB_A_COUNT] = {};
    int dtype[WENO_SB_A_COUNT] = {};
    double* sum_scratch = nullptr;  // kSumBlocks partials + 1 result
    int device = 0;
    // Per direction: whether each of the five coefficient arrays was last set
    // by weno_sb_upload with the same values on every face (then the sweeps
    // take them from kernel parameters), and face 0's values.
    bool coef_uniform[3][5] = {};
    weno_sb_face_coefs face0[3] = {};
    // weno_sb_upload_async of v_vf: the copy runs on copy_stream one
    // variable at a time, var_ready[q] recorded after variable q; while
    // vf_pending, folded sweeps wait per variable and every other use of the
    // handle waits for all of them (await_vf)
    cudaStream_t copy_stream = nullptr;
    std::vector<cudaEvent_t> var_ready;
    cudaEvent_t main_done = nullptr;
    bool vf_pending = false;
};

// Make the handle's stream wait for an asynchronous upload of v_vf.
void await_vf(Handle* H) {
    if (!H->vf_pending) return;
    for (cudaEvent_t e : H->var_ready) cudaStreamWaitEvent(H->stream, e, 0);
    H->vf_pending = false;
}

std::mutex g_mu;
std::vector<Handle*> g_handles;

Handle* get_handle(int h) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (h < 1 || h > (int)g_handles.size()) return nullptr;
    return g_handles[h - 1];
}

// Record whether an uploaded coefficient array is the same on every face.
void note_coefficients(Handle* H, int which, const double* host) {
    const int kind = (which - WENO_SB_A_POLYL(0)) / 3;  // 0 polyL 1 polyR 2 dL 3 dR 4 beta
    const int dir = (which - WENO_SB_A_POLYL(0)) % 3;
    long long ns, c1, c2;
    sweep_ext(H->dims, dir, &ns, &c1, &c2);
    const long long nc = ns - 6;
    weno_sb_face_coefs& f = H->face0[dir];
    bool uni = true;
    if (kind <= 1 || kind == 4) {  // (nc, 5, S) arrays
        const int S = (kind == 4) ? 6 : 3;
        for (int s = 0; s < S; ++s)
            for (int r = 0; r < 5; ++r) {
                const double* col = host + nc * (r + 5 * s);
                for (long long cc = 1; cc < nc && uni; ++cc) uni = (col[cc] == col[0]);
                if (kind == 0) f.polyL[s][r] = col[0];
                else if (kind == 1) f.polyR[s][r] = col[0];
                else f.beta_coef[s][r] = col[0];
            }
    } else {  // (5, nc)
        for (int r = 0; r < 5; ++r) {
            for (long long cc = 1; cc < nc && uni; ++cc) uni = (host[r + 5 * cc] == host[r]);
            if (kind == 2) f.dL[r] = host[r];
            else f.dR[r] = host[r];
        }
    }
    H->coef_uniform[dir][kind] = uni;
}

void free_handle_arrays(Handle* H) {
    if (H->copy_stream) cudaStreamSynchronize(H->copy_stream);
    for (int i = 0; i < WENO_SB_A_COUNT; ++i)
        if (H->arr[i]) cudaFree(H->arr[i]);
    if (H->sum_scratch) cudaFree(H->sum_scratch);
    for (cudaEvent_t e : H->var_ready) cudaEventDestroy(e);
    if (H->main_done) cudaEventDestroy(H->main_done);
    if (H->copy_stream) cudaStreamDestroy(H->copy_stream);
    if (H->stream) cudaStreamDestroy(H->stream);
}

}  // namespace

// ======================================================================
// C ABI
// ======================================================================
extern "C" {

int weno_sb_version(void) { return WENO_SB_VERSION; }

const char* weno_sb_last_error_string(void) { return g_last_error.c_str(); }

int weno_sb_extents(const weno_sb_grid* g, int dir, int64_t* ns, int64_t* c1, int64_t* c2) {
    Dims d;
    int rc = check_grid(g, &d);
    if (rc) return rc;
    if ((rc = check_dir(dir))) return rc;
    long long a, b, c;
    sweep_ext(d, dir, &a, &b, &c);
    if (ns) *ns = a;
    if (c1) *c1 = b;
    if (c2) *c2 = c;
    return WENO_SB_OK;
}

int weno_sb_init(const weno_sb_grid* g, int precision, int* handle) {
    WSB_FAULT("init");
    if (!handle) return set_err(WENO_SB_ERR_ARG, "handle pointer is NULL");
    Dims d;
    int rc = check_grid(g, &d);
    if (rc) return rc;
    if ((rc = check_dtype(precision))) return rc;
    Handle* H = new Handle;
    H->grid = *g;
    H->dims = d;
    H->precision = precision;
    cudaGetDevice(&H->device);
    const size_t fsz = precision == WENO_SB_FP32 ? sizeof(float) : sizeof(double);
    auto alloc = [&](int which, long long n, bool field) -> int {
        H->n[which] = n;
        H->dtype[which] = field ? precision : WENO_SB_FP64;
        const size_t bytes = (size_t)n * (field ? fsz : sizeof(double));
        cudaError_t e = cudaMalloc(&H->arr[which], bytes);
        if (e != cudaSuccess) return cuda_err(e, "cudaMalloc");
        e = cudaMemset(H->arr[which], 0, bytes);
        return cuda_err(e, "cudaMemset");
    };
    rc = cuda_err(cudaStreamCreateWithFlags(&H->stream, cudaStreamNonBlocking), "cudaStreamCreate");
    if (!rc) rc = alloc(WENO_SB_A_V_VF, d.E[0] * d.E[1] * d.E[2] * d.nv, false);
    for (int dir = 0; dir < 3 && !rc; ++dir) {
        long long ns, c1, c2;
        sweep_ext(d, dir, &ns, &c1, &c2);
        const long long nc = ns - 6;
        if (!rc) rc = alloc(WENO_SB_A_RS(dir), (ns + 6) * c1 * c2 * d.nv, true);
        if (!rc) rc = alloc(WENO_SB_A_VL(dir), ns * c1 * c2 * d.nv, true);
        if (!rc) rc = alloc(WENO_SB_A_VR(dir), ns * c1 * c2 * d.nv, true);
        if (!rc) rc = alloc(WENO_SB_A_POLYL(dir), nc * 15, false);
        if (!rc) rc = alloc(WENO_SB_A_POLYR(dir), nc * 15, false);
        if (!rc) rc = alloc(WENO_SB_A_DL(dir), nc * 5, false);
        if (!rc) rc = alloc(WENO_SB_A_DR(dir), nc * 5, false);
        if (!rc) rc = alloc(WENO_SB_A_BETA(dir), nc * 30, false);
    }
    if (!rc) rc = cuda_err(cudaMalloc((void**)&H->sum_scratch, sizeof(double) * (kSumBlocks + 1)), "cudaMalloc");
    if (rc) {
        free_handle_arrays(H);
        delete H;
        return rc;
    }
    std::lock_guard<std::mutex> lk(g_mu);
    g_handles.push_back(H);
    *handle = (int)g_handles.size();
    return WENO_SB_OK;
}

int weno_sb_finalize(int handle) {
    Handle* H = get_handle(handle);
    if (!H) return set_err(WENO_SB_ERR_HANDLE, "unknown handle %d", handle);
    cudaStreamSynchronize(H->stream);
    free_handle_arrays(H);
    {
        std::lock_guard<std::mutex> lk(g_mu);
        g_handles[handle - 1] = nullptr;
    }
    delete H;
    return WENO_SB_OK;
}

int weno_sb_array_info(int handle, int which, void** dev_ptr, int64_t* n_elem, int* dtype) {
    Handle* H = get_handle(handle);
    if (!H) return set_err(WENO_SB_ERR_HANDLE, "unknown handle %d", handle);
    await_vf(H);
    if (which < 0 || which >= WENO_SB_A_COUNT) return set_err(WENO_SB_ERR_ARG, "unknown array id %d", which);
    if (dev_ptr) *dev_ptr = H->arr[which];
    // the caller may now write the array directly: stop trusting the
    // uniformity recorded at upload
    if (dev_ptr && which >= WENO_SB_A_POLYL(0))
        H->coef_uniform[(which - WENO_SB_A_POLYL(0)) % 3][(which - WENO_SB_A_POLYL(0)) / 3] = false;
    if (n_elem) *n_elem = H->n[which];
    if (dtype) *dtype = H->dtype[which];
    return WENO_SB_OK;
}

int weno_sb_upload(int handle, int which, const double* host) {
    WSB_FAULT("upload");
    Handle* H = get_handle(handle);
    if (!H) return set_err(WENO_SB_ERR_HANDLE, "unknown handle %d", handle);
    if (which < 0 || which >= WENO_SB_A_COUNT) return set_err(WENO_SB_ERR_ARG, "unknown array id %d", which);
    if (!host) return set_err(WENO_SB_ERR_ARG, "host pointer is NULL");
    await_vf(H);
    const long long n = H->n[which];
    if (which >= WENO_SB_A_POLYL(0)) note_coefficients(H, which, host);
    if (H->dtype[which] == WENO_SB_FP64) {
        WSB_CUDA(cudaMemcpyAsync(H->arr[which], host, sizeof(double) * n, cudaMemcpyHostToDevice, H->stream));
    } else {
        std::vector<float> tmp((size_t)n);
        for (long long i = 0; i < n; ++i) tmp[i] = (float)host[i];
        WSB_CUDA(cudaMemcpyAsync(H->arr[which], tmp.data(), sizeof(float) * n, cudaMemcpyHostToDevice, H->stream));
        WSB_CUDA(cudaStreamSynchronize(H->stream));
    }
    return cuda_err(cudaStreamSynchronize(H->stream), "upload");
}

int weno_sb_download(int handle, int which, double* host) {
    WSB_FAULT("download");
    Handle* H = get_handle(handle);
    if (!H) return set_err(WENO_SB_ERR_HANDLE, "unknown handle %d", handle);
    if (which < 0 || which >= WENO_SB_A_COUNT) return set_err(WENO_SB_ERR_ARG, "unknown array id %d", which);
    if (!host) return set_err(WENO_SB_ERR_ARG, "host pointer is NULL");
    await_vf(H);
    const long long n = H->n[which];
    if (H->dtype[which] == WENO_SB_FP64) {
        WSB_CUDA(cudaMemcpyAsync(host, H->arr[which], sizeof(double) * n, cudaMemcpyDeviceToHost, H->stream));
        return cuda_err(cudaStreamSynchronize(H->stream), "download");
    }
    std::vector<float> tmp((size_t)n);
    WSB_CUDA(cudaMemcpyAsync(tmp.data(), H->arr[which], sizeof(float) * n, cudaMemcpyDeviceToHost, H->stream));
    WSB_CUDA(cudaStreamSynchronize(H->stream));
    for (long long i = 0; i < n; ++i) host[i] = (double)tmp[i];
    return WENO_SB_OK;
}

int weno_sb_stream(int handle, void** stream) {
    Handle* H = get_handle(handle);
    if (!H) return set_err(WENO_SB_ERR_HANDLE, "unknown handle %d", handle);
    await_vf(H);
    if (stream) *stream = (void*)H->stream;
    return WENO_SB_OK;
}

int weno_sb_upload_async(int handle, int which, const double* host) {
    WSB_FAULT("upload");
    Handle* H = get_handle(handle);
    if (!H) return set_err(WENO_SB_ERR_HANDLE, "unknown handle %d", handle);
    if (which < 0 || which >= WENO_SB_A_COUNT) return set_err(WENO_SB_ERR_ARG, "unknown array id %d", which);
    if (!host) return set_err(WENO_SB_ERR_ARG, "host pointer is NULL");
    // only v_vf of an FP64 handle is pipelined; the rest is weno_sb_upload
    if (which != WENO_SB_A_V_VF || H->dtype[which] != WENO_SB_FP64) return weno_sb_upload(handle, which, host);
    const int nv = H->dims.nv;
    if (!H->copy_stream) {
        WSB_CUDA(cudaStreamCreateWithFlags(&H->copy_stream, cudaStreamNonBlocking));
        WSB_CUDA(cudaEventCreateWithFlags(&H->main_done, cudaEventDisableTiming));
        H->var_ready.resize(nv, nullptr);
        for (int q = 0; q < nv; ++q) WSB_CUDA(cudaEventCreateWithFlags(&H->var_ready[q], cudaEventDisableTiming));
    }
    await_vf(H);
    // the new copy must not overwrite v_vf while earlier work still reads it
    WSB_CUDA(cudaEventRecord(H->main_done, H->stream));
    WSB_CUDA(cudaStreamWaitEvent(H->copy_stream, H->main_done, 0));
    const long long per = H->n[which] / nv;
    double* dst = (double*)H->arr[which];
    for (int q = 0; q < nv; ++q) {
        WSB_CUDA(cudaMemcpyAsync(dst + per * q, host + per * q, sizeof(double) * per, cudaMemcpyHostToDevice,
                                 H->copy_stream));
        WSB_CUDA(cudaEventRecord(H->var_ready[q], H->copy_stream));
    }
    H->vf_pending = true;
    return WENO_SB_OK;
}

int weno_sb_sync(int handle) {
    WSB_FAULT("sync");
    Handle* H = get_handle(handle);
    if (!H) return set_err(WENO_SB_ERR_HANDLE, "unknown handle %d", handle);
    await_vf(H);
    int rc = cuda_err(cudaStreamSynchronize(H->stream), "cudaStreamSynchronize");
    if (rc) return rc;
    return weno_sb_check_device(H->stream);
}

int weno_sb_check_device(void* stream) {
    const int v = pipe_check_device_error((cudaStream_t)stream);
    if (v == 0) return WENO_SB_OK;
    if (v == WENO_SB_ERR_TIMEOUT)
        return set_err(v, "a pipelined sweep gave up a bounded wait for its staged data (device timeout)");
    if (v < 1000) return cuda_err((cudaError_t)v, "device check");
    return set_err(v, "device error flag %d", v);
}

int weno_sb_reshape_dev(const weno_sb_grid* g, int dir, int dtype, const double* v_vf, void* v_rs_ws,
                        void* stream) {
    WSB_FAULT("launch");
    Dims d;
    int rc = check_grid(g, &d);
    if (rc || (rc = check_dir(dir)) || (rc = check_dtype(dtype))) return rc;
    if (!v_vf || !v_rs_ws) return set_err(WENO_SB_ERR_ARG, "NULL array pointer");
    cudaStream_t st = (cudaStream_t)stream;
    if (dtype == WENO_SB_FP64) return launch_reshape<double>(d, dir, v_vf, (double*)v_rs_ws, st);
    return launch_reshape<float>(d, dir, v_vf, (float*)v_rs_ws, st);
}

int weno_sb_order1_dev(const weno_sb_grid* g, int dir, int dtype, const double* v_vf, void* vL,
                       void* vR, void* stream) {
    WSB_FAULT("launch");
    Dims d;
    int rc = check_grid(g, &d);
    if (rc || (rc = check_dir(dir)) || (rc = check_dtype(dtype))) return rc;
    if (!v_vf || !vL || !vR) return set_err(WENO_SB_ERR_ARG, "NULL array pointer");
    cudaStream_t st = (cudaStream_t)stream;
    if (dtype == WENO_SB_FP64) return launch_order1<double>(d, dir, v_vf, (double*)vL, (double*)vR, st);
    return launch_order1<float>(d, dir, v_vf, (float*)vL, (float*)vR, st);
}

int weno_sb_weno_dev(const weno_sb_grid* g, int dir, int order, unsigned flags, int dtype,
                     const void* v_in, const weno_sb_coefs* coefs, void* vL, void* vR, void* stream) {
    WSB_FAULT("launch");
    Dims d;
    int rc = check_grid(g, &d);
    if (rc || (rc = check_dir(dir)) || (rc = check_dtype(dtype))) return rc;
    if (order != 3 && order != 5 && order != 7)
        return set_err(WENO_SB_ERR_ARG, "order must be 3, 5 or 7 for weno_sb_weno_dev (got %d)", order);
    if (flags & ~(WENO_SB_F_SPLIT | WENO_SB_F_SPECIALIZED | WENO_SB_F_MP | WENO_SB_F_FOLDED))
        return set_err(WENO_SB_ERR_ARG, "unknown flag bits 0x%x", flags);
    if (!v_in || !vL || !vR || !coefs || !coefs->polyL || !coefs->polyR || !coefs->dL || !coefs->dR ||
        !coefs->beta_coef)
        return set_err(WENO_SB_ERR_ARG, "NULL array pointer");
    if ((flags & WENO_SB_F_FOLDED) && dtype != WENO_SB_FP64)
        return set_err(WENO_SB_ERR_UNSUPPORTED, "the folded form reads the FP64 v_vf; use dtype FP64");
    cudaStream_t st = (cudaStream_t)stream;
    if (dtype == WENO_SB_FP64)
        return run_weno<double>(d, g, dir, order, flags, (const double*)v_in, coefs, (double*)vL, (double*)vR, st);
    return run_weno<float>(d, g, dir, order, flags, (const float*)v_in, coefs, (float*)vL, (float*)vR, st);
}

int weno_sb_weno_uniform_dev(const weno_sb_grid* g, int dir, int order, unsigned flags, int dtype,
                             const void* v_in, const weno_sb_face_coefs* face, void* vL, void* vR, void* stream) {
    WSB_FAULT("launch");
    Dims d;
    int rc = check_grid(g, &d);
    if (rc || (rc = check_dir(dir)) || (rc = check_dtype(dtype))) return rc;
    if (order != 3 && order != 5 && order != 7)
        return set_err(WENO_SB_ERR_ARG, "order must be 3, 5 or 7 (got %d)", order);
    if (flags & ~(WENO_SB_F_SPLIT | WENO_SB_F_SPECIALIZED | WENO_SB_F_MP | WENO_SB_F_FOLDED))
        return set_err(WENO_SB_ERR_ARG, "unknown flag bits 0x%x", flags);
    if (!v_in || !vL || !vR || !face) return set_err(WENO_SB_ERR_ARG, "NULL pointer");
    if ((flags & WENO_SB_F_FOLDED) && dtype != WENO_SB_FP64)
        return set_err(WENO_SB_ERR_UNSUPPORTED, "the folded form reads the FP64 v_vf; use dtype FP64");
    double ucf[56];
    build_ucf(order, face, ucf);
    cudaStream_t st = (cudaStream_t)stream;
    if (dtype == WENO_SB_FP64)
        return run_weno<double>(d, g, dir, order, flags, (const double*)v_in, nullptr, (double*)vL, (double*)vR, st,
                                ucf);
    return run_weno<float>(d, g, dir, order, flags, (const float*)v_in, nullptr, (float*)vL, (float*)vR, st, ucf);
}

int weno_sb_vjp_dev(const weno_sb_grid* g, int dir, int order, unsigned flags, const double* v_in,
                    const weno_sb_coefs* coefs, const weno_sb_face_coefs* face, const double* gL, const double* gR,
                    double* gv, void* stream) {
    WSB_FAULT("launch");
    Dims d;
    int rc = check_grid(g, &d);
    if (rc || (rc = check_dir(dir))) return rc;
    if (order != 3 && order != 5 && order != 7)
        return set_err(WENO_SB_ERR_ARG, "order must be 3, 5 or 7 (got %d)", order);
    if (flags & ~(WENO_SB_F_SPLIT | WENO_SB_F_SPECIALIZED | WENO_SB_F_MP | WENO_SB_F_FOLDED | WENO_SB_F_ACCUMULATE))
        return set_err(WENO_SB_ERR_ARG, "unknown flag bits 0x%x", flags);
    if (g->scheme != WENO_SB_JS && g->scheme != WENO_SB_TENO)
        return set_err(WENO_SB_ERR_UNSUPPORTED, "the adjoint covers the JS and TENO weights (scheme %d)", g->scheme);
    if (order == 3 && g->scheme == WENO_SB_TENO)
        return set_err(WENO_SB_ERR_UNSUPPORTED, "WENO3 has no TENO weights (its forward output is NaN)");
    if (!v_in || !gL || !gR || !gv) return set_err(WENO_SB_ERR_ARG, "NULL pointer");
    if ((coefs == nullptr) == (face == nullptr))
        return set_err(WENO_SB_ERR_ARG, "pass exactly one of coefs (device arrays) and face (host values)");
    CoefPtrs cp{nullptr, nullptr, nullptr, nullptr, nullptr};
    double ucf[56];
    const double* up = nullptr;
    if (coefs) {
        if (!coefs->polyL || !coefs->polyR || !coefs->dL || !coefs->dR || !coefs->beta_coef)
            return set_err(WENO_SB_ERR_ARG, "NULL coefficient pointer");
        cp = CoefPtrs{coefs->polyL, coefs->polyR, coefs->dL, coefs->dR, coefs->beta_coef};
    } else {
        build_ucf(order, face, ucf);
        up = ucf;
    }
    return launch_vjp(d, g, dir, order, flags, v_in, cp, up, gL, gR, gv, (cudaStream_t)stream);
}

int weno_sb_preserve_monotonicity_dev(const weno_sb_grid* g, int dir, int dtype, const void* v_rs_ws,
                                      void* vL, void* vR, void* stream) {
    WSB_FAULT("launch");
    Dims d;
    int rc = check_grid(g, &d);
    if (rc || (rc = check_dir(dir)) || (rc = check_dtype(dtype))) return rc;
    if (!v_rs_ws || !vL || !vR) return set_err(WENO_SB_ERR_ARG, "NULL array pointer");
    SweepGeom sg = make_geom(d, dir, false);
    CoefPtrs cp{nullptr, nullptr, nullptr, nullptr, nullptr};
    WenoParams wp{g->scheme, g->weno_eps, g->teno_CT};
    cudaStream_t st = (cudaStream_t)stream;
    if (dtype == WENO_SB_FP64)
        return launch_generic<double>(sg, 0, true, (const double*)v_rs_ws, (double*)vL, (double*)vR, cp, wp, st);
    return launch_generic<float>(sg, 0, true, (const float*)v_rs_ws, (float*)vL, (float*)vR, cp, wp, st);
}

size_t weno_sb_checksum_scratch_bytes(int64_t n) {
    (void)n;
    return sizeof(double) * kSumBlocks;
}

int weno_sb_checksum_dev(int dtype, const void* arr, int64_t n, void* scratch, double* d_result,
                         void* stream) {
    WSB_FAULT("launch");
    int rc = check_dtype(dtype);
    if (rc) return rc;
    if (n < 0) return set_err(WENO_SB_ERR_ARG, "negative element count");
    if ((n > 0 && !arr) || !scratch || !d_result) return set_err(WENO_SB_ERR_ARG, "NULL pointer");
    cudaStream_t st = (cudaStream_t)stream;
    double* part = (double*)scratch;
    if (dtype == WENO_SB_FP64)
        abs_sum_partial_kernel<double><<<kSumBlocks, kSumThreads, 0, st>>>((const double*)arr, n, part);
    else
        abs_sum_partial_kernel<float><<<kSumBlocks, kSumThreads, 0, st>>>((const float*)arr, n, part);
    abs_sum_final_kernel<<<1, kSumThreads, 0, st>>>(part, kSumBlocks, d_result);
    return cuda_err(cudaGetLastError(), "checksum launch");
}

// ---------------- handle-based wrappers ----------------

int weno_sb_initialize_weno(int handle, int dir) {
    Handle* H = get_handle(handle);
    if (!H) return set_err(WENO_SB_ERR_HANDLE, "unknown handle %d", handle);
    await_vf(H);
    int rc = check_dir(dir);
    if (rc) return rc;
    return weno_sb_reshape_dev(&H->grid, dir, H->precision, (const double*)H->arr[WENO_SB_A_V_VF],
                               H->arr[WENO_SB_A_RS(dir)], H->stream);
}

int weno_sb_weno(int handle, int dir, int order, unsigned flags) {
    Handle* H = get_handle(handle);
    if (!H) return set_err(WENO_SB_ERR_HANDLE, "unknown handle %d", handle);
    int rc = check_dir(dir);
    if (rc) return rc;
    const bool folded = (flags & WENO_SB_F_FOLDED) != 0;
    if (H->vf_pending && (order == 1 || !folded || (order != 3 && order != 5 && order != 7))) await_vf(H);
    if (order == 1)
        return weno_sb_order1_dev(&H->grid, dir, H->precision, (const double*)H->arr[WENO_SB_A_V_VF],
                                  H->arr[WENO_SB_A_VL(dir)], H->arr[WENO_SB_A_VR(dir)], H->stream);
    weno_sb_coefs cf{(const double*)H->arr[WENO_SB_A_POLYL(dir)], (const double*)H->arr[WENO_SB_A_POLYR(dir)],
                     (const double*)H->arr[WENO_SB_A_DL(dir)], (const double*)H->arr[WENO_SB_A_DR(dir)],
                     (const double*)H->arr[WENO_SB_A_BETA(dir)]};
    const void* in = folded ? H->arr[WENO_SB_A_V_VF] : H->arr[WENO_SB_A_RS(dir)];
    bool uni = true;
    for (int k = 0; k < 5; ++k) uni = uni && H->coef_uniform[dir][k];
    if (H->vf_pending) {
        // v_vf is still arriving: one sweep per variable, each after its
        // variable's copy (the variables of v_vf and of the face states are
        // contiguous blocks, so a variable is a block of v_size 1)
        weno_sb_grid g1 = H->grid;
        g1.v_size = 1;
        const long long per_in = H->n[WENO_SB_A_V_VF] / H->dims.nv;
        const long long per_out = H->n[WENO_SB_A_VL(dir)] / H->dims.nv;
        for (int q = 0; q < H->dims.nv; ++q) {
            WSB_CUDA(cudaStreamWaitEvent(H->stream, H->var_ready[q], 0));
            const double* inq = (const double*)in + per_in * q;
            double* Lq = (double*)H->arr[WENO_SB_A_VL(dir)] + per_out * q;
            double* Rq = (double*)H->arr[WENO_SB_A_VR(dir)] + per_out * q;
            rc = (uni && getenv("WENO_SB_PER_FACE") == nullptr)
                     ? weno_sb_weno_uniform_dev(&g1, dir, order, flags, WENO_SB_FP64, inq, &H->face0[dir], Lq, Rq,
                                                H->stream)
                     : weno_sb_weno_dev(&g1, dir, order, flags, WENO_SB_FP64, inq, &cf, Lq, Rq, H->stream);
            if (rc) return rc;
        }
        return WENO_SB_OK;
    }
    if (uni && getenv("WENO_SB_PER_FACE") == nullptr)
        return weno_sb_weno_uniform_dev(&H->grid, dir, order, flags, H->precision, in, &H->face0[dir],
                                        H->arr[WENO_SB_A_VL(dir)], H->arr[WENO_SB_A_VR(dir)], H->stream);
    return weno_sb_weno_dev(&H->grid, dir, order, flags, H->precision, in, &cf, H->arr[WENO_SB_A_VL(dir)],
                            H->arr[WENO_SB_A_VR(dir)], H->stream);
}

int weno_sb_vjp(int handle, int dir, int order, unsigned flags, const double* gL, const double* gR, double* gv) {
    Handle* H = get_handle(handle);
    if (!H) return set_err(WENO_SB_ERR_HANDLE, "unknown handle %d", handle);
    await_vf(H);
    int rc = check_dir(dir);
    if (rc) return rc;
    if (H->precision != WENO_SB_FP64) return set_err(WENO_SB_ERR_UNSUPPORTED, "the adjoint is FP64 (FP32-bulk handle)");
    const void* in = (flags & WENO_SB_F_FOLDED) ? H->arr[WENO_SB_A_V_VF] : H->arr[WENO_SB_A_RS(dir)];
    bool uni = true;
    for (int k = 0; k < 5; ++k) uni = uni && H->coef_uniform[dir][k];
    if (uni && getenv("WENO_SB_PER_FACE") == nullptr)
        return weno_sb_vjp_dev(&H->grid, dir, order, flags, (const double*)in, nullptr, &H->face0[dir], gL, gR, gv,
                               H->stream);
    weno_sb_coefs cf{(const double*)H->arr[WENO_SB_A_POLYL(dir)], (const double*)H->arr[WENO_SB_A_POLYR(dir)],
                     (const double*)H->arr[WENO_SB_A_DL(dir)], (const double*)H->arr[WENO_SB_A_DR(dir)],
                     (const double*)H->arr[WENO_SB_A_BETA(dir)]};
    return weno_sb_vjp_dev(&H->grid, dir, order, flags, (const double*)in, &cf, nullptr, gL, gR, gv, H->stream);
}

int weno_sb_preserve_monotonicity(int handle, int dir) {
    Handle* H = get_handle(handle);
    if (!H) return set_err(WENO_SB_ERR_HANDLE, "unknown handle %d", handle);
    int rc = check_dir(dir);
    if (rc) return rc;
    return weno_sb_preserve_monotonicity_dev(&H->grid, dir, H->precision, H->arr[WENO_SB_A_RS(dir)],
                                             H->arr[WENO_SB_A_VL(dir)], H->arr[WENO_SB_A_VR(dir)], H->stream);
}

int weno_sb_checksum(int handle, int which, double* result) {
    Handle* H = get_handle(handle);
    if (!H) return set_err(WENO_SB_ERR_HANDLE, "unknown handle %d", handle);
    await_vf(H);
    if (which < 0 || which >= WENO_SB_A_COUNT) return set_err(WENO_SB_ERR_ARG, "unknown array id %d", which);
    if (!result) return set_err(WENO_SB_ERR_ARG, "result pointer is NULL");
    int rc = weno_sb_checksum_dev(H->dtype[which], H->arr[which], H->n[which], H->sum_scratch,
                                  H->sum_scratch + kSumBlocks, H->stream);
    if (rc) return rc;
    WSB_CUDA(cudaMemcpyAsync(result, H->sum_scratch + kSumBlocks, sizeof(double), cudaMemcpyDeviceToHost, H->stream));
    return cuda_err(cudaStreamSynchronize(H->stream), "checksum");
}

// ---------------- coefficients for arbitrary cell widths ----------------
int weno_sb_coefficients(int order, int64_t ns, const double* x_cb, double* polyL, double* polyR, double* dL,
                         double* dR, double* beta_coef) {
    if (order != 3 && order != 5 && order != 7)
        return set_err(WENO_SB_ERR_ARG, "order must be 3, 5 or 7 (got %d)", order);
    if (ns < 7) return set_err(WENO_SB_ERR_ARG, "need at least 7 cells along the sweep (got %lld)", (long long)ns);
    if (!x_cb || !polyL || !polyR || !dL || !dR || !beta_coef) return set_err(WENO_SB_ERR_ARG, "NULL pointer");
    for (int64_t k = 0; k <= ns; ++k) {
        if (!std::isfinite(x_cb[k])) return set_err(WENO_SB_ERR_ARG, "cell boundary %lld is not finite", (long long)k);
        if (k > 0 && !(x_cb[k] > x_cb[k - 1]))
            return set_err(WENO_SB_ERR_ARG, "cell boundaries must increase (x_cb[%lld] <= x_cb[%lld])", (long long)k,
                           (long long)(k - 1));
    }
    if (wsb::coef::generate(order, ns, x_cb, polyL, polyR, dL, dR, beta_coef) != 0)
        return set_err(WENO_SB_ERR_ARG, "degenerate stencil in the cell boundaries");
    return 0;
}

// ---------------- checksum without allocation ----------------
// Partial sums for weno_sb_checksum_noalloc: kSumBlocks doubles for each of
// up to kNoAllocMaxArrays arrays (74 KB), resident on every GPU that loads
// the library until the process exits.  Host code may not use the symbol
// as a device address: the address comes from cudaGetSymbolAddress, looked
// up on a device's first call and again whenever the device's current
// context is a different one (after cudaDeviceReset the module loads anew,
// possibly at another address).  Contexts are told apart by cuCtxGetId,
// which never repeats within a process.
static constexpr int kNoAllocMaxArrays = 16;
static __device__ __align__(256) double g_noalloc_partials[kNoAllocMaxArrays * kSumBlocks];
static constexpr int kNoAllocMaxDevices = 64;
static std::mutex g_noalloc_mu;
static double* g_noalloc_addr[kNoAllocMaxDevices] = {};
static unsigned long long g_noalloc_ctx[kNoAllocMaxDevices] = {};

// Id of the calling thread's current context, 0 when there is none or the
// driver entry points are unavailable.
static unsigned long long current_context_id() {
    typedef CUresult (*GetCurrentFn)(CUcontext*);
    typedef CUresult (*GetIdFn)(CUcontext, unsigned long long*);
    static GetCurrentFn get_current = nullptr;
    static GetIdFn get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = (GetCurrentFn)p;
        p = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = (GetIdFn)p;
    });
    if (!get_current || !get_id) return 0;
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (get_current(&ctx) != CUDA_SUCCESS || !ctx || get_id(ctx, &id) != CUDA_SUCCESS) return 0;
    return id;
}

int weno_sb_checksum_noalloc(int dtype, const void* const* arrays, const int64_t* n, int count,
                             double* d_results, void* stream) {
    WSB_FAULT("launch");
    int rc = check_dtype(dtype);
    if (rc) return rc;
    if (count < 1 || count > kNoAllocMaxArrays)
        return set_err(WENO_SB_ERR_ARG,
                       "count must be 1..%d: the static scratch holds the partial sums of at most %d arrays (got %d)",
                       kNoAllocMaxArrays, kNoAllocMaxArrays, count);
    if (!arrays || !n || !d_results) return set_err(WENO_SB_ERR_ARG, "NULL pointer");
    for (int a = 0; a < count; ++a) {
        if (n[a] < 0) return set_err(WENO_SB_ERR_ARG, "negative element count for array %d", a);
        if (n[a] > 0 && !arrays[a]) return set_err(WENO_SB_ERR_ARG, "NULL device pointer for array %d", a);
    }
    int dev = 0;
    WSB_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kNoAllocMaxDevices)
        return set_err(WENO_SB_ERR_UNSUPPORTED, "device ordinal %d beyond %d", dev, kNoAllocMaxDevices);
    double* scratch = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_noalloc_mu);
        // a thread with no current context yet (the runtime creates it on
        // first use) gets one from the lookup below, and its id after it
        const unsigned long long ctx = current_context_id();
        if (!g_noalloc_addr[dev] || ctx == 0 || ctx != g_noalloc_ctx[dev]) {
            void* p = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_partials);
            if (e != cudaSuccess) return cuda_err(e, "cudaGetSymbolAddress(g_noalloc_partials)");
            g_noalloc_addr[dev] = (double*)p;
            g_noalloc_ctx[dev] = current_context_id();
        }
        scratch = g_noalloc_addr[dev];
    }
    cudaStream_t st = (cudaStream_t)stream;
    for (int a = 0; a < count; ++a) {
        double* part = scratch + (size_t)a * kSumBlocks;
        // every one of the kSumBlocks partials is rewritten before it is read,
        // so nothing left by an earlier call needs clearing
        if (dtype == WENO_SB_FP64)
            abs_sum_partial_kernel<double><<<kSumBlocks, kSumThreads, 0, st>>>((const double*)arrays[a], n[a], part);
        else
            abs_sum_partial_kernel<float><<<kSumBlocks, kSumThreads, 0, st>>>((const float*)arrays[a], n[a], part);
        abs_sum_final_kernel<<<1, kSumThreads, 0, st>>>(part, kSumBlocks, d_results + a);
    }
    return cuda_err(cudaGetLastError(), "checksum (no-alloc) launch");
}

// Face-independent coefficients of a batch block: reads its coefficient
// arrays back once (batch set-up) and, when every face holds face 0's
// values, writes them in the Coef<order> layout.  False otherwise.
bool batch_coefs_uniform(const weno_sb_coefs& cf, long long nc, int order, double* ucf) {
    if (nc < 1) return false;
    std::vector<double> pL(nc * 15), pR(nc * 15), dL(5 * nc), dR(5 * nc), bc(nc * 30);
    if (cudaMemcpy(pL.data(), cf.polyL, sizeof(double) * pL.size(), cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(pR.data(), cf.polyR, sizeof(double) * pR.size(), cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(dL.data(), cf.dL, sizeof(double) * dL.size(), cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(dR.data(), cf.dR, sizeof(double) * dR.size(), cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(bc.data(), cf.beta_coef, sizeof(double) * bc.size(), cudaMemcpyDeviceToHost) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    // (nc, 5, S) arrays: face c of column (r, s) at c + nc (r + 5 s); (5, nc): r + 5 c
    auto same_cols = [&](const std::vector<double>& a, int S) {
        for (int k = 0; k < 5 * S; ++k)
            for (long long c = 1; c < nc; ++c)
                if (a[c + nc * k] != a[nc * k]) return false;
        return true;
    };
    auto same_rows = [&](const std::vector<double>& a) {
        for (long long c = 1; c < nc; ++c)
            for (int r = 0; r < 5; ++r)
                if (a[r + 5 * c] != a[r]) return false;
        return true;
    };
    if (!same_cols(pL, 3) || !same_cols(pR, 3) || !same_cols(bc, 6) || !same_rows(dL) || !same_rows(dR)) return false;
    weno_sb_face_coefs f{};
    for (int r = 0; r < 5; ++r) {
        for (int q = 0; q < 3; ++q) {
            f.polyL[q][r] = pL[nc * (r + 5 * q)];
            f.polyR[q][r] = pR[nc * (r + 5 * q)];
        }
        for (int q = 0; q < 6; ++q) f.beta_coef[q][r] = bc[nc * (r + 5 * q)];
        f.dL[r] = dL[r];
        f.dR[r] = dR[r];
    }
    build_ucf(order, &f, ucf);
    return true;
}

// Release everything a batch owns (also a half-built one).
void batch_free(Batch* B) {
    if (B->cap) cudaStreamSynchronize(B->cap);
    batch_release_graph(B);
    batch_free_groups(B);
    if (B->d_entries) cudaFree(B->d_entries);
    if (B->d_counter) cudaFree(B->d_counter);
    if (B->d_margs) cudaFree(B->d_margs);
    for (int k = 0; k < kBatchMaxBranches; ++k) {
        if (B->br[k]) cudaStreamDestroy(B->br[k]);
        if (B->join[k]) cudaEventDestroy(B->join[k]);
    }
    if (B->fork) cudaEventDestroy(B->fork);
    if (B->cap) cudaStreamDestroy(B->cap);
    delete B;
}

int weno_sb_batch_create(const weno_sb_block* blocks, int n, int* batch) {
    WSB_FAULT("init");
    if (!blocks || n < 1 || !batch) return set_err(WENO_SB_ERR_ARG, "need at least one block and a batch pointer");
    Batch* B = new Batch;
    cudaGetDevice(&B->device);
    for (int i = 0; i < n; ++i) {
        const weno_sb_block& b = blocks[i];
        Dims d;
        int rc = check_grid(&b.grid, &d);
        if (!rc) rc = check_dir(b.dir);
        if (!rc) rc = check_dtype(b.dtype);
        if (!rc && b.order != 3 && b.order != 5 && b.order != 7)
            rc = set_err(WENO_SB_ERR_ARG, "block %d: order must be 3, 5 or 7", i);
        if (!rc && (b.flags & ~(WENO_SB_F_MP | WENO_SB_F_FOLDED | WENO_SB_F_SPLIT | WENO_SB_F_SPECIALIZED)))
            rc = set_err(WENO_SB_ERR_ARG, "block %d: unknown flag bits 0x%x", i, b.flags);
        if (!rc && (!b.v_in || !b.vL || !b.vR || !b.coefs.polyL || !b.coefs.polyR || !b.coefs.dL ||
                    !b.coefs.dR || !b.coefs.beta_coef))
            rc = set_err(WENO_SB_ERR_ARG, "block %d: NULL pointer", i);
        if (rc) {
            delete B;
            return rc;
        }
        BatchEntry e{};
        e.g = make_geom(d, b.dir, (b.flags & WENO_SB_F_FOLDED) != 0);
        e.in = b.v_in;
        e.vL = b.vL;
        e.vR = b.vR;
        e.cp = CoefPtrs{b.coefs.polyL, b.coefs.polyR, b.coefs.dL, b.coefs.dR, b.coefs.beta_coef};
        e.wp = WenoParams{b.grid.scheme, b.grid.weno_eps, b.grid.teno_CT};
        e.order = b.order;
        e.mp = (b.flags & WENO_SB_F_MP) ? 1 : 0;
        e.fp32 = b.dtype == WENO_SB_FP32;
        e.o_first = (b.order == 3) ? 0 : 3;
        e.nf = (int)((b.order == 3) ? e.g.ns : e.g.nc);
        // marching items for the orders and weights a marching engine covers,
        // when the block's coefficients are the same on every face
        const bool js = b.grid.scheme == WENO_SB_JS;
        const bool teno = b.grid.scheme == WENO_SB_TENO;
        double ucf[56];
        const bool uni = batch_coefs_uniform(b.coefs, e.g.nc, b.order, ucf);
        B->ucf.push_back(uni ? std::vector<double>(ucf, ucf + 56) : std::vector<double>());
        if (uni && kernel_choice() != 1 && ((b.order == 5 || b.order == 7) && (js || teno) || (b.order == 3 && js)) &&
            march_weights_ok(ucf, b.order)) {
            B->margs.push_back(make_march_args(e.g, b.v_in, b.vL, b.vR, e.wp, ucf, b.order));
            e.march = (int)B->margs.size();
        }
        B->blocks.push_back(b);
        B->entries.push_back(e);
    }
    int rc = cuda_err(cudaMalloc((void**)&B->d_entries, sizeof(BatchEntry) * n), "cudaMalloc");
    if (!rc) rc = cuda_err(cudaMalloc((void**)&B->d_counter, sizeof(unsigned long long)), "cudaMalloc");
    if (!rc && !B->margs.empty()) {
        rc = cuda_err(cudaMalloc((void**)&B->d_margs, sizeof(MarchArgs) * B->margs.size()), "cudaMalloc");
        if (!rc)
            rc = cuda_err(cudaMemcpy(B->d_margs, B->margs.data(), sizeof(MarchArgs) * B->margs.size(),
                                     cudaMemcpyHostToDevice),
                          "cudaMemcpy");
    }
    if (!rc) rc = cuda_err(cudaStreamCreateWithFlags(&B->cap, cudaStreamNonBlocking), "cudaStreamCreate");
    for (int k = 0; !rc && k < kBatchMaxBranches; ++k) {
        rc = cuda_err(cudaStreamCreateWithFlags(&B->br[k], cudaStreamNonBlocking), "cudaStreamCreate");
        if (!rc) rc = cuda_err(cudaEventCreateWithFlags(&B->join[k], cudaEventDisableTiming), "cudaEventCreate");
    }
    if (!rc) rc = cuda_err(cudaEventCreateWithFlags(&B->fork, cudaEventDisableTiming), "cudaEventCreate");
    if (!rc) rc = batch_layout(B, 128, 8);
    if (!rc) rc = batch_plan_groups(B, B->seg_faces);
    if (rc) {
        batch_free(B);
        return rc;
    }
    std::lock_guard<std::mutex> lk(g_batch_mu);
    g_batches.push_back(B);
    *batch = (int)g_batches.size();
    return WENO_SB_OK;
}

// Time the ways of running the batch -- the persistent kernel over its
// tile shapes (CTA width x columns per item), the graph of specialised
// sweeps over its branch counts, the grouped sweeps over segment lengths
// and branch counts -- and keep the fastest.  Each candidate is captured
// into its graph, launched once to warm up and three times timed.  With
// WENO_SB_TUNE_CACHE naming a file, a batch of the same composition reuses
// the recorded choice (one line: signature, threads, columns per item,
// milliseconds, mode, branches, faces per grouped work item).
int weno_sb_batch_autotune(int batch, void* stream, int* threads, int* cols_per_item, double* best_ms) {
    Batch* B = get_batch(batch);
    if (!B) return set_err(WENO_SB_ERR_HANDLE, "unknown batch %d", batch);
    cudaStream_t st = (cudaStream_t)stream;
    const unsigned long long sig = batch_signature(B);
    const char* cache = getenv("WENO_SB_TUNE_CACHE");
    auto report = [&](double ms) {
        if (threads) *threads = B->threads;
        if (cols_per_item) *cols_per_item = B->U;
        if (best_ms) *best_ms = ms;
    };
    if (cache && *cache) {
        std::ifstream f(cache);
        std::string line;
        while (std::getline(f, line)) {
            std::istringstream ls(line);
            unsigned long long h;
            int t, u, mode = 0, nb = 8, sf = 64;
            double ms;
            if ((ls >> std::hex >> h >> std::dec >> t >> u >> ms) && h == sig) {
                if (!(ls >> mode >> nb)) { mode = 0; nb = 8; }
                if (!(ls >> sf) || sf < 8 || sf > 4096) sf = 64;
                int rc = batch_layout(B, t, u);
                if (!rc && mode == 2 && sf != B->seg_faces) rc = batch_plan_groups(B, sf);
                if (rc) return rc;
                B->mode = (mode == 1 || mode == 2) ? mode : 0;
                B->branches = std::max(1, std::min(nb, kBatchMaxBranches));
                batch_release_graph(B);
                report(ms);
                return WENO_SB_OK;
            }
        }
    }
    struct Cand { int mode, t, u, nb, sf; };
    std::vector<Cand> cands;
    for (int t : {64, 128, 256})
        for (int u : {4, 8, 16, 32}) cands.push_back({0, t, u, 0, 0});
    for (int nb : {1, 2, 4, 8, 16}) cands.push_back({1, 128, 8, nb, 0});
    if (!B->groups.empty())
        for (int sf : {32, 64, 128})
            for (int nb : {1, 2, 4}) cands.push_back({2, 128, 8, nb, sf});
    cudaEvent_t e0, e1;
    WSB_CUDA(cudaEventCreate(&e0));
    WSB_CUDA(cudaEventCreate(&e1));
    float best = 1e30f;
    Cand bc = cands[0];
    int rc = 0;
    for (const Cand& c : cands) {
        rc = batch_layout(B, c.t, c.u);
        if (!rc && c.mode == 2 && c.sf != B->seg_faces) rc = batch_plan_groups(B, c.sf);
        if (rc) break;
        B->mode = c.mode;
        B->branches = c.mode != 0 ? c.nb : B->branches;
        rc = batch_build_graph(B);
        if (!rc) rc = cuda_err(cudaGraphLaunch(B->exec, st), "cudaGraphLaunch");  // warm-up
        if (rc) break;
        cudaEventRecord(e0, st);
        for (int r = 0; r < 3; ++r) cudaGraphLaunch(B->exec, st);
        cudaEventRecord(e1, st);
        rc = cuda_err(cudaEventSynchronize(e1), "autotune");
        if (rc) break;
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        ms /= 3.f;
        if (ms < best) {
            best = ms;
            bc = c;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    rc = batch_layout(B, bc.t, bc.u);
    if (!rc && bc.mode == 2 && bc.sf != B->seg_faces) rc = batch_plan_groups(B, bc.sf);
    if (rc) return rc;
    B->mode = bc.mode;
    if (bc.mode != 0) B->branches = bc.nb;
    batch_release_graph(B);
    if (cache && *cache) {
        std::ofstream f(cache, std::ios::app);
        f << std::hex << sig << std::dec << " " << bc.t << " " << bc.u << " " << best << " " << bc.mode << " "
          << B->branches << " " << B->seg_faces << "\n";
    }
    report(best);
    return WENO_SB_OK;
}

int weno_sb_batch_launch(int batch, void* stream) {
    WSB_FAULT("launch");
    Batch* B = get_batch(batch);
    if (!B) return set_err(WENO_SB_ERR_HANDLE, "unknown batch %d", batch);
    if (!B->exec) {
        int rc = batch_build_graph(B);
        if (rc) return rc;
    }
    return cuda_err(cudaGraphLaunch(B->exec, (cudaStream_t)stream), "cudaGraphLaunch");
}

int weno_sb_batch_destroy(int batch) {
    Batch* B = get_batch(batch);
    if (!B) return set_err(WENO_SB_ERR_HANDLE, "unknown batch %d", batch);
    {
        std::lock_guard<std::mutex> lk(g_batch_mu);
        g_batches[batch - 1] = nullptr;
    }
    batch_free(B);
    return WENO_SB_OK;
}

int weno_sb_batch_configure(int batch, int mode, int threads, int cols_per_item, int branches) {
    Batch* B = get_batch(batch);
    if (!B) return set_err(WENO_SB_ERR_HANDLE, "unknown batch %d", batch);
    if (mode < 0 || mode > 2)
        return set_err(WENO_SB_ERR_ARG, "mode must be 0 (persistent), 1 (graph of sweeps) or 2 (grouped sweeps)");
    if (mode == 0) {
        if (threads != 64 && threads != 128 && threads != 256)
            return set_err(WENO_SB_ERR_ARG, "threads must be 64, 128 or 256 (got %d)", threads);
        if (cols_per_item < 1 || cols_per_item > 64)
            return set_err(WENO_SB_ERR_ARG, "cols_per_item must be 1..64 (got %d)", cols_per_item);
        B->mode = 0;
        return batch_layout(B, threads, cols_per_item);
    }
    if (branches < 1 || branches > kBatchMaxBranches)
        return set_err(WENO_SB_ERR_ARG, "branches must be 1..%d (got %d)", kBatchMaxBranches, branches);
    if (mode == 2) {
        if (cols_per_item < 8 || cols_per_item > 4096)
            return set_err(WENO_SB_ERR_ARG, "mode 2: cols_per_item (faces per work item) must be 8..4096 (got %d)",
                           cols_per_item);
        if (cols_per_item != B->seg_faces) {
            const int rc = batch_plan_groups(B, cols_per_item);
            if (rc) return rc;
        }
    }
    B->mode = mode;
    B->branches = branches;
    batch_release_graph(B);
    return WENO_SB_OK;
}

int weno_sb_batch_query(int batch, int* mode, int* threads, int* cols_per_item, int* branches) {
    Batch* B = get_batch(batch);
    if (!B) return set_err(WENO_SB_ERR_HANDLE, "unknown batch %d", batch);
    if (mode) *mode = B->mode;
    if (threads) *threads = B->threads;
    if (cols_per_item) *cols_per_item = B->mode == 2 ? B->seg_faces : B->U;
    if (branches) *branches = B->branches;
    return WENO_SB_OK;
}

int weno_sb_selftest_rcp(const double* d_x, double* d_fast, double* d_ieee, int64_t n, void* stream) {
    if (n < 0 || (n > 0 && (!d_x || !d_fast || !d_ieee))) return set_err(WENO_SB_ERR_ARG, "bad self-test arguments");
    if (n == 0) return WENO_SB_OK;
    selftest_rcp_kernel<<<(unsigned)std::min<int64_t>((n + 255) / 256, 4096), 256, 0, (cudaStream_t)stream>>>(
        d_x, d_fast, d_ieee, n);
    return cuda_err(cudaGetLastError(), "self-test launch");
}

int weno_sb_selftest_timeout(int64_t limit_cycles, void* stream) {
    if (limit_cycles < 0 || limit_cycles > 100000000LL)
        return set_err(WENO_SB_ERR_ARG, "limit_cycles must be in [0, 1e8]");
    selftest_timeout_kernel<<<1, 32, 0, (cudaStream_t)stream>>>((long long)limit_cycles);
    int rc = cuda_err(cudaGetLastError(), "self-test launch");
    if (rc) return rc;
    return weno_sb_check_device(stream);
}

}  // extern "C"
