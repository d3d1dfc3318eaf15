/*
 * weno_sb.h -- C ABI of the B200 WENO library (libweno_sb.so).
 *
 * Drop-in replacement for the device loops of the reference WENO harness
 * wilfonba/WenoStandalone (inputs/weno_standalone.f90, "f90:" below), which
 * in turn restate MFC's src/simulation/m_weno.fpp.  Every entry point says
 * which reference routine it replaces.  All calls return an int status:
 *   0                      success
 *   1 .. 999               a cudaError_t from the CUDA runtime
 *   WENO_SB_ERR_* (>=1000) an argument or library error
 * weno_sb_last_error_string() describes the last failure of this thread.
 *
 * Array layouts are the reference's Fortran allocations (column-major,
 * first index fastest, variable index slowest), passed as base addresses
 * (c_loc of the first element):
 *   v_vf        (N1+6, N2+6, N3+6, V)      f90:163-165  cell field, 3 pad cells
 *   v_rs_ws_d   (Ns+6, C1, C2, V)          f90:167-169  sweep-ordered field
 *   vL_d, vR_d  (Ns,   C1, C2, V)          f90:1779-1784 face states
 *   polyL/R_d   (NC, 5, 3)                 f90:171-176
 *   dL/R_d      (5, NC)                    f90:178-183
 *   beta_coef_d (NC, 5, 6)                 f90:185-187
 * with Nd = cells_d + 2*buff_size, NC = Ns - 6 core faces, and per
 * direction (Ns, C1, C2) = x: (N1,N2,N3), y: (N2,N1,N3), z: (N3,N2,N1).
 * For m=n=p these are exactly the harness's arrays; other block shapes use
 * the general (Ns, C1, C2) extents above.
 */
#ifndef WENO_SB_H
#define WENO_SB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define WENO_SB_VERSION 1

/* ---- status codes (>= 1000; smaller positive values are cudaError_t) ---- */
#define WENO_SB_OK 0
#define WENO_SB_ERR_ARG 1001         /* invalid argument / shape             */
#define WENO_SB_ERR_HANDLE 1002      /* unknown or finalized handle          */
#define WENO_SB_ERR_UNSUPPORTED 1003 /* valid request this build cannot do   */
#define WENO_SB_ERR_INJECTED 1004    /* failure injected via WENO_SB_FAULT   */
#define WENO_SB_ERR_TIMEOUT 1005     /* a bounded device wait gave up        */
#define WENO_SB_ERR_ALIGN 1006       /* pointer alignment requirement unmet  */
#define WENO_SB_ERR_HOST 1007        /* host allocation failed               */

/* ---- nonlinear weight families (f90:64-75: wenojs, mapped_weno, wenoz, teno) */
#define WENO_SB_JS 0     /* wenojs = .true.                                  */
#define WENO_SB_MAPPED 1 /* mapped_weno (compile-time .false. in the harness) */
#define WENO_SB_Z 2      /* wenoz       (compile-time .false. in the harness) */
#define WENO_SB_TENO 3   /* teno: wenojs = .false. with teno = .true.         */
#define WENO_SB_NONE 4   /* wenojs = .false. with every family disabled: the
                            shipped harness; alpha stays 0 and outputs NaN   */

/* ---- storage precision of sweep fields and face states ---- */
#define WENO_SB_FP64 0 /* everything FP64 (the reference)                    */
#define WENO_SB_FP32 1 /* FP32-bulk: FP32 storage and stencil sums, FP64 beta
                          differences and weight normalisation               */

/* ---- flags for weno_sb_weno / weno_sb_weno_dev ---- */
#define WENO_SB_F_SPLIT 1u       /* WENO5_SPLIT_KERNELS=1 (f90:1410-1412)    */
#define WENO_SB_F_SPECIALIZED 2u /* WENO5_SPECIALIZED_COMBINED=1 (f90:1721)  */
#define WENO_SB_F_MP 4u          /* fuse s_preserve_monotonicity (f90:1544)  */
#define WENO_SB_F_FOLDED 8u      /* read v_vf directly: reshape folded into
                                    the sweep (no v_rs_ws needed)            */
#define WENO_SB_F_ACCUMULATE 16u /* adjoint: add into gv instead of writing it */

/* ---- array ids for the handle API (the harness's module arrays) ---- */
#define WENO_SB_A_V_VF 0
#define WENO_SB_A_RS(d) (1 + (d))     /* v_rs_ws_{x,y,z}                     */
#define WENO_SB_A_VL(d) (4 + (d))     /* vL_{x,y,z}                          */
#define WENO_SB_A_VR(d) (7 + (d))     /* vR_{x,y,z}                          */
#define WENO_SB_A_POLYL(d) (10 + (d)) /* poly_coef_cbL_{x,y,z}               */
#define WENO_SB_A_POLYR(d) (13 + (d)) /* poly_coef_cbR_{x,y,z}               */
#define WENO_SB_A_DL(d) (16 + (d))    /* d_cbL_{x,y,z}                       */
#define WENO_SB_A_DR(d) (19 + (d))    /* d_cbR_{x,y,z}                       */
#define WENO_SB_A_BETA(d) (22 + (d))  /* beta_coef_{x,y,z}                   */
#define WENO_SB_A_COUNT 25

/* Grid and scheme parameters: the &grid_params namelist (f90:117-118). */
typedef struct weno_sb_grid {
    int32_t m_cells, n_cells, p_cells; /* m, n, p (cells - 1 per axis)        */
    int32_t v_size;                    /* number of variables                 */
    int32_t buff_size;                 /* ghost layers per side (>= 3)        */
    int32_t scheme;                    /* WENO_SB_JS / _MAPPED / _Z / _TENO / _NONE */
    double weno_eps;                   /* regulariser added to beta           */
    double teno_CT;                    /* TENO cutoff                         */
} weno_sb_grid;

/* Device pointers to one direction's coefficients (layouts above). */
typedef struct weno_sb_coefs {
    const double *polyL, *polyR, *dL, *dR, *beta_coef;
} weno_sb_coefs;

/* One face's coefficients, on the host, for grids where every face uses the
 * same values (uniform spacing, and the harness's synthetic data):
 * polyL[s][r] = polyL(j,r,s), dL[r] = dL(r,j), beta_coef[s][r] =
 * beta_coef(j,r,s) for any core face j. */
typedef struct weno_sb_face_coefs {
    double polyL[3][5], polyR[3][5];
    double dL[5], dR[5];
    double beta_coef[6][5];
} weno_sb_face_coefs;

/* ===================================================================== */
/* Library                                                                */
/* ===================================================================== */
int weno_sb_version(void);
const char *weno_sb_last_error_string(void);
/* Extents helper: (Ns, C1, C2) of direction dir, and NC = Ns - 6. */
int weno_sb_extents(const weno_sb_grid *g, int dir, int64_t *ns, int64_t *c1, int64_t *c2);

/* ===================================================================== */
/* Handle API: the harness's module state on one GPU.                     */
/* ===================================================================== */

/* Allocate device mirrors of every array of f90:163-187 plus vL/vR_{x,y,z}
 * (f90:1779-1790) and a private stream: replaces s_initialize_data's
 * `target enter data map(alloc:...)` (f90:194-197, 1790).  `precision` is
 * WENO_SB_FP64 or WENO_SB_FP32 (v_rs_ws and vL/vR stored as float). */
int weno_sb_init(const weno_sb_grid *g, int precision, int *handle);
/* Release everything: replaces s_finalize_data (f90:207-219). */
int weno_sb_finalize(int handle);
/* Host <-> device copies of one array, always FP64 on the host side
 * (converted on the fly for FP32 handles): replace `target update to/from`
 * (f90:199-203, 1791, 1831).  Synchronous. */
int weno_sb_upload(int handle, int which, const double *host);
int weno_sb_download(int handle, int which, double *host);
/* weno_sb_upload of v_vf without waiting for it -- no counterpart in the
 * reference, whose `target update to` is synchronous.  The copy runs on a
 * copy stream of the handle one variable at a time, and the folded sweeps
 * (weno_sb_weno with WENO_SB_F_FOLDED, orders 3/5/7) launch one variable at
 * a time, each waiting only for its own variable, so the sweeps of the first
 * variables run while the later ones are still crossing PCIe.  Every other
 * call on the handle waits for the whole copy first.  The host buffer must
 * not change until weno_sb_sync, weno_sb_download or weno_sb_checksum
 * returns (they wait for the copy); it overlaps nothing unless page-locked
 * (cudaHostAlloc / cudaHostRegister).  Other arrays, and FP32 handles, take
 * the synchronous weno_sb_upload. */
int weno_sb_upload_async(int handle, int which, const double *host);
/* Device address, element count and storage dtype (WENO_SB_FP64/FP32).
 * After weno_sb_upload_async, call weno_sb_sync before reading v_vf there. */
int weno_sb_array_info(int handle, int which, void **dev_ptr, int64_t *n_elem, int *dtype);
/* s_initialize_weno_{x,y,z} (f90:281-330): reshape v_vf into v_rs_ws_dir. */
int weno_sb_initialize_weno(int handle, int dir);
/* s_weno: order 1 = s_order1_copy_dir (f90:332-390); 3 = s_weno3_kernel
 * (f90:392-475); 5 = s_weno5_kernel_dispatch / s_weno5_kernel_dir
 * (f90:477-1417); 7 = s_weno7_kernel (f90:1419-1542).  flags: WENO_SB_F_*. */
int weno_sb_weno(int handle, int dir, int order, unsigned flags);
/* s_preserve_monotonicity (f90:1544-1615) on vL/vR_dir, in place. */
int weno_sb_preserve_monotonicity(int handle, int dir);
/* Adjoint of weno_sb_weno(handle, dir, order, flags) for order 3/5/7 -- no
 * counterpart in the reference.  Reads the handle's v_rs_ws_dir (or v_vf
 * with WENO_SB_F_FOLDED) and coefficients; gL, gR (face layout) and gv
 * (layout of the input) are device pointers of the caller.  See
 * weno_sb_vjp_dev for the flags and the meaning of gv.  FP64 handles. */
int weno_sb_vjp(int handle, int dir, int order, unsigned flags, const double *gL, const double *gR, double *gv);
/* f_checksum (f90:1617-1620): sum(|a|) of one array, computed on the GPU. */
int weno_sb_checksum(int handle, int which, double *result);
/* Wait for all work queued on the handle's stream; also reports a device
 * timeout (WENO_SB_ERR_TIMEOUT) raised by a pipelined sweep. */
int weno_sb_sync(int handle);
/* Synchronise `stream` (a cudaStream_t) and report, then clear, the device
 * error flag that pipelined sweeps set when a bounded wait for staged data
 * expires (WENO_SB_ERR_TIMEOUT).  Device-pointer callers use it where the
 * handle API uses weno_sb_sync. */
int weno_sb_check_device(void *stream);
/* The handle's cudaStream_t (as void*), for callers that order their own
 * work after the library's. */
int weno_sb_stream(int handle, void **stream);

/* ===================================================================== */
/* Device-pointer API: MFC-style calls on caller-owned device arrays.      */
/* `stream` is a cudaStream_t (NULL = legacy default stream).  FP32-bulk  */
/* arrays (v_rs_ws, vL, vR) are float when dtype == WENO_SB_FP32; v_vf    */
/* and the coefficients are always double.                                */
/* ===================================================================== */

/* s_initialize_weno_dir (f90:281-330). */
int weno_sb_reshape_dev(const weno_sb_grid *g, int dir, int dtype, const double *v_vf,
                        void *v_rs_ws, void *stream);
/* s_order1_copy_dir (f90:332-390). */
int weno_sb_order1_dev(const weno_sb_grid *g, int dir, int dtype, const double *v_vf,
                       void *vL, void *vR, void *stream);
/* Reconstruction, order 3/5/7 (f90:392-1542).  v_in is v_rs_ws_dir, or
 * v_vf when flags has WENO_SB_F_FOLDED.  Per-face coefficient arrays take a
 * per-face table, allocated and freed stream-ordered on `stream`
 * (cudaMallocAsync). */
int weno_sb_weno_dev(const weno_sb_grid *g, int dir, int order, unsigned flags, int dtype,
                     const void *v_in, const weno_sb_coefs *coefs, void *vL, void *vR,
                     void *stream);
/* The same reconstruction for face-independent coefficients given on the
 * host (MFC on a uniform grid; the harness's synthetic coefficients, which
 * f90:256-277 fills identically for every face): the kernels take them from
 * the kernel-parameter bank instead of per-thread registers.  The handle
 * API uses this path by itself when the uploaded coefficient arrays are
 * face-independent.  Allocates nothing. */
int weno_sb_weno_uniform_dev(const weno_sb_grid *g, int dir, int order, unsigned flags, int dtype,
                             const void *v_in, const weno_sb_face_coefs *face, void *vL, void *vR,
                             void *stream);
/* Adjoint (vector-Jacobian product) of one sweep -- no counterpart in the
 * reference, which has no derivatives.  With the sweep's outputs
 * (vL, vR) = F(v_in) for order 3/5/7, JS or TENO weights (the grid's
 * scheme) and the MP limiter when flags has WENO_SB_F_MP, it computes
 * gv = (dF/dv)^T (gL, gR), recomputing beta and the weights from v_in
 * instead of storing them.  gL, gR have the face layout; v_in and gv the
 * layout of v_rs_ws, or of v_vf with WENO_SB_F_FOLDED.  gv is overwritten
 * (the cells no face reads get 0) unless WENO_SB_F_ACCUMULATE adds into it,
 * so the three folded sweeps can sum into one gv.  Coefficients come either
 * per face (coefs) or face-independent (face); pass exactly one.  FP64. */
int weno_sb_vjp_dev(const weno_sb_grid *g, int dir, int order, unsigned flags, const double *v_in,
                    const weno_sb_coefs *coefs, const weno_sb_face_coefs *face, const double *gL,
                    const double *gR, double *gv, void *stream);
/* s_preserve_monotonicity (f90:1544-1615). */
int weno_sb_preserve_monotonicity_dev(const weno_sb_grid *g, int dir, int dtype,
                                      const void *v_rs_ws, void *vL, void *vR, void *stream);
/* f_checksum (f90:1617-1620) of n values on the device.  `scratch` is a
 * caller-owned device buffer of weno_sb_checksum_scratch_bytes(n) bytes;
 * the sum is written to the device double *d_result. */
size_t weno_sb_checksum_scratch_bytes(int64_t n);
int weno_sb_checksum_dev(int dtype, const void *arr, int64_t n, void *scratch,
                         double *d_result, void *stream);

/* f_checksum of up to 16 arrays in one call, allocating nothing.
 * No counterpart in the reference.  For callers that cannot allocate device
 * memory: Fortran drivers whose device heap belongs to the OpenMP/OpenACC
 * offload runtime (as in MFC), and time-step loops that must not call
 * cudaMalloc/cudaFree because those calls can synchronise the whole device.
 * arrays[a] (device pointers) and n[a] are host arrays of `count` entries;
 * sum(|arrays[a]|) is written to the device double d_results[a].  The
 * scratch is a static device array of 16 x 592 doubles (74 KB) in the
 * library, held on every GPU that loads it until exit: count > 16 is
 * rejected with WENO_SB_ERR_ARG.  The first call on a device looks up the
 * array's device address (cudaGetSymbolAddress), and so does the first call
 * after the device's context changes (cudaDeviceReset); make those calls
 * before any stream capture.  All calls share the one array, so calls that overlap
 * on the GPU (different streams, or host threads) race; each call rewrites
 * every partial it reads, so nothing needs clearing between calls. */
int weno_sb_checksum_noalloc(int dtype, const void *const *arrays, const int64_t *n, int count,
                             double *d_results, void *stream);

/* Coefficients of WENO-JS reconstruction, order 3/5/7, for a grid with any
 * cell widths -- MFC's s_compute_weno_coefficients, for which the reference
 * substitutes synthetic values (f90:246-279).  x_cb[0..ns] are the cell
 * boundaries along one sweep (ns = the direction's Ns, ghost cells
 * included, increasing); the outputs are HOST arrays in the layouts above
 * with NC = ns - 6 core faces (core face c is sweep cell c + 3), entries
 * the order does not use set to 0.  Follows C.-W. Shu, ICASE Report 97-65
 * (1997), sections 2.1-2.2 (stencil values from the primitive function,
 * linear weights) and Jiang & Shu, JCP 126 (1996) (smoothness indicators).
 * Host computation only (set-up time): upload the arrays, or pass them to
 * weno_sb_weno_dev after copying them to the device. */
int weno_sb_coefficients(int order, int64_t ns, const double *x_cb, double *polyL, double *polyR,
                         double *dL, double *dR, double *beta_coef);

/* ===================================================================== */
/* Batches of uneven blocks (no counterpart in the reference, which runs   */
/* one block): one CUDA graph launch of all the blocks' sweeps.            */
/* ===================================================================== */
typedef struct weno_sb_block {
    weno_sb_grid grid;     /* this block's extents, v_size and weights      */
    int32_t dir, order;    /* sweep direction 0/1/2, order 3/5/7            */
    uint32_t flags;        /* WENO_SB_F_MP, WENO_SB_F_FOLDED                */
    int32_t dtype;         /* WENO_SB_FP64, or WENO_SB_FP32: v_in, vL, vR are
                              float (for a folded FP32 entry v_in is an FP32
                              copy of v_vf)                                 */
    const void *v_in;      /* v_rs_ws_dir, or v_vf with WENO_SB_F_FOLDED     */
    weno_sb_coefs coefs;   /* per-face coefficient arrays (device)           */
    void *vL, *vR;         /* face states (device)                           */
} weno_sb_block;

/* Validate the blocks and build the device work list (allocates).  The
 * coefficient arrays are read back once here: blocks whose arrays hold the
 * same values on every face get the face-independent kernels, so their
 * coefficients must not change while the batch lives. */
int weno_sb_batch_create(const weno_sb_block *blocks, int n, int *batch);
/* Time the ways of running the batch on `stream` and keep the fastest:
 * mode 0, one persistent kernel over all blocks (candidate tile shapes:
 * CTA width x columns per work item); mode 1, every block's sweep by the
 * sweep kernel specialised for it, spread over 1..16 parallel branches of
 * the graph (candidate branch counts); mode 2, the blocks with
 * face-independent coefficients that a marching engine covers grouped by
 * kernel and coefficients, one TMA marching launch per group over all its
 * blocks' work items (candidate faces per work item and branch counts),
 * the other blocks as in mode 1.  With WENO_SB_TUNE_CACHE naming a file, a
 * batch of the same composition reuses the recorded choice.
 * threads / cols_per_item report the persistent layout. */
int weno_sb_batch_autotune(int batch, void *stream, int *threads, int *cols_per_item, double *best_ms);
/* Choose the way explicitly: mode 0 with threads (64/128/256) and
 * cols_per_item (1..64); mode 1 with branches (1..16); or mode 2 (grouped
 * marching sweeps: one launch per group of blocks with the same kernel and
 * coefficients) with cols_per_item = faces per work item (8..4096) and
 * branches (1..16).  weno_sb_batch_query reports the faces per work item
 * in cols_per_item for mode 2. */
int weno_sb_batch_configure(int batch, int mode, int threads, int cols_per_item, int branches);
/* The current choice (any pointer may be NULL). */
int weno_sb_batch_query(int batch, int *mode, int *threads, int *cols_per_item, int *branches);
/* Run every block's sweep: one graph launch, captured on first use after
 * the choice last changed. */
int weno_sb_batch_launch(int batch, void *stream);
int weno_sb_batch_destroy(int batch);

/* ===================================================================== */
/* Diagnostics (no counterpart in the reference; used by the test suite).  */
/* ===================================================================== */
/* fast[i] = the library's Newton-refined reciprocal of x[i], ieee[i] = 1/x[i]
 * by IEEE division, for n device doubles (normal, positive x). */
int weno_sb_selftest_rcp(const double *d_x, double *d_fast, double *d_ieee, int64_t n, void *stream);
/* Launch one bounded mbarrier wait that nothing completes, with a limit of
 * limit_cycles SM clocks (<= 1e8), and return what weno_sb_check_device
 * reports afterwards: WENO_SB_ERR_TIMEOUT when the bound works. */
int weno_sb_selftest_timeout(int64_t limit_cycles, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* WENO_SB_H */
