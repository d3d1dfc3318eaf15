/*
 * weno_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of the WENO harness kernels of wilfonba/WenoStandalone
 * (inputs/weno_standalone.f90).  It is the checker that the CUDA library is
 * compared against; nothing in the product links it.  Only tests/, the smoke
 * check and the bench's CPU-baseline / reference arm may load it.
 *
 * Array conventions (all Fortran column-major, first index fastest, flat
 * 0-based here):
 *   sweep input  v_rs_ws : (ns+6) x c1 x c2 x nv   (sweep axis with +-3 halo)
 *   sweep output vL, vR  :  ns    x c1 x c2 x nv
 *   poly{L,R}            :  nc x 5 x 3              (nc = ns - 6 core faces)
 *   d{L,R}               :  5 x nc
 *   beta_coef            :  nc x 5 x 6
 * For the x sweep (ns,c1,c2) = (N1,N2,N3); y: (N2,N1,N3); z: (N3,N2,N1),
 * with Nd = cells + 2*buff_size.  For m=n=p this is byte-identical to the
 * harness's own allocations (f90:163-187).
 */
#ifndef WENO_ORACLE_H
#define WENO_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

enum { WO_JS = 0, WO_MAPPED = 1, WO_Z = 2, WO_TENO = 3, WO_NONE = 4 };

void wo_fill_input_field(int m, int n, int p, int nv, int buff, double *v_vf);
void wo_fill_coefficients(int nc, double offset, double *polyL, double *polyR,
                          double *dL, double *dR, double *beta);
int wo_reshape(int m, int n, int p, int nv, int buff, int dir,
               const double *v_vf, double *v_rs_ws);
int wo_order1_copy(int m, int n, int p, int nv, int buff, int dir,
                   const double *v_vf, double *vL, double *vR);
int wo_reconstruct(int ns, int c1, int c2, int nv, int order, int scheme,
                   double eps, double teno_ct, const double *v_rs_ws,
                   const double *polyL, const double *polyR, const double *dL,
                   const double *dR, const double *beta, double *vL, double *vR);
int wo_teno_margin(int ns, int c1, int c2, int nv, int order, double eps, double teno_ct,
                   const double *v_rs_ws, const double *beta, double *margin);
int wo_preserve_monotonicity(int ns, int c1, int c2, int nv,
                             const double *v_rs_ws, double *vL, double *vR);
double wo_checksum(long long n, const double *a);
int wo_harness_run(int m, int n, int p, int nv, int buff, double eps,
                   int scheme, double teno_ct, int all_mode, double out[4]);
void wo_set_threads(int nthreads);
int wo_get_threads(void);

#ifdef __cplusplus
}
#endif
#endif
