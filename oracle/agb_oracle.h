/*
 * agb_oracle.h -- TEST INFRASTRUCTURE ONLY (the oracle).
 *
 * A plain-C, one-point-at-a-time restatement of the reference's evaluation
 * algorithms, used by tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline as the checker.  The product never links or calls it.
 *
 * Layouts are the reference's: SoA x, y, z; Multipole poly[(c*n_int+k)*6+j]
 * with lm_l/lm_m sorted by (|m|, l, cos before sin); CylSpline
 * node_arr[((h*nR+iR)*nz+iz)*4+q] with m_arr ascending.  Outputs are Phi,
 * gradient of Phi (AoS 3), Hessian of Phi (AoS 6: xx, yy, zz, xy, yz, xz) and
 * density, i.e. the reference kernels' raw outputs.
 */
#ifndef AGB_ORACLE_H
#define AGB_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* mode: 0 potential, 1 potential+gradient, 2 +Hessian, 3 density */
int oracle_multipole(int mode, const double* x, const double* y, const double* z,
                     const double* poly, const double* scalars /* 10: logr_min, dlogr,
                     inv_dlogr, invPhi0, in_s, in_U, in_W, out_s, out_U, out_W */,
                     int n_int, int n_lm, int lmax, const int* lm_l, const int* lm_m,
                     int log_scaling, double* phi, double* grad, double* hess, double* rho,
                     int64_t n, int nthreads);

/* mode: 0, 1, 2 as above; 3 density = -(Hxx+Hyy+Hzz)/(4 pi G) as the reference's wrapper */
int oracle_cylspline(int mode, const double* x, const double* y, const double* z,
                     double Rscale, const double* lR, int nR, const double* lz, int nz,
                     const double* node_arr, int n_harm, const int* m_arr, int log_scaling,
                     const double* W_outer, double r0_outer, int lmax_outer, int mmax_outer,
                     double* phi, double* grad, double* hess, double* rho, int64_t n,
                     int nthreads);

/* kind: 10 NFW, 11 Plummer, 12 Hernquist, 13 Dehnen, 14 Isochrone, 15 MiyamotoNagai,
   16 LogHalo, 17 DiskAnsatz, 18 UniformAcceleration; p[] as in include/agb.h's users */
int oracle_analytic(int kind, const double* p, int mode, const double* x, const double* y,
                    const double* z, double* phi, double* grad, double* hess, double* rho,
                    int64_t n);

#ifdef __cplusplus
}
#endif
#endif
