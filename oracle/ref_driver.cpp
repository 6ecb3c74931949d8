/*
 * ref_driver.cpp -- test infrastructure only (oracle).
 *
 * Host driver for the reference's own kernels compiled as C++ through
 * ref_shim.h.  Each entry point runs the reference kernel once per point
 * (threadIdx.x = i, blockIdx.x = 0, blockDim.x = 1) under OpenMP.  The
 * argument lists are the reference's kernel signatures verbatim:
 *   _multipole_potential_kernel.cu:415-455 (potential/force),
 *   :466-483 (hess), :809-826 (density);
 *   _cylspl_potential_kernel.cu:871-972 (potential/force/hess).
 * Nothing in the product links this file.
 */
#include "ref_shim.h"
#include <omp.h>

thread_local ref_dim3 threadIdx;
thread_local ref_dim3 blockIdx;
thread_local ref_dim3 blockDim;

#define MP_ARGS                                                              \
    const double* x, const double* y, const double* z, const double* poly,   \
    double logr_min, double dlogr, double inv_dlogr, int n_intervals,        \
    int n_lm, int lmax, const int* lm_l, const int* lm_m, int log_scaling,    \
    double invPhi0, double inner_s, double inner_U, double inner_W,          \
    double outer_s, double outer_U, double outer_W
#define MP_PASS x, y, z, poly, logr_min, dlogr, inv_dlogr, n_intervals, n_lm, \
    lmax, lm_l, lm_m, log_scaling, invPhi0, inner_s, inner_U, inner_W,        \
    outer_s, outer_U, outer_W

extern "C" void multipole_potential_kernel(MP_ARGS, double* phi, double* grad, int N);
extern "C" void multipole_force_kernel(MP_ARGS, double* phi, double* grad, int N);
extern "C" void multipole_hess_kernel(MP_ARGS, double* phi, double* grad, double* hess, int N);
extern "C" void multipole_density_kernel(MP_ARGS, double inv_4piG, double* rho, int N);

#define CS_ARGS                                                               \
    const double* x, const double* y, const double* z, double Rscale,         \
    const double* lR_grid, int nR, const double* lz_grid, int nz,             \
    const double* node_arr, int n_harm, const int* m_arr, int mmax,           \
    int log_scaling, const double* W_outer, double r0_outer, int lmax_outer,  \
    int mmax_outer
#define CS_PASS x, y, z, Rscale, lR_grid, nR, lz_grid, nz, node_arr, n_harm,  \
    m_arr, mmax, log_scaling, W_outer, r0_outer, lmax_outer, mmax_outer

extern "C" void cylspl_potential_kernel(CS_ARGS, double* phi, int N);
extern "C" void cylspl_force_kernel(CS_ARGS, double* phi, double* grad, int N);
extern "C" void cylspl_hess_kernel(CS_ARGS, double* phi, double* grad, double* hess, int N);

#define FOR_POINTS(N, CALL)                                  \
    _Pragma("omp parallel for schedule(static)")             \
    for (int i = 0; i < (N); i++) {                          \
        threadIdx.x = (unsigned)i; blockIdx.x = 0; blockDim.x = 1; \
        CALL;                                                \
    }

/* mode: 0 = potential, 1 = potential+gradient, 2 = +hessian, 3 = density */
extern "C" int ref_multipole_eval(int mode, MP_ARGS, double inv_4piG,
                                  double* phi, double* grad, double* hess,
                                  double* rho, int N, int nthreads)
{
    if (nthreads > 0) omp_set_num_threads(nthreads);
    switch (mode) {
    case 0: FOR_POINTS(N, multipole_potential_kernel(MP_PASS, phi, grad, N)); break;
    case 1: FOR_POINTS(N, multipole_force_kernel(MP_PASS, phi, grad, N)); break;
    case 2: FOR_POINTS(N, multipole_hess_kernel(MP_PASS, phi, grad, hess, N)); break;
    case 3: FOR_POINTS(N, multipole_density_kernel(MP_PASS, inv_4piG, rho, N)); break;
    default: return -1;
    }
    return 0;
}

/* mode: 0 = potential, 1 = potential+gradient, 2 = +hessian */
extern "C" int ref_cylspl_eval(int mode, CS_ARGS, double* phi, double* grad,
                               double* hess, int N, int nthreads)
{
    if (nthreads > 0) omp_set_num_threads(nthreads);
    switch (mode) {
    case 0: FOR_POINTS(N, cylspl_potential_kernel(CS_PASS, phi, N)); break;
    case 1: FOR_POINTS(N, cylspl_force_kernel(CS_PASS, phi, grad, N)); break;
    case 2: FOR_POINTS(N, cylspl_hess_kernel(CS_PASS, phi, grad, hess, N)); break;
    default: return -1;
    }
    return 0;
}

extern "C" int ref_max_threads(void) { return omp_get_max_threads(); }
