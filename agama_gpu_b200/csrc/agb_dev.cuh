// agb_dev.cuh -- device-side descriptors and small helpers shared by the
// Multipole, CylSpline and analytic evaluators.
#pragma once
#include <stdint.h>
#include "../../include/agb.h"
#include "legendre_tables.cuh"

#define AGB_G_AGAMA   4.30091727067736e-06                 // kpc (km/s)^2 / Msol
#define AGB_INV_4PIG  (1.0 / (4.0 * 3.141592653589793 * AGB_G_AGAMA))

// Component as the kernels see it (built on the host from agb_component or
// from the arguments of a kernel-signature entry).
struct DevComp {
    int kind;
    int n_lm;          // harmonics (Multipole) / harmonics (CylSpline)
    int n_int;         // radial intervals (Multipole) / nR (CylSpline)
    int nz;            // CylSpline z nodes
    int lmax;
    int log_scaling;
    int layout;        // Multipole: AGB_LAYOUT_*; CylSpline: 0 reference, 1 cell-major
    int lm_split;      // 1: harmonic list given as separate l[] and m[] arrays
    int structure;     // Multipole: AGB_STRUCT_* (column structure of the table)
    int pad_;
    const double*  table;
    const float*   table32;
    const int32_t* lm;     // packed (l<<16 | m&0xffff), or l[] when lm_split
    const int32_t* lm_m;   // m[] when lm_split
    const double*  grid_a;
    const double*  grid_b;
    const double*  extra;
    double p[16];
};

struct DevLeaf {
    int    comp;
    int    pad;
    double sigma;
    double g0, g1, g2;
    double ampl;
};

struct EvalArgs {
    long long n;
    int n_leaves;
    int out_flags;
    int soa;                 // 1: x, y, z separate arrays (kernel-signature entries)
    int pad;
    long long chunk;         // points per block: block b evaluates [b*chunk, (b+1)*chunk)
    const double* xyz;       // AoS N x 3 when !soa (sorted copy when perm != null)
    const int* perm;         // binned order: point pos is input point perm[pos]
    const double* x;
    const double* y;
    const double* z;
    double* phi;
    double* grad;
    double* hess;
    double* rho;
    double* stage;           // binned calls: outputs in sorted order, [pos][rec] (or null)
    const int* dest;         // binned calls: sorted position of input point i
    const double* gphi;      // VJP mode: dL/dPhi [N] (may be null)
    const double* gforce;    // VJP mode: dL/dF [N,3] (may be null)
    const DevLeaf* dleaves;  // leaves in device memory (agb_eval_timed), else null
    DevComp comps[AGB_MAX_COMPONENTS];
    DevLeaf leaves[AGB_MAX_LEAVES];
};

// Result of one component at one point (component frame, un-negated).
struct PointOut {
    double phi;
    double g[3];
    double h[6];           // Hxx, Hyy, Hzz, Hxy, Hyz, Hxz
    double rho;
};

// Hessian slot -> (i, j) in the output order Hxx, Hyy, Hzz, Hxy, Hyz, Hxz.
__device__ __forceinline__ int hess_i(int p) { return p < 3 ? p : (p == 4 ? 1 : 0); }
__device__ __forceinline__ int hess_j(int p) { return p < 3 ? p : (p == 3 ? 1 : 2); }

// Spherically symmetric Phi(r) given dPhi/dr and d2Phi/dr2 as radial terms:
// H_ij = A x_i x_j + B delta_ij with A = (d2 - d1/r)/r^2, B = d1/r.
__device__ __forceinline__ void hess_radial(double A, double B, double x, double y,
                                            double z, double* h)
{
    h[0] = A * x * x + B;
    h[1] = A * y * y + B;
    h[2] = A * z * z + B;
    h[3] = A * x * y;
    h[4] = A * y * z;
    h[5] = A * x * z;
}
