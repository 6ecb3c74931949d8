// adjoint_steps.cuh -- the per-step vector updates of the leapfrog adjoint, one
// launch each instead of three (kick) or two (reverse drift) elementwise passes.
//
// Kick after the VJP of substep g (gx = (dF/dx)^T gF at x_{g+1}):
//     lx += gx;   lv += dt_g lx;   gF = c lv          (c = h_g + h_{g-1})
// Reverse drift of the time-reversed substep (F = F(x_{g+1})):
//     vh -= k F;  x -= dt_g vh
// Both are HBM streams over 3N doubles: grid-stride, 2 elements per thread-step.
#pragma once
#include "agb_dev.cuh"

__global__ void __launch_bounds__(256)
adjoint_kick_kernel(double* __restrict__ lx, double* __restrict__ lv, const double* __restrict__ gx,
                    double* __restrict__ gF, long long m, double dt, double c)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride) {
        const double x = lx[i] + gx[i];
        const double v = fma(dt, x, lv[i]);
        lx[i] = x;
        lv[i] = v;
        gF[i] = c * v;
    }
}

__global__ void __launch_bounds__(256)
reverse_drift_kernel(double* __restrict__ x, double* __restrict__ vh, const double* __restrict__ F,
                     long long m, double k, double dt)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride) {
        const double v = fma(-k, F[i], vh[i]);
        vh[i] = v;
        x[i] = fma(-dt, v, x[i]);
    }
}
