// time_plan.cuh -- time-dependent leaf transforms evaluated on the device.
//
// A leaf program (agb_leaf_prog) maps the time t to one leaf (component,
// sigma, gamma, ampl) through the modifier chain of its component, innermost
// modifier first, with the arithmetic of the host path operation by
// operation:
//   * Shifted centre (gpu_potential.py:1716-1734): a cubic spline inside
//     [t0, tN] evaluated like scipy's PPoly (interval by bisection with
//     x[i] <= t, the last interval at t = tN; sum of c_k s^k with s^k formed
//     by repeated multiplication), the end value plus slope times (t - t_end)
//     outside; gamma += sigma * c;
//   * Scaled (gpu_potential.py:1845-1871): s = 1/scale(t), a = ampl(t) (a spline
//     or the static value) the same way; sigma *= s, ampl = (a*s)*ampl;
//   * Evolving (gpu_potential.py:1559-1612): the bisection bracket and
//     alpha = (t - t_i)/(t_i+1 - t_i), or the nearest snapshot (first minimum
//     of |t_j - t|); ampl *= weight.
// Every product and sum is rounded on its own (no FMA contraction), so the
// device leaves equal the host leaves bit for bit; the same functions compile
// for the host (agb_time_plan_leaves_host).
#pragma once
#include <math.h>
#include "agb_dev.cuh"

__host__ __device__ __forceinline__ double tp_mul(double a, double b)
{
#ifdef __CUDA_ARCH__
    return __dmul_rn(a, b);
#else
    return a * b;
#endif
}
__host__ __device__ __forceinline__ double tp_add(double a, double b)
{
#ifdef __CUDA_ARCH__
    return __dadd_rn(a, b);
#else
    return a + b;
#endif
}
__host__ __device__ __forceinline__ double tp_sub(double a, double b)
{
#ifdef __CUDA_ARCH__
    return __dsub_rn(a, b);
#else
    return a - b;
#endif
}
__host__ __device__ __forceinline__ double tp_div(double a, double b)
{
#ifdef __CUDA_ARCH__
    return __ddiv_rn(a, b);
#else
    return a / b;
#endif
}

// largest i in [0, T-2] with x[i] <= t, for x[0] <= t <= x[T-1]
__host__ __device__ __forceinline__ int tp_interval(const double* x, int T, double t)
{
    int lo = 0, hi = T - 2;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (x[mid] <= t) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// component j of a piecewise cubic (c[4][T-1][dim], highest power first) at t
__host__ __device__ __forceinline__ double tp_cubic(const double* c, int T, int dim, int i, int j,
                                                    double s)
{
    const long long stride = (long long)(T - 1) * dim;
    double res = 0.0, z = 1.0;
    for (int kp = 0; kp < 4; ++kp) {
        res = tp_add(res, tp_mul(c[(3 - kp) * stride + (long long)i * dim + j], z));
        if (kp < 3) z = tp_mul(z, s);
    }
    return res;
}

// a spline value with linear extension: end value e0/eN and slope d0/dN
__host__ __device__ __forceinline__ double tp_spline1(const double* x, const double* c, int T,
                                                      double t0, double tN, double e0, double eN,
                                                      double d0, double dN, double t)
{
    if (t < t0) return tp_add(e0, tp_mul(d0, tp_sub(t, t0)));
    if (t > tN) return tp_add(eN, tp_mul(dN, tp_sub(t, tN)));
    const int i = tp_interval(x, T, t);
    return tp_cubic(c, T, 1, i, 0, tp_sub(t, x[i]));
}

// the leaf of one program at time t (agb_leaf layout: comp, pair flag, sigma,
// gamma[3], ampl)
__host__ __device__ inline void tp_leaf(const agb_leaf_prog& pg, const double* tab, double t,
                                        DevLeaf& o)
{
    int comp = pg.comp;
    double sigma = 1.0, g0 = 0.0, g1 = 0.0, g2 = 0.0, ampl = 1.0;
    for (int k = 0; k < pg.n_ops; ++k) {
        const double* d = tab + pg.arg[k];
        if (pg.op[k] == AGB_OP_SHIFT) {
            double c0, c1, c2;
            if (d[0] == 0.0) {
                c0 = d[1]; c1 = d[2]; c2 = d[3];
            } else {
                const int T = (int)d[1];
                const double t0 = d[2], tN = d[3];
                const double* p0 = d + 4; const double* pN = d + 7;
                const double* v0 = d + 10; const double* vN = d + 13;
                const double* x = d + 16;
                const double* cc = x + T;
                if (t < t0) {
                    const double dt = tp_sub(t, t0);
                    c0 = tp_add(p0[0], tp_mul(v0[0], dt));
                    c1 = tp_add(p0[1], tp_mul(v0[1], dt));
                    c2 = tp_add(p0[2], tp_mul(v0[2], dt));
                } else if (t > tN) {
                    const double dt = tp_sub(t, tN);
                    c0 = tp_add(pN[0], tp_mul(vN[0], dt));
                    c1 = tp_add(pN[1], tp_mul(vN[1], dt));
                    c2 = tp_add(pN[2], tp_mul(vN[2], dt));
                } else {
                    const int i = tp_interval(x, T, t);
                    const double s = tp_sub(t, x[i]);
                    c0 = tp_cubic(cc, T, 3, i, 0, s);
                    c1 = tp_cubic(cc, T, 3, i, 1, s);
                    c2 = tp_cubic(cc, T, 3, i, 2, s);
                }
            }
            g0 = tp_add(g0, tp_mul(sigma, c0));
            g1 = tp_add(g1, tp_mul(sigma, c1));
            g2 = tp_add(g2, tp_mul(sigma, c2));
        } else if (pg.op[k] == AGB_OP_SCALE) {
            double s, a;
            if (d[0] == 0.0) {
                s = tp_div(1.0, d[1]);
                a = d[2];
            } else {
                const int T = (int)d[1];
                const double t0 = d[2], tN = d[3];
                const double* x = d + 14;
                const double* cs = x + T;
                s = tp_div(1.0, tp_spline1(x, cs, T, t0, tN, d[4], d[5], d[6], d[7], t));
                if (d[8] != 0.0) {
                    const double* ca = cs + 4LL * (T - 1);
                    a = tp_spline1(x, ca, T, t0, tN, d[10], d[11], d[12], d[13], t);
                } else {
                    a = d[9];
                }
            }
            sigma = tp_mul(sigma, s);
            ampl = tp_mul(tp_mul(a, s), ampl);
        } else if (pg.op[k] == AGB_OP_EVOLVE) {
            const int n = (int)d[0];
            const bool interp = d[1] != 0.0;
            const double* tt = d + 2;
            int pick = 0;
            double w = 1.0;
            if (n == 1 || !interp) {
                double best = fabs(tp_sub(tt[0], t));
                for (int j = 1; j < n; ++j) {
                    const double e = fabs(tp_sub(tt[j], t));
                    if (e < best) { best = e; pick = j; }
                }
            } else {
                int i;
                double alpha;
                if (t <= tt[0]) {
                    i = 0; alpha = 0.0;
                } else if (t >= tt[n - 1]) {
                    i = n - 2; alpha = 1.0;
                } else {
                    int lo = 0, hi = n - 2;
                    while (lo < hi) {
                        const int mid = (lo + hi) / 2;
                        if (tt[mid + 1] <= t) lo = mid + 1;
                        else hi = mid;
                    }
                    i = lo;
                    alpha = tp_div(tp_sub(t, tt[i]), tp_sub(tt[i + 1], tt[i]));
                }
                if (pg.slot == 0) {
                    pick = i;
                    w = alpha == 0.0 ? 1.0 : (alpha == 1.0 ? 0.0 : tp_sub(1.0, alpha));
                } else {
                    pick = i + 1;
                    w = alpha == 0.0 ? 0.0 : (alpha == 1.0 ? 1.0 : alpha);
                }
            }
            comp += pick;
            ampl = tp_mul(ampl, w);
        }
    }
    o.comp = comp;
    o.pad = pg.pair;
    o.sigma = sigma;
    o.g0 = g0; o.g1 = g1; o.g2 = g2;
    o.ampl = ampl;
}

#define AGB_TP_MAX AGB_MAX_LEAVES

struct TimeLeafArgs {
    agb_leaf_prog progs[AGB_TP_MAX];
    int n;
    const double* table;
    const long long* step;       // null: step 0
    double t0, dt, off;
    DevLeaf* out;
};

__global__ void __launch_bounds__(32)
time_leaves_kernel(const __grid_constant__ TimeLeafArgs a)
{
    const int i = threadIdx.x;
    if (i >= a.n) return;
    const double st = a.step ? (double)(*a.step) : 0.0;
    const double t = tp_add(tp_add(a.t0, tp_mul(st, a.dt)), a.off);
    DevLeaf o;
    tp_leaf(a.progs[i], a.table, t, o);
    a.out[i] = o;
}

// leapfrog boundary update: v = fma(h1, F, v); v = fma(h2, F, v); x = fma(dt, v, x)
__global__ void __launch_bounds__(256)
kick_drift_kernel(double* __restrict__ x, double* __restrict__ v, const double* __restrict__ F,
                  long long m, double h1, double h2, double dt, int flags, long long* step)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    const long long i0 = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    for (long long i = i0; i < m; i += stride) {
        double vi = v[i];
        const double f = F[i];
        if (flags & 1) vi = fma(h1, f, vi);
        if (flags & 2) vi = fma(h2, f, vi);
        if (flags & 3) v[i] = vi;
        if (flags & 4) x[i] = fma(dt, vi, x[i]);
    }
    if ((flags & 8) && step && i0 == 0) *step += 1;
}
