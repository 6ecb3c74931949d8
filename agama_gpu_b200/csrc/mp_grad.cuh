// mp_grad.cuh -- gradient of a loss with respect to a Multipole's quintic
// coefficients (the table-gradient half of the backward pass).
//
// For one Multipole leaf (component frame x' = sigma x - gamma, output factor
// A), with cotangents gPhi = dL/dPhi and gF = dL/dF of the composite's
// outputs, the loss depends on the leaf's Phi(x') and grad Phi(x') through
//   alpha = gPhi A,   w = -A sigma gF,   beta_r,theta,phi = w . (u_r, u_theta, u_phi)
// where grad Phi = Phi_r u_r + Phi_theta u_theta + Phi_os u_phi.  Inside the
// radial grid and with the log-scaling factor F(log r):
//   dL/da_{c,j} = s^j U_c + j s^(j-1) V_c                               (c >= 1)
//   U_c = (alpha F + beta_r dF) W_c + beta_theta F dW_c + beta_phi F Q_c
//   V_c = beta_r F inv_dlogr W_c
// with W = Y T, dW = dY/dtheta T, Q = (Y/sin theta) dT/dphi, and for the
// monopole column through F and dF (chain rule written out in the kernel).
// Each warp reduces its lanes' six values per harmonic with shuffles when all
// of its points share one interval (the points are binned by interval), else
// every lane adds its own; FP64 atomics accumulate into grad[k][c][j].
//
// The scalars the table builder derives from the nodes get their gradient too
// (gconst, 8 doubles: invPhi0, inner s, U, W, outer eps, T, S (below), 0).  A point
// inside the grid depends on invPhi0 through F = 1/(invPhi0 - e^c0):
//   dL/dinvPhi0 = -F^2 QF - 2 F dF QdF,
// QF and QdF the weights of F and dF in the point's loss (those of the monopole
// column below).  A point beyond the grid has Phi = MP0 p0(log r) and
// grad Phi = MP0 d1 x / r^2 with p0 = U e^(s dlr) + W (inside the first node) or
// W e^(-dlr) + U e^(s dlr) (beyond the last) and d1 = dp0/dlog r, so
//   dL/dc = MP0 (alpha dp0/dc + beta_r dd1/dc),  beta_r = w . x / r^2.
// The outer fit is usually degenerate: its power s = -1 + eps with eps at the
// rounding level and U ~ -W ~ 1e16 (the builder's two roots coincide), so its
// gradient is taken in the well-conditioned variables eps = s + 1,
// T = U eps, S = U + W:  p0 = e^(-dlr) (S + T phi),  phi = expm1(eps dlr) / eps,
// d1 = e^(-dlr) (T e^(eps dlr) - S - T phi).
#pragma once
#include "multipole.cuh"

#ifndef AGB_MP_NCONST
#define AGB_MP_NCONST 8
#endif

// one point's contributions to the gradient of the builder's scalars (zeros for a
// point inside the grid except v[0], which the caller sets)
__device__ __forceinline__ void mp_const_extrap(const DevComp& c, double r, double alpha,
                                                double br, double v[AGB_MP_NCONST])
{
    const double MP0 = AGB_MUL0 * AGB_PREFACT[0];
    const double logr_min = c.p[0], dlogr = c.p[1];
    if (!(r >= 1.0e-300)) {                 // the origin: Phi = MP0 W_in, no force
        v[3] += MP0 * alpha;
        return;
    }
    const double logr = log(r);
    if (logr < logr_min) {
        const double s = c.p[4], U = c.p[5];
        const double dlr = logr - logr_min;
        const double rs = (s != 0.0) ? exp(s * dlr) : 1.0;
        // p0 = U rs + W, d1 = U s rs
        v[1] += MP0 * (alpha * U * dlr * rs + br * U * rs * (1.0 + s * dlr));
        v[2] += MP0 * (alpha * rs + br * s * rs);
        v[3] += MP0 * alpha;
        return;
    }
    const int k = (int)((logr - logr_min) * c.p[2]);
    if (k < c.n_int) return;
    const double eps = c.p[7] + 1.0, T = c.p[8] * eps, S = c.p[8] + c.p[9];
    const double dlr = logr - (logr_min + c.n_int * dlogr);
    const double en = exp(-dlr), x = eps * dlr, ex = exp(x);
    double ph, dph;                         // phi and dphi/deps (series near eps = 0)
    if (fabs(x) < 1.0e-4) {
        ph = dlr * (1.0 + x * (0.5 + x * (1.0 / 6.0)));
        dph = dlr * dlr * (0.5 + x * (1.0 / 3.0 + x * 0.125));
    } else {
        ph = expm1(x) / eps;
        dph = (dlr * ex * eps - expm1(x)) / (eps * eps);
    }
    v[4] += MP0 * en * T * (alpha * dph + br * (dlr * ex - dph));     // d/deps
    v[5] += MP0 * en * (alpha * ph + br * (ex - ph));                 // d/dT
    v[6] += MP0 * en * (alpha - br);                                  // d/dS
}

__device__ __forceinline__ double warp_sum(double v)
{
    #pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Warp reduce-scatter of eight values: lane L returns the warp sum of value
// 4*b4 + 2*b3 + b2 (b = bits of L); 9 shuffles instead of 40 for eight
// independent butterflies.
template <typename T>
__device__ __forceinline__ T warp_rs8(const T v[8], int lane)
{
    const bool h16 = lane & 16, h8 = lane & 8, h4 = lane & 4;
    T w[4], u[2];
    #pragma unroll
    for (int q = 0; q < 4; ++q) {
        const T keep = h16 ? v[q + 4] : v[q];
        const T send = h16 ? v[q] : v[q + 4];
        w[q] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
    }
    #pragma unroll
    for (int q = 0; q < 2; ++q) {
        const T keep = h8 ? w[q + 2] : w[q];
        const T send = h8 ? w[q] : w[q + 2];
        u[q] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
    }
    T z = (h4 ? u[1] : u[0]) + __shfl_xor_sync(0xffffffffu, h4 ? u[0] : u[1], 4);
    z += __shfl_xor_sync(0xffffffffu, z, 2);
    z += __shfl_xor_sync(0xffffffffu, z, 1);
    return z;
}

// add the warp's eight constant gradients (lane values v) into g: one atomic each
__device__ __forceinline__ void mp_const_flush(double* g, const double v[AGB_MP_NCONST], int lane)
{
    const double z = warp_rs8<double>(v, lane);
    const int idx = ((lane >> 4) & 1) * 4 + ((lane >> 3) & 1) * 2 + ((lane >> 2) & 1);
    if ((lane & 3) == 0 && z != 0.0) atomicAdd(g + idx, z);
}

// add six per-lane values into gk[col][0..5]; gk is the interval's row of the
// gradient (null when no lane of a uniform warp is inside the grid)
__device__ __forceinline__ void grad_add6(double* __restrict__ gk, int col, const double v[6],
                                          bool uniform, int lane, bool active)
{
    if (uniform) {
        double s[6];
        #pragma unroll
        for (int j = 0; j < 6; ++j) s[j] = warp_sum(active ? v[j] : 0.0);
        if (lane == 0 && gk) {
            #pragma unroll
            for (int j = 0; j < 6; ++j) atomicAdd(gk + (long long)col * 6 + j, s[j]);
        }
    } else if (active && gk) {
        #pragma unroll
        for (int j = 0; j < 6; ++j) atomicAdd(gk + (long long)col * 6 + j, v[j]);
    }
}

struct MPGradArgs {
    long long n;
    const double* xyz;        // sorted copy when perm != null
    const int* perm;
    const double* gphi;       // [N] or null
    const double* gforce;     // [N,3] or null
    double* grad;             // [n_int][n_lm][6], accumulated
    double* gconst;           // [AGB_MP_NCONST] or null, accumulated
    DevComp c;
    DevLeaf leaf;
};

// one warp-synchronous pass over all points (every lane runs the same loop trip count)
__global__ void __launch_bounds__(256, 1)
mp_grad_kernel(const __grid_constant__ MPGradArgs a)
{
    const DevComp& c = a.c;
    const int lane = threadIdx.x & 31;
    const long long warp0 = ((long long)blockIdx.x * blockDim.x + threadIdx.x) - lane;
    const long long wstride = (long long)gridDim.x * blockDim.x;
    const double logr_min = c.p[0], dlogr = c.p[1], inv_dlogr = c.p[2], invPhi0 = c.p[3];
    const double MP0 = AGB_MUL0 * AGB_PREFACT[0];
    for (long long base = warp0; base < a.n; base += wstride) {
        const long long pos = base + lane;
        bool active = pos < a.n;
        long long i = pos;
        double px = 0.0, py = 0.0, pz = 1.0, gp = 0.0, gf0 = 0.0, gf1 = 0.0, gf2 = 0.0;
        if (active) {
            i = a.perm ? (long long)a.perm[pos] : pos;
            const double X = a.xyz[3 * pos], Yv = a.xyz[3 * pos + 1], Z = a.xyz[3 * pos + 2];
            px = a.leaf.sigma * X - a.leaf.g0;
            py = a.leaf.sigma * Yv - a.leaf.g1;
            pz = a.leaf.sigma * Z - a.leaf.g2;
            gp = a.gphi ? a.gphi[i] : 0.0;
            if (a.gforce) { gf0 = a.gforce[3 * i]; gf1 = a.gforce[3 * i + 1]; gf2 = a.gforce[3 * i + 2]; }
        }
        const double r2 = px * px + py * py + pz * pz;
        const double r = sqrt(r2);
        const double Rc = sqrt(px * px + py * py);
        int k = -1;
        double s = 0.0;
        if (active && r >= 1.0e-300) {
            const double logr = log(r);
            if (logr >= logr_min) {
                int kk = (int)((logr - logr_min) * inv_dlogr);
                if (kk < 0) kk = 0;
                if (kk < c.n_int) {
                    k = kk;
                    s = fmin(fmax((logr - (logr_min + kk * dlogr)) * inv_dlogr, 0.0), 1.0);
                }
            }
        }
        active = active && k >= 0;
        // lanes outside the grid walk with zero weights at a valid interval
        const int kw = active ? k : 0;
        const double inv_r = active ? 1.0 / r : 0.0;
        const double cth = active ? pz * inv_r : 1.0;
        const double sth = active ? Rc * inv_r : 0.0;
        const double cph = (Rc > 1.0e-300) ? px / Rc : 1.0;
        const double sph = (Rc > 1.0e-300) ? py / Rc : 0.0;

        // forward quantities
        double c0, c0s, c0ss;
        mp_quintic0(c, kw, s, c0, c0s, c0ss);
        const double dc0 = c0s * inv_dlogr;
        double F = 1.0, dF = 0.0, F1 = 0.0, ex = 0.0;
        if (c.log_scaling) {
            ex = exp(c0);
            F = 1.0 / (invPhi0 - ex);
            F1 = F * F * ex;
            dF = F1 * dc0;
        }
        MPSums t = {};
        if (c.structure == AGB_STRUCT_EVEN)
            mp_harmonics_reg<AGB_MODE_GRAD, double, 2>(c, kw, s, cth, sth, cph, sph, t);
        else if (c.structure == AGB_STRUCT_ALL)
            mp_harmonics_reg<AGB_MODE_GRAD, double, 1>(c, kw, s, cth, sth, cph, sph, t);
        else
            mp_harmonics<AGB_MODE_GRAD, double>(c, kw, s, cth, sth, cph, sph, t);
        const double Bp = t.B * inv_dlogr;

        // per-point weights
        const double As = a.leaf.ampl * a.leaf.sigma;
        const double w0 = -As * gf0, w1 = -As * gf1, w2 = -As * gf2;
        const double inv_r2 = inv_r * inv_r;
        const double alpha = active ? gp * a.leaf.ampl : 0.0;
        const double br = active ? (w0 * px + w1 * py + w2 * pz) * inv_r2 : 0.0;
        const double bt = active ? (w0 * cth * cph + w1 * cth * sph - w2 * sth) * inv_r : 0.0;
        const double bp = active ? (-w0 * sph + w1 * cph) * inv_r : 0.0;
        const double P1 = alpha * F + br * dF, P2 = br * F * inv_dlogr, P3 = bt * F, P4 = bp * F;

        // uniform interval across the warp?
        const int kmax = __reduce_max_sync(0xffffffffu, k);
        const bool uniform = __all_sync(0xffffffffu, k == kmax || k < 0);
        const double sp[6] = {1.0, s, s * s, s * s * s, s * s * s * s, s * s * s * s * s};
        const double dw[6] = {0.0, 1.0, 2.0 * s, 3.0 * s * s, 4.0 * s * s * s, 5.0 * s * s * s * s};

        // monopole column
        {
            double v[6];
            if (c.log_scaling) {
                const double QF = alpha * (MP0 + t.A) + br * Bp + bt * t.Th + bp * t.Pos;
                const double QdF = br * (MP0 + t.A);
                const double dFdc0 = F1 * (1.0 + 2.0 * F * ex) * dc0;
                #pragma unroll
                for (int j = 0; j < 6; ++j)
                    v[j] = QF * F1 * sp[j] + QdF * (dFdc0 * sp[j] + F1 * inv_dlogr * dw[j]);
            } else {
                #pragma unroll
                for (int j = 0; j < 6; ++j)
                    v[j] = alpha * MP0 * sp[j] + br * MP0 * inv_dlogr * dw[j];
            }
            const int kk = uniform ? kmax : k;
            grad_add6((kk >= 0) ? a.grad + (long long)kk * c.n_lm * 6 : nullptr, 0, v, uniform,
                      lane, active);
            if (a.gconst) {             // the builder's scalars (warp-uniform branch)
                double cv[AGB_MP_NCONST] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
                if (active && c.log_scaling) {
                    const double QF = alpha * (MP0 + t.A) + br * Bp + bt * t.Th + bp * t.Pos;
                    const double QdF = br * (MP0 + t.A);
                    cv[0] = -F * F * QF - 2.0 * F * dF * QdF;
                } else if (!active && pos < a.n) {
                    const double brx = -As * (gf0 * px + gf1 * py + gf2 * pz) / r2;
                    mp_const_extrap(c, r, gp * a.leaf.ampl, r2 > 0.0 ? brx : 0.0, cv);
                }
                mp_const_flush(a.gconst, cv, lane);
            }
        }

        // harmonic columns: the same regular / list walk as the forward
        const bool near_pole = sth < 1.0e-10;
        const double inv_sth = near_pole ? 0.0 : 1.0 / sth;
        const int kk = uniform ? kmax : k;
        double* gbase = (kk >= 0) ? a.grad + (long long)kk * c.n_lm * 6 : nullptr;
        double cm = 1.0, sm = 0.0, sinpow = 1.0, sinpow_m1 = 0.0;
        int col = 1;
        const int par = (c.structure == AGB_STRUCT_EVEN) ? 2 : 1;
        if (c.structure == AGB_STRUCT_LIST) {
            // list walk: one column at a time, (l, m) from the harmonic list
            int cur = 0, lc = 0;
            double Pc = AGB_SEED[0], Pp = 0.0, dPc = 0.0, dPp = 0.0;
            for (int ci = 1; ci < c.n_lm; ++ci) {
                int l, m;
                mp_decode(c, ci, l, m);
                const int am = m < 0 ? -m : m;
                if (l > AGB_MAX_LMAX || am > l || am < cur || (am == cur && l < lc)) continue;
                if (am != cur) {
                    for (int q = cur; q < am; ++q) {
                        const double tt = cm * cph - sm * sph;
                        sm = sm * cph + cm * sph; cm = tt;
                        sinpow_m1 = sinpow; sinpow *= sth;
                    }
                    cur = am;
                    Pc = AGB_SEED[am] * sinpow; Pp = 0.0; dPp = 0.0;
                    dPc = (am == 0) ? 0.0 : (am == 1 ? AGB_SEED[1] * cth
                          : (near_pole ? 0.0 : (double)am * AGB_SEED[am] * sinpow_m1 * cth));
                    lc = am;
                }
                while (lc < l) {
                    ++lc;
                    const int ti = am * AGB_LEG_N + lc;
                    const double Pn = AGB_ALPHA[ti] * (cth * Pc) - AGB_BETA[ti] * Pp;
                    const double dPn = AGB_ALPHA[ti] * (cth * dPc - sth * Pc) - AGB_BETA[ti] * dPp;
                    Pp = Pc; Pc = Pn; dPp = dPc; dPc = dPn;
                }
                const double T = m >= 0 ? cm : sm;
                const double dT = m >= 0 ? -(double)am * sm : (double)am * cm;
                const double Pos = (am == 0) ? 0.0 : (!near_pole ? Pc * inv_sth : (am == 1 ? dPc : 0.0));
                const double U = T * (P1 * Pc + P3 * dPc) + dT * P4 * Pos;
                const double V = P2 * Pc * T;
                double v[6];
                #pragma unroll
                for (int j = 0; j < 6; ++j) v[j] = sp[j] * U + dw[j] * V;
                grad_add6(gbase, ci, v, uniform, lane, active);
            }
        } else {
            for (int m = 0; m <= c.lmax; ++m) {
                if (m > 0) {
                    const double tt = cm * cph - sm * sph;
                    sm = sm * cph + cm * sph; cm = tt;
                    sinpow_m1 = sinpow; sinpow *= sth;
                }
                int l0 = (par == 2) ? (m + (m & 1)) : m;
                if (m == 0) l0 = par;
                if (l0 > c.lmax) continue;
                const double q1 = (near_pole && m == 1) ? 1.0 : 0.0;
                double Pc = AGB_SEED[m] * sinpow, Pp = 0.0, dPp = 0.0;
                double dPc = (m == 0) ? 0.0 : (m == 1 ? AGB_SEED[1] * cth
                             : (near_pole ? 0.0 : (double)m * AGB_SEED[m] * sinpow_m1 * cth));
                const int tb = m * AGB_LEG_N;
                int l = m;
                for (;;) {
                    while (l < l0) {
                        ++l;
                        const double Pn = AGB_ALPHA[tb + l] * (cth * Pc) - AGB_BETA[tb + l] * Pp;
                        const double dPn = AGB_ALPHA[tb + l] * (cth * dPc - sth * Pc) - AGB_BETA[tb + l] * dPp;
                        Pp = Pc; Pc = Pn; dPp = dPc; dPc = dPn;
                    }
                    const double Pos = Pc * inv_sth + q1 * dPc;
                    const double base_c = P1 * Pc + P3 * dPc;
                    const double dTc = -(double)m * sm, dTs = (double)m * cm;
                    {
                        const double U = cm * base_c + dTc * P4 * Pos, V = P2 * Pc * cm;
                        double v[6];
                        #pragma unroll
                        for (int j = 0; j < 6; ++j) v[j] = sp[j] * U + dw[j] * V;
                        grad_add6(gbase, col, v, uniform, lane, active);
                        ++col;
                    }
                    if (m > 0) {
                        const double U = sm * base_c + dTs * P4 * Pos, V = P2 * Pc * sm;
                        double v[6];
                        #pragma unroll
                        for (int j = 0; j < 6; ++j) v[j] = sp[j] * U + dw[j] * V;
                        grad_add6(gbase, col, v, uniform, lane, active);
                        ++col;
                    }
                    l0 = l + par;
                    if (l0 > c.lmax) break;
                }
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Fused adjoint of one Multipole leaf: position VJP and coefficient gradient in
// one walk over the harmonics (regular column structures).
// ---------------------------------------------------------------------------

// add six per-lane gradient values of one column into gk[col][0..5]; when the
// warp is uniform and sk (the warp's shared-memory accumulator for this
// interval) is given, the reduced values go there instead of to global memory
template <typename T>
__device__ __forceinline__ void grad_emit6(double* __restrict__ gk, double* sk, int col,
                                           const T v6[6], bool uniform, int lane, bool active)
{
    if (uniform) {
        const T v[8] = {active ? v6[0] : T(0), active ? v6[1] : T(0), active ? v6[2] : T(0),
                        active ? v6[3] : T(0), active ? v6[4] : T(0), active ? v6[5] : T(0),
                        T(0), T(0)};
        const T z = warp_rs8<T>(v, lane);
        const int idx = ((lane >> 4) & 1) * 4 + ((lane >> 3) & 1) * 2 + ((lane >> 2) & 1);
        if ((lane & 3) == 0 && idx < 6) {
            if (sk) sk[col * 6 + idx] += (double)z;
            else if (gk) atomicAdd(gk + (long long)col * 6 + idx, (double)z);
        }
    } else if (active && gk) {
        #pragma unroll
        for (int j = 0; j < 6; ++j) atomicAdd(gk + (long long)col * 6 + j, (double)v6[j]);
    }
}

struct MPAdjArgs {
    long long n;
    const double* xyz;        // sorted copy when perm != null
    const int* perm;
    const double* gphi;       // [N] or null
    const double* gforce;     // [N,3] or null
    double* gx;               // [N,3], accumulated (+=)
    double* grad;             // [n_int][n_lm][6], accumulated
    long long chunk;          // points per warp (multiple of 32)
    int warp_smem;            // bytes of dynamic shared memory per warp
    int staged;               // 1: interval sums staged in shared memory
    double* force;            // [N,3] or null: this leaf's force added (+=)
    double* stage;            // binned calls: per sorted position the 3 (6 with force)
                              // values to add, gathered back by adj_unpermute_add
    int stage_rec;            // 3, or 6 with the force
    double* gconst;           // [AGB_MP_NCONST] or null, accumulated
    double gforce_scale;      // the force cotangent is gforce_scale * gforce
    DevComp c;
    DevLeaf leaf;
};

// Coefficient gradient of one interval k for a warp whose 32 points all lie
// in k: dL/da_{c,j} = sum_p (s_p^j U_c(p) + j s_p^(j-1) V_c(p)).  Instead of
// reducing 6 values across the warp for every column, the walk writes each
// point's (U, V) of the column into a shared tile [point][column], and every
// 32 columns the lanes switch roles: lane q takes column q of the tile and
// contracts it with the points' powers of s (broadcast reads), 10 FMAs per
// point, then adds its 6 sums to the interval's accumulator.
template <typename R> struct AdjVec;
template <> struct AdjVec<float> {
    typedef float2 T2;
    // a point's 9 weights (s..s^5, 2s, 3s^2, 4s^3, 5s^4) from its 16-byte aligned row
    static __device__ __forceinline__ void weights(const float* w, float o[9])
    {
        const float4 a = *reinterpret_cast<const float4*>(w);
        const float4 b = *reinterpret_cast<const float4*>(w + 4);
        o[0] = a.x; o[1] = a.y; o[2] = a.z; o[3] = a.w;
        o[4] = b.x; o[5] = b.y; o[6] = b.z; o[7] = b.w; o[8] = w[8];
    }
};
template <> struct AdjVec<double> {
    typedef double2 T2;
    static __device__ __forceinline__ void weights(const double* w, double o[9])
    {
        #pragma unroll
        for (int j = 0; j < 4; ++j) {
            const double2 v = *reinterpret_cast<const double2*>(w + 2 * j);
            o[2 * j] = v.x; o[2 * j + 1] = v.y;
        }
        o[8] = w[8];
    }
};

#define AGB_ADJ_TILE_STRIDE 33          // tile row length (columns + 1: no bank conflicts)
#define AGB_ADJ_SPW 12                  // per-point powers: s..s^5, 2s, 3s^2, 4s^3, 5s^4, pad

template <typename R>
__host__ __device__ constexpr int adj_tile_bytes()
{
    return (32 * AGB_ADJ_TILE_STRIDE * 2 + 32 * AGB_ADJ_SPW) * (int)sizeof(R);
}

template <typename R>
struct AdjTile {
    typename AdjVec<R>::T2* uv;   // [32 points][AGB_ADJ_TILE_STRIDE]
    R* spw;                       // [32 points][AGB_ADJ_SPW]
    double* acc;                  // interval accumulator [n_lm][6]: shared (staged) or global
    int nb, col0;
    bool on;                      // warp-uniform: this warp's points share one interval
    bool shared_acc;
};

template <typename R>
__device__ __forceinline__ void adj_contract(AdjTile<R>& T, int lane)
{
    __syncwarp();
    if (lane < T.nb) {
        R g0 = R(0), g1 = R(0), g2 = R(0), g3 = R(0), g4 = R(0), g5 = R(0);
        #pragma unroll 4
        for (int p = 0; p < 32; ++p) {
            const typename AdjVec<R>::T2 uv = T.uv[p * AGB_ADJ_TILE_STRIDE + lane];
            R w[9];
            AdjVec<R>::weights(T.spw + p * AGB_ADJ_SPW, w);
            g0 += uv.x;
            g1 = fma(w[0], uv.x, g1 + uv.y);
            g2 = fma(w[1], uv.x, fma(w[5], uv.y, g2));
            g3 = fma(w[2], uv.x, fma(w[6], uv.y, g3));
            g4 = fma(w[3], uv.x, fma(w[7], uv.y, g4));
            g5 = fma(w[4], uv.x, fma(w[8], uv.y, g5));
        }
        double* d = T.acc + (long long)(T.col0 + lane) * 6;
        if (T.shared_acc) {
            d[0] += (double)g0; d[1] += (double)g1; d[2] += (double)g2;
            d[3] += (double)g3; d[4] += (double)g4; d[5] += (double)g5;
        } else {
            atomicAdd(d, (double)g0); atomicAdd(d + 1, (double)g1); atomicAdd(d + 2, (double)g2);
            atomicAdd(d + 3, (double)g3); atomicAdd(d + 4, (double)g4); atomicAdd(d + 5, (double)g5);
        }
    }
    __syncwarp();
    T.col0 += T.nb;
    T.nb = 0;
}

// one column's (U, V) of this lane's point.  EMIT: 0 decides per column (tile
// when the warp shares one interval, else atomics), 1 writes the tile without a
// flush check (the caller flushes per |m| group), 2 always uses atomics.
template <typename R, int EMIT = 0>
__device__ __forceinline__ void adj_put(AdjTile<R>& T, double* __restrict__ gk, int col,
                                        const R sp[6], const R dw[6], R U, R V, int lane,
                                        bool active)
{
    if (EMIT == 1) {
        typename AdjVec<R>::T2 uv;
        uv.x = U;
        uv.y = V;
        T.uv[lane * AGB_ADJ_TILE_STRIDE + T.nb] = uv;
        ++T.nb;
        return;
    }
    if (EMIT == 2) {
        if (active && gk) {
            #pragma unroll
            for (int j = 0; j < 6; ++j) atomicAdd(gk + (long long)col * 6 + j, (double)fma(sp[j], U, dw[j] * V));
        }
        return;
    }
    if (T.on) {
        typename AdjVec<R>::T2 uv;
        uv.x = U;
        uv.y = V;
        T.uv[lane * AGB_ADJ_TILE_STRIDE + T.nb] = uv;
        if (++T.nb == 32) adj_contract(T, lane);
    } else if (active && gk) {
        #pragma unroll
        for (int j = 0; j < 6; ++j) atomicAdd(gk + (long long)col * 6 + j, (double)fma(sp[j], U, dw[j] * V));
    }
}

template <typename R, int PAR, int EMIT>
__device__ __forceinline__ void mp_adj_walk(const DevComp& c, int kw, R s, double cth_d,
                                            double sth_d, double cph, double sph, R P1, R P2,
                                            R P3, R P4, double* gbase, AdjTile<R>& T, int lane,
                                            bool active, MPSums& tot)
{
    constexpr int MODE = AGB_MODE_HESS;
    const bool near_pole = sth_d < 1.0e-10;
    R sp[6], dw[6], ew[6];
    sp[0] = R(1); sp[1] = s; sp[2] = s * s; sp[3] = sp[2] * s; sp[4] = sp[2] * sp[2]; sp[5] = sp[4] * s;
    dw[0] = R(0); dw[1] = R(1); dw[2] = R(2) * s; dw[3] = R(3) * sp[2]; dw[4] = R(4) * sp[3]; dw[5] = R(5) * sp[4];
    ew[0] = R(0); ew[1] = R(0); ew[2] = R(2); ew[3] = R(6) * s; ew[4] = R(12) * sp[2]; ew[5] = R(20) * sp[3];
    const R cth = (R)cth_d, sth = (R)sth_d;
    const R c2 = (R)(cth_d * cth_d), w2 = (R)(-2.0 * cth_d * sth_d);   // two-step walk
    const R inv_sth = near_pole ? R(0) : (R)(1.0 / sth_d);
    const R cot = near_pole ? R(0) : (R)(cth_d / sth_d);
    const R np1 = near_pole ? R(0) : R(1);
    const R* rec = MPPtr<R>::base(c, kw) + MPPtr<R>::REC;
    double cm = 1.0, sm = 0.0, sinpow = 1.0, sinpow_m1 = 0.0;
    int col = 1;
    for (int m = 0; m <= c.lmax; ++m) {
        if (m > 0) {
            const double t = cm * cph - sm * sph;
            sm = sm * cph + cm * sph;
            cm = t;
            sinpow_m1 = sinpow;
            sinpow *= sth_d;
        }
        int l0 = (PAR == 2) ? (m + (m & 1)) : m;
        if (m == 0) l0 = PAR;
        if (l0 > c.lmax) continue;
        if (EMIT == 1) {
            // even l, lmax <= 32: a group holds at most 32 columns; flush before it
            // when it would not fit, so the loop below never branches to flush
            const int ncols = (m == 0 ? 1 : 2) * ((c.lmax - l0) / PAR + 1);
            if (T.nb + ncols > 32) adj_contract(T, lane);
        }
        const R q1 = (near_pole && m == 1) ? R(1) : R(0);
        const R m2 = R(m * m) * inv_sth * inv_sth;
        const R Tc = (R)cm, Ts = (R)sm, dTc = -R(m) * Ts, dTs = R(m) * Tc;
        R Pc = (R)(AGB_SEED[m] * sinpow), Pp = R(0), dPp = R(0);
        R dPc = (m == 0) ? R(0) : ((m == 1) ? (R)(AGB_SEED[1] * cth_d)
                : (near_pole ? R(0) : (R)((double)m * AGB_SEED[m] * sinpow_m1 * cth_d)));
        MPCol<R> gc, gs;
        gc.zero();
        gs.zero();
        const int tb = m * AGB_LEG_N;
        // the rescaled recurrence of the regular tables (multipole.cuh); the emitted
        // gradients are then w.r.t. the rescaled coefficients (the host multiplies
        // each column by its scale)
        auto step = [&](int L) {
            const R nb = MPConst<R>::nbetaq(tb + L);
            const R Pn = fma(cth, Pc, nb * Pp);
            const R dPn = fma(cth, dPc, fma(-sth, Pc, nb * dPp));
            dPp = dPc; dPc = dPn; Pp = Pc; Pc = Pn;
        };
        auto acc = [&](int L) {
            const R ll1 = R(L * (L + 1));
            const R Pos = fma(Pc, inv_sth, q1 * dPc);
            const R base = fma(P3, dPc, P1 * Pc);
            const R Pq = P4 * Pos;
            // FP32 m>0 records are interleaved (cos, sin): both come in one load;
            // FP64 loads the sin record only when it is needed (register pressure)
            constexpr bool F32 = std::is_same<R, float>::value;
            R a[6], b[6];
            if (F32 && m > 0) MPPtr<R>::load_cs(rec, a, b);
            else MPPtr<R>::load(rec, a);
            mp_col_acc<MODE, R>(gc, a, sp, dw, ew, Pc, dPc, ll1);
            adj_put<R, EMIT>(T, gbase, col++, sp, dw, fma(Tc, base, dTc * Pq), P2 * Pc * Tc, lane,
                             active);
            if (m > 0) {
                if (!F32) MPPtr<R>::load(rec + MPPtr<R>::REC, b);
                mp_col_acc<MODE, R>(gs, b, sp, dw, ew, Pc, dPc, ll1);
                adj_put<R, EMIT>(T, gbase, col++, sp, dw, fma(Ts, base, dTs * Pq), P2 * Pc * Ts, lane,
                           active);
            }
            rec += (m > 0 ? 2 : 1) * MPPtr<R>::REC;
        };
        const R seed = Pc;
        int l = m;
        while (l < l0) step(++l);
        acc(l);
        if (PAR == 2) {
            // even l: Q_l = (cos^2 + A_l) Q_{l-2} + B_l Q_{l-4} (multipole.cuh)
            const int ts = m * AGB_SKIP_N;
            Pp = (m == 0) ? seed : R(0);
            dPp = R(0);
            #pragma unroll 4
            for (l = l0 + 2; l <= c.lmax; l += 2) {
                const auto ab = MPConst<R>::skip(ts + (l >> 1));
                const R t = c2 + (R)ab.x;
                const R Pn = fma(t, Pc, (R)ab.y * Pp);
                const R dPn = fma(w2, Pc, fma(t, dPc, (R)ab.y * dPp));
                dPp = dPc; dPc = dPn; Pp = Pc; Pc = Pn;
                acc(l);
            }
        } else {
            for (l = l0 + 1; l <= c.lmax; ++l) {
                step(l);
                acc(l);
            }
        }
        mp_col_finish<MODE, R>(gc, inv_sth, q1, np1, cot, m2);
        mp_col_finish<MODE, R>(gs, inv_sth, q1, np1, cot, m2);
        const double md = (double)m;
        const double ddTc = -md * sm, ddTs = md * cm;
        tot.A += (double)gc.V * cm + (double)gs.V * sm;
        tot.B += (double)gc.VR * cm + (double)gs.VR * sm;
        tot.D += (double)gc.VRR * cm + (double)gs.VRR * sm;
        tot.Th += (double)gc.VT * cm + (double)gs.VT * sm;
        tot.Pos += (double)gc.VP * ddTc + (double)gs.VP * ddTs;
        tot.Thth += (double)gc.VTT * cm + (double)gs.VTT * sm;
        tot.BTh += (double)gc.VRT * cm + (double)gs.VRT * sm;
        tot.Ph += (double)gc.V * ddTc + (double)gs.V * ddTs;
        tot.Phph += -md * md * ((double)gc.V * cm + (double)gs.V * sm);
        tot.BPh += (double)gc.VR * ddTc + (double)gs.VR * ddTs;
        tot.ThPh += (double)gc.VT * ddTc + (double)gs.VT * ddTs;
    }
    if (T.on && T.nb) adj_contract(T, lane);
}

// Each warp owns `chunk` consecutive (interval-sorted) points and a slice of
// dynamic shared memory: the (U, V) tile and powers of s above, and when
// `staged`, an accumulator of n_lm x 6 doubles for the interval its points are
// in, flushed to global memory (one atomic per value) only when the interval
// changes and at the end.  Without `staged` the tile contractions add to
// global memory directly.  Warps whose points straddle intervals add each
// lane's six values with atomics.
template <typename R>
__global__ void __launch_bounds__(64, 4)
mp_adjoint_kernel(const __grid_constant__ MPAdjArgs a)
{
    extern __shared__ __align__(16) unsigned char agb_adj_smem[];
    const DevComp& c = a.c;
    const int lane = threadIdx.x & 31;
    const long long gwarp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nval = c.n_lm * 6;
    unsigned char* wbase = agb_adj_smem + (size_t)(threadIdx.x >> 5) * a.warp_smem;
    AdjTile<R> T;
    T.uv = reinterpret_cast<typename AdjVec<R>::T2*>(wbase);
    T.spw = reinterpret_cast<R*>(wbase + 32 * AGB_ADJ_TILE_STRIDE * sizeof(typename AdjVec<R>::T2));
    double* swarp = a.staged ? reinterpret_cast<double*>(wbase + adj_tile_bytes<R>()) : nullptr;
    const long long lo = gwarp * a.chunk;
    const long long hi = lo + a.chunk < a.n ? lo + a.chunk : a.n;
    if (swarp)
        for (int q = lane; q < nval; q += 32) swarp[q] = 0.0;
    // this warp's sums of the builder-scalar gradients (the last 64 bytes of its slice)
    double* wc = a.gconst ? reinterpret_cast<double*>(wbase + a.warp_smem - 64) : nullptr;
    if (wc && lane < AGB_MP_NCONST) wc[lane] = 0.0;
    __syncwarp();
    int cur_k = -1;                      // interval held in swarp
    auto flush = [&]() {
        __syncwarp();
        if (cur_k >= 0) {
            double* g = a.grad + (long long)cur_k * nval;
            for (int q = lane; q < nval; q += 32) {
                const double v = swarp[q];
                if (v != 0.0) atomicAdd(g + q, v);
                swarp[q] = 0.0;
            }
        }
        cur_k = -1;
        __syncwarp();
    };
    const double logr_min = c.p[0], dlogr = c.p[1], inv_dlogr = c.p[2], invPhi0 = c.p[3];
    const double MP0 = AGB_MUL0 * AGB_PREFACT[0];
    const double A = a.leaf.ampl, sg = a.leaf.sigma;
    for (long long base = lo; base < hi; base += 32) {
        const long long pos = base + lane;
        const bool valid = pos < hi;
        long long i = pos;
        double px = 0.0, py = 0.0, pz = 1.0, gp = 0.0, gf0 = 0.0, gf1 = 0.0, gf2 = 0.0;
        if (valid) {
            i = a.perm ? (long long)a.perm[pos] : pos;
            px = sg * a.xyz[3 * pos] - a.leaf.g0;
            py = sg * a.xyz[3 * pos + 1] - a.leaf.g1;
            pz = sg * a.xyz[3 * pos + 2] - a.leaf.g2;
            gp = a.gphi ? a.gphi[i] : 0.0;
            if (a.gforce) {
                const double sc = a.gforce_scale;
                gf0 = sc * a.gforce[3 * i]; gf1 = sc * a.gforce[3 * i + 1]; gf2 = sc * a.gforce[3 * i + 2];
            }
        }
        const double r2 = px * px + py * py + pz * pz;
        const double r = sqrt(r2);
        const double Rc = sqrt(px * px + py * py);
        int k = -1;
        double s = 0.0;
        if (valid && r >= 1.0e-300) {
            const double logr = log(r);
            if (logr >= logr_min) {
                int kk = (int)((logr - logr_min) * inv_dlogr);
                if (kk < 0) kk = 0;
                if (kk < c.n_int) {
                    k = kk;
                    s = fmin(fmax((logr - (logr_min + kk * dlogr)) * inv_dlogr, 0.0), 1.0);
                }
            }
        }
        const bool inside = k >= 0;
        const int kw = inside ? k : 0;
        const double inv_r = inside ? 1.0 / r : 0.0;
        const double cth = inside ? pz * inv_r : 1.0;
        const double sth = inside ? Rc * inv_r : 0.0;
        const double cph = (Rc > 1.0e-300) ? px / Rc : 1.0;
        const double sph = (Rc > 1.0e-300) ? py / Rc : 0.0;
        // monopole and log-scaling factor
        double c0, c0s, c0ss;
        mp_quintic0(c, kw, s, c0, c0s, c0ss);
        const double dc0 = c0s * inv_dlogr, d2c0 = c0ss * inv_dlogr * inv_dlogr;
        double F = 1.0, dF = 0.0, d2F = 0.0, F1 = 0.0, ex = 0.0, mono, dmono, d2mono;
        if (c.log_scaling) {
            ex = exp(c0);
            F = 1.0 / (invPhi0 - ex);
            F1 = F * F * ex;
            dF = F1 * dc0;
            d2F = F1 * (d2c0 + dc0 * dc0 * F * (invPhi0 + ex));
            mono = MP0 * F; dmono = MP0 * dF; d2mono = MP0 * d2F;
        } else {
            mono = MP0 * c0; dmono = MP0 * dc0; d2mono = MP0 * d2c0;
        }
        // weights of the coefficient gradient
        const double w0 = -A * sg * gf0, w1 = -A * sg * gf1, w2 = -A * sg * gf2;
        const double inv_r2 = inv_r * inv_r;
        const double alpha = inside ? gp * A : 0.0;
        const double br = inside ? (w0 * px + w1 * py + w2 * pz) * inv_r2 : 0.0;
        const double bt = inside ? (w0 * cth * cph + w1 * cth * sph - w2 * sth) * inv_r : 0.0;
        const double bp = inside ? (-w0 * sph + w1 * cph) * inv_r : 0.0;
        const R P1 = (R)(alpha * F + br * dF), P2 = (R)(br * F * inv_dlogr);
        const R P3 = (R)(bt * F), P4 = (R)(bp * F);
        const int kmax = __reduce_max_sync(0xffffffffu, k);
        const bool uniform = __all_sync(0xffffffffu, k == kmax || k < 0);
        const int kk = uniform ? kmax : k;
        double* gbase = (kk >= 0) ? a.grad + (long long)kk * c.n_lm * 6 : nullptr;
        double* sk = nullptr;
        T.on = uniform && kk >= 0;
        T.nb = 0;
        T.col0 = 1;
        T.shared_acc = false;
        T.acc = gbase;
        if (T.on) {
            if (swarp) {
                if (kk != cur_k) {
                    flush();
                    cur_k = kk;
                }
                sk = swarp;
                T.acc = swarp;
                T.shared_acc = true;
            }
            // this lane's powers of s (zeros for points outside the grid)
            const R sr = inside ? (R)s : R(0);
            const R s2 = sr * sr, s3 = s2 * sr, s4 = s2 * s2;
            R* w = T.spw + lane * AGB_ADJ_SPW;
            w[0] = sr; w[1] = s2; w[2] = s3; w[3] = s4; w[4] = s4 * sr;
            w[5] = R(2) * sr; w[6] = R(3) * s2; w[7] = R(4) * s3; w[8] = R(5) * s4;
        }
        MPSums tw = {};
        // warp-uniform choice: tile emission (all 32 points in one interval) or atomics
        if (c.structure == AGB_STRUCT_EVEN) {
            if (T.on)
                mp_adj_walk<R, 2, 1>(c, kw, (R)s, cth, sth, cph, sph, P1, P2, P3, P4, gbase, T, lane, inside, tw);
            else
                mp_adj_walk<R, 2, 2>(c, kw, (R)s, cth, sth, cph, sph, P1, P2, P3, P4, gbase, T, lane, inside, tw);
        } else {
            if (T.on)
                mp_adj_walk<R, 1, 0>(c, kw, (R)s, cth, sth, cph, sph, P1, P2, P3, P4, gbase, T, lane, inside, tw);
            else
                mp_adj_walk<R, 1, 2>(c, kw, (R)s, cth, sth, cph, sph, P1, P2, P3, P4, gbase, T, lane, inside, tw);
        }
        const MPSums t = tw;
        // monopole column of the coefficient gradient
        {
            const double Bp = t.B * inv_dlogr;
            double v[6];
            const double sp[6] = {1.0, s, s * s, s * s * s, s * s * s * s, s * s * s * s * s};
            const double dw[6] = {0.0, 1.0, 2.0 * s, 3.0 * s * s, 4.0 * s * s * s, 5.0 * s * s * s * s};
            if (c.log_scaling) {
                const double QF = alpha * (MP0 + t.A) + br * Bp + bt * t.Th + bp * t.Pos;
                const double QdF = br * (MP0 + t.A);
                const double dFdc0 = F1 * (1.0 + 2.0 * F * ex) * dc0;
                #pragma unroll
                for (int j = 0; j < 6; ++j)
                    v[j] = QF * F1 * sp[j] + QdF * (dFdc0 * sp[j] + F1 * inv_dlogr * dw[j]);
            } else {
                #pragma unroll
                for (int j = 0; j < 6; ++j) v[j] = alpha * MP0 * sp[j] + br * MP0 * inv_dlogr * dw[j];
            }
            grad_emit6<double>(gbase, sk, 0, v, uniform, lane, inside);
            if (wc) {                   // the builder's scalars (warp-uniform branch)
                double gi = 0.0;
                if (inside && c.log_scaling) {
                    const double QF = alpha * (MP0 + t.A) + br * Bp + bt * t.Th + bp * t.Pos;
                    const double QdF = br * (MP0 + t.A);
                    gi = -F * F * QF - 2.0 * F * dF * QdF;
                }
                gi = warp_sum(gi);
                if (lane == 0) wc[0] += gi;
                if (valid && !inside) {     // beyond the grid: few points, shared atomics
                    double cv[AGB_MP_NCONST] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
                    const double brx = (w0 * px + w1 * py + w2 * pz) / r2;
                    mp_const_extrap(c, r, gp * A, r2 > 0.0 ? brx : 0.0, cv);
                    #pragma unroll
                    for (int q = 1; q < 7; ++q)
                        if (cv[q] != 0.0) atomicAdd(wc + q, cv[q]);
                }
            }
        }
        if (!valid) continue;
        // position VJP of this leaf: A sigma (gPhi grad - sigma H gF)
        PointOut o;
        o.phi = 0.0; o.rho = 0.0;
        o.g[0] = o.g[1] = o.g[2] = 0.0;
        #pragma unroll
        for (int q = 0; q < 6; ++q) o.h[q] = 0.0;
        if (inside)
            mp_finish<AGB_MODE_HESS>(t, inv_dlogr, F, dF, d2F, mono, dmono, d2mono, px, py, pz,
                                     inv_r, Rc, cth, sth, cph, sph, o);
        else
            multipole_point<AGB_MODE_HESS, R>(c, px, py, pz, o);
        const double As = A * sg, s2 = sg;
        const double* h = o.h;
        const double v0 = As * (gp * o.g[0] - s2 * (h[0] * gf0 + h[3] * gf1 + h[5] * gf2));
        const double v1 = As * (gp * o.g[1] - s2 * (h[3] * gf0 + h[1] * gf1 + h[4] * gf2));
        const double v2 = As * (gp * o.g[2] - s2 * (h[5] * gf0 + h[4] * gf1 + h[2] * gf2));
        if (a.stage) {
            // sorted order: consecutive lanes write consecutive records
            double* r = a.stage + a.stage_rec * pos;
            r[0] = v0; r[1] = v1; r[2] = v2;
            if (a.stage_rec == 6) { r[3] = -As * o.g[0]; r[4] = -As * o.g[1]; r[5] = -As * o.g[2]; }
            continue;
        }
        a.gx[3 * i] += v0;
        a.gx[3 * i + 1] += v1;
        a.gx[3 * i + 2] += v2;
        if (a.force) {
            a.force[3 * i] -= As * o.g[0];
            a.force[3 * i + 1] -= As * o.g[1];
            a.force[3 * i + 2] -= As * o.g[2];
        }
    }
    if (swarp) flush();
    if (wc) {
        __syncwarp();
        if (lane < AGB_MP_NCONST && wc[lane] != 0.0) atomicAdd(a.gconst + lane, wc[lane]);
    }
}

// the staged records of a binned adjoint added back in input order: point i's
// record sits at its sorted position dest[i] (coalesced writes, one gather read)
template <int REC>
__global__ void __launch_bounds__(256)
adj_unpermute_add(const int* __restrict__ dest, const double* __restrict__ stage, long long n,
                  double* __restrict__ gx, double* __restrict__ force)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const double* t = stage + (long long)REC * __ldg(dest + i);
        gx[3 * i] += t[0]; gx[3 * i + 1] += t[1]; gx[3 * i + 2] += t[2];
        if (REC == 6) { force[3 * i] += t[3]; force[3 * i + 1] += t[4]; force[3 * i + 2] += t[5]; }
    }
}
