// mp_grad.cuh -- gradient of a loss with respect to a Multipole's quintic
// coefficients (the table-gradient half of the backward pass).
//
// For one Multipole leaf (component frame x' = sigma x - gamma, output factor
// A), with cotangents gPhi = dL/dPhi and gF = dL/dF of the composite's
// outputs, the loss depends on the leaf's Phi(x') and grad Phi(x') through
//   alpha = gPhi A,   w = -A sigma gF,   beta_r,theta,phi = w . (u_r, u_theta, u_phi)
// where grad Phi = Phi_r u_r + Phi_theta u_theta + Phi_os u_phi.  Inside the
// radial grid (extrapolated points depend only on the extrapolation
// constants, which are held fixed) and with the log-scaling factor F(log r):
//   dL/da_{c,j} = s^j U_c + j s^(j-1) V_c                               (c >= 1)
//   U_c = (alpha F + beta_r dF) W_c + beta_theta F dW_c + beta_phi F Q_c
//   V_c = beta_r F inv_dlogr W_c
// with W = Y T, dW = dY/dtheta T, Q = (Y/sin theta) dT/dphi, and for the
// monopole column through F and dF (chain rule written out in the kernel).
// Each warp reduces its lanes' six values per harmonic with shuffles when all
// of its points share one interval (the points are binned by interval), else
// every lane adds its own; FP64 atomics accumulate into grad[k][c][j].
#pragma once
#include "multipole.cuh"

__device__ __forceinline__ double warp_sum(double v)
{
    #pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
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
