// cylspline.cuh -- per-point evaluation of an Agama CylSpline expansion.
//
// Follows the reference (_cylspl_potential_kernel.cu):
//   * asinh-scaled coordinates lR = asinh(R/Rscale), lz = asinh(z/Rscale) and
//     their Jacobians (:426-440);
//   * points outside the (lR, lz) grid go to the lmax=8 PowerLaw multipole
//     asymptote whose gradient omits the theta term and whose Hessian is
//     monopole-only (:181-383, :445-458);
//   * cell search (:73-96, :463-469), per-harmonic bicubic Hermite evaluation
//     with the corner offset for round-off (:524-591), first in z for the four
//     R-node functions, then in R (:147-169, :110-128);
//   * Fourier sum with log-scaling of m=0 (log(-Phi0)) and Phi_m/Phi0 ratios
//     (:592-700), un-scaling (:706-750), cylindrical -> Cartesian gradient and
//     Hessian with the R=0 rules (:764-862).
// Node tables come in two layouts: the reference's [harm][iR][iz][4]
// (kernel-signature entries) and a cell-major one where the 16 values a
// harmonic needs in one cell are contiguous (the fused path).
#pragma once
#include <type_traits>
#include "agb_dev.cuh"

__device__ __forceinline__ int cs_cell(double x, const double* __restrict__ g, int n)
{
    // index i with g[i] <= x < g[i+1], clamped to [0, n-2]
    int lo = 0, hi = n - 1;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(g + mid) > x) hi = mid; else lo = mid;
    }
    return lo;
}

// Cubic Hermite on [xl, xh] from end values and end slopes (Agama's form).
template <typename T>
__device__ __forceinline__ void cs_hermite(T t, T Tm, T tT, T h, T fl, T fh, T f1l, T f1h,
                                           T* f, T* df, T* d2f)
{
    const T dif = fh - fl;
    const T Q = T(3) * (f1l + f1h) - T(6) * dif / h;
    if (f) *f = fl * Tm + fh * t + (dif * (t - Tm) + (f1l * Tm - f1h * t) * h) * tT;
    if (df) *df = f1l * Tm + f1h * t - Q * tT;
    if (d2f) *d2f = (f1h - f1l + Q * (t - Tm)) / h;
}

// One harmonic's bicubic Hermite in a cell: value and lR/lz derivatives from the
// 16 node values v (layout of cs_load), first along z, then along R.
template <typename T, bool DO_G, bool DO_H>
__device__ __forceinline__ void cs_bicubic(const T v[16], T tR, T TR, T tTR, T hR, T tz, T Tz,
                                           T tTz, T hz, T& val, T& vR, T& vRR, T& vz, T& vRz,
                                           T& vzz)
{
    T F[4], dF[4], d2F[4];
    const int lo_i[4] = {0, 2, 4, 6}, hi_i[4] = {1, 3, 5, 7};
    #pragma unroll
    for (int q = 0; q < 4; ++q)
        cs_hermite<T>(tz, Tz, tTz, hz, v[lo_i[q]], v[hi_i[q]], v[8 + lo_i[q]], v[8 + hi_i[q]],
                      &F[q], DO_G ? &dF[q] : nullptr, DO_H ? &d2F[q] : nullptr);
    cs_hermite<T>(tR, TR, tTR, hR, F[0], F[1], F[2], F[3], &val, DO_G ? &vR : nullptr,
                  DO_H ? &vRR : nullptr);
    if (DO_G)
        cs_hermite<T>(tR, TR, tTR, hR, dF[0], dF[1], dF[2], dF[3], &vz, DO_H ? &vRz : nullptr, nullptr);
    if (DO_H)
        cs_hermite<T>(tR, TR, tTR, hR, d2F[0], d2F[1], d2F[2], d2F[3], &vzz, nullptr, nullptr);
}

// Outer PowerLaw multipole (W_outer, r0) evaluated with the reference's
// simplifications (no theta term in the gradient, monopole-only Hessian) and
// its angular basis (see legendre.outer_asymptote_basis on the host side).
template <int MODE>
__device__ void cs_outer(const DevComp& c, double x, double y, double z, PointOut& o)
{
    const double* __restrict__ W = c.extra;
    const double r0 = c.p[1];
    const int lmax = c.lmax;
    const int mmax = (int)c.p[2];
    const double R2 = x * x + y * y;
    const double R = sqrt(R2);
    const double r = sqrt(R2 + z * z);
    const double rinv = 1.0 / r;
    const double ct = z * rinv, st = R * rinv;
    const double cph = (R > 0.0) ? x / R : 1.0;
    const double sph = (R > 0.0) ? y / R : 0.0;
    const double rr = r0 * rinv;

    double phi = 0.0, dr = 0.0, dphi = 0.0;
    double cm = 1.0, sm = 0.0, sinpow = 1.0;
    for (int m = 0; m <= mmax; ++m) {
        const double MUL = (m == 0) ? AGB_MUL0 : AGB_MUL1;
        // the reference's basis: true P_m^m and P_{m+1}^m, then a three-term
        // recurrence whose oldest slot lags one order (0 at l = m+2)
        const double Ymm = AGB_COEF[m] * sinpow;
        double p2 = 0.0, p1 = Ymm / AGB_PREFACT[m], p = ct * (double)(2 * m + 1) * p1;
        double pw = rr;                               // (r0/r)^(m+1)
        for (int q = 0; q < m; ++q) pw *= rr;
        for (int l = m; l <= lmax; ++l) {
            double Pl;
            if (l == m) {
                Pl = Ymm;
            } else if (l == m + 1) {
                Pl = p * AGB_NORM[m * AGB_LEG_N + l];
                pw *= rr;
            } else {
                const double nw = (ct * (double)(2 * l - 1) * p - (double)(l + m - 1) * p2) / (double)(l - m);
                p2 = p1; p1 = p; p = nw;
                Pl = nw * AGB_NORM[m * AGB_LEG_N + l];
                pw *= rr;
            }
            const double Yb = Pl * MUL;
            if (m == 0) {
                const double w = __ldg(W + l * (l + 1));
                phi += w * pw * Yb;
                dr += w * (double)(-(l + 1)) * rinv * pw * Yb;
            } else {
                const double wc = __ldg(W + l * (l + 1) + m);
                const double ws = __ldg(W + l * (l + 1) - m);
                const double contrib = pw * Yb * (wc * cm + ws * sm);
                phi += contrib;
                dr += (double)(-(l + 1)) * rinv * contrib;
                dphi += pw * Yb * (wc * (-(double)m * sm) + ws * ((double)m * cm));
            }
        }
        const double t = cm * cph - sm * sph;
        sm = sm * cph + cm * sph;
        cm = t;
        sinpow *= st;
    }
    o.phi = phi;
    if (MODE == AGB_MODE_GRAD || MODE == AGB_MODE_HESS) {
        const double dphx = (R > 1e-30) ? -y / R2 : 0.0;
        const double dphy = (R > 1e-30) ? x / R2 : 0.0;
        o.g[0] = dr * (x * rinv) + dphi * dphx;
        o.g[1] = dr * (y * rinv) + dphi * dphy;
        o.g[2] = dr * (z * rinv);
    }
    if (MODE == AGB_MODE_HESS || MODE == AGB_MODE_DENS) {
        const double W0 = __ldg(W) * AGB_MUL0;
        const double p0 = W0 * rr;
        const double Pr = -p0 * rinv;
        const double Prr = 2.0 * p0 * rinv * rinv;
        const double C1 = (Prr - Pr * rinv) / (r * r);
        const double C2 = Pr * rinv;
        hess_radial(C1, C2, x, y, z, o.h);
    }
}

// Load the 16 node values of harmonic h in cell (iR, iz):
// v[0..3] fval at (lo,lo) (lo,hi) (hi,lo) (hi,hi) [R first, z second],
// v[4..7] fx, v[8..11] fy, v[12..15] fxy.
__device__ __forceinline__ void cs_load(const DevComp& c, int h, int iR, int iz, double v[16])
{
    const int nR = c.n_int, nz = c.nz;
    if (c.layout == 1) {
        const double2* p = reinterpret_cast<const double2*>(
            c.table + (((long long)iR * (nz - 1) + iz) * c.n_lm + h) * 16);
        #pragma unroll
        for (int q = 0; q < 8; ++q) {
            const double2 w = __ldg(p + q);
            v[2 * q] = w.x; v[2 * q + 1] = w.y;
        }
    } else {
        const long long base = (long long)h * nR * nz;
        const long long idx[4] = {base + (long long)iR * nz + iz, base + (long long)iR * nz + iz + 1,
                                  base + (long long)(iR + 1) * nz + iz,
                                  base + (long long)(iR + 1) * nz + iz + 1};
        #pragma unroll
        for (int q = 0; q < 4; ++q) {
            const double2* p = reinterpret_cast<const double2*>(c.table + idx[q] * 4);
            const double2 a = __ldg(p), b = __ldg(p + 1);
            v[q] = a.x; v[4 + q] = a.y; v[8 + q] = b.x; v[12 + q] = b.y;
        }
    }
}

// EXACT: add the dPhi/dphi * d2(phi)/dx_i dx_j terms of the Cartesian Hessian,
// which the reference's conversion omits (_cylspl_potential_kernel.cu:836-852);
// used for derivatives (the VJP), not for forceDeriv, which keeps the
// reference's values.
// Mixed precision: the FP32 record (see prep_cylspline.cell_major_f32) holds the
// corner value f00 in FP64 and the rest relative to it in FP32; the Hermite runs
// in FP32 and f00 is added back in FP64.
__device__ __forceinline__ double cs_load32(const DevComp& c, int h, int iR, int iz, float v[16])
{
    const float4* p = reinterpret_cast<const float4*>(
        c.table32 + (((long long)iR * (c.nz - 1) + iz) * c.n_lm + h) * 20);
    const float4 q0 = __ldg(p), q1 = __ldg(p + 1), q2 = __ldg(p + 2), q3 = __ldg(p + 3),
                 q4 = __ldg(p + 4);
    v[0] = 0.0f; v[1] = q0.z; v[2] = q0.w; v[3] = q1.x;
    v[4] = q1.y; v[5] = q1.z; v[6] = q1.w; v[7] = q2.x;
    v[8] = q2.y; v[9] = q2.z; v[10] = q2.w; v[11] = q3.x;
    v[12] = q3.y; v[13] = q3.z; v[14] = q3.w; v[15] = q4.x;
    return __hiloint2double(__float_as_int(q0.y), __float_as_int(q0.x));
}

template <int MODE, bool EXACT = false, typename RT = double>
__device__ __forceinline__ void cylspline_point(const DevComp& c, double px, double py,
                                                double pz, PointOut& o)
{
    constexpr bool F32 = std::is_same<RT, float>::value;   // mixed precision
    constexpr bool DO_G = MODE != AGB_MODE_POT;
    constexpr bool DO_H = MODE == AGB_MODE_HESS || MODE == AGB_MODE_DENS;
    const double Rs = c.p[0];
    const double* __restrict__ lRg = c.grid_a;
    const double* __restrict__ lzg = c.grid_b;
    const int nR = c.n_int, nz = c.nz;

    const double R2 = px * px + py * py;
    const double R = sqrt(R2);
    const double lR = asinh(R / Rs);
    const double lz = asinh(pz / Rs);
    const double dlRdR = 1.0 / sqrt(R2 + Rs * Rs);
    const double dlzdz = 1.0 / sqrt(pz * pz + Rs * Rs);
    const double d2lRdR2 = -R * dlRdR * dlRdR * dlRdR;
    const double d2lzdz2 = -pz * dlzdz * dlzdz * dlzdz;

    if (lR < __ldg(lRg) || lR > __ldg(lRg + nR - 1) || lz < __ldg(lzg) || lz > __ldg(lzg + nz - 1)) {
        cs_outer<MODE>(c, px, py, pz, o);
        if (MODE == AGB_MODE_DENS) o.rho = -(o.h[0] + o.h[1] + o.h[2]) * AGB_INV_4PIG;
        return;
    }
    int iR = cs_cell(lR, lRg, nR);
    int iz = cs_cell(lz, lzg, nz);
    const double lR_lo = __ldg(lRg + iR), lR_hi = __ldg(lRg + iR + 1);
    const double lz_lo = __ldg(lzg + iz), lz_hi = __ldg(lzg + iz + 1);
    const double hR = lR_hi - lR_lo, hz = lz_hi - lz_lo;
    const double tR = (lR - lR_lo) / hR, TR = 1.0 - tR, tTR = tR * TR;
    const double tz = (lz - lz_lo) / hz, Tz = 1.0 - tz, tTz = tz * Tz;
    const bool R_at_hi = (lR == lR_hi), z_at_hi = (lz == lz_hi);

    const double cph = (R > 0.0) ? px / R : 1.0;
    const double sph = (R > 0.0) ? py / R : 0.0;

    const int ls = c.log_scaling;
    double S = ls ? 1.0 : 0.0, S_R = 0.0, S_z = 0.0, S_RR = 0.0, S_Rz = 0.0, S_zz = 0.0;
    double S_p = 0.0, S_pp = 0.0, S_Rp = 0.0, S_zp = 0.0;
    double f0 = 0.0, f0R = 0.0, f0z = 0.0, f0RR = 0.0, f0Rz = 0.0, f0zz = 0.0;

    int cur = 0;
    double cm = 1.0, sm = 0.0;
    for (int h = 0; h < c.n_lm; ++h) {
        const int m = __ldg(c.lm + h);
        double val, vR = 0.0, vRR = 0.0, vz = 0.0, vRz = 0.0, vzz = 0.0;
        if (F32 && c.table32) {
            float w[16];
            const double f00 = cs_load32(c, h, iR, iz, w);
            float a, aR = 0.0f, aRR = 0.0f, az = 0.0f, aRz = 0.0f, azz = 0.0f;
            cs_bicubic<float, DO_G, DO_H>(w, (float)tR, (float)TR, (float)tTR, (float)hR,
                                          (float)tz, (float)Tz, (float)tTz, (float)hz,
                                          a, aR, aRR, az, aRz, azz);
            val = f00 + (double)a;
            vR = aR; vRR = aRR; vz = az; vRz = aRz; vzz = azz;
        } else {
            double v[16];
            cs_load(c, h, iR, iz, v);
            const double off = R_at_hi ? (z_at_hi ? v[3] : v[2]) : (z_at_hi ? v[1] : v[0]);
            v[0] -= off; v[1] -= off; v[2] -= off; v[3] -= off;
            cs_bicubic<double, DO_G, DO_H>(v, tR, TR, tTR, hR, tz, Tz, tTz, hz, val, vR, vRR, vz,
                                           vRz, vzz);
            val += off;
        }

        double T = 1.0, dT = 0.0, d2T = 0.0;
        if (m != 0) {
            const int am = m < 0 ? -m : m;
            if (am < cur) { cur = 0; cm = 1.0; sm = 0.0; }
            for (; cur < am; ++cur) {
                const double t = cm * cph - sm * sph;
                sm = sm * cph + cm * sph;
                cm = t;
            }
            if (m > 0) { T = cm; dT = -(double)am * sm; d2T = -(double)(am * am) * cm; }
            else       { T = sm; dT = (double)am * cm; d2T = -(double)(am * am) * sm; }
        }
        if (m == 0) {
            f0 = val; f0R = vR; f0z = vz; f0RR = vRR; f0Rz = vRz; f0zz = vzz;
            if (!ls) {
                S += val; S_R += vR; S_z += vz;
                if (DO_H) { S_RR += vRR; S_Rz += vRz; S_zz += vzz; }
            }
        } else {
            S += val * T; S_R += vR * T; S_z += vz * T; S_p += val * dT;
            if (DO_H) {
                S_RR += vRR * T; S_Rz += vRz * T; S_zz += vzz * T;
                S_Rp += vR * dT; S_zp += vz * dT; S_pp += val * d2T;
            }
        }
    }

    double P, PR = 0.0, Pz = 0.0, Pp = S_p, PRR = 0.0, PRz = 0.0, Pzz = 0.0;
    double PRp = 0.0, Pzp = 0.0, Ppp = S_pp;
    if (ls) {
        const double P0 = -exp(f0);
        const double P0R = P0 * f0R, P0z = P0 * f0z;
        P = P0 * S;
        if (DO_G) { PR = P0 * S_R + P0R * S; Pz = P0 * S_z + P0z * S; Pp = P0 * S_p; }
        if (DO_H) {
            const double P0RR = P0 * (f0RR + f0R * f0R);
            const double P0zz = P0 * (f0zz + f0z * f0z);
            const double P0Rz = P0 * (f0Rz + f0R * f0z);
            PRR = P0 * S_RR + 2.0 * P0R * S_R + P0RR * S;
            Pzz = P0 * S_zz + 2.0 * P0z * S_z + P0zz * S;
            PRz = P0 * S_Rz + P0R * S_z + P0z * S_R + P0Rz * S;
            PRp = P0 * S_Rp + P0R * S_p;
            Pzp = P0 * S_zp + P0z * S_p;
            Ppp = P0 * S_pp;
        }
    } else {
        P = S; PR = S_R; Pz = S_z;
        if (DO_H) { PRR = S_RR; Pzz = S_zz; PRz = S_Rz; PRp = S_Rp; Pzp = S_zp; }
    }
    o.phi = P;
    if (!DO_G) return;

    const double dPdR = PR * dlRdR;
    const double dPdz = Pz * dlzdz;
    double gx = 0.0, gy = 0.0;
    if (R > 1e-30) {
        const double Ri = 1.0 / R, R2i = Ri * Ri;
        gx = dPdR * (px * Ri) - Pp * (py * R2i);
        gy = dPdR * (py * Ri) + Pp * (px * R2i);
    }
    o.g[0] = gx; o.g[1] = gy; o.g[2] = dPdz;
    if (!DO_H) return;

    const double H_RR = PRR * (dlRdR * dlRdR) + PR * d2lRdR2;
    const double H_zz = Pzz * (dlzdz * dlzdz) + Pz * d2lzdz2;
    const double H_Rz = PRz * dlRdR * dlzdz;
    const double H_pp = Ppp;
    const double H_Rp = PRp * dlRdR;
    const double H_zp = Pzp * dlzdz;
    if (R > 1e-30) {
        const double Ri = 1.0 / R, R2i = Ri * Ri, R3i = R2i * Ri;
        const double x = px, y = py, x2 = x * x, y2 = y * y, xy = x * y;
        o.h[0] = H_RR * x2 * R2i - 2.0 * H_Rp * xy * R3i + H_pp * y2 * R2i * R2i + dPdR * y2 * R3i;
        o.h[1] = H_RR * y2 * R2i + 2.0 * H_Rp * xy * R3i + H_pp * x2 * R2i * R2i + dPdR * x2 * R3i;
        o.h[2] = H_zz;
        o.h[3] = H_RR * xy * R2i + H_Rp * (x2 - y2) * R3i - H_pp * xy * R2i * R2i - dPdR * xy * R3i;
        o.h[4] = H_Rz * (y * Ri) + H_zp * (x * R2i);
        o.h[5] = H_Rz * (x * Ri) - H_zp * (y * R2i);
        if (EXACT) {
            const double R4i = R2i * R2i;
            o.h[0] += 2.0 * Pp * xy * R4i;
            o.h[1] -= 2.0 * Pp * xy * R4i;
            o.h[3] += Pp * (y2 - x2) * R4i;
        }
    } else {
        o.h[0] = H_RR; o.h[1] = H_RR; o.h[2] = H_zz;
        o.h[3] = 0.0; o.h[4] = 0.0; o.h[5] = 0.0;
    }
    // the reference's CylSpline density is -(Hxx+Hyy+Hzz)/(4 pi G)
    // (gpu_potential.py:1389-1395); kept for parity
    if (MODE == AGB_MODE_DENS) o.rho = -(o.h[0] + o.h[1] + o.h[2]) * AGB_INV_4PIG;
}
