// analytic.cuh -- closed-form profiles (Phi, grad, Hessian, density).
//
// Same formulas and the same r floors as the reference's ElementwiseKernel
// bodies (_analytic_potentials.py): NFW :176-243, Plummer :288-340,
// Hernquist :383-444, Dehnen (spherical) :486-549, Isochrone :603-676,
// Miyamoto-Nagai :720-793, LogHalo (triaxial) :842-892, DiskAnsatz with inner
// cutoff :950-1052 (always the exponential vertical profile with |h|, as the
// reference's kernels are), UniformAcceleration :1112-1165.
// Parameters p[] per kind are set by the Python layer (analytic.py).
#pragma once
#include "agb_dev.cuh"

#define AGB_4PI 12.566370614359172
#define AGB_2PI 6.283185307179586

// NFW: p = {GM, rs, M}
template <int MODE>
__device__ __forceinline__ void nfw_point(const double* p, double x, double y, double z, PointOut& o)
{
    const double GM = p[0], rs = p[1], M = p[2];
    const double r2raw = x * x + y * y + z * z;
    const double rraw = sqrt(r2raw);
    const double r = rraw < 1e-300 ? 1e-300 : rraw;
    if (MODE == AGB_MODE_DENS) {
        const double rrs = r + rs;
        o.rho = M / (AGB_4PI * r * rrs * rrs);
        return;
    }
    o.phi = -GM * log1p(r / rs) / r;
    if (MODE == AGB_MODE_GRAD) {
        const double d1 = GM * (log1p(r / rs) / (r * r) - 1.0 / (r * (r + rs)));
        const double ir = 1.0 / r;
        o.g[0] = d1 * x * ir; o.g[1] = d1 * y * ir; o.g[2] = d1 * z * ir;
    }
    if (MODE == AGB_MODE_HESS) {
        {   // gradient exactly as the grad kernel computes it
            const double d1 = GM * (log1p(r / rs) / (r * r) - 1.0 / (r * (r + rs)));
            const double ir = 1.0 / r;
            o.g[0] = d1 * x * ir; o.g[1] = d1 * y * ir; o.g[2] = d1 * z * ir;
        }
        const double r2 = r2raw < 1e-300 ? 1e-300 : r2raw;
        const double rh = sqrt(r2);
        const double rrs = rh + rs;
        const double ln = log1p(rh / rs);
        const double d1 = GM * (ln / r2 - 1.0 / (rh * rrs));
        const double d2 = GM * (-2.0 * ln / (r2 * rh) + 1.0 / (r2 * rrs) + (2.0 * rh + rs) / (r2 * rrs * rrs));
        const double d1r = d1 / rh;
        hess_radial((d2 - d1r) / r2, d1r, x, y, z, o.h);
    }
}

// Plummer: p = {GM, b2, M}
template <int MODE>
__device__ __forceinline__ void plummer_point(const double* p, double x, double y, double z, PointOut& o)
{
    const double GM = p[0], b2 = p[1], M = p[2];
    const double s2 = x * x + y * y + z * z + b2;
    if (MODE == AGB_MODE_DENS) {
        o.rho = (3.0 * M / AGB_4PI) * b2 / pow(s2, 2.5);
        return;
    }
    const double s = sqrt(s2);
    o.phi = -GM / s;
    if (MODE == AGB_MODE_GRAD || MODE == AGB_MODE_HESS) {
        const double c = GM / (s2 * s);
        o.g[0] = c * x; o.g[1] = c * y; o.g[2] = c * z;
    }
    if (MODE == AGB_MODE_HESS) {
        const double s3 = s2 * s, s5 = s3 * s2;
        hess_radial(-3.0 * GM / s5, GM / s3, x, y, z, o.h);
    }
}

// Hernquist: p = {GM, a, M}
template <int MODE>
__device__ __forceinline__ void hernquist_point(const double* p, double x, double y, double z, PointOut& o)
{
    const double GM = p[0], a = p[1], M = p[2];
    const double r2raw = x * x + y * y + z * z;
    const double rraw = sqrt(r2raw);
    const double r = rraw < 1e-300 ? 1e-300 : rraw;
    if (MODE == AGB_MODE_DENS) {
        o.rho = (M * a) / (AGB_2PI * r * pow(r + a, 3));
        return;
    }
    o.phi = -GM / (rraw + a);
    if (MODE == AGB_MODE_GRAD || MODE == AGB_MODE_HESS) {
        const double ra = r + a;
        const double f = GM / (ra * ra * r);
        o.g[0] = f * x; o.g[1] = f * y; o.g[2] = f * z;
    }
    if (MODE == AGB_MODE_HESS) {
        const double r2 = r2raw < 1e-300 ? 1e-300 : r2raw;
        const double rh = sqrt(r2);
        const double ra = rh + a;
        const double d1 = GM / (ra * ra);
        const double d2 = -2.0 * GM / (ra * ra * ra);
        const double d1r = d1 / rh;
        hess_radial((d2 - d1r) / r2, d1r, x, y, z, o.h);
    }
}

// Dehnen (spherical): p = {GM, a, gamma, 2-gamma, M}
template <int MODE>
__device__ __forceinline__ void dehnen_point(const double* p, double x, double y, double z, PointOut& o)
{
    const double GM = p[0], a = p[1], g = p[2], ex = p[3], M = p[4];
    const double r = sqrt(x * x + y * y + z * z);
    const double sr = r < 1e-300 ? 1e-300 : r;
    if (MODE == AGB_MODE_DENS) {
        const double t1 = (3.0 - g) * M / (AGB_4PI * a * a * a);
        o.rho = t1 * pow(sr / a, -g) * pow(1.0 + sr / a, g - 4.0);
        return;
    }
    const double u = sr / (sr + a);
    o.phi = -(GM / a) * (1.0 - pow(u, ex)) / ex;
    if (MODE == AGB_MODE_GRAD || MODE == AGB_MODE_HESS) {
        const double ra = sr + a;
        const double d1 = GM * pow(sr, 1.0 - g) * pow(ra, g - 3.0);
        const double c = d1 / sr;
        o.g[0] = c * x; o.g[1] = c * y; o.g[2] = c * z;
        if (MODE == AGB_MODE_HESS) {
            const double d2 = d1 * ((1.0 - g) / sr + (g - 3.0) / ra);
            hess_radial((d2 - c) / (sr * sr), c, x, y, z, o.h);
        }
    }
}

// Isochrone: p = {GM, b}
template <int MODE>
__device__ __forceinline__ void isochrone_point(const double* p, double x, double y, double z, PointOut& o)
{
    const double GM = p[0], b = p[1];
    const double r2raw = x * x + y * y + z * z;
    if (MODE == AGB_MODE_DENS || MODE == AGB_MODE_HESS) {
        const double r2 = r2raw < 1e-300 ? 1e-300 : r2raw;
        const double s = sqrt(r2 + b * b);
        const double bs = b + s;
        const double d1r = GM / (s * bs * bs);
        if (MODE == AGB_MODE_DENS) {
            const double A = -GM * (b + 3.0 * s) / (pow(s, 3) * pow(bs, 3));
            o.rho = (A * r2 + 3.0 * d1r) * AGB_INV_4PIG;
            return;
        }
        const double A = -GM * (b + 3.0 * s) / (s * s * s * bs * bs * bs);
        hess_radial(A, d1r, x, y, z, o.h);
    }
    const double s = sqrt(r2raw + b * b);
    o.phi = -GM / (b + s);
    if (MODE == AGB_MODE_GRAD || MODE == AGB_MODE_HESS) {
        const double bs = b + s;
        const double c = GM / (s * bs * bs);
        o.g[0] = c * x; o.g[1] = c * y; o.g[2] = c * z;
    }
}

// Miyamoto-Nagai: p = {GM, a, b}
template <int MODE>
__device__ __forceinline__ void mn_point(const double* p, double x, double y, double z, PointOut& o)
{
    const double GM = p[0], a = p[1], b = p[2];
    const double R2 = x * x + y * y;
    const double D = sqrt(z * z + b * b);
    const double aD = a + D;
    const double S2 = R2 + aD * aD;
    if (MODE == AGB_MODE_DENS) {
        const double D3 = D * D * D;
        const double S5 = pow(S2, 2.5);
        o.rho = (GM * b * b * AGB_INV_4PIG) * (a * R2 + (a + 3.0 * D) * aD * aD) / (D3 * S5);
        return;
    }
    o.phi = -GM / sqrt(x * x + y * y + aD * aD);
    if (MODE == AGB_MODE_GRAD || MODE == AGB_MODE_HESS) {
        const double S3 = S2 * sqrt(S2);
        const double c = GM / S3;
        o.g[0] = c * x; o.g[1] = c * y; o.g[2] = c * aD * z / D;
    }
    if (MODE == AGB_MODE_HESS) {
        const double D2 = D * D;
        const double S = sqrt(S2);
        const double S3 = S2 * S, S5 = S3 * S2;
        o.h[0] = GM * (1.0 / S3 - 3.0 * x * x / S5);
        o.h[1] = GM * (1.0 / S3 - 3.0 * y * y / S5);
        o.h[3] = -3.0 * GM * x * y / S5;
        const double daD = z / D;
        const double t1 = ((daD * D - aD * z / D) * z + aD * D) / (D2 * S3);
        const double t2 = 3.0 * aD * z * (aD * z / D) / (D * S5);
        o.h[2] = GM * (t1 - t2);
        const double oz = -3.0 * GM * aD * z / (D * S5);
        o.h[5] = oz * x;
        o.h[4] = oz * y;
    }
}

// LogHalo: p = {v0^2, rc^2, p^2, q^2}
template <int MODE>
__device__ __forceinline__ void loghalo_point(const double* p, double x, double y, double z, PointOut& o)
{
    const double v02 = p[0], rc2 = p[1], p2 = p[2], q2 = p[3];
    const double m2 = rc2 + x * x + y * y / p2 + z * z / q2;
    if (MODE == AGB_MODE_DENS) {
        const double m4 = m2 * m2;
        const double t1 = (1.0 + 1.0 / p2 + 1.0 / q2) / m2;
        const double t2 = 2.0 * (x * x + y * y / (p2 * p2) + z * z / (q2 * q2)) / m4;
        o.rho = v02 * (t1 - t2) * AGB_INV_4PIG;
        return;
    }
    o.phi = (v02 * 0.5) * log(m2);
    if (MODE == AGB_MODE_GRAD || MODE == AGB_MODE_HESS) {
        const double c = v02 / m2;
        o.g[0] = c * x; o.g[1] = c * y / p2; o.g[2] = c * z / q2;
    }
    if (MODE == AGB_MODE_HESS) {
        const double m4 = m2 * m2;
        o.h[0] = v02 * (1.0 / m2 - 2.0 * x * x / m4);
        o.h[1] = v02 * (1.0 / (m2 * p2) - 2.0 * y * y / (m4 * p2 * p2));
        o.h[2] = v02 * (1.0 / (m2 * q2) - 2.0 * z * z / (m4 * q2 * q2));
        const double cm = -2.0 * v02 / m4;
        o.h[3] = cm * x * y / p2;
        o.h[4] = cm * y * z / (p2 * q2);
        o.h[5] = cm * x * z / q2;
    }
}

// DiskAnsatz: p = {Sigma*G, hr, |hz|, hin}
template <int MODE>
__device__ __forceinline__ void diskansatz_point(const double* p, double x, double y, double z, PointOut& o)
{
    const double Sig = p[0], hr = p[1], hz = p[2], hin = p[3];
    const double r = sqrt(x * x + y * y + z * z);
    const double sr = r < 1e-300 ? 1e-300 : r;
    const double ir = 1.0 / sr;
    const double f = AGB_4PI * Sig * exp(-sr / hr - hin / sr);
    const double abz = fabs(z);
    const double u = abz / hz;
    const double eu = exp(-u);
    const double H = (hz / 2.0) * (eu - 1.0 + u);
    if (MODE == AGB_MODE_POT) { o.phi = f * H; return; }
    const double fdo = -1.0 / hr + hin * ir * ir;
    const double f1 = f * fdo;
    const double sgn = (double)((z > 0) - (z < 0));
    const double H1 = 0.5 * sgn * (1.0 - eu);
    if (MODE == AGB_MODE_GRAD) {
        o.phi = f * H;
        const double cm = H * f1 * ir;
        o.g[0] = cm * x; o.g[1] = cm * y; o.g[2] = cm * z + H1 * f;
        return;
    }
    const double f2 = f * (fdo * fdo - 2.0 * hin * ir * ir * ir);
    const double H2 = 0.5 * eu / hz;
    if (MODE == AGB_MODE_DENS) {
        const double zr = z * ir;
        o.rho = (H * (f2 + 2.0 * f1 * ir) + 2.0 * f1 * H1 * zr + f * H2) * AGB_INV_4PIG;
        return;
    }
    o.phi = f * H;
    {
        const double cm = H * f1 * ir;
        o.g[0] = cm * x; o.g[1] = cm * y; o.g[2] = cm * z + H1 * f;
    }
    const double xr = x * ir, yr = y * ir, zr = z * ir;
    const double A = H * (f2 - f1 * ir);
    const double B = H * f1 * ir;
    o.h[0] = A * xr * xr + B;
    o.h[1] = A * yr * yr + B;
    o.h[2] = H * (f2 * zr * zr + f1 * (1.0 - zr * zr) * ir) + 2.0 * f1 * H1 * zr + f * H2;
    o.h[3] = A * xr * yr;
    o.h[4] = A * yr * zr + f1 * H1 * yr;
    o.h[5] = A * xr * zr + f1 * H1 * xr;
}

// UniformAcceleration: p = {ax, ay, az}
template <int MODE>
__device__ __forceinline__ void uniform_point(const double* p, double x, double y, double z, PointOut& o)
{
    const double ax = p[0], ay = p[1], az = p[2];
    if (MODE == AGB_MODE_DENS) { o.rho = 0.0; return; }
    o.phi = -(ax * x + ay * y + az * z);
    if (MODE == AGB_MODE_GRAD || MODE == AGB_MODE_HESS) { o.g[0] = -ax; o.g[1] = -ay; o.g[2] = -az; }
    if (MODE == AGB_MODE_HESS) for (int q = 0; q < 6; ++q) o.h[q] = 0.0;
}
