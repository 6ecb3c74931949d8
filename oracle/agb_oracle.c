/*
 * agb_oracle.c -- TEST INFRASTRUCTURE ONLY (the oracle).  See agb_oracle.h.
 *
 * A scalar FP64 restatement of the reference's per-point algorithms, written
 * the way the reference computes them (un-normalised Legendre recurrence with
 * a normalisation update per order, atan2 + direct cos/sin(m phi), the
 * log-scaling chain applied per harmonic) so that it checks the CUDA
 * kernels' reformulations independently.  Pinned against vectors produced by
 * the reference itself (tests/golden/).
 */
#include "agb_oracle.h"
#include <math.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define MUL0 3.5449077018110318      /* 2 sqrt(pi) */
#define MUL1 5.0132565706694072      /* the reference's m != 0 factor */
#define G_AGAMA 4.30091727067736e-06
#define PI_ 3.141592653589793
#define INV_4PIG (1.0 / (4.0 * PI_ * G_AGAMA))

static double PREF[33], COEF[33];
static int tables_ready = 0;

static void init_tables(void)
{
    if (tables_ready) return;
    double fact2m = 1.0, dfact = 1.0;     /* (2m)!, (2m-1)!! */
    for (int m = 0; m <= 32; ++m) {
        if (m > 0) {
            fact2m *= (double)(2 * m - 1) * (double)(2 * m);
            dfact *= (double)(2 * m - 1);
        }
        PREF[m] = sqrt((2.0 * m + 1.0) / (4.0 * PI_ * fact2m));
        COEF[m] = ((m & 1) ? -1.0 : 1.0) * dfact * PREF[m];
    }
    tables_ready = 1;
}

/* quintic on s in [0,1]: value and d/ds, d2/ds2 (_multipole_potential_kernel.cu:100-118) */
static void quintic(const double* a, double s, double* v, double* d1, double* d2)
{
    *v = a[0] + s * (a[1] + s * (a[2] + s * (a[3] + s * (a[4] + s * a[5]))));
    *d1 = a[1] + s * (2 * a[2] + s * (3 * a[3] + s * (4 * a[4] + s * 5 * a[5])));
    *d2 = 2 * a[2] + s * (6 * a[3] + s * (12 * a[4] + s * 20 * a[5]));
}

static void hess_from_radial(double A, double B, double x, double y, double z, double* h)
{
    h[0] = A * x * x + B; h[1] = A * y * y + B; h[2] = A * z * z + B;
    h[3] = A * x * y; h[4] = A * y * z; h[5] = A * x * z;
}

/* ---------------------------------------------------------------- Multipole */
/* spherical derivatives: value, d/dlogr, d2/dlogr2, theta, phi and mixed */
typedef struct {
    double P, Pr, Prr, Pt, Ptt, Prt, Pp, Ppp, Prp, Ptp, Pos, lap;
} sph_t;

/* One point; follows _multipole_potential_kernel.cu:140-410 (Phi, grad),
   :466-800 (Hessian) and :809-958 (density). */
static void mp_point(int mode, double px, double py, double pz, const double* poly,
                     const double* sc, int n_int, int n_lm, const int* lm_l, const int* lm_m,
                     int log_scaling, double* phi, double* g, double* h, double* rho)
{
    const double logr_min = sc[0], dlogr = sc[1], inv_dlogr = sc[2], invPhi0 = sc[3];
    const double in_s = sc[4], in_U = sc[5], in_W = sc[6];
    const double out_s = sc[7], out_U = sc[8], out_W = sc[9];
    const double c00 = MUL0 * PREF[0];
    const double r2 = px * px + py * py + pz * pz, r = sqrt(r2), Rc = sqrt(px * px + py * py);
    int q;
    if (r < 1e-300) {
        if (phi) *phi = c00 * in_W;
        if (g) g[0] = g[1] = g[2] = 0.0;
        if (h) for (q = 0; q < 6; ++q) h[q] = 0.0;
        if (rho) *rho = 0.0;
        return;
    }
    const double logr = log(r);
    double p0, d1, d2;
    int region = 0;
    if (logr < logr_min) {
        const double t = logr - logr_min;
        const double e = (in_s != 0.0) ? exp(in_s * t) : 1.0;
        p0 = in_U * e + in_W; d1 = in_U * in_s * e; d2 = in_U * in_s * in_s * e;
        region = 1;
    }
    int k = (int)((logr - logr_min) * inv_dlogr);
    if (k < 0) k = 0;
    if (!region && k >= n_int) {
        const double t = logr - (logr_min + n_int * dlogr);
        const double en = exp(-t), es = exp(out_s * t);
        p0 = out_W * en + out_U * es;
        d1 = -out_W * en + out_s * out_U * es;
        d2 = out_W * en + out_s * out_s * out_U * es;
        region = 2;
    }
    if (region) {
        if (mode == 3) {
            *rho = (region == 1) ? c00 * (d2 + d1) / (r * r) * INV_4PIG : 0.0;
            return;
        }
        if (phi) *phi = c00 * p0;
        if (mode >= 1) {
            const double gg = c00 * d1 / r2;
            g[0] = gg * px; g[1] = gg * py; g[2] = gg * pz;
        }
        if (mode == 2) hess_from_radial(c00 * (d2 - d1) / (r2 * r2), c00 * d1 / r2, px, py, pz, h);
        return;
    }
    double s = (logr - (logr_min + k * dlogr)) * inv_dlogr;
    if (s < 0.0) s = 0.0;
    if (s > 1.0) s = 1.0;
    const double ct = pz / r, st = Rc / r, ph = atan2(py, px);
    const int near_pole = st < 1e-10;

    /* monopole with the log-scaling inverse */
    double C0, C0s, C0ss;
    quintic(poly + ((long)0 * n_int + k) * 6, s, &C0, &C0s, &C0ss);
    double F = C0, dF = C0s * inv_dlogr, d2F = C0ss * inv_dlogr * inv_dlogr;
    if (log_scaling) {
        const double ex = exp(C0), P0 = 1.0 / (invPhi0 - ex), dPdX = P0 * P0 * ex;
        const double dC = dF, d2C = d2F;
        F = P0;
        dF = dPdX * dC;
        d2F = dPdX * (d2C + dC * dC * P0 * (invPhi0 + ex));
    }
    sph_t S;
    memset(&S, 0, sizeof(S));
    S.P = c00 * F; S.Pr = c00 * dF; S.Prr = c00 * d2F;
    S.lap = (d2F + dF) / r2 * c00;

    int cur = -1, lcur = 0;
    double v0 = 0, v1 = 0, dv0 = 0, dv1 = 0, pf = 0;   /* un-normalised P_{l-1}, P_l (or seed) */
    for (int c = 1; c < n_lm; ++c) {
        const int l = lm_l[c], m = lm_m[c], am = m < 0 ? -m : m;
        if (am != cur) {
            cur = am;
            lcur = am;
            pf = PREF[am];
            const double sp = pow(st, (double)am);
            if (am == 0) { v0 = 1.0; dv0 = 0.0; }
            else if (am == 1) { v0 = -st; dv0 = -ct; }
            else {
                v0 = COEF[am] * sp / pf;
                dv0 = near_pole ? 0.0 : am * ct / st * v0;
            }
            v1 = v0 * ct * (2 * am + 1);
            dv1 = (2 * am + 1) * (ct * dv0 - st * v0);
        }
        while (lcur < l) {
            const int L = lcur + 1;
            if (L > am + 1) {
                const double nv = ((2 * L - 1) * ct * v1 - (L + am - 1) * v0) / (L - am);
                const double nd = ((2 * L - 1) * (ct * dv1 - st * v1) - (L + am - 1) * dv0) / (L - am);
                v0 = v1; v1 = nv; dv0 = dv1; dv1 = nd;
            }
            pf *= sqrt((2.0 * L + 1) / (2.0 * L - 1) * (double)(L - am) / (double)(L + am));
            lcur = L;
        }
        const double Y = ((l == am) ? v0 : v1) * pf;
        const double dY = ((l == am) ? dv0 : dv1) * pf;
        double Cs, Cd, Cdd;
        quintic(poly + ((long)c * n_int + k) * 6, s, &Cs, &Cd, &Cdd);
        double Cv = Cs, dv = Cd * inv_dlogr, d2v = Cdd * inv_dlogr * inv_dlogr;
        if (log_scaling) {
            const double d1c = dv, d2c = d2v;
            d2v = d2c * F + 2.0 * d1c * dF + Cs * d2F;
            dv = d1c * F + Cs * dF;
            Cv = Cs * F;
        }
        const double mul = am == 0 ? MUL0 : MUL1;
        const double T = m >= 0 ? cos(am * ph) : sin(am * ph);
        const double dT = m >= 0 ? -am * sin(am * ph) : am * cos(am * ph);
        const double d2T = -(double)(am * am) * T;
        const double d2Y = near_pole ? 0.0 : (-ct / st * dY - (l * (l + 1.0) - am * am / (st * st)) * Y);
        const double Pos = am == 0 ? 0.0 : (!near_pole ? Y / st : (am == 1 ? dY : 0.0));
        S.P += mul * Cv * Y * T;
        S.Pr += mul * dv * Y * T;
        S.Prr += mul * d2v * Y * T;
        S.Pt += mul * Cv * dY * T;
        S.Ptt += mul * Cv * d2Y * T;
        S.Prt += mul * dv * dY * T;
        S.Pp += mul * Cv * Y * dT;
        S.Ppp += mul * Cv * Y * d2T;
        S.Prp += mul * dv * Y * dT;
        S.Ptp += mul * Cv * dY * dT;
        S.Pos += mul * Cv * Pos * dT;
        S.lap += mul * (d2v + dv - l * (l + 1.0) * Cv) / r2 * Y * T;
    }
    if (mode == 3) { *rho = S.lap * INV_4PIG; return; }
    if (phi) *phi = S.P;
    if (mode == 0) return;
    const double ir = 1.0 / r, ir2 = ir * ir;
    const double cp = Rc > 1e-300 ? px / Rc : 1.0, sp = Rc > 1e-300 ? py / Rc : 0.0;
    g[0] = S.Pr * px * ir2 + S.Pt * ct * cp * ir - S.Pos * sp * ir;
    g[1] = S.Pr * py * ir2 + S.Pt * ct * sp * ir + S.Pos * cp * ir;
    g[2] = S.Pr * pz * ir2 - S.Pt * st * ir;
    if (mode == 1) return;
    /* Cartesian Hessian by the chain rule through (log r, theta, phi) */
    const double X[3] = {px, py, pz};
    const double iR = Rc > 1e-300 ? 1.0 / Rc : 0.0;
    const double jr[3] = {px * ir2, py * ir2, pz * ir2};
    const double jt[3] = {ct * cp * ir, ct * sp * ir, -st * ir};
    const double jp[3] = {-sp * iR, cp * iR, 0.0};
    const double ir3 = ir2 * ir, ir4 = ir2 * ir2, ir5 = ir4 * ir;
    const double is = st > 1e-14 ? 1.0 / st : 0.0;
    const int I[6] = {0, 1, 2, 0, 1, 0}, J[6] = {0, 1, 2, 1, 2, 2};
    for (q = 0; q < 6; ++q) {
        const int i = I[q], j = J[q];
        const double dij = i == j ? 1.0 : 0.0;
        const double hr = dij * ir2 - 2.0 * X[i] * X[j] * ir4;
        /* theta = acos(z/r) */
        const double dfi = (i == 2 ? ir : 0.0) - pz * X[i] * ir3;
        const double dfj = (j == 2 ? ir : 0.0) - pz * X[j] * ir3;
        const double d2f = -((i == 2 ? X[j] : 0.0) + (j == 2 ? X[i] : 0.0) + dij * pz) * ir3
                         + 3.0 * pz * X[i] * X[j] * ir5;
        const double ht = -d2f * is - dfi * dfj * ct * is * is * is;
        double hp = 0.0;
        if (Rc > 1e-14) {
            const double iR4 = iR * iR * iR * iR;
            if (q == 0) hp = 2.0 * px * py * iR4;
            else if (q == 1) hp = -2.0 * px * py * iR4;
            else if (q == 3) hp = (py * py - px * px) * iR4;
        }
        h[q] = S.Prr * jr[i] * jr[j] + S.Prt * (jr[i] * jt[j] + jr[j] * jt[i])
             + S.Prp * (jr[i] * jp[j] + jr[j] * jp[i]) + S.Ptt * jt[i] * jt[j]
             + S.Ptp * (jt[i] * jp[j] + jt[j] * jp[i]) + S.Ppp * jp[i] * jp[j]
             + S.Pr * hr + S.Pt * ht + S.Pp * hp;
    }
}

int oracle_multipole(int mode, const double* x, const double* y, const double* z,
                     const double* poly, const double* sc, int n_int, int n_lm, int lmax,
                     const int* lm_l, const int* lm_m, int log_scaling, double* phi,
                     double* grad, double* hess, double* rho, int64_t n, int nthreads)
{
    (void)lmax;
    init_tables();
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i)
        mp_point(mode, x[i], y[i], z[i], poly, sc, n_int, n_lm, lm_l, lm_m, log_scaling,
                 phi ? phi + i : 0, grad ? grad + 3 * i : 0, hess ? hess + 6 * i : 0,
                 rho ? rho + i : 0);
    return 0;
}

/* ---------------------------------------------------------------- CylSpline */
static int cell_of(double v, const double* g, int n)
{
    int lo = 0, hi = n - 1;
    while (hi - lo > 1) {
        const int mid = (lo + hi) / 2;
        if (g[mid] > v) hi = mid; else lo = mid;
    }
    return lo;
}

/* cubic Hermite value/derivatives on one interval (_cylspl_potential_kernel.cu:110-128) */
static void herm(double xv, double xl, double xh, double fl, double fh, double dl, double dh,
                 double* f, double* df, double* d2f)
{
    const double hh = xh - xl, t = (xv - xl) / hh, T = 1.0 - t, tT = t * T, dif = fh - fl;
    const double Q = 3.0 * (dl + dh) - 6.0 * dif / hh;
    *f = fl * T + fh * t + (dif * (t - T) + (dl * T - dh * t) * hh) * tT;
    *df = dl * T + dh * t - Q * tT;
    *d2f = (dh - dl + Q * (t - T)) / hh;
}

/* exterior asymptote (_cylspl_potential_kernel.cu:181-383), including the
   reference's lagged three-term recurrence for orders l >= m+2 */
static void cs_outer(int mode, double x, double y, double z, const double* W, double r0,
                     int lmax, int mmax, double* phi, double* g, double* h)
{
    const double R2 = x * x + y * y, R = sqrt(R2), r = sqrt(R2 + z * z), ri = 1.0 / r;
    const double ct = z * ri, st = R * ri, ph = atan2(y, x);
    double P = 0, Pr = 0, Pp = 0;
    double buf[33];
    for (int m = 0; m <= mmax; ++m) {
        double pref = PREF[m];
        buf[0] = COEF[m] * pow(st, (double)m);
        if (lmax > m) {
            double p1 = buf[0] / pref, p = ct * (2 * m + 1) * p1, p2 = 0.0;
            pref *= sqrt((double)(2 * m + 3) / (2 * m + 1) / (2.0 * m + 1.0));
            buf[1] = p * pref;
            for (int l = m + 2; l <= lmax; ++l) {
                const double nv = (ct * (2 * l - 1) * p - (double)(l + m - 1) * p2) / (l - m);
                pref *= sqrt((double)(2 * l + 1) / (2 * l - 1) * (double)(l - m) / (l + m));
                buf[l - m] = nv * pref;
                p2 = p1; p1 = p; p = nv;
            }
        }
        const double MUL = m == 0 ? MUL0 : MUL1;
        const double cm = cos(m * ph), sm = sin(m * ph);
        for (int l = m; l <= lmax; ++l) {
            const double pw = pow(r0 * ri, (double)(l + 1));
            const double Yb = buf[l - m] * MUL;
            if (m == 0) {
                P += W[l * (l + 1)] * pw * Yb;
                Pr += W[l * (l + 1)] * (-(l + 1)) * ri * pw * Yb;
            } else {
                const double wc = W[l * (l + 1) + m], ws = W[l * (l + 1) - m];
                const double cc = pw * Yb * (wc * cm + ws * sm);
                P += cc;
                Pr += -(l + 1) * ri * cc;
                Pp += pw * Yb * (-wc * m * sm + ws * m * cm);
            }
        }
    }
    if (phi) *phi = P;
    if (mode >= 1 && g) {
        g[0] = Pr * x * ri + Pp * (R > 1e-30 ? -y / R2 : 0.0);
        g[1] = Pr * y * ri + Pp * (R > 1e-30 ? x / R2 : 0.0);
        g[2] = Pr * z * ri;
    }
    if (mode >= 2 && h) {
        const double p0 = W[0] * MUL0 * r0 * ri, d1 = -p0 * ri, d2 = 2.0 * p0 * ri * ri;
        hess_from_radial((d2 - d1 * ri) / (r * r), d1 * ri, x, y, z, h);
    }
}

static void cs_point(int mode, double px, double py, double pz, double Rs, const double* lRg,
                     int nR, const double* lzg, int nz, const double* nodes, int n_harm,
                     const int* m_arr, int ls, const double* W, double r0, int lmax_o,
                     int mmax_o, double* phi, double* g, double* h, double* rho)
{
    const int need_h = mode >= 2;
    const double R2 = px * px + py * py, R = sqrt(R2), ph = atan2(py, px);
    const double lR = asinh(R / Rs), lz = asinh(pz / Rs);
    const double jR = 1.0 / sqrt(R2 + Rs * Rs), jz = 1.0 / sqrt(pz * pz + Rs * Rs);
    const double jRR = -R * jR * jR * jR, jzz = -pz * jz * jz * jz;
    double hh[6], gg[3];
    if (lR < lRg[0] || lR > lRg[nR - 1] || lz < lzg[0] || lz > lzg[nz - 1]) {
        cs_outer(mode >= 2 ? 2 : mode, px, py, pz, W, r0, lmax_o, mmax_o, phi, g ? g : gg, need_h ? (h ? h : hh) : 0);
        if (mode == 3) { const double* H = h ? h : hh; *rho = -(H[0] + H[1] + H[2]) * INV_4PIG; }
        return;
    }
    const int iR = cell_of(lR, lRg, nR), iz = cell_of(lz, lzg, nz);
    double S = ls ? 1.0 : 0.0, SR = 0, Sz = 0, SRR = 0, SRz = 0, Szz = 0, Sp = 0, Spp = 0, SRp = 0, Szp = 0;
    double f0 = 0, f0R = 0, f0z = 0, f0RR = 0, f0Rz = 0, f0zz = 0;
    for (int hm = 0; hm < n_harm; ++hm) {
        const int m = m_arr[hm];
        const double* nd = nodes + (long)hm * nR * nz * 4;
#define NODE(a, b, qq) nd[((long)(a) * nz + (b)) * 4 + (qq)]
        double fll = NODE(iR, iz, 0), flu = NODE(iR, iz + 1, 0);
        double ful = NODE(iR + 1, iz, 0), fuu = NODE(iR + 1, iz + 1, 0);
        const double off = (lR == lRg[iR + 1]) ? ((lz == lzg[iz + 1]) ? fuu : ful)
                                               : ((lz == lzg[iz + 1]) ? flu : fll);
        fll -= off; flu -= off; ful -= off; fuu -= off;
        double F[4], dF[4], d2F[4];
        herm(lz, lzg[iz], lzg[iz + 1], fll, flu, NODE(iR, iz, 2), NODE(iR, iz + 1, 2), &F[0], &dF[0], &d2F[0]);
        herm(lz, lzg[iz], lzg[iz + 1], ful, fuu, NODE(iR + 1, iz, 2), NODE(iR + 1, iz + 1, 2), &F[1], &dF[1], &d2F[1]);
        herm(lz, lzg[iz], lzg[iz + 1], NODE(iR, iz, 1), NODE(iR, iz + 1, 1), NODE(iR, iz, 3), NODE(iR, iz + 1, 3), &F[2], &dF[2], &d2F[2]);
        herm(lz, lzg[iz], lzg[iz + 1], NODE(iR + 1, iz, 1), NODE(iR + 1, iz + 1, 1), NODE(iR + 1, iz, 3), NODE(iR + 1, iz + 1, 3), &F[3], &dF[3], &d2F[3]);
#undef NODE
        double v, vR, vRR, vz, vRz, vzz, dum;
        herm(lR, lRg[iR], lRg[iR + 1], F[0], F[1], F[2], F[3], &v, &vR, &vRR);
        v += off;
        herm(lR, lRg[iR], lRg[iR + 1], dF[0], dF[1], dF[2], dF[3], &vz, &vRz, &dum);
        herm(lR, lRg[iR], lRg[iR + 1], d2F[0], d2F[1], d2F[2], d2F[3], &vzz, &dum, &dum);
        if (m == 0) {
            f0 = v; f0R = vR; f0z = vz; f0RR = vRR; f0Rz = vRz; f0zz = vzz;
            if (!ls) { S += v; SR += vR; Sz += vz; SRR += vRR; SRz += vRz; Szz += vzz; }
        } else {
            const int am = m < 0 ? -m : m;
            const double T = m > 0 ? cos(am * ph) : sin(am * ph);
            const double dT = m > 0 ? -am * sin(am * ph) : am * cos(am * ph);
            const double d2T = -(double)(am * am) * T;
            S += v * T; SR += vR * T; Sz += vz * T; Sp += v * dT;
            SRR += vRR * T; SRz += vRz * T; Szz += vzz * T; SRp += vR * dT; Szp += vz * dT; Spp += v * d2T;
        }
    }
    double P, PR, Pz, Pp, PRR, PRz, Pzz, PRp, Pzp, Ppp;
    if (ls) {
        const double P0 = -exp(f0), P0R = P0 * f0R, P0z = P0 * f0z;
        P = P0 * S; PR = P0 * SR + P0R * S; Pz = P0 * Sz + P0z * S; Pp = P0 * Sp;
        PRR = P0 * SRR + 2 * P0R * SR + P0 * (f0RR + f0R * f0R) * S;
        Pzz = P0 * Szz + 2 * P0z * Sz + P0 * (f0zz + f0z * f0z) * S;
        PRz = P0 * SRz + P0R * Sz + P0z * SR + P0 * (f0Rz + f0R * f0z) * S;
        PRp = P0 * SRp + P0R * Sp; Pzp = P0 * Szp + P0z * Sp; Ppp = P0 * Spp;
    } else {
        P = S; PR = SR; Pz = Sz; Pp = Sp; PRR = SRR; PRz = SRz; Pzz = Szz; PRp = SRp; Pzp = Szp; Ppp = Spp;
    }
    if (phi) *phi = P;
    if (mode == 0) return;
    const double dR = PR * jR, dz = Pz * jz;
    double* G = g ? g : gg;
    G[0] = R > 1e-30 ? dR * px / R - Pp * py / R2 : 0.0;
    G[1] = R > 1e-30 ? dR * py / R + Pp * px / R2 : 0.0;
    G[2] = dz;
    if (mode == 1) return;
    double* H = h ? h : hh;
    const double HRR = PRR * jR * jR + PR * jRR, Hzz = Pzz * jz * jz + Pz * jzz;
    const double HRz = PRz * jR * jz, Hpp = Ppp, HRp = PRp * jR, Hzp = Pzp * jz;
    if (R > 1e-30) {
        const double x = px, y = py, R3 = R2 * R;
        H[0] = HRR * x * x / R2 - 2 * HRp * x * y / R3 + Hpp * y * y / (R2 * R2) + dR * y * y / R3;
        H[1] = HRR * y * y / R2 + 2 * HRp * x * y / R3 + Hpp * x * x / (R2 * R2) + dR * x * x / R3;
        H[2] = Hzz;
        H[3] = HRR * x * y / R2 + HRp * (x * x - y * y) / R3 - Hpp * x * y / (R2 * R2) - dR * x * y / R3;
        H[4] = HRz * y / R + Hzp * x / R2;
        H[5] = HRz * x / R - Hzp * y / R2;
    } else {
        H[0] = HRR; H[1] = HRR; H[2] = Hzz; H[3] = H[4] = H[5] = 0.0;
    }
    if (mode == 3) *rho = -(H[0] + H[1] + H[2]) * INV_4PIG;
}

int oracle_cylspline(int mode, const double* x, const double* y, const double* z, double Rscale,
                     const double* lR, int nR, const double* lz, int nz, const double* node_arr,
                     int n_harm, const int* m_arr, int log_scaling, const double* W_outer,
                     double r0_outer, int lmax_outer, int mmax_outer, double* phi, double* grad,
                     double* hess, double* rho, int64_t n, int nthreads)
{
    init_tables();
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i)
        cs_point(mode, x[i], y[i], z[i], Rscale, lR, nR, lz, nz, node_arr, n_harm, m_arr,
                 log_scaling, W_outer, r0_outer, lmax_outer, mmax_outer, phi ? phi + i : 0,
                 grad ? grad + 3 * i : 0, hess ? hess + 6 * i : 0, rho ? rho + i : 0);
    return 0;
}

/* ---------------------------------------------------------------- analytic */
/* _analytic_potentials.py: closed forms of each profile */
static void an_point(int kind, const double* p, int mode, double x, double y, double z,
                     double* phi, double* g, double* h, double* rho)
{
    const double r2 = x * x + y * y + z * z, r = sqrt(r2);
    const double sr = r < 1e-300 ? 1e-300 : r, sr2 = r2 < 1e-300 ? 1e-300 : r2, rh = sqrt(sr2);
    double P = 0, d1 = 0, d2 = 0, dens = 0;     /* spherical: Phi(r), dPhi/dr, d2Phi/dr2 */
    int spherical = 1;
    double gg[3] = {0, 0, 0}, hh[6] = {0, 0, 0, 0, 0, 0};
    switch (kind) {
    case 10: { /* NFW: GM, rs, M */
        const double GM = p[0], rs = p[1], M = p[2];
        P = -GM * log1p(sr / rs) / sr;
        const double g1 = GM * (log1p(sr / rs) / (sr * sr) - 1.0 / (sr * (sr + rs)));
        gg[0] = g1 * x / sr; gg[1] = g1 * y / sr; gg[2] = g1 * z / sr;
        const double ln = log1p(rh / rs), rr = rh + rs;
        d1 = GM * (ln / sr2 - 1.0 / (rh * rr));
        d2 = GM * (-2.0 * ln / (sr2 * rh) + 1.0 / (sr2 * rr) + (2.0 * rh + rs) / (sr2 * rr * rr));
        hess_from_radial((d2 - d1 / rh) / sr2, d1 / rh, x, y, z, hh);
        dens = M / (4.0 * PI_ * sr * (sr + rs) * (sr + rs));
        spherical = 0;
        break; }
    case 11: { /* Plummer: GM, b2, M */
        const double GM = p[0], b2 = p[1], M = p[2], s2 = r2 + b2, s = sqrt(s2);
        P = -GM / s;
        gg[0] = GM / (s2 * s) * x; gg[1] = GM / (s2 * s) * y; gg[2] = GM / (s2 * s) * z;
        hess_from_radial(-3.0 * GM / (s2 * s2 * s), GM / (s2 * s), x, y, z, hh);
        dens = 3.0 * M / (4.0 * PI_) * b2 / pow(s2, 2.5);
        spherical = 0;
        break; }
    case 12: { /* Hernquist: GM, a, M */
        const double GM = p[0], a = p[1], M = p[2];
        P = -GM / (r + a);
        const double f = GM / ((sr + a) * (sr + a) * sr);
        gg[0] = f * x; gg[1] = f * y; gg[2] = f * z;
        const double e1 = GM / ((rh + a) * (rh + a)), e2 = -2.0 * GM / ((rh + a) * (rh + a) * (rh + a));
        hess_from_radial((e2 - e1 / rh) / sr2, e1 / rh, x, y, z, hh);
        dens = M * a / (2.0 * PI_ * sr * pow(sr + a, 3));
        spherical = 0;
        break; }
    case 13: { /* Dehnen: GM, a, gamma, 2-gamma, M */
        const double GM = p[0], a = p[1], ga = p[2], ex = p[3], M = p[4];
        P = -(GM / a) * (1.0 - pow(sr / (sr + a), ex)) / ex;
        const double e1 = GM * pow(sr, 1.0 - ga) * pow(sr + a, ga - 3.0);
        gg[0] = e1 / sr * x; gg[1] = e1 / sr * y; gg[2] = e1 / sr * z;
        const double e2 = e1 * ((1.0 - ga) / sr + (ga - 3.0) / (sr + a));
        hess_from_radial((e2 - e1 / sr) / (sr * sr), e1 / sr, x, y, z, hh);
        dens = (3.0 - ga) * M / (4.0 * PI_ * a * a * a) * pow(sr / a, -ga) * pow(1.0 + sr / a, ga - 4.0);
        spherical = 0;
        break; }
    case 14: { /* Isochrone: GM, b */
        const double GM = p[0], b = p[1];
        const double s = sqrt(r2 + b * b);
        P = -GM / (b + s);
        const double c = GM / (s * (b + s) * (b + s));
        gg[0] = c * x; gg[1] = c * y; gg[2] = c * z;
        const double sh = sqrt(sr2 + b * b), bs = b + sh, d1r = GM / (sh * bs * bs);
        hess_from_radial(-GM * (b + 3.0 * sh) / (sh * sh * sh * bs * bs * bs), d1r, x, y, z, hh);
        dens = (-GM * (b + 3.0 * sh) / (pow(sh, 3) * pow(bs, 3)) * sr2 + 3.0 * d1r) * INV_4PIG;
        spherical = 0;
        break; }
    case 15: { /* Miyamoto-Nagai: GM, a, b */
        const double GM = p[0], a = p[1], b = p[2], R2 = x * x + y * y, D = sqrt(z * z + b * b);
        const double aD = a + D, S2 = R2 + aD * aD, S = sqrt(S2), S3 = S2 * S, S5 = S3 * S2;
        P = -GM / S;
        gg[0] = GM / S3 * x; gg[1] = GM / S3 * y; gg[2] = GM / S3 * aD * z / D;
        hh[0] = GM * (1.0 / S3 - 3.0 * x * x / S5);
        hh[1] = GM * (1.0 / S3 - 3.0 * y * y / S5);
        hh[2] = GM * (aD / (D * S3) - z * z * aD / (D * D * D * S3) + z * z / (D * D * S3)
                      - 3.0 * aD * aD * z * z / (D * D * S5));
        hh[3] = -3.0 * GM * x * y / S5;
        hh[4] = -3.0 * GM * aD * z / (D * S5) * y;
        hh[5] = -3.0 * GM * aD * z / (D * S5) * x;
        dens = GM * b * b * INV_4PIG * (a * R2 + (a + 3.0 * D) * aD * aD) / (D * D * D * pow(S2, 2.5));
        spherical = 0;
        break; }
    case 16: { /* LogHalo: v0^2, rc^2, p^2, q^2 */
        const double v2 = p[0], rc2 = p[1], p2 = p[2], q2 = p[3];
        const double m2 = rc2 + x * x + y * y / p2 + z * z / q2, m4 = m2 * m2;
        P = 0.5 * v2 * log(m2);
        gg[0] = v2 / m2 * x; gg[1] = v2 / m2 * y / p2; gg[2] = v2 / m2 * z / q2;
        hh[0] = v2 * (1.0 / m2 - 2.0 * x * x / m4);
        hh[1] = v2 * (1.0 / (m2 * p2) - 2.0 * y * y / (m4 * p2 * p2));
        hh[2] = v2 * (1.0 / (m2 * q2) - 2.0 * z * z / (m4 * q2 * q2));
        hh[3] = -2.0 * v2 / m4 * x * y / p2;
        hh[4] = -2.0 * v2 / m4 * y * z / (p2 * q2);
        hh[5] = -2.0 * v2 / m4 * x * z / q2;
        dens = v2 * ((1.0 + 1.0 / p2 + 1.0 / q2) / m2 - 2.0 * (x * x + y * y / (p2 * p2) + z * z / (q2 * q2)) / m4) * INV_4PIG;
        spherical = 0;
        break; }
    case 17: { /* DiskAnsatz: Sigma*G, hr, |hz|, hin (exponential vertical law) */
        const double Sg = p[0], hr = p[1], hz = p[2], hin = p[3], ir = 1.0 / sr;
        const double f = 4.0 * PI_ * Sg * exp(-sr / hr - hin / sr);
        const double fo = -1.0 / hr + hin * ir * ir, f1 = f * fo;
        const double f2 = f * (fo * fo - 2.0 * hin * ir * ir * ir);
        const double u = fabs(z) / hz, eu = exp(-u);
        const double H = 0.5 * hz * (eu - 1.0 + u);
        const double H1 = 0.5 * ((z > 0) - (z < 0)) * (1.0 - eu), H2 = 0.5 * eu / hz;
        P = f * H;
        gg[0] = H * f1 * ir * x; gg[1] = H * f1 * ir * y; gg[2] = H * f1 * ir * z + H1 * f;
        const double xr = x * ir, yr = y * ir, zr = z * ir, A = H * (f2 - f1 * ir), B = H * f1 * ir;
        hh[0] = A * xr * xr + B; hh[1] = A * yr * yr + B;
        hh[2] = H * (f2 * zr * zr + f1 * (1.0 - zr * zr) * ir) + 2.0 * f1 * H1 * zr + f * H2;
        hh[3] = A * xr * yr; hh[4] = A * yr * zr + f1 * H1 * yr; hh[5] = A * xr * zr + f1 * H1 * xr;
        dens = (H * (f2 + 2.0 * f1 * ir) + 2.0 * f1 * H1 * zr + f * H2) * INV_4PIG;
        spherical = 0;
        break; }
    case 18: /* UniformAcceleration: ax, ay, az */
        P = -(p[0] * x + p[1] * y + p[2] * z);
        gg[0] = -p[0]; gg[1] = -p[1]; gg[2] = -p[2];
        dens = 0.0;
        spherical = 0;
        break;
    default:
        break;
    }
    (void)spherical;
    if (mode == 3) { *rho = dens; return; }
    if (phi) *phi = P;
    if (mode >= 1 && g) { g[0] = gg[0]; g[1] = gg[1]; g[2] = gg[2]; }
    if (mode >= 2 && h) for (int q = 0; q < 6; ++q) h[q] = hh[q];
}

int oracle_analytic(int kind, const double* p, int mode, const double* x, const double* y,
                    const double* z, double* phi, double* grad, double* hess, double* rho,
                    int64_t n)
{
    if (kind < 10 || kind > 18) return -1;
    for (int64_t i = 0; i < n; ++i)
        an_point(kind, p, mode, x[i], y[i], z[i], phi ? phi + i : 0, grad ? grad + 3 * i : 0,
                 hess ? hess + 6 * i : 0, rho ? rho + i : 0);
    return 0;
}
