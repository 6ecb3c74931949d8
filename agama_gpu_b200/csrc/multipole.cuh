// multipole.cuh -- per-point evaluation of an Agama Multipole expansion.
//
// Follows the reference's kernels (_multipole_potential_kernel.cu):
//   * log-r interval lookup, s clamp and the r < 1e-300 origin rule (:160-216);
//   * inner power-law l=0 extrapolation U (r/r0)^s + W (:177-193, :492-520,
//     :836-847) and outer W (r/rN)^-1 + U (r/rN)^s (:197-214, :522-549);
//   * quintic Horner value/derivatives on s in [0,1] (:100-118);
//   * Agama log-scaling: c=0 stores log(invPhi0 - 1/Phi0), c>0 store Phi_c/Phi0
//     (:239-258, :566-585);
//   * pole-safe gradient (:388-409), full Cartesian Hessian chain rule (:713-799),
//     Laplacian density with zero density beyond the grid (:851, :915).
// Differences in form, not in result:
//   * Legendre functions come from the normalised recurrence with tabulated
//     ALPHA/BETA (legendre_tables.cuh) instead of an un-normalised recurrence
//     with a sqrt per step; cos/sin(m phi) from x/R, y/R and a rotation instead
//     of atan2 + sincos;
//   * the log-scaling chain rule is factored out of the harmonic loop: the loop
//     accumulates sums of C_c Y T, dC_c Y T, ... and the monopole factor is
//     applied once per point;
//   * the loop is templated on the real type R: double (plain FP64) or float
//     (mixed: FP32 recurrences and polynomials, per-|m| FP32 partial sums
//     promoted to FP64, FP64 everywhere else).
#pragma once
#include <type_traits>
#include "agb_dev.cuh"

// Radial sums of one Multipole at one point (component frame).
struct MPSums {
    double A, B, D, L;              // sum C Y T, dC/ds Y T, d2C/ds2 Y T, l(l+1) C Y T
    double Th, Pos;                 // C dY T, C (Y/sin) dT
    double Thth, BTh, Ph, Phph, BPh, ThPh;
};

template <typename R> struct MPGroup {
    R A, B, D, L, Th, Pos, Thth, BTh, Ph, Phph, BPh, ThPh;
    __device__ __forceinline__ void zero() {
        A = B = D = L = Th = Pos = Thth = BTh = Ph = Phph = BPh = ThPh = R(0);
    }
};

template <int MODE, typename R>
__device__ __forceinline__ void mp_flush(MPSums& t, MPGroup<R>& g)
{
    t.A += (double)g.A;
    if (MODE != AGB_MODE_POT) t.B += (double)g.B;
    if (MODE == AGB_MODE_HESS || MODE == AGB_MODE_DENS) t.D += (double)g.D;
    if (MODE == AGB_MODE_DENS) t.L += (double)g.L;
    if (MODE == AGB_MODE_GRAD || MODE == AGB_MODE_HESS) {
        t.Th += (double)g.Th;
        t.Pos += (double)g.Pos;
    }
    if (MODE == AGB_MODE_HESS) {
        t.Thth += (double)g.Thth; t.BTh += (double)g.BTh; t.Ph += (double)g.Ph;
        t.Phph += (double)g.Phph; t.BPh += (double)g.BPh; t.ThPh += (double)g.ThPh;
    }
    g.zero();
}

template <typename R> struct MPConst;
template <> struct MPConst<double> {
    static __device__ __forceinline__ double alpha(int i) { return AGB_ALPHA[i]; }
    static __device__ __forceinline__ double beta(int i) { return AGB_BETA[i]; }
    static __device__ __forceinline__ double nbetaq(int i) { return AGB_NBETAQ[i]; }
    static __device__ __forceinline__ double2 skip(int i) { return AGB_SKIP[i]; }
};
template <> struct MPConst<float> {
    static __device__ __forceinline__ float alpha(int i) { return AGB_ALPHA_F[i]; }
    static __device__ __forceinline__ float beta(int i) { return AGB_BETA_F[i]; }
    static __device__ __forceinline__ float nbetaq(int i) { return AGB_NBETAQ_F[i]; }
    static __device__ __forceinline__ float2 skip(int i) { return AGB_SKIP_F[i]; }
};

// Quintic coefficients of harmonic c in radial interval k.
template <typename R> struct MPRec;
template <> struct MPRec<double> {
    static __device__ __forceinline__ void load(const DevComp& c, int ci, int k, double a[6])
    {
        const long long off = (c.layout == AGB_LAYOUT_INTERVAL_MAJOR)
            ? ((long long)k * c.n_lm + ci) * 6
            : ((long long)ci * c.n_int + k) * 6;
        const double2* p = reinterpret_cast<const double2*>(c.table + off);
        double2 v0 = __ldg(p), v1 = __ldg(p + 1), v2 = __ldg(p + 2);
        a[0] = v0.x; a[1] = v0.y; a[2] = v1.x; a[3] = v1.y; a[4] = v2.x; a[5] = v2.y;
    }
};
template <> struct MPRec<float> {
    // FP32 table is interval-major with 8-float records (a0..a5, 0, 0).
    static __device__ __forceinline__ void load(const DevComp& c, int ci, int k, float a[6])
    {
        const float4* p = reinterpret_cast<const float4*>(c.table32 + ((long long)k * c.n_lm + ci) * 8);
        float4 v0 = __ldg(p), v1 = __ldg(p + 1);
        a[0] = v0.x; a[1] = v0.y; a[2] = v0.z; a[3] = v0.w; a[4] = v1.x; a[5] = v1.y;
    }
};

__device__ __forceinline__ void mp_decode(const DevComp& c, int ci, int& l, int& m)
{
    if (c.lm_split) {
        l = __ldg(c.lm + ci);
        m = __ldg(c.lm_m + ci);
    } else {
        const int v = __ldg(c.lm + ci);
        l = v >> 16;
        m = (int)(short)(v & 0xffff);
    }
}

// Harmonic sums over c = 1 .. n_lm-1 (c = 0 is the monopole, done in FP64).
template <int MODE, typename R>
__device__ __forceinline__ void mp_harmonics(const DevComp& c, int k, double s_d,
                                             double cth_d, double sth_d,
                                             double cph, double sph, MPSums& tot)
{
    constexpr bool NEED_B = MODE != AGB_MODE_POT;
    constexpr bool NEED_D = MODE == AGB_MODE_HESS || MODE == AGB_MODE_DENS;
    constexpr bool NEED_ANG = MODE == AGB_MODE_GRAD || MODE == AGB_MODE_HESS;
    constexpr bool NEED_ANG2 = MODE == AGB_MODE_HESS;

    const bool near_pole = sth_d < 1.0e-10;
    const R s = (R)s_d;
    const R cth = (R)cth_d;
    const R sth = (R)sth_d;
    const R inv_sth = near_pole ? R(0) : (R)(1.0 / sth_d);
    const R cot = near_pole ? R(0) : (R)(cth_d / sth_d);

    double cm = 1.0, sm = 0.0;        // cos, sin of (cur * phi)
    double sinpow = 1.0, sinpow_m1 = 0.0;
    int cur = 0;
    R Tc = R(1), Ts = R(0);
    R Pp = R(0), Pc = (R)AGB_SEED[0], dPp = R(0), dPc = R(0);
    int lc = 0;

    MPGroup<R> g;
    g.zero();

    for (int ci = 1; ci < c.n_lm; ++ci) {
        int l, m;
        mp_decode(c, ci, l, m);
        const int am = m < 0 ? -m : m;
        // a harmonic outside 0 <= |m| <= l <= 32, or out of the sorted order,
        // cannot be evaluated: skip it rather than index past the tables
        if (l > AGB_MAX_LMAX || am > l || am < cur || (am == cur && l < lc)) continue;
        if (am != cur) {
            mp_flush<MODE, R>(tot, g);
            for (int q = cur; q < am; ++q) {
                const double t = cm * cph - sm * sph;
                sm = sm * cph + cm * sph;
                cm = t;
                sinpow_m1 = sinpow;
                sinpow *= sth_d;
            }
            cur = am;
            Tc = (R)cm;
            Ts = (R)sm;
            Pc = (R)(AGB_SEED[am] * sinpow);
            Pp = R(0);
            dPp = R(0);
            if (NEED_ANG) {
                if (am == 1)
                    dPc = (R)(AGB_SEED[1] * cth_d);
                else
                    dPc = near_pole ? R(0) : (R)((double)am * AGB_SEED[am] * sinpow_m1 * cth_d);
            }
            lc = am;
        }
        while (lc < l) {
            ++lc;
            const int ti = am * AGB_LEG_N + lc;
            const R a = MPConst<R>::alpha(ti);
            const R b = MPConst<R>::beta(ti);
            const R Pn = a * (cth * Pc) - b * Pp;
            if (NEED_ANG) {
                const R dPn = a * (cth * dPc - sth * Pc) - b * dPp;
                dPp = dPc;
                dPc = dPn;
            }
            Pp = Pc;
            Pc = Pn;
        }

        R q[6];
        MPRec<R>::load(c, ci, k, q);
        const R C = fma(s, fma(s, fma(s, fma(s, fma(s, q[5], q[4]), q[3]), q[2]), q[1]), q[0]);
        R dC = R(0), d2C = R(0);
        if (NEED_B)
            dC = fma(s, fma(s, fma(s, fma(s, R(5) * q[5], R(4) * q[4]), R(3) * q[3]), R(2) * q[2]), q[1]);
        if (NEED_D)
            d2C = fma(s, fma(s, fma(s, R(20) * q[5], R(12) * q[4]), R(6) * q[3]), R(2) * q[2]);

        const bool is_cos = m >= 0;
        const R T = is_cos ? Tc : Ts;
        const R YT = Pc * T;
        g.A += C * YT;
        if (NEED_B) g.B += dC * YT;
        if (NEED_D) g.D += d2C * YT;
        if (MODE == AGB_MODE_DENS) g.L += R(l * (l + 1)) * (C * YT);
        if (NEED_ANG) {
            const R dT = is_cos ? -R(am) * Ts : R(am) * Tc;
            g.Th += C * (dPc * T);
            R Pos = R(0);
            if (am != 0) Pos = !near_pole ? Pc * inv_sth : (am == 1 ? dPc : R(0));
            g.Pos += C * (Pos * dT);
            if (NEED_ANG2) {
                const R d2Y = near_pole ? R(0)
                    : (-cot * dPc - (R(l * (l + 1)) - R(am * am) * inv_sth * inv_sth) * Pc);
                g.Thth += C * (d2Y * T);
                g.BTh  += dC * (dPc * T);
                g.Ph   += C * (Pc * dT);
                g.Phph += C * (Pc * (-R(am * am) * T));
                g.BPh  += dC * (Pc * dT);
                g.ThPh += C * (dPc * dT);
            }
        }
    }
    mp_flush<MODE, R>(tot, g);
}

// ---------------------------------------------------------------------------
// Regular column structure (AGB_STRUCT_ALL / AGB_STRUCT_EVEN): every (l, m) up
// to lmax (or every even l) has a column, in (|m|, l, cos, sin) order, so the
// walk needs no harmonic list.  Per |m| group the sums over l are formed
// without cos/sin(m phi): the group's cos-column and sin-column sums are
// multiplied by cos(m phi), sin(m phi) (and their phi derivatives) once, in FP64.
// The quintic is evaluated in the power basis with the powers of s (and the
// derivative weights j s^(j-1), j (j-1) s^(j-2)) formed once per point.
// ---------------------------------------------------------------------------
template <typename R> struct MPPtr;
template <> struct MPPtr<double> {
    static constexpr int REC = 6;
    static __device__ __forceinline__ const double* base(const DevComp& c, int k)
    {
        return c.table + (long long)k * c.n_lm * 6;
    }
    template <bool GEN = false>
    static __device__ __forceinline__ void load(const double* p, double a[6])
    {
        const double2* q = reinterpret_cast<const double2*>(p);
        const double2 v0 = GEN ? q[0] : __ldg(q), v1 = GEN ? q[1] : __ldg(q + 1),
                      v2 = GEN ? q[2] : __ldg(q + 2);
        a[0] = v0.x; a[1] = v0.y; a[2] = v1.x; a[3] = v1.y; a[4] = v2.x; a[5] = v2.y;
    }
    // the cos and sin records of an m>0 harmonic (consecutive columns)
    template <bool GEN = false>
    static __device__ __forceinline__ void load_cs(const double* p, double c[6], double s[6])
    {
        load<GEN>(p, c);
        load<GEN>(p + REC, s);
    }
};
template <> struct MPPtr<float> {
    static constexpr int REC = 8;
    static __device__ __forceinline__ const float* base(const DevComp& c, int k)
    {
        return c.table32 + (long long)k * c.n_lm * 8;
    }
    // GEN: p may point to shared memory (a staged slab): generic loads, not __ldg
    template <bool GEN = false>
    static __device__ __forceinline__ float4 ld4(const float4* q) { return GEN ? *q : __ldg(q); }
    template <bool GEN = false>
    static __device__ __forceinline__ void load(const float* p, float a[6])
    {
        const float4* q = reinterpret_cast<const float4*>(p);
        const float4 v0 = ld4<GEN>(q), v1 = ld4<GEN>(q + 1);
        a[0] = v0.x; a[1] = v0.y; a[2] = v0.z; a[3] = v0.w; a[4] = v1.x; a[5] = v1.y;
    }
    // an m>0 harmonic's cos and sin records, stored interleaved in the FP32
    // table of a regular structure: c0 s0 c1 s1 ... c5 s5 (+4 pads)
    template <bool GEN = false>
    static __device__ __forceinline__ void load_cs(const float* p, float c[6], float s[6])
    {
        const float4* q = reinterpret_cast<const float4*>(p);
        const float4 v0 = ld4<GEN>(q), v1 = ld4<GEN>(q + 1), v2 = ld4<GEN>(q + 2);
        c[0] = v0.x; s[0] = v0.y; c[1] = v0.z; s[1] = v0.w;
        c[2] = v1.x; s[2] = v1.y; c[3] = v1.z; s[3] = v1.w;
        c[4] = v2.x; s[4] = v2.y; c[5] = v2.z; s[5] = v2.w;
    }
};

template <typename R> struct MPCol {         // per-group sums of one trig column (cos or sin)
    R V, VR, VRR, VT, VTT, VRT, VP, L;
    __device__ __forceinline__ void zero() { V = VR = VRR = VT = VTT = VRT = VP = L = R(0); }
};

// Per l the walk accumulates C*Y, C'*Y, C*dY (and C''*Y, C'*dY, l(l+1) C*Y for
// the second derivatives); the two angular sums that need Y/sin(theta) and
// d2Y/dtheta2 follow from those once per |m| group, because inside a group
//   Y/sin         = Y inv_sth + q1 dY              (q1: the m=1 pole rule)
//   d2Y/dtheta2   = np1 (-cot dY - (l(l+1) - m^2/sin^2) Y)
// (the Legendre equation) have coefficients that do not depend on l.
template <int MODE, typename R>
__device__ __forceinline__ void mp_col_acc(MPCol<R>& g, const R a[6], const R sp[6],
                                           const R dw[6], const R ew[6], R Y, R dY, R ll1)
{
    constexpr bool NEED_B = MODE != AGB_MODE_POT;
    constexpr bool NEED_D = MODE == AGB_MODE_HESS || MODE == AGB_MODE_DENS;
    constexpr bool NEED_ANG = MODE == AGB_MODE_GRAD || MODE == AGB_MODE_HESS;
    // C = sum a_j s^j.  FP32: one Horner pass carries C, C' and C''/2 together
    // (5 + 4 + 3 FMAs against 5 + 5 + 5 for separate sums); the C''/2 sum is doubled
    // once per group in mp_col_finish.  FP64: two short chains per sum, where the
    // longer dependent DFMA chain costs more than it saves
    R C, dC = R(0), d2C = R(0);
    if (std::is_same<R, float>::value) {
        const R x = sp[1];
        R p = fma(a[5], x, a[4]), d = a[5], e = a[5];
        d = fma(d, x, p); p = fma(p, x, a[3]);
        if (NEED_D) e = fma(e, x, d);
        d = fma(d, x, p); p = fma(p, x, a[2]);
        if (NEED_D) e = fma(e, x, d);
        d = fma(d, x, p); p = fma(p, x, a[1]);
        if (NEED_D) e = fma(e, x, d);
        d = fma(d, x, p); p = fma(p, x, a[0]);
        C = p;
        dC = d;
        d2C = e;
    } else {
        C = fma(a[2], sp[2], fma(a[1], sp[1], a[0])) + fma(a[5], sp[5], fma(a[4], sp[4], a[3] * sp[3]));
        if (NEED_B) dC = fma(a[2], dw[2], a[1]) + fma(a[5], dw[5], fma(a[4], dw[4], a[3] * dw[3]));
        if (NEED_D) d2C = fma(a[3], ew[3], R(2) * a[2]) + fma(a[5], ew[5], a[4] * ew[4]);
    }
    g.V = fma(C, Y, g.V);
    if (NEED_B) {
        g.VR = fma(dC, Y, g.VR);
        if (MODE == AGB_MODE_HESS) g.VRT = fma(dC, dY, g.VRT);
    }
    if (NEED_D) g.VRR = fma(d2C, Y, g.VRR);
    if (MODE == AGB_MODE_DENS || MODE == AGB_MODE_HESS) g.L = fma(ll1 * C, Y, g.L);
    if (NEED_ANG) g.VT = fma(C, dY, g.VT);
}

// the group's Y/sin and d2Y/dtheta2 sums from its accumulators (see above)
template <int MODE, typename R>
__device__ __forceinline__ void mp_col_finish(MPCol<R>& g, R inv_sth, R q1, R np1, R cot, R m2)
{
    if (MODE == AGB_MODE_GRAD || MODE == AGB_MODE_HESS) g.VP = fma(g.V, inv_sth, q1 * g.VT);
    if (MODE == AGB_MODE_HESS) g.VTT = np1 * (fma(-cot, g.VT, m2 * g.V) - g.L);
    if ((MODE == AGB_MODE_HESS || MODE == AGB_MODE_DENS) && std::is_same<R, float>::value)
        g.VRR *= R(2);                                          // the FP32 walk sums C''/2
}

// GEN: the interval's records come from `slab` (this interval's row of a staged
// copy of the FP32 table, possibly in shared memory) instead of the table itself
template <int MODE, typename R, int PAR, bool GEN = false>
__device__ __forceinline__ void mp_harmonics_reg(const DevComp& c, int k, double s_d,
                                                 double cth_d, double sth_d,
                                                 double cph, double sph, MPSums& tot,
                                                 const R* slab = nullptr)
{
    constexpr bool NEED_ANG = MODE == AGB_MODE_GRAD || MODE == AGB_MODE_HESS;
    constexpr bool NEED_ANG2 = MODE == AGB_MODE_HESS;
    const bool near_pole = sth_d < 1.0e-10;
    const R s = (R)s_d;
    R sp[6], dw[6], ew[6];
    sp[0] = R(1); sp[1] = s; sp[2] = s * s; sp[3] = sp[2] * s; sp[4] = sp[2] * sp[2]; sp[5] = sp[4] * s;
    dw[0] = R(0); dw[1] = R(1); dw[2] = R(2) * s; dw[3] = R(3) * sp[2]; dw[4] = R(4) * sp[3]; dw[5] = R(5) * sp[4];
    ew[0] = R(0); ew[1] = R(0); ew[2] = R(2); ew[3] = R(6) * s; ew[4] = R(12) * sp[2]; ew[5] = R(20) * sp[3];
    const R cth = (R)cth_d, sth = (R)sth_d;
    const R c2 = (R)(cth_d * cth_d), w2 = (R)(-2.0 * cth_d * sth_d);   // two-step walk
    const R inv_sth = near_pole ? R(0) : (R)(1.0 / sth_d);
    const R cot = near_pole ? R(0) : (R)(cth_d / sth_d);
    const R np1 = near_pole ? R(0) : R(1);
    const int lmax = c.lmax;
    // column 1 (column 0 = monopole)
    const R* rec = (GEN ? slab : MPPtr<R>::base(c, k)) + MPPtr<R>::REC;

    double cm = 1.0, sm = 0.0, sinpow = 1.0, sinpow_m1 = 0.0;
    for (int m = 0; m <= lmax; ++m) {
        if (m > 0) {
            const double t = cm * cph - sm * sph;
            sm = sm * cph + cm * sph;
            cm = t;
            sinpow_m1 = sinpow;
            sinpow *= sth_d;
        }
        int l0 = (PAR == 2) ? (m + (m & 1)) : m;
        if (m == 0) l0 = PAR;                                   // column 0 is the monopole
        if (l0 > lmax) continue;
        const R q1 = (near_pole && m == 1) ? R(1) : R(0);       // pole rule for Y/sin(theta)
        const R m2 = R(m * m) * inv_sth * inv_sth;
        R Pc = (R)(AGB_SEED[m] * sinpow), Pp = R(0), dPc = R(0), dPp = R(0);
        if (NEED_ANG && m > 0)
            dPc = (m == 1) ? (R)(AGB_SEED[1] * cth_d)
                           : (near_pole ? R(0) : (R)((double)m * AGB_SEED[m] * sinpow_m1 * cth_d));
        MPCol<R> gc, gs;
        gc.zero();
        gs.zero();
        const int tb = m * AGB_LEG_N;
        // rescaled recurrence (Q_l = Ybar_l / C_l, the C_l folded into the regular
        // tables): Q_l = cos Q_{l-1} - betaq Q_{l-2}, dQ_l = cos dQ_{l-1} - sin Q_{l-1} - betaq dQ_{l-2}
        auto step = [&](int L) {
            const R nb = MPConst<R>::nbetaq(tb + L);
            const R Pn = fma(cth, Pc, nb * Pp);
            if (NEED_ANG) {
                const R dPn = fma(cth, dPc, fma(-sth, Pc, nb * dPp));
                dPp = dPc;
                dPc = dPn;
            }
            Pp = Pc;
            Pc = Pn;
        };
        // one l: both trig columns' records are loaded before any arithmetic so
        // the loads of a loop body issue together (no branch inside the body)
        auto acc = [&](int L, auto has_sin) {
            R ac[6], as[6];
            if (has_sin) MPPtr<R>::template load_cs<GEN>(rec, ac, as);
            else MPPtr<R>::template load<GEN>(rec, ac);
            rec += has_sin ? 2 * MPPtr<R>::REC : MPPtr<R>::REC;
            const R ll1 = R(L * (L + 1));
            mp_col_acc<MODE, R>(gc, ac, sp, dw, ew, Pc, dPc, ll1);
            if (has_sin) mp_col_acc<MODE, R>(gs, as, sp, dw, ew, Pc, dPc, ll1);
        };
        // even l only: Q_l = (cos^2 + A_l) Q_{l-2} + B_l Q_{l-4} (one step per stored l)
        const int ts = m * AGB_SKIP_N;
        auto skip2 = [&](int L) {
            const auto ab = MPConst<R>::skip(ts + (L >> 1));
            const R t = c2 + (R)ab.x;
            const R Pn = fma(t, Pc, (R)ab.y * Pp);
            if (NEED_ANG) {
                const R dPn = fma(w2, Pc, fma(t, dPc, (R)ab.y * dPp));
                dPp = dPc;
                dPc = dPn;
            }
            Pp = Pc;
            Pc = Pn;
        };
        const R seed = Pc;
        auto walk = [&](auto has_sin) {
            int l = m;
            while (l < l0) step(++l);
            acc(l, has_sin);
            if (PAR == 2) {
                // the two-step state (Q_l0, Q_l0-2): Q_0 for m = 0, zero otherwise
                Pp = (m == 0) ? seed : R(0);
                dPp = R(0);
                #pragma unroll 4
                for (l = l0 + 2; l <= lmax; l += 2) {
                    skip2(l);
                    acc(l, has_sin);
                }
            } else {
                #pragma unroll 4
                for (l = l0 + 1; l <= lmax; ++l) {
                    step(l);
                    acc(l, has_sin);
                }
            }
        };
        if (m == 0) walk(std::false_type());
        else walk(std::true_type());
        mp_col_finish<MODE, R>(gc, inv_sth, q1, np1, cot, m2);
        mp_col_finish<MODE, R>(gs, inv_sth, q1, np1, cot, m2);
        // combine the group's cos and sin sums with cos/sin(m phi) in FP64
        const double md = (double)m;
        const double dTc = -md * sm, dTs = md * cm;
        tot.A += (double)gc.V * cm + (double)gs.V * sm;
        if (MODE != AGB_MODE_POT) tot.B += (double)gc.VR * cm + (double)gs.VR * sm;
        if (MODE == AGB_MODE_HESS || MODE == AGB_MODE_DENS)
            tot.D += (double)gc.VRR * cm + (double)gs.VRR * sm;
        if (MODE == AGB_MODE_DENS) tot.L += (double)gc.L * cm + (double)gs.L * sm;
        if (NEED_ANG) {
            tot.Th += (double)gc.VT * cm + (double)gs.VT * sm;
            tot.Pos += (double)gc.VP * dTc + (double)gs.VP * dTs;
        }
        if (NEED_ANG2) {
            tot.Thth += (double)gc.VTT * cm + (double)gs.VTT * sm;
            tot.BTh += (double)gc.VRT * cm + (double)gs.VRT * sm;
            tot.Ph += (double)gc.V * dTc + (double)gs.V * dTs;
            tot.Phph += -md * md * ((double)gc.V * cm + (double)gs.V * sm);
            tot.BPh += (double)gc.VR * dTc + (double)gs.VR * dTs;
            tot.ThPh += (double)gc.VT * dTc + (double)gs.VT * dTs;
        }
    }
}

// The same walk for two tables with one column structure, lmax and radial grid (the
// two bracketing snapshots of an Evolving potential): the geometry, the Legendre and
// m-phi recurrences are shared, each table keeps its own sums.  Per table the
// arithmetic is that of mp_harmonics_reg.
template <int MODE, typename R, int PAR>
__device__ __forceinline__ void mp_harmonics_reg2(const DevComp& c1, const DevComp& c2, int k,
                                                  double s_d, double cth_d, double sth_d,
                                                  double cph, double sph, MPSums& tot1,
                                                  MPSums& tot2)
{
    constexpr bool NEED_ANG = MODE == AGB_MODE_GRAD || MODE == AGB_MODE_HESS;
    constexpr bool NEED_ANG2 = MODE == AGB_MODE_HESS;
    const bool near_pole = sth_d < 1.0e-10;
    const R s = (R)s_d;
    R sp[6], dw[6], ew[6];
    sp[0] = R(1); sp[1] = s; sp[2] = s * s; sp[3] = sp[2] * s; sp[4] = sp[2] * sp[2]; sp[5] = sp[4] * s;
    dw[0] = R(0); dw[1] = R(1); dw[2] = R(2) * s; dw[3] = R(3) * sp[2]; dw[4] = R(4) * sp[3]; dw[5] = R(5) * sp[4];
    ew[0] = R(0); ew[1] = R(0); ew[2] = R(2); ew[3] = R(6) * s; ew[4] = R(12) * sp[2]; ew[5] = R(20) * sp[3];
    const R cth = (R)cth_d, sth = (R)sth_d;
    const R cc2 = (R)(cth_d * cth_d), w2 = (R)(-2.0 * cth_d * sth_d);
    const R inv_sth = near_pole ? R(0) : (R)(1.0 / sth_d);
    const R cot = near_pole ? R(0) : (R)(cth_d / sth_d);
    const R np1 = near_pole ? R(0) : R(1);
    const int lmax = c1.lmax;
    const R* rec1 = MPPtr<R>::base(c1, k) + MPPtr<R>::REC;
    const R* rec2 = MPPtr<R>::base(c2, k) + MPPtr<R>::REC;

    double cm = 1.0, sm = 0.0, sinpow = 1.0, sinpow_m1 = 0.0;
    for (int m = 0; m <= lmax; ++m) {
        if (m > 0) {
            const double t = cm * cph - sm * sph;
            sm = sm * cph + cm * sph;
            cm = t;
            sinpow_m1 = sinpow;
            sinpow *= sth_d;
        }
        int l0 = (PAR == 2) ? (m + (m & 1)) : m;
        if (m == 0) l0 = PAR;
        if (l0 > lmax) continue;
        const R q1 = (near_pole && m == 1) ? R(1) : R(0);
        const R m2 = R(m * m) * inv_sth * inv_sth;
        R Pc = (R)(AGB_SEED[m] * sinpow), Pp = R(0), dPc = R(0), dPp = R(0);
        if (NEED_ANG && m > 0)
            dPc = (m == 1) ? (R)(AGB_SEED[1] * cth_d)
                           : (near_pole ? R(0) : (R)((double)m * AGB_SEED[m] * sinpow_m1 * cth_d));
        MPCol<R> gc1, gs1, gc2, gs2;
        gc1.zero(); gs1.zero(); gc2.zero(); gs2.zero();
        const int tb = m * AGB_LEG_N;
        auto step = [&](int L) {
            const R nb = MPConst<R>::nbetaq(tb + L);
            const R Pn = fma(cth, Pc, nb * Pp);
            if (NEED_ANG) {
                const R dPn = fma(cth, dPc, fma(-sth, Pc, nb * dPp));
                dPp = dPc;
                dPc = dPn;
            }
            Pp = Pc;
            Pc = Pn;
        };
        auto acc = [&](int L, auto has_sin) {
            R ac1[6], as1[6], ac2[6], as2[6];
            if (has_sin) {
                MPPtr<R>::load_cs(rec1, ac1, as1);
                MPPtr<R>::load_cs(rec2, ac2, as2);
            } else {
                MPPtr<R>::load(rec1, ac1);
                MPPtr<R>::load(rec2, ac2);
            }
            rec1 += has_sin ? 2 * MPPtr<R>::REC : MPPtr<R>::REC;
            rec2 += has_sin ? 2 * MPPtr<R>::REC : MPPtr<R>::REC;
            const R ll1 = R(L * (L + 1));
            mp_col_acc<MODE, R>(gc1, ac1, sp, dw, ew, Pc, dPc, ll1);
            mp_col_acc<MODE, R>(gc2, ac2, sp, dw, ew, Pc, dPc, ll1);
            if (has_sin) {
                mp_col_acc<MODE, R>(gs1, as1, sp, dw, ew, Pc, dPc, ll1);
                mp_col_acc<MODE, R>(gs2, as2, sp, dw, ew, Pc, dPc, ll1);
            }
        };
        const int ts = m * AGB_SKIP_N;
        auto skip2 = [&](int L) {
            const auto ab = MPConst<R>::skip(ts + (L >> 1));
            const R t = cc2 + (R)ab.x;
            const R Pn = fma(t, Pc, (R)ab.y * Pp);
            if (NEED_ANG) {
                const R dPn = fma(w2, Pc, fma(t, dPc, (R)ab.y * dPp));
                dPp = dPc;
                dPc = dPn;
            }
            Pp = Pc;
            Pc = Pn;
        };
        const R seed = Pc;
        auto walk = [&](auto has_sin) {
            int l = m;
            while (l < l0) step(++l);
            acc(l, has_sin);
            if (PAR == 2) {
                Pp = (m == 0) ? seed : R(0);
                dPp = R(0);
                #pragma unroll 2
                for (l = l0 + 2; l <= lmax; l += 2) {
                    skip2(l);
                    acc(l, has_sin);
                }
            } else {
                #pragma unroll 2
                for (l = l0 + 1; l <= lmax; ++l) {
                    step(l);
                    acc(l, has_sin);
                }
            }
        };
        if (m == 0) walk(std::false_type());
        else walk(std::true_type());
        const double md = (double)m;
        const double dTc = -md * sm, dTs = md * cm;
        auto combine = [&](MPSums& tot, MPCol<R>& gc, MPCol<R>& gs) {
            mp_col_finish<MODE, R>(gc, inv_sth, q1, np1, cot, m2);
            mp_col_finish<MODE, R>(gs, inv_sth, q1, np1, cot, m2);
            tot.A += (double)gc.V * cm + (double)gs.V * sm;
            if (MODE != AGB_MODE_POT) tot.B += (double)gc.VR * cm + (double)gs.VR * sm;
            if (MODE == AGB_MODE_HESS || MODE == AGB_MODE_DENS)
                tot.D += (double)gc.VRR * cm + (double)gs.VRR * sm;
            if (MODE == AGB_MODE_DENS) tot.L += (double)gc.L * cm + (double)gs.L * sm;
            if (NEED_ANG) {
                tot.Th += (double)gc.VT * cm + (double)gs.VT * sm;
                tot.Pos += (double)gc.VP * dTc + (double)gs.VP * dTs;
            }
            if (NEED_ANG2) {
                tot.Thth += (double)gc.VTT * cm + (double)gs.VTT * sm;
                tot.BTh += (double)gc.VRT * cm + (double)gs.VRT * sm;
                tot.Ph += (double)gc.V * dTc + (double)gs.V * dTs;
                tot.Phph += -md * md * ((double)gc.V * cm + (double)gs.V * sm);
                tot.BPh += (double)gc.VR * dTc + (double)gs.VR * dTs;
                tot.ThPh += (double)gc.VT * dTc + (double)gs.VT * dTs;
            }
        };
        combine(tot1, gc1, gs1);
        combine(tot2, gc2, gs2);
    }
}

__device__ __forceinline__ void mp_quintic0(const DevComp& c, int k, double s,
                                            double& v, double& d1, double& d2)
{
    double q[6];
    MPRec<double>::load(c, 0, k, q);
    v = fma(s, fma(s, fma(s, fma(s, fma(s, q[5], q[4]), q[3]), q[2]), q[1]), q[0]);
    d1 = fma(s, fma(s, fma(s, fma(s, 5.0 * q[5], 4.0 * q[4]), 3.0 * q[3]), 2.0 * q[2]), q[1]);
    d2 = fma(s, fma(s, fma(s, 20.0 * q[5], 12.0 * q[4]), 6.0 * q[3]), 2.0 * q[2]);
}

// l=0 power-law extrapolation written as Phi(log r) with its two log-r derivatives.
__device__ __forceinline__ void mp_extrap_out(int MODE_, double p0, double d1, double d2,
                                              double px, double py, double pz, double r2,
                                              PointOut& o)
{
    const double MP0 = AGB_MUL0 * AGB_PREFACT[0];
    const double inv_r2 = 1.0 / r2;
    o.phi = MP0 * p0;
    if (MODE_ == AGB_MODE_GRAD || MODE_ == AGB_MODE_HESS) {
        const double gg = MP0 * d1;
        o.g[0] = gg * (px * inv_r2);
        o.g[1] = gg * (py * inv_r2);
        o.g[2] = gg * (pz * inv_r2);
    }
    if (MODE_ == AGB_MODE_HESS) {
        const double A = MP0 * (d2 - d1) * inv_r2 * inv_r2;
        const double B = MP0 * d1 * inv_r2;
        hess_radial(A, B, px, py, pz, o.h);
    }
}

// Phi, gradient, Hessian or density of one Multipole point from its harmonic
// sums, the log-scaling factor F(log r) with its log-r derivatives, the
// monopole terms and the point's geometry (the conversion of
// _multipole_potential_kernel.cu:388-409 and :713-799).
template <int MODE>
__device__ __forceinline__ void mp_finish(const MPSums& t, double inv_dlogr, double F, double dF,
                                          double d2F, double mono, double dmono, double d2mono,
                                          double px, double py, double pz, double inv_r,
                                          double Rc, double cth, double sth, double cph,
                                          double sph, PointOut& o)
{
    const double Bp = t.B * inv_dlogr;
    const double Dp = t.D * inv_dlogr * inv_dlogr;
    o.phi = mono + F * t.A;
    if (MODE == AGB_MODE_POT) return;

    const double Pr = dmono + F * Bp + dF * t.A;
    if (MODE == AGB_MODE_DENS) {
        const double inv_r2 = inv_r * inv_r;
        const double lap = (d2mono + dmono) * inv_r2
            + (F * (Dp + Bp - t.L) + dF * (2.0 * Bp + t.A) + d2F * t.A) * inv_r2;
        o.rho = lap * AGB_INV_4PIG;
        return;
    }
    const double Pth = F * t.Th;
    const double Pos = F * t.Pos;
    const double inv_r2 = inv_r * inv_r;
    o.g[0] = Pr * (px * inv_r2) + Pth * (cth * cph * inv_r) + Pos * (-sph * inv_r);
    o.g[1] = Pr * (py * inv_r2) + Pth * (cth * sph * inv_r) + Pos * (cph * inv_r);
    o.g[2] = Pr * (pz * inv_r2) + Pth * (-sth * inv_r);
    if (MODE != AGB_MODE_HESS) return;

    // second derivatives in (log r, theta, phi)
    const double Prr = d2mono + F * Dp + 2.0 * dF * Bp + d2F * t.A;
    const double Pthth = F * t.Thth;
    const double Prth = F * (t.BTh * inv_dlogr) + dF * t.Th;
    const double Pph = F * t.Ph;
    const double Pphph = F * t.Phph;
    const double Prph = F * (t.BPh * inv_dlogr) + dF * t.Ph;
    const double Pthph = F * t.ThPh;

    // first and second derivatives of (log r, theta, phi) w.r.t. x, y, z
    const double inv_R = (Rc > 1.0e-300) ? 1.0 / Rc : 0.0;
    const double X[3] = {px, py, pz};
    const double dlr[3] = {px * inv_r2, py * inv_r2, pz * inv_r2};
    const double dth[3] = {cth * cph * inv_r, cth * sph * inv_r, -sth * inv_r};
    const double dph[3] = {-sph * inv_R, cph * inv_R, 0.0};
    const double inv_r3 = inv_r2 * inv_r, inv_r4 = inv_r2 * inv_r2, inv_r5 = inv_r4 * inv_r;
    const double inv_s = (sth > 1.0e-14) ? 1.0 / sth : 0.0;
    const double cos3 = cth * inv_s * inv_s * inv_s;
    // f = cos(theta) = z / r
    const double df[3] = {-pz * px * inv_r3, -pz * py * inv_r3, inv_r - pz * pz * inv_r3};
    double d2ph_xx = 0.0, d2ph_xy = 0.0, d2ph_yy = 0.0;
    if (Rc > 1.0e-14) {
        const double iR4 = inv_R * inv_R * inv_R * inv_R;
        d2ph_xx = 2.0 * px * py * iR4;
        d2ph_xy = (py * py - px * px) * iR4;
        d2ph_yy = -2.0 * px * py * iR4;
    }
    #pragma unroll
    for (int p = 0; p < 6; ++p) {
        const int i = hess_i(p), j = hess_j(p);
        const double dij = (i == j) ? 1.0 : 0.0;
        const double d2lr = dij * inv_r2 - 2.0 * X[i] * X[j] * inv_r4;
        // d2 f / dx_i dx_j = -(delta_ij z + delta_iz x_j + delta_jz x_i)/r^3 + 3 z x_i x_j / r^5
        const double d2f = -(dij * pz + (i == 2 ? X[j] : 0.0) + (j == 2 ? X[i] : 0.0)) * inv_r3
                         + 3.0 * pz * X[i] * X[j] * inv_r5;
        const double d2th = -d2f * inv_s - df[i] * df[j] * cos3;
        double d2ph = 0.0;
        if (p == 0) d2ph = d2ph_xx;
        else if (p == 1) d2ph = d2ph_yy;
        else if (p == 3) d2ph = d2ph_xy;
        o.h[p] = Prr * dlr[i] * dlr[j]
               + Prth * (dlr[i] * dth[j] + dlr[j] * dth[i])
               + Prph * (dlr[i] * dph[j] + dlr[j] * dph[i])
               + Pthth * dth[i] * dth[j]
               + Pthph * (dth[i] * dph[j] + dth[j] * dph[i])
               + Pphph * dph[i] * dph[j]
               + Pr * d2lr + Pth * d2th + Pph * d2ph;
    }
}

// STAGED: the records of intervals [k0, k1] are also in `slab` (a staged copy of
// those rows of the FP32 table, in shared memory): a point in that range reads them
// there (FP32 walks of regular structures; other points read the table)
template <int MODE, typename R, bool STAGED = false>
__device__ __forceinline__ void multipole_point(const DevComp& c, double px, double py,
                                                double pz, PointOut& o,
                                                const float* slab = nullptr, int k0 = 0,
                                                int k1 = -1)
{
    const double logr_min = c.p[0], dlogr = c.p[1], inv_dlogr = c.p[2], invPhi0 = c.p[3];
    const double in_s = c.p[4], in_U = c.p[5], in_W = c.p[6];
    const double out_s = c.p[7], out_U = c.p[8], out_W = c.p[9];
    const double MP0 = AGB_MUL0 * AGB_PREFACT[0];

    const double r2 = px * px + py * py + pz * pz;
    const double r = sqrt(r2);
    const double Rc = sqrt(px * px + py * py);

    if (r < 1.0e-300) {                          // origin: Phi = W, zero derivatives
        o.phi = (MODE == AGB_MODE_DENS) ? 0.0 : MP0 * in_W;
        o.g[0] = o.g[1] = o.g[2] = 0.0;
        for (int p = 0; p < 6; ++p) o.h[p] = 0.0;
        o.rho = 0.0;
        return;
    }
    const double logr = log(r);

    if (logr < logr_min) {                       // inner l=0 power law
        const double dlr = logr - logr_min;
        const double rs = (in_s != 0.0) ? exp(in_s * dlr) : 1.0;
        const double p0 = in_U * rs + in_W;
        const double d1 = in_U * in_s * rs;
        const double d2 = in_U * in_s * in_s * rs;
        if (MODE == AGB_MODE_DENS) {
            o.rho = MP0 * ((d2 + d1) / (r * r)) * AGB_INV_4PIG;
            return;
        }
        mp_extrap_out(MODE, p0, d1, d2, px, py, pz, r2, o);
        return;
    }
    int k = (int)((logr - logr_min) * inv_dlogr);
    if (k < 0) k = 0;
    if (k >= c.n_int) {                          // outer l=0 power law
        if (MODE == AGB_MODE_DENS) { o.rho = 0.0; return; }
        const double dlr = logr - (logr_min + c.n_int * dlogr);
        const double en = exp(-dlr);
        const double es = exp(out_s * dlr);
        const double p0 = out_W * en + out_U * es;
        const double d1 = -out_W * en + out_s * out_U * es;
        const double d2 = out_W * en + out_s * out_s * out_U * es;
        mp_extrap_out(MODE, p0, d1, d2, px, py, pz, r2, o);
        return;
    }
    double s = (logr - (logr_min + k * dlogr)) * inv_dlogr;
    s = fmin(fmax(s, 0.0), 1.0);

    const double inv_r = 1.0 / r;
    const double cth = pz * inv_r;
    const double sth = Rc * inv_r;
    const double cph = (Rc > 1.0e-300) ? px / Rc : 1.0;
    const double sph = (Rc > 1.0e-300) ? py / Rc : 0.0;

    MPSums t = {};
    bool staged = false;
    if constexpr (STAGED && std::is_same<R, float>::value) {
        if (k >= k0 && k <= k1 && c.structure != AGB_STRUCT_LIST) {
            const float* row = slab + (long long)(k - k0) * c.n_lm * 8;
            if (c.structure == AGB_STRUCT_EVEN)
                mp_harmonics_reg<MODE, R, 2, true>(c, k, s, cth, sth, cph, sph, t, row);
            else
                mp_harmonics_reg<MODE, R, 1, true>(c, k, s, cth, sth, cph, sph, t, row);
            staged = true;
        }
    }
    if (!staged) {
        if (c.structure == AGB_STRUCT_EVEN)
            mp_harmonics_reg<MODE, R, 2>(c, k, s, cth, sth, cph, sph, t);
        else if (c.structure == AGB_STRUCT_ALL)
            mp_harmonics_reg<MODE, R, 1>(c, k, s, cth, sth, cph, sph, t);
        else
            mp_harmonics<MODE, R>(c, k, s, cth, sth, cph, sph, t);
    }

    // monopole (FP64) and the log-scaling factor F(log r) with derivatives, after the
    // walk so that its values are not live across it (FP64 kernel 7.22 -> 6.96 ms)
    double c0, c0s, c0ss;
    mp_quintic0(c, k, s, c0, c0s, c0ss);
    const double dc0 = c0s * inv_dlogr;
    const double d2c0 = c0ss * inv_dlogr * inv_dlogr;
    double F = 1.0, dF = 0.0, d2F = 0.0, mono, dmono, d2mono;
    if (c.log_scaling) {
        const double ex = exp(c0);
        const double P0 = 1.0 / (invPhi0 - ex);
        const double dPdX = P0 * P0 * ex;
        F = P0;
        dF = dPdX * dc0;
        d2F = dPdX * (d2c0 + dc0 * dc0 * P0 * (invPhi0 + ex));
        mono = MP0 * F; dmono = MP0 * dF; d2mono = MP0 * d2F;
    } else {
        mono = MP0 * c0; dmono = MP0 * dc0; d2mono = MP0 * d2c0;
    }

    mp_finish<MODE>(t, inv_dlogr, F, dF, d2F, mono, dmono, d2mono, px, py, pz, inv_r, Rc,
                    cth, sth, cph, sph, o);
}

// Two Multipoles on one radial grid and column structure at the same point (the two
// bracketing snapshots of an Evolving potential, same transform): one geometry and one
// shared walk (mp_harmonics_reg2); each keeps its monopole, log-scaling and
// extrapolation.  Off the grid each is evaluated alone.
template <int MODE, typename R>
__device__ __forceinline__ void multipole_pair_point(const DevComp& c1, const DevComp& c2,
                                                     double px, double py, double pz,
                                                     PointOut& o1, PointOut& o2)
{
    const double logr_min = c1.p[0], dlogr = c1.p[1], inv_dlogr = c1.p[2];
    const double MP0 = AGB_MUL0 * AGB_PREFACT[0];
    const double r2 = px * px + py * py + pz * pz;
    const double r = sqrt(r2);
    const double logr = r < 1.0e-300 ? 0.0 : log(r);
    const int kk = r < 1.0e-300 || logr < logr_min ? -1 : (int)((logr - logr_min) * inv_dlogr);
    if (kk < 0 || kk >= c1.n_int) {
        multipole_point<MODE, R>(c1, px, py, pz, o1);
        multipole_point<MODE, R>(c2, px, py, pz, o2);
        return;
    }
    const int k = kk;
    const double Rc = sqrt(px * px + py * py);
    double s = (logr - (logr_min + k * dlogr)) * inv_dlogr;
    s = fmin(fmax(s, 0.0), 1.0);
    const double inv_r = 1.0 / r;
    const double cth = pz * inv_r;
    const double sth = Rc * inv_r;
    const double cph = (Rc > 1.0e-300) ? px / Rc : 1.0;
    const double sph = (Rc > 1.0e-300) ? py / Rc : 0.0;
    MPSums t1 = {}, t2 = {};
    if (c1.structure == AGB_STRUCT_EVEN)
        mp_harmonics_reg2<MODE, R, 2>(c1, c2, k, s, cth, sth, cph, sph, t1, t2);
    else
        mp_harmonics_reg2<MODE, R, 1>(c1, c2, k, s, cth, sth, cph, sph, t1, t2);
    auto finish = [&](const DevComp& c, const MPSums& t, PointOut& o) {
        const double invPhi0 = c.p[3];
        double c0, c0s, c0ss;
        mp_quintic0(c, k, s, c0, c0s, c0ss);
        const double dc0 = c0s * inv_dlogr;
        const double d2c0 = c0ss * inv_dlogr * inv_dlogr;
        double F = 1.0, dF = 0.0, d2F = 0.0, mono, dmono, d2mono;
        if (c.log_scaling) {
            const double ex = exp(c0);
            const double P0 = 1.0 / (invPhi0 - ex);
            const double dPdX = P0 * P0 * ex;
            F = P0;
            dF = dPdX * dc0;
            d2F = dPdX * (d2c0 + dc0 * dc0 * P0 * (invPhi0 + ex));
            mono = MP0 * F; dmono = MP0 * dF; d2mono = MP0 * d2F;
        } else {
            mono = MP0 * c0; dmono = MP0 * dc0; d2mono = MP0 * d2c0;
        }
        mp_finish<MODE>(t, inv_dlogr, F, dF, d2F, mono, dmono, d2mono, px, py, pz, inv_r, Rc,
                        cth, sth, cph, sph, o);
    };
    finish(c1, t1, o1);
    finish(c2, t2, o2);
}
