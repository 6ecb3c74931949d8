// cs_grad.cuh -- gradient of a loss with respect to a CylSpline's node table.
//
// Inside the (lR, lz) grid a harmonic's value and its lR / lz derivatives are
// linear in the 16 node values of the point's cell (a tensor product of cubic
// Hermite bases, first along z, then along R).  With cotangents gPhi and gF of
// the potential and force, and the chain through the Fourier sum, the
// log-scaling of m=0 and the cylindrical -> Cartesian conversion of the
// forward (cylspline.cuh), each point adds to every harmonic's cell record
//   dL/dv_j = A_h W_j + B_h W^R_j + C_h W^z_j
// where W, W^R, W^z are the basis weights of node value j in val, d val/dlR and
// d val/dlz, and A_h, B_h, C_h = dL/d(val_h, vR_h, vz_h).  FP64, one thread per
// point, atomic adds into the cell-major gradient [cell][harmonic][16] (the
// layout of the FP64 table; the host folds it onto the nodes).  Points outside
// the grid contribute nothing: the outer asymptote (fitted to the boundary
// nodes) and Rscale are held fixed.
#pragma once
#include "cylspline.cuh"

struct CSGradArgs {
    long long n;
    const double* xyz;
    const double* gphi;       // [N] or null
    const double* gforce;     // [N,3] or null
    double* grad;             // [(nR-1)(nz-1)][n_harm][16], accumulated
    DevComp c;
    DevLeaf leaf;
};

// value and derivative weights of (fl, fh, f1l, f1h) in cs_hermite
__device__ __forceinline__ void cs_basis(double t, double h, double wv[4], double wd[4])
{
    const double T = 1.0 - t, tT = t * T;
    wv[0] = T - (t - T) * tT;
    wv[1] = t + (t - T) * tT;
    wv[2] = T * h * tT;
    wv[3] = -t * h * tT;
    wd[0] = -6.0 * tT / h;
    wd[1] = 6.0 * tT / h;
    wd[2] = T - 3.0 * tT;
    wd[3] = t - 3.0 * tT;
}

__global__ void __launch_bounds__(256)
cs_grad_kernel(const __grid_constant__ CSGradArgs a)
{
    const DevComp& c = a.c;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += stride) {
        const double sg = a.leaf.sigma, A = a.leaf.ampl;
        const double px = sg * a.xyz[3 * i] - a.leaf.g0;
        const double py = sg * a.xyz[3 * i + 1] - a.leaf.g1;
        const double pz = sg * a.xyz[3 * i + 2] - a.leaf.g2;
        const double gp = a.gphi ? a.gphi[i] : 0.0;
        double gf0 = 0.0, gf1 = 0.0, gf2 = 0.0;
        if (a.gforce) { gf0 = a.gforce[3 * i]; gf1 = a.gforce[3 * i + 1]; gf2 = a.gforce[3 * i + 2]; }
        const double Rs = c.p[0];
        const double* __restrict__ lRg = c.grid_a;
        const double* __restrict__ lzg = c.grid_b;
        const int nR = c.n_int, nz = c.nz, H = c.n_lm;
        const double R2 = px * px + py * py;
        const double R = sqrt(R2);
        const double lR = asinh(R / Rs);
        const double lz = asinh(pz / Rs);
        if (!(lR >= __ldg(lRg) && lR <= __ldg(lRg + nR - 1) && lz >= __ldg(lzg) &&
              lz <= __ldg(lzg + nz - 1)))
            continue;
        const double dlRdR = 1.0 / sqrt(R2 + Rs * Rs);
        const double dlzdz = 1.0 / sqrt(pz * pz + Rs * Rs);
        const int iR = cs_cell(lR, lRg, nR), iz = cs_cell(lz, lzg, nz);
        const double lR_lo = __ldg(lRg + iR), hR = __ldg(lRg + iR + 1) - lR_lo;
        const double lz_lo = __ldg(lzg + iz), hz = __ldg(lzg + iz + 1) - lz_lo;
        const double tR = (lR - lR_lo) / hR, tz = (lz - lz_lo) / hz;
        double wRv[4], wRd[4], wZv[4], wZd[4];
        cs_basis(tR, hR, wRv, wRd);
        cs_basis(tz, hz, wZv, wZd);
        const double cph = (R > 0.0) ? px / R : 1.0;
        const double sph = (R > 0.0) ? py / R : 0.0;
        // cotangent weights of P, dP/dlR, dP/dlz, dP/dphi (leaf amplitude and scale folded in)
        const double al = A * gp;
        const double w0 = A * sg * gf0, w1 = A * sg * gf1, w2 = A * sg * gf2;
        double bR = 0.0, bp = 0.0;
        if (R > 1e-30) {
            bR = -dlRdR * (w0 * px + w1 * py) / R;
            bp = -(w1 * px - w0 * py) / R2;
        }
        const double bz = -dlzdz * w2;
        const long long rec0 = ((long long)iR * (nz - 1) + iz) * H;

        // pass 1 (log-scaling only): the forward sums that the m=0 chain needs
        const int ls = c.log_scaling;
        double P0 = 0.0, S = 1.0, f0R = 0.0, f0z = 0.0, Ltot = 0.0;
        if (ls) {
            double f0 = 0.0, S_R = 0.0, S_z = 0.0, S_p = 0.0;
            int cur = 0;
            double cm = 1.0, sm = 0.0;
            for (int h = 0; h < H; ++h) {
                const int m = __ldg(c.lm + h);
                double v[16];
                cs_load(c, h, iR, iz, v);
                double val, vR = 0.0, vRR = 0.0, vz = 0.0, vRz = 0.0, vzz = 0.0;
                cs_bicubic<double, true, false>(v, tR, 1.0 - tR, tR * (1.0 - tR), hR, tz, 1.0 - tz,
                                                tz * (1.0 - tz), hz, val, vR, vRR, vz, vRz, vzz);
                if (m == 0) { f0 = val; f0R = vR; f0z = vz; continue; }
                const int am = m < 0 ? -m : m;
                if (am < cur) { cur = 0; cm = 1.0; sm = 0.0; }
                for (; cur < am; ++cur) {
                    const double t = cm * cph - sm * sph;
                    sm = sm * cph + cm * sph;
                    cm = t;
                }
                const double T = m > 0 ? cm : sm, dT = m > 0 ? -(double)am * sm : (double)am * cm;
                S += val * T; S_R += vR * T; S_z += vz * T; S_p += val * dT;
            }
            P0 = -exp(f0);
            const double P = P0 * S, PR = P0 * S_R + P0 * f0R * S, Pz = P0 * S_z + P0 * f0z * S;
            const double Pp = P0 * S_p;
            Ltot = al * P + bR * PR + bz * Pz + bp * Pp;
        }

        // pass 2: per harmonic, dL/d(val, vR, vz) and the scatter onto its cell record
        int cur = 0;
        double cm = 1.0, sm = 0.0;
        for (int h = 0; h < H; ++h) {
            const int m = __ldg(c.lm + h);
            double T = 1.0, dT = 0.0;
            if (m != 0) {
                const int am = m < 0 ? -m : m;
                if (am < cur) { cur = 0; cm = 1.0; sm = 0.0; }
                for (; cur < am; ++cur) {
                    const double t = cm * cph - sm * sph;
                    sm = sm * cph + cm * sph;
                    cm = t;
                }
                T = m > 0 ? cm : sm;
                dT = m > 0 ? -(double)am * sm : (double)am * cm;
            }
            double Ah, Bh, Ch;
            if (!ls) {
                Ah = al * T + bp * dT; Bh = bR * T; Ch = bz * T;
            } else if (m == 0) {
                Ah = Ltot; Bh = bR * P0 * S; Ch = bz * P0 * S;
            } else {
                Ah = P0 * ((al + bR * f0R + bz * f0z) * T + bp * dT);
                Bh = bR * P0 * T; Ch = bz * P0 * T;
            }
            double* g = a.grad + (rec0 + h) * 16;
            // q: R-node function (f lo, f hi, fx lo, fx hi) with its R-basis role q
            #pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int lo = (q & 1) ? 2 + 4 * (q >> 1) : 4 * (q >> 1);   // 0, 2, 4, 6
                const double aw = Ah * wRv[q] + Bh * wRd[q];     // weight of F_q
                const double cz = Ch * wRv[q];                    // weight of dF_q/dlz
                // z roles: fl = v[lo], fh = v[lo+1], f1l = v[8+lo], f1h = v[9+lo]
                const int js[4] = {lo, lo + 1, 8 + lo, 9 + lo};
                #pragma unroll
                for (int r = 0; r < 4; ++r) {
                    const double gv = aw * wZv[r] + cz * wZd[r];
                    if (gv != 0.0) atomicAdd(g + js[r], gv);
                }
            }
        }
    }
}
