"""Host preprocessing of a CylSpline expansion into bicubic node tables.

Restates the reference's builder (gpu_potential.py:943-1253), which replicates
Agama's CylSpline constructor:

* a z >= 0 grid is mirrored to the full range (gpu_potential.py:1168-1190);
* the outer asymptote: an lmax=8 exterior multipole W_lm (r0/r)^(l+1) Y_lm fitted
  by least squares to the grid boundary nodes, per m (gpu_potential.py:1001-1095),
  with the reference's angular basis (legendre.outer_asymptote_basis);
* Rscale = -Mtot/Phi(0,0) from the asymptote's monopole (gpu_potential.py:1192-1207);
* asinh-scaled grids lR = asinh(R/Rscale), lz = asinh(z/Rscale);
* log-scaling when every m=0 node is negative: m=0 stores log(-Phi0), m!=0 store
  Phi_m/Phi0 (gpu_potential.py:1213-1233);
* per-harmonic CubicSpline2d node derivatives (fx, fy, fxy): natural cubic
  splines in lz, splines in lR with zero slope at R=0 and a natural right end
  (gpu_potential.py:1098-1140).

The kernels read a cell-major copy: for cell (iR, iz) and harmonic h the 16
values {fval, fx, fy, fxy} at the corners (lo,lo), (lo,hi), (hi,lo), (hi,hi)
are contiguous (128 bytes), harmonics ordered by (|m|, cos before sin).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
from scipy.interpolate import CubicSpline
from scipy.linalg import lstsq

from .legendre import MUL0, MUL1, outer_asymptote_basis

LMAX_OUTER = 8


@dataclass
class CylSplineTables:
    Rscale: float
    lR_grid: np.ndarray        # (nR,)
    lz_grid: np.ndarray        # (nz,)
    node_arr: np.ndarray       # (n_harm, nR, nz, 4) reference layout, m ascending
    m_arr: np.ndarray          # (n_harm,) int32, ascending
    mmax: int
    log_scaling: int
    W_outer: np.ndarray        # ((LMAX_OUTER+1)^2,)
    r0_outer: float
    lmax_outer: int
    mmax_outer: int

    @property
    def n_harm(self) -> int:
        return int(len(self.m_arr))

    def harmonic_order(self) -> np.ndarray:
        """Harmonic permutation used by the cell-major table: (|m|, cos before sin)."""
        m = self.m_arr.astype(np.int64)
        return np.lexsort((m < 0, np.abs(m)))

    def cell_major(self) -> np.ndarray:
        """((nR-1)*(nz-1)*n_harm*16,) FP64 cell-major node table."""
        order = self.harmonic_order()
        nd = self.node_arr[order]                       # (H, nR, nz, 4)
        H, nR, nz, _ = nd.shape
        corners = [nd[:, :-1, :-1], nd[:, :-1, 1:], nd[:, 1:, :-1], nd[:, 1:, 1:]]
        # (H, nR-1, nz-1, 4 corners, 4 quantities) -> quantities major within a record
        c = np.stack(corners, axis=3)                   # (H, nR-1, nz-1, 4c, 4q)
        c = c.transpose(1, 2, 0, 4, 3)                  # (nR-1, nz-1, H, 4q, 4c)
        return np.ascontiguousarray(c.reshape(-1))

    def cell_major_f32(self) -> np.ndarray:
        """FP32 cell-major records for the mixed-precision kernel, 20 floats (80 bytes)
        per (cell, harmonic): the (lo,lo) corner value f00 as one FP64 in the first 8
        bytes, then f - f00 at the (lo,hi), (hi,lo), (hi,hi) corners, f_R, f_z and
        f_Rz at the four corners (FP32), 3 pads.  Values relative to the corner keep
        FP32's 24 bits for the variation across the cell, which the derivatives need."""
        rec64 = self.cell_major().reshape(-1, 16)
        out = np.zeros((rec64.shape[0], 20), dtype=np.float32)
        out.view(np.float64)[:, 0] = rec64[:, 0]
        out[:, 2:5] = (rec64[:, 1:4] - rec64[:, 0:1]).astype(np.float32)
        out[:, 5:17] = rec64[:, 4:16].astype(np.float32)
        return np.ascontiguousarray(out.reshape(-1))

    def m_sorted(self) -> np.ndarray:
        return np.ascontiguousarray(self.m_arr[self.harmonic_order()].astype(np.int32))


def _boundary_points(R: np.ndarray, z: np.ndarray):
    """Grid-boundary nodes used by the asymptote fit (gpu_potential.py:1032-1047)."""
    nR, nz = len(R), len(z)
    zsym = z[0] == 0
    Rp, zp, iRp, izp = [], [], [], []
    for iR in range(nR - 1):
        Rp.append(R[iR]); zp.append(z[nz - 1]); iRp.append(iR); izp.append(nz - 1)
        if zsym:
            Rp.append(R[iR]); zp.append(-z[nz - 1]); iRp.append(iR); izp.append(nz - 1)
        else:
            Rp.append(R[iR]); zp.append(z[0]); iRp.append(iR); izp.append(0)
    for iz in range(nz):
        Rp.append(R[nR - 1]); zp.append(z[iz]); iRp.append(nR - 1); izp.append(iz)
        if zsym and iz > 0:
            Rp.append(R[nR - 1]); zp.append(-z[iz]); iRp.append(nR - 1); izp.append(iz)
    return (np.array(Rp, dtype=np.float64), np.array(zp, dtype=np.float64),
            np.array(iRp), np.array(izp))


def fit_outer_asymptote(R: np.ndarray, z: np.ndarray, phi: dict, mmax: int,
                        lmax_fit: int = LMAX_OUTER):
    """Least-squares exterior multipole on the grid boundary (Agama determineAsympt)."""
    Rp, zp, iRp, izp = _boundary_points(R, z)
    rp = np.hypot(Rp, zp)
    ct, st = zp / rp, Rp / rp
    r0 = min(float(R[-1]), float(np.max(np.abs(z))))
    W = np.zeros((lmax_fit + 1) ** 2)
    for m in range(-min(lmax_fit, mmax), min(lmax_fit, mmax) + 1):
        if m not in phi:
            continue
        am = abs(m)
        P = outer_asymptote_basis(lmax_fit, am, ct, st)          # (npts, lmax-am+1)
        ls = np.arange(am, lmax_fit + 1)
        M = P * (rp[:, None] / r0) ** (-(ls[None, :] + 1)) * (MUL0 if m == 0 else MUL1)
        rhs = phi[m][iRp, izp]
        sol = lstsq(M, rhs)[0]
        W[ls * (ls + 1) + m] = sol
    if not np.isfinite(W[0]):
        avg = float(np.mean(phi[0][iRp, izp] * rp / r0)) if 0 in phi else 0.0
        W[:] = 0.0
        W[0] = avg
    return W, float(r0)


def _node_derivatives(lR: np.ndarray, lz: np.ndarray, f: np.ndarray) -> np.ndarray:
    """(nR, nz, 4) = {f, df/dlR, df/dlz, d2f/dlR dlz} (Agama CubicSpline2d nodes)."""
    fy = CubicSpline(lz, f, axis=1, bc_type="natural")(lz, 1)
    bc = ((1, np.zeros(f.shape[1])), "natural")
    fx = CubicSpline(lR, f, axis=0, bc_type=bc)(lR, 1)
    fxy = CubicSpline(lR, fy, axis=0, bc_type=bc)(lR, 1)
    return np.stack([f, fx, fy, fxy], axis=-1).astype(np.float64)


def build_cylspline_tables(coefs) -> CylSplineTables:
    R = np.asarray(coefs.R_grid, dtype=np.float64)
    z0 = np.asarray(coefs.z_grid, dtype=np.float64)
    tabs = {int(m): np.asarray(v, dtype=np.float64) for m, v in coefs.phi.items()}
    if 0 not in tabs:
        raise ValueError("CylSpline coefficients need an m=0 harmonic")
    nR = len(R)
    mmax = max(abs(m) for m in tabs)

    if z0[0] == 0:                                   # half-space grid: mirror
        nz0 = len(z0)
        z = np.concatenate([-z0[:0:-1], z0])
        phi = {}
        for m, t in tabs.items():
            full = np.empty((nR, 2 * nz0 - 1))
            full[:, nz0 - 1:] = t
            full[:, :nz0] = t[:, ::-1]
            phi[m] = full
        Phi0 = phi[0][0, nz0 - 1]
    else:
        z = z0
        phi = tabs
        Phi0 = phi[0][0, (len(z) + 1) // 2]

    W, r0 = fit_outer_asymptote(R, z, phi, mmax)
    Mtot = -W[0] * r0 * MUL0
    Rscale = -Mtot / Phi0 if (Phi0 < 0.0 and Mtot > 0.0) else float(R[nR // 2])
    lR = np.arcsinh(R / Rscale)
    lz = np.arcsinh(z / Rscale)
    log_scaling = bool(np.all(phi[0] < 0.0))

    m_values = sorted(phi)
    nodes = []
    for m in m_values:
        f = phi[m]
        if log_scaling:
            f = np.log(-f) if m == 0 else f / phi[0]
        nodes.append(_node_derivatives(lR, lz, f))
    return CylSplineTables(Rscale=float(Rscale), lR_grid=lR, lz_grid=lz,
                           node_arr=np.ascontiguousarray(np.stack(nodes, axis=0)),
                           m_arr=np.array(m_values, dtype=np.int32), mmax=int(mmax),
                           log_scaling=int(log_scaling), W_outer=W, r0_outer=r0,
                           lmax_outer=LMAX_OUTER, mmax_outer=min(LMAX_OUTER, mmax))
