"""Host preprocessing of a Multipole expansion into quintic-spline tables.

Restates the reference's table builder (gpu_potential.py:183-631), which in
turn replicates Agama's MultipoleInterp1d:

* l=0 inner power-law extrapolation U (r/r0)^s + W with s from a Lambert-W
  solve, the constant-density-core test that may override s to 2, and the
  log-scaling constant invPhi0 = 1/W (gpu_potential.py:183-263);
* l=0 outer extrapolation W (r/rN)^-1 + U (r/rN)^s (gpu_potential.py:266-328);
* resampling onto a log-uniform grid with a cubic Hermite spline when the grid
  spacing varies by more than 1e-3 (gpu_potential.py:468-496);
* sort of the harmonics by (|m|, l, cos before sin) and removal of all-zero
  columns (gpu_potential.py:513-537);
* log-scaling: c=0 stores log(invPhi0 - 1/Phi0), c>0 store Phi_c/Phi0
  (gpu_potential.py:539-570);
* quintic C2 spline: the tridiagonal system for second derivatives with zero
  fourth derivative at both ends (gpu_potential.py:331-405), then six Horner
  coefficients per (harmonic, interval) (gpu_potential.py:572-605).

The result carries the reference's harmonic-major table plus the layouts the
B200 kernels read: interval-major FP64 [k][c][6] and interval-major FP32
[k][c][8] (a0..a5 and two zeros, 32-byte records).
"""
from __future__ import annotations

import warnings
from dataclasses import dataclass

import numpy as np
from scipy.interpolate import CubicHermiteSpline
from scipy.linalg import solve_banded
from scipy.special import lambertw

_EPS = np.finfo(np.float64).eps


@dataclass
class MultipoleTables:
    poly: np.ndarray          # (n_lm, n_int, 6) harmonic-major (reference layout)
    lm_l: np.ndarray          # (n_lm,) int32
    lm_m: np.ndarray          # (n_lm,) int32
    logr_min: float
    dlogr: float
    inv_dlogr: float
    n_int: int
    lmax: int
    log_scaling: int
    invPhi0: float
    inner_s: float
    inner_U: float
    inner_W: float
    outer_s: float
    outer_U: float
    outer_W: float
    r_grid: np.ndarray
    node_phi: np.ndarray = None      # (nR, n_lm) Phi at the nodes, builder's harmonic order
    node_dphi_dr: np.ndarray = None  # (nR, n_lm) dPhi/dr at the nodes
    node_cols: np.ndarray = None     # (n_lm,) column of each harmonic in the coefficient file
    resampled: bool = False          # the input grid was not log-uniform and was resampled

    @property
    def n_lm(self) -> int:
        return int(self.poly.shape[0])

    def interval_major(self) -> np.ndarray:
        """(n_int, n_lm, 6) FP64, contiguous."""
        return np.ascontiguousarray(self.poly.transpose(1, 0, 2))

    def interval_major_f32(self) -> np.ndarray:
        """(n_int, n_lm, 8) FP32 with two zero pads per record."""
        out = np.zeros((self.n_int, self.n_lm, 8), dtype=np.float32)
        out[:, :, :6] = self.poly.transpose(1, 0, 2).astype(np.float32)
        return out

    def lm_packed(self) -> np.ndarray:
        return ((self.lm_l.astype(np.int64) << 16) | (self.lm_m.astype(np.int64) & 0xFFFF)).astype(np.int32)

    def regular(self, max_ratio: float = 1.5):
        """Column structure for the kernels' regular walk.

        Returns (structure, poly_reg) where structure is 1 (every l) or 2 (even l
        only) and poly_reg (n_reg, n_int, 6) holds every (l, m) with l <= lmax of
        that parity in (|m|, l, cos before sin) order -- the order the table
        builder sorts by -- with zero columns for harmonics the builder pruned;
        or (0, None) when the regular layout would exceed max_ratio times the
        pruned column count.
        """
        L = self.lmax
        even = bool(np.all(self.lm_l % 2 == 0))
        order = []
        for am in range(L + 1):
            for l in range(am, L + 1):
                if even and l % 2:
                    continue
                order.append((l, am))
                if am > 0:
                    order.append((l, -am))
        if len(order) > max_ratio * self.n_lm:
            return 0, None
        pos = {lm: i for i, lm in enumerate(order)}
        reg = np.zeros((len(order), self.n_int, 6))
        for c, (l, m) in enumerate(zip(self.lm_l.tolist(), self.lm_m.tolist())):
            reg[pos[(l, m)]] = self.poly[c]
        return (2 if even else 1), reg

    def scalars(self) -> list:
        return [self.logr_min, self.dlogr, self.inv_dlogr, self.invPhi0, self.inner_s,
                self.inner_U, self.inner_W, self.outer_s, self.outer_U, self.outer_W]


def _lambert(x: float, branch: int) -> float:
    return float(np.real(lambertw(x, k=branch)))


def inner_extrapolation(phi0: np.ndarray, dphi0_dr: np.ndarray, r: np.ndarray):
    """(invPhi0, s, U, W) for the l=0 term inside the first node.

    Agama's computeExtrapolationCoefs for v = 0 (as restated at
    gpu_potential.py:183-263): Phi(r) = U (r/r1)^s + W fitted to Phi, dPhi/dr at
    r1 and Phi at r2; s solves  s ln(r2/r1) = A (1 - exp(-s ln(r2/r1)))  via the
    Lambert W function.
    """
    P1, P2 = phi0[0], phi0[1]
    d1, d2 = dphi0_dr[0], dphi0_dr[1]
    r1, r2 = r[0], r[1]
    lnr = np.log(r2 / r1)
    g1 = r1 * d1                                      # dPhi/dlog r at r1
    tiny = 100.0 * _EPS
    if abs(g1) == 0.0 or abs(P1 - P2) < tiny * max(abs(P1), abs(P2)):
        return 0.0, 0.0, 0.0, P1
    A = lnr * g1 / (P1 - P2)
    if not np.isfinite(A) or A >= 0.0:
        return 0.0, 0.0, 0.0, P1
    if abs(A + 1.0) < np.sqrt(_EPS):
        s = 0.0
    else:
        w = _lambert(A * np.exp(A), 0 if A > -1.0 else -1)
        s = (A - w) / lnr
    if not np.isfinite(s):
        s = 2.0
    if s != 0:
        U = (r1 * d1 - 0 * P1) / (s - 0)
        W = (r1 * d1 - s * P1) / (0 - s)
    else:
        U = r1 * d1 - 0 * P1
        W = P1
    # constant-density-core check: prefer s = 2 when a cubic predicts dPhi(r2) better
    pred_pow = U * s * np.exp(s * lnr) / r2 if s != 0 else r1 * d1 / r2
    pred_cub = (r2 / r1 * (6.0 * r1 * (P2 - P1) / (r2 - r1) - d1 * (2 * r1 + r2))) / (2 * r2 + r1)
    if abs(d2 - pred_cub) < abs(d2 - pred_pow):
        s = 2.0
        U = 0.5 * r1 * d1
        W = P1 - U
    if s <= 0.0:
        return 0.0, float(s), float(U), float(W)
    inv = 1.0 / W
    if np.any(phi0 * inv >= 1.0):
        inv = 0.0
    return float(inv), float(s), float(U), float(W)


def outer_extrapolation(phi0: np.ndarray, dphi0_dr: np.ndarray, r: np.ndarray):
    """(s, U, W) for the l=0 term beyond the last node (v = -1, Keplerian W term).

    Restates gpu_potential.py:266-328 (Agama computeExtrapolationCoefs, outer).
    """
    v = -1
    P1, P2 = float(phi0[-1]), float(phi0[-2])
    d1 = float(dphi0_dr[-1])
    r1, r2 = float(r[-1]), float(r[-2])
    lnr = np.log(r2 / r1)
    num1, num2 = r1 * d1, v * P1
    den1, den2 = P1, P2 * np.exp(-v * lnr)
    tiny = 100.0 * _EPS
    roundoff = (abs(num1 - num2) < max(abs(num1), abs(num2)) * tiny or
                abs(den1 - den2) < max(abs(den1), abs(den2)) * tiny)
    if not np.isfinite(P1) or roundoff or den1 == den2:
        return 0.0, 0.0, P1
    A = lnr * (num1 - num2) / (den1 - den2)
    if not np.isfinite(A) or A >= 0:
        return 0.0, 0.0, P1
    if abs(A + 1) < np.sqrt(_EPS):
        s = float(v)
    else:
        s = v + (A - _lambert(A * np.exp(A), 0 if A > -1 else -1)) / lnr
    if not np.isfinite(s) or s >= 0:
        s = -2.0
    if s != v:
        U = (r1 * d1 - v * P1) / (s - v)
        W = (r1 * d1 - s * P1) / (v - s)
    else:
        U = r1 * d1 - v * P1
        W = P1
    return float(s), float(U), float(W)


def quintic_second_derivatives(x: np.ndarray, f: np.ndarray, df: np.ndarray) -> np.ndarray:
    """Second derivatives of the C2 quintic spline through (f, df) at nodes x.

    Agama's constructQuinticSpline (restated at gpu_potential.py:331-405): for
    each interior node the continuity of the third derivative gives a
    tridiagonal row; the end rows impose a zero fourth derivative.
    f, df: (n, ncol).  Returns (n, ncol).
    """
    n = x.shape[0]
    h = 1.0 / np.diff(x)                                  # inverse widths, (n-1,)
    diag = np.zeros(n)
    upper = np.zeros(n)                                   # A[i, i+1]
    lower = np.zeros(n)                                   # A[i, i-1]
    rhs = np.zeros((n, f.shape[1]))
    for i in range(n):
        if i > 0:
            hi = h[i - 1]
            diag[i] += 3.0 * hi
            upper[i - 1] = -hi
            rhs[i] -= (20.0 * (f[i] - f[i - 1]) * hi - 12.0 * df[i] - 8.0 * df[i - 1]) * hi * hi
        if i < n - 1:
            hi = h[i]
            diag[i] += 3.0 * hi
            lower[i + 1] = -hi
            rhs[i] += (20.0 * (f[i + 1] - f[i]) * hi - 12.0 * df[i] - 8.0 * df[i + 1]) * hi * hi
    h0, hn = h[0], h[-1]
    upper[0] = -2.0 * h0
    rhs[0] = (30.0 * (f[1] - f[0]) * h0 - 14.0 * df[1] - 16.0 * df[0]) * h0 * h0
    lower[n - 1] = -2.0 * hn
    rhs[n - 1] = (-30.0 * (f[n - 1] - f[n - 2]) * hn + 14.0 * df[n - 2] + 16.0 * df[n - 1]) * hn * hn
    band = np.zeros((3, n))
    band[0, 1:] = upper[:n - 1]
    band[1, :] = diag
    band[2, :n - 1] = lower[1:]
    return solve_banded((1, 1), band, rhs)


def quintic_coefficients(f: np.ndarray, df: np.ndarray, d2f: np.ndarray, h: float) -> np.ndarray:
    """Horner coefficients a0..a5 of each interval on s in [0, 1].

    The quintic matching value, first and second derivative at both ends
    (gpu_potential.py:572-605).  Inputs (n, ncol) in log r; returns (ncol, n-1, 6).
    """
    f0, f1 = f[:-1], f[1:]
    m0, m1 = df[:-1] * h, df[1:] * h
    q0, q1 = d2f[:-1] * (h * h), d2f[1:] * (h * h)
    dd = f1 - f0
    a = np.stack([f0, m0, 0.5 * q0,
                  10.0 * dd - 6.0 * m0 - 4.0 * m1 - 1.5 * q0 + 0.5 * q1,
                  -15.0 * dd + 8.0 * m0 + 7.0 * m1 + 1.5 * q0 - q1,
                  6.0 * dd - 3.0 * m0 - 3.0 * m1 + 0.5 * (q1 - q0)], axis=-1)
    return np.ascontiguousarray(a.transpose(1, 0, 2)).astype(np.float64)


def build_multipole_tables(coefs, prune_threshold: float = 1e-16) -> MultipoleTables:
    """Quintic-spline tables for one Multipole coefficient set (see module doc)."""
    if coefs.dphi_dr is None:
        raise ValueError(
            "MultipoleCoefs.dphi_dr is None; dPhi/dr data is required.\n"
            "Use a .coef_mul_DR file (not plain .coef_mul).")
    r = np.asarray(coefs.R_grid, dtype=np.float64)
    phi = np.asarray(coefs.phi, dtype=np.float64)
    dphi_dr = np.asarray(coefs.dphi_dr, dtype=np.float64)
    nR, n_lm = len(r), phi.shape[1]
    if nR < 2:
        raise ValueError(f"Need at least 2 radial grid points, got {nR}.")

    logr = np.log(r)
    steps = np.diff(logr)
    dlogr = float(steps.mean())
    spread = float(np.max(np.abs(steps - dlogr)) / dlogr)
    dphi_dlogr = dphi_dr * r[:, None]
    d0_dr = dphi_dr[:, 0]

    resampled = spread > 1e-3
    if resampled:
        n_new = max(nR, 1000)
        logr_new = np.linspace(logr[0], logr[-1], n_new)
        r_new = np.exp(logr_new)
        herm = CubicHermiteSpline(logr, phi, dphi_dlogr)
        phi = herm(logr_new)
        dphi_dlogr = herm(logr_new, 1)
        d0_dr = dphi_dlogr[:, 0] / r_new
        r, logr, nR = r_new, logr_new, n_new
        steps = np.diff(logr)
        dlogr = float(steps.mean())
    elif spread > 1e-6:
        warnings.warn(f"Radial grid is not perfectly log-uniform (max relative spacing error = "
                      f"{spread:.2e}). O(1) grid lookup may be slightly inaccurate.", stacklevel=3)

    logr_min = float(logr[0])
    inv_dlogr = 1.0 / dlogr
    n_int = nR - 1
    out_s, out_U, out_W = outer_extrapolation(phi[:, 0], d0_dr, r)

    lm_l = np.array([l for l, _ in coefs.lm_labels], dtype=np.int32)
    lm_m = np.array([m for _, m in coefs.lm_labels], dtype=np.int32)
    lmax = int(lm_l.max())
    if lmax > 32:
        raise ValueError(f"lmax={lmax} exceeds the kernel's compile-time limit of 32.")
    order = np.lexsort((lm_m < 0, lm_l, np.abs(lm_m)))
    lm_l, lm_m = lm_l[order], lm_m[order]
    phi, dphi_dlogr = phi[:, order], dphi_dlogr[:, order]
    cols = order.copy()

    keep = np.ones(n_lm, dtype=bool)
    if prune_threshold > 0:
        keep[1:] = np.any(np.abs(phi[:, 1:]) >= prune_threshold, axis=0)
    if not keep.all():
        phi, dphi_dlogr = phi[:, keep], dphi_dlogr[:, keep]
        lm_l, lm_m = lm_l[keep], lm_m[keep]
        cols = cols[keep]
        lmax = int(lm_l.max())

    p0 = phi[:, 0]
    log_scaling = bool(np.all(p0 < 0.0))
    invPhi0, in_s, in_U, in_W = 0.0, 0.0, 0.0, float(p0[0])
    if log_scaling:
        invPhi0, in_s, in_U, in_W = inner_extrapolation(p0, d0_dr, r)

    f = phi.copy()
    df = dphi_dlogr.copy()
    if log_scaling:
        f[:, 0] = np.log(invPhi0 - 1.0 / p0)
        df[:, 0] = dphi_dlogr[:, 0] / (p0 * (invPhi0 * p0 - 1.0))
        ratio = phi[:, 1:] / p0[:, None]
        f[:, 1:] = ratio
        df[:, 1:] = (dphi_dlogr[:, 1:] - ratio * dphi_dlogr[:, 0:1]) / p0[:, None]

    d2f = quintic_second_derivatives(logr, f, df)
    poly = quintic_coefficients(f, df, d2f, dlogr)
    return MultipoleTables(poly=poly, lm_l=lm_l, lm_m=lm_m, logr_min=logr_min, dlogr=dlogr,
                           inv_dlogr=inv_dlogr, n_int=n_int, lmax=lmax,
                           log_scaling=int(log_scaling), invPhi0=float(invPhi0),
                           inner_s=float(in_s), inner_U=float(in_U), inner_W=float(in_W),
                           outer_s=float(out_s), outer_U=float(out_U), outer_W=float(out_W),
                           r_grid=r, node_phi=np.ascontiguousarray(phi),
                           node_dphi_dr=np.ascontiguousarray(dphi_dlogr / r[:, None]),
                           node_cols=cols, resampled=bool(resampled))
