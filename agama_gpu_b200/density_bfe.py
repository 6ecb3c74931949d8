"""Multipole expansions from a density: the Poisson solve behind the Spheroid,
King, triaxial / gamma = 2 Dehnen and Disk types.

The reference builds these types with Agama's CPU library and loads the
exported Multipole (gpu_potential.py:1936-2052).  This module builds the same
kind of object -- node tables Phi_lm(r_i), dPhi_lm/dr(r_i) on a log-uniform
radial grid, handed to MultipolePotentialGPU -- from the density itself:

1. angular projection on the device: the density is sampled on
   (radius) x (Gauss-Legendre cos theta) x (uniform phi) and projected onto the
   evaluator's own angular functions Y_c (normalised Legendre x MUL0/MUL1 x
   cos/sin m phi) with the discrete dual weights, so that
   rho(r, theta, phi) = sum_c rho_c(r) Y_c(theta, phi) in the convention the
   kernels evaluate;
2. radial integrals per harmonic, on composite Gauss-Legendre sub-intervals of
   the log-radius grid with power-law tails beyond both ends:

       Phi_c(r)   = -4 pi G / (2l+1) (P(r) + Q(r))
       dPhi_c/dr  = -4 pi G / (2l+1) (-(l+1) P(r) + l Q(r)) / r
       P(r) = r^-(l+1) int_0^r rho_c s^(l+2) ds,  Q(r) = r^l int_r^inf rho_c s^(1-l) ds

   accumulated as scaled recurrences (P and Q stay O(rho r^2) at every l, so
   lmax = 32 does not overflow).  Each Y_c is an eigenfunction of the angular
   Laplacian (eigenvalue -l(l+1)), so the normalisation of the basis drops out.

Densities are torch callables rho(x, y, z) -> tensor evaluated where the
samples live (the GPU when there is one).  Agama is not needed; where the
result can differ from Agama's own expansion (grid choice, quadrature), the
differences are at the level of the expansion's truncation error.
"""
from __future__ import annotations

import math
from typing import Callable, List, Optional, Sequence, Tuple

import numpy as np
import torch

from .coefs import MultipoleCoefs
from .legendre import MUL0, MUL1, legendre_normalised
from .potentials import G_AGAMA

DensityFn = Callable[[torch.Tensor, torch.Tensor, torch.Tensor], torch.Tensor]

_GL_ORDER = 6
_SUB_PER_NODE = 8


def _labels(lmax: int, mmax: int, symmetry: str) -> List[Tuple[int, int]]:
    out = []
    for l in range(lmax + 1):
        for m in range(-l, l + 1):
            if abs(m) > mmax:
                continue
            if symmetry == "spherical" and l > 0:
                continue
            if symmetry in ("axisymmetric", "triaxial") and (l % 2 or m % 2 or m < 0):
                continue
            if symmetry == "axisymmetric" and m != 0:
                continue
            out.append((l, m))
    return out


def angular_basis(labels: Sequence[Tuple[int, int]], ct: np.ndarray, st: np.ndarray,
                  ph: np.ndarray) -> np.ndarray:
    """(n_points, n_labels) angular functions Y_c of the evaluator at the given points."""
    lmax = max(l for l, _ in labels)
    cache = {}
    out = np.zeros((len(ct), len(labels)))
    for c, (l, m) in enumerate(labels):
        am = abs(m)
        if am not in cache:
            cache[am] = legendre_normalised(lmax, am, ct, st)
        Y = cache[am][:, l - am] * (MUL0 if am == 0 else MUL1)
        T = np.cos(am * ph) if m >= 0 else np.sin(am * ph)
        out[:, c] = Y * T
    return out


def _angular_grid(lmax: int, mmax: int, n_phi: Optional[int], n_theta: Optional[int] = None):
    n_th = max(2 * lmax + 2, int(n_theta or 0))
    ct, wt = np.polynomial.legendre.leggauss(n_th)
    if n_phi is None:
        n_phi = 4 * mmax + 4 if mmax > 0 else 8
    ph = (np.arange(n_phi) + 0.5) * (2.0 * np.pi / n_phi)
    CT, PH = np.meshgrid(ct, ph, indexing="ij")
    W = np.repeat(wt[:, None], n_phi, axis=1) * (2.0 * np.pi / n_phi)
    CT, PH, W = CT.ravel(), PH.ravel(), W.ravel()
    return CT, np.sqrt(np.maximum(0.0, 1.0 - CT * CT)), PH, W


def _radial_samples(logr_nodes: np.ndarray, ext_in: float, ext_out: float):
    """Sub-interval boundaries (in log r) and the GL abscissae/weights inside each."""
    d = (logr_nodes[1] - logr_nodes[0]) / _SUB_PER_NODE
    n_in = int(math.ceil(ext_in / d))
    n_out = int(math.ceil(ext_out / d))
    n_mid = (len(logr_nodes) - 1) * _SUB_PER_NODE
    b = logr_nodes[0] + d * np.arange(-n_in, n_mid + n_out + 1, dtype=np.float64)
    b[n_in::_SUB_PER_NODE][:len(logr_nodes)] = logr_nodes        # nodes exactly
    x, w = np.polynomial.legendre.leggauss(_GL_ORDER)
    lo, hi = b[:-1, None], b[1:, None]
    s = 0.5 * (lo + hi) + 0.5 * (hi - lo) * x[None, :]
    ws = 0.5 * (hi - lo) * w[None, :]
    return b, s, ws, n_in


def project_density(rho: DensityFn, labels, r: np.ndarray, lmax: int, mmax: int,
                    device, n_phi: Optional[int] = None, n_theta: Optional[int] = None,
                    chunk: int = 64) -> np.ndarray:
    """rho_c(r) for every label at radii r: (len(r), n_labels)."""
    ct, st, ph, w = _angular_grid(lmax, mmax, n_phi, n_theta)
    Y = angular_basis(labels, ct, st, ph)                         # (n_ang, n_lab)
    norm = (w[:, None] * Y * Y).sum(0)
    dual = torch.as_tensor(w[:, None] * Y / norm[None, :], dtype=torch.float64, device=device)
    ux = torch.as_tensor(st * np.cos(ph), dtype=torch.float64, device=device)
    uy = torch.as_tensor(st * np.sin(ph), dtype=torch.float64, device=device)
    uz = torch.as_tensor(ct, dtype=torch.float64, device=device)
    out = np.empty((len(r), len(labels)))
    rt = torch.as_tensor(r, dtype=torch.float64, device=device)
    for i in range(0, len(r), chunk):
        rr = rt[i:i + chunk, None]
        vals = rho(rr * ux[None, :], rr * uy[None, :], rr * uz[None, :])
        out[i:i + chunk] = (vals.to(torch.float64) @ dual).cpu().numpy()
    return out


def _tail_slope(r1, r2, f1, f2):
    ok = (f1 * f2 > 0)
    with np.errstate(divide="ignore", invalid="ignore"):
        g = np.where(ok, np.log(np.abs(f2 / np.where(ok, f1, 1.0))) / math.log(r2 / r1), 0.0)
    return g, ok


def solve_poisson(rho_c: np.ndarray, s: np.ndarray, ws: np.ndarray, b: np.ndarray,
                  ls: np.ndarray, n_in: int, node_idx: np.ndarray):
    """Phi_c and dPhi_c/dr at the boundaries b[node_idx] from rho_c at the GL samples.

    rho_c: (n_sub, n_gl, n_lab) at radii exp(s) (n_sub, n_gl), weights ws in log r."""
    n_sub = s.shape[0]
    R = np.exp(s)                                                 # (n_sub, n_gl)
    eb = np.exp(b)
    l = ls[None, None, :].astype(np.float64)
    # P recurrence: P(b_{j+1}) = (b_j / b_{j+1})^(l+1) P(b_j) + sum w rho s^2 (s / b_{j+1})^(l+1)
    IP = (ws[:, :, None] * rho_c * (R * R)[:, :, None]
          * (R[:, :, None] / eb[1:, None, None]) ** (l + 1)).sum(1)           # (n_sub, n_lab)
    IQ = (ws[:, :, None] * rho_c * (R * R)[:, :, None]
          * (eb[:-1, None, None] / R[:, :, None]) ** l).sum(1)
    ratio = np.exp(b[:-1] - b[1:])                                            # (n_sub,)
    nl = len(ls)
    P = np.zeros((n_sub + 1, nl))
    Q = np.zeros((n_sub + 1, nl))
    # inner tail: rho_c ~ A s^g below exp(b_0)
    g, ok = _tail_slope(R[0, 0], R[0, -1], rho_c[0, 0], rho_c[0, -1])
    den = g + ls + 3.0
    A = np.where(ok & (den > 0), rho_c[0, 0] * R[0, 0] ** 2 * (eb[0] / R[0, 0]) ** (g + 2.0), 0.0)
    P[0] = np.where(den > 0, A / np.where(den > 0, den, 1.0), 0.0)
    for j in range(n_sub):
        P[j + 1] = ratio[j] ** (ls + 1.0) * P[j] + IP[j]
    # outer tail: rho_c ~ A s^g above exp(b_end)
    g, ok = _tail_slope(R[-1, 0], R[-1, -1], rho_c[-1, 0], rho_c[-1, -1])
    den = ls - g - 2.0
    A = np.where(ok & (den > 0), rho_c[-1, -1] * R[-1, -1] ** 2 * (eb[-1] / R[-1, -1]) ** (g + 2.0), 0.0)
    Q[-1] = np.where(den > 0, A / np.where(den > 0, den, 1.0), 0.0)
    for j in range(n_sub - 1, -1, -1):
        Q[j] = ratio[j] ** ls * Q[j + 1] + IQ[j]
    k = -4.0 * math.pi * G_AGAMA / (2.0 * ls + 1.0)
    Pn, Qn = P[node_idx], Q[node_idx]
    rn = eb[node_idx][:, None]
    phi = k[None, :] * (Pn + Qn)
    dphi = k[None, :] * (-(ls + 1.0) * Pn + ls * Qn) / rn
    return phi, dphi


def _auto_range(rho: DensityFn, device, hint: float = 1.0, n_theta: int = 512) -> Tuple[float, float]:
    """rmin, rmax enclosing mass fractions 1e-4 .. 1 - 1e-4 of the spherically averaged
    density in a window 1e-6 .. 1e6 x hint (1e-3 .. 1e3 x its half-mass radius when the
    mass diverges).  The average takes n_theta nodes in cos theta, enough for a disk."""
    r = hint * np.exp(np.linspace(math.log(1e-6), math.log(1e6), 481))
    rc = project_density(rho, [(0, 0)], r, 0, 0, device, n_phi=8, n_theta=n_theta)[:, 0]
    dm = 4.0 * math.pi * rc * r ** 3                     # dM / dln r
    dl = np.log(r[1] / r[0])
    M = np.concatenate([[0.0], np.cumsum(0.5 * (dm[1:] + dm[:-1]) * dl)])
    tot = M[-1]
    if not (tot > 0 and np.isfinite(tot)):
        raise ValueError("density has no positive finite mass in its sampling window")
    r_half = float(np.interp(0.5 * tot, M, r))
    if dm[-1] * 5.0 > 1e-3 * tot:                      # still growing: mass diverges
        return 1e-3 * r_half, 1e3 * r_half
    rmin = float(np.interp(1e-4 * tot, M, r))
    rmax = float(np.interp((1 - 1e-4) * tot, M, r))
    return rmin, rmax


def multipole_from_density(rho: DensityFn, lmax: int = 6, mmax: Optional[int] = None,
                           gridSizeR: int = 60, rmin: Optional[float] = None,
                           rmax: Optional[float] = None, symmetry: str = "none",
                           n_phi: Optional[int] = None, n_theta: Optional[int] = None,
                           device=None, length_hint: float = 1.0) -> MultipoleCoefs:
    """MultipoleCoefs (Phi_lm and dPhi_lm/dr on a log-uniform grid) of the potential of
    ``rho`` (Msol / kpc^3 as a function of x, y, z in kpc).

    symmetry: 'spherical' (l = 0), 'axisymmetric' (m = 0, even l), 'triaxial' (even l,
    even m >= 0) or 'none' (every l <= lmax, |m| <= mmax).  n_theta: Gauss-Legendre nodes
    in cos theta (at least 2 lmax + 2; raise it for densities thinner in angle than
    pi / (2 lmax), e.g. disks); n_phi: uniform azimuths (1 is exact for an axisymmetric
    density)."""
    if symmetry not in ("spherical", "axisymmetric", "triaxial", "none"):
        raise ValueError(f"unknown symmetry {symmetry!r}")
    lmax = 0 if symmetry == "spherical" else int(lmax)
    mmax = lmax if mmax is None else min(int(mmax), lmax)
    if symmetry == "axisymmetric":
        mmax = 0
    dev = torch.device(device) if device is not None else (
        torch.device("cuda") if torch.cuda.is_available() else torch.device("cpu"))
    if rmin is None or rmax is None:
        a, bmax = _auto_range(rho, dev, length_hint)
        rmin = a if rmin is None else rmin
        rmax = bmax if rmax is None else rmax
    if not (0 < rmin < rmax) or gridSizeR < 3:
        raise ValueError("need 0 < rmin < rmax and gridSizeR >= 3")
    labels = _labels(lmax, mmax, symmetry)
    logr = np.linspace(math.log(rmin), math.log(rmax), int(gridSizeR))
    b, s, ws, n_in = _radial_samples(logr, ext_in=math.log(1e4), ext_out=math.log(1e4))
    if n_phi is None and symmetry in ("spherical", "axisymmetric") and getattr(
            rho, "symmetry", None) in ("spherical", "axisymmetric"):
        n_phi = 1
    rc = project_density(rho, labels, np.exp(s.ravel()), lmax, mmax, dev, n_phi=n_phi,
                         n_theta=n_theta)
    rc = rc.reshape(s.shape + (len(labels),))
    ls = np.array([l for l, _ in labels], dtype=np.float64)
    node_idx = n_in + _SUB_PER_NODE * np.arange(len(logr))
    phi, dphi = solve_poisson(rc, s, ws, b, ls, n_in, node_idx)
    return MultipoleCoefs(np.exp(logr), phi, dphi, labels,
                          {"type": "Multipole", "gridSizeR": str(int(gridSizeR)),
                           "lmax": str(lmax), "symmetry": symmetry})


# -- densities of the Agama-routed types -------------------------------------------------

def spheroid_density(densityNorm: float = None, mass: float = None, scaleRadius: float = 1.0,
                     gamma: float = 1.0, beta: float = 4.0, alpha: float = 1.0,
                     axisRatioY: float = 1.0, axisRatioZ: float = 1.0,
                     outerCutoffRadius: float = 0.0, cutoffStrength: float = 2.0) -> DensityFn:
    """Double power law with an optional exponential cutoff (Agama's Spheroid):
    rho = rho0 (s/a)^-gamma (1 + (s/a)^alpha)^((gamma-beta)/alpha) exp(-(s/rcut)^xi),
    s = sqrt(x^2 + (y/p)^2 + (z/q)^2).  ``mass`` fixes rho0 from the total mass."""
    a, p, q = float(scaleRadius), float(axisRatioY), float(axisRatioZ)
    g, bt, al = float(gamma), float(beta), float(alpha)
    rc, xi = float(outerCutoffRadius), float(cutoffStrength)

    def shape(sv):
        u = sv / a
        f = u.pow(-g) * (1.0 + u.pow(al)).pow((g - bt) / al)
        if rc > 0:
            f = f * torch.exp(-(sv / rc).pow(xi))
        return f

    if densityNorm is not None and mass is not None:
        raise ValueError("give densityNorm or mass, not both")
    if mass is not None:
        if rc <= 0 and bt <= 3.0:
            raise ValueError("total mass is infinite for beta <= 3 without an outer cutoff")
        # M = 4 pi p q int shape(s) s^2 ds (log-r trapezoid over 24 decades)
        sv = a * torch.exp(torch.linspace(math.log(1e-12), math.log(1e12), 24001, dtype=torch.float64))
        integrand = shape(sv) * sv ** 3
        I = float(torch.trapezoid(integrand, torch.log(sv)))
        rho0 = float(mass) / (4.0 * math.pi * p * q * I)
    else:
        rho0 = 1.0 if densityNorm is None else float(densityNorm)

    def rho(x, y, z):
        sv = torch.sqrt(x * x + (y / p) ** 2 + (z / q) ** 2)
        return rho0 * shape(sv)

    rho.symmetry = "spherical" if (p == 1.0 and q == 1.0) else (
        "axisymmetric" if p == 1.0 else "triaxial")
    rho.length = a
    return rho


def disk_density(surfaceDensity: float = None, mass: float = None, scaleRadius: float = 1.0,
                 scaleHeight: float = 0.1, innerCutoffRadius: float = 0.0,
                 sersicIndex: float = 1.0) -> DensityFn:
    """Agama's Disk density Sigma(R) h(z): Sigma = Sigma0 exp(-(R/Rd)^(1/n) - Rin/R);
    h = exp(-|z|/h)/(2h) (h > 0) or sech^2(z/2|h|)/(4|h|) (h < 0)."""
    Rd, hz, Rin, n = float(scaleRadius), float(scaleHeight), float(innerCutoffRadius), float(sersicIndex)
    if abs(hz) < 1e-10:
        raise ValueError("a razor-thin disk (scaleHeight = 0) has no volume density to expand")

    def sigma(R):
        e = (R / Rd).pow(1.0 / n)
        if Rin > 0:
            e = e + Rin / torch.clamp(R, min=1e-300)
        return torch.exp(-e)

    if surfaceDensity is not None and mass is not None:
        raise ValueError("give surfaceDensity or mass, not both")
    if mass is not None:
        Rv = Rd * torch.exp(torch.linspace(math.log(1e-10), math.log(1e4), 20001, dtype=torch.float64))
        I = float(torch.trapezoid(2.0 * math.pi * sigma(Rv) * Rv * Rv, torch.log(Rv)))
        s0 = float(mass) / I
    else:
        s0 = 1.0 if surfaceDensity is None else float(surfaceDensity)

    def rho(x, y, z):
        R = torch.sqrt(x * x + y * y)
        az = torch.abs(z)
        if hz > 0:
            h = torch.exp(-az / hz) / (2.0 * hz)
        else:
            hh = -hz
            c = torch.cosh(az / (2.0 * hh))
            h = 1.0 / (4.0 * hh * c * c)
        return s0 * sigma(R) * h

    rho.symmetry = "axisymmetric"
    rho.length = Rd
    rho.sigma0 = s0
    return rho


def disk_residual_density(rho_disk: DensityFn, sigma0: float, scaleRadius: float,
                          scaleHeight: float, innerCutoffRadius: float = 0.0) -> DensityFn:
    """rho_disk minus the density of DiskAnsatzPotentialGPU(sigma0, scaleRadius,
    scaleHeight, innerCutoffRadius): the part a Multipole carries in Agama's Disk
    decomposition.  The ansatz density is the Laplacian of its potential
    f(r) H(z) / (4 pi G) with f = 4 pi G Sigma0 exp(-r/Rd - Rin/r) (r spherical),
    H = (h/2)(exp(-|z|/h) - 1 + |z|/h) (the exponential law with |h|):
        (H (f'' + 2 f'/r) + 2 f' H' z/r + f H'') / (4 pi G)."""
    hr, hz, hin = float(scaleRadius), abs(float(scaleHeight)), float(innerCutoffRadius)
    s0 = float(sigma0)

    def rho(x, y, z):
        r = torch.sqrt(x * x + y * y + z * z).clamp(min=1e-300)
        ir = 1.0 / r
        f = s0 * torch.exp(-r / hr - hin * ir)              # f / (4 pi G)
        fdo = -1.0 / hr + hin * ir * ir
        f1 = f * fdo
        f2 = f * (fdo * fdo - 2.0 * hin * ir * ir * ir)
        u = torch.abs(z) / hz
        eu = torch.exp(-u)
        H = 0.5 * hz * (eu - 1.0 + u)
        H1 = 0.5 * torch.sign(z) * (1.0 - eu)
        H2 = 0.5 * eu / hz
        ans = H * (f2 + 2.0 * f1 * ir) + 2.0 * f1 * H1 * z * ir + f * H2
        return rho_disk(x, y, z) - ans

    rho.symmetry = "axisymmetric"
    rho.length = hr
    return rho


def king_multipole(mass: float = 1.0, scaleRadius: float = 1.0, W0: float = 5.0,
                   trunc: float = 1.0, gridSizeR: int = 40) -> MultipoleCoefs:
    """Spherical Multipole (l = 0) of a lowered-isothermal (generalised King) model.

    Density as a function of the dimensionless potential W: rho ~ exp(W) P(trunc + 3/2, W)
    (P the regularised lower incomplete gamma function; trunc = 1 is King 1966).  In units
    of the King radius r0 = scaleRadius, W'' + 2 W'/r = -9 rho(W)/rho(W0), W(0) = W0,
    integrated to the tidal radius where W = 0; sigma^2 follows from the total mass:
    M = -sigma^2 r0 rt^2 W'(rt) / G.  Phi = -sigma^2 W - G M / r_t inside, -G M / r outside."""
    from scipy.integrate import solve_ivp
    from scipy.special import gammainc
    W0, g = float(W0), float(trunc)
    if not (W0 > 0 and 0 <= g < 3.5):
        raise ValueError("King model needs W0 > 0 and 0 <= trunc < 3.5")
    r0, M = float(scaleRadius), float(mass)
    a = g + 1.5
    rho0 = math.exp(W0) * gammainc(a, W0)

    def rhohat(W):
        W = max(W, 0.0)
        return math.exp(W) * gammainc(a, W) / rho0

    def rhs(r, y):
        return [y[1], -9.0 * rhohat(y[0]) - 2.0 * y[1] / r]

    def hit(r, y):
        return y[0]
    hit.terminal, hit.direction = True, -1
    r_start = 1e-6
    y0 = [W0 - 1.5 * r_start ** 2, -3.0 * r_start]
    sol = solve_ivp(rhs, (r_start, 1e6), y0, method="DOP853", rtol=1e-12, atol=1e-14,
                    events=hit, dense_output=True)
    if not sol.t_events[0].size:
        raise RuntimeError("King model: W did not reach 0")
    rt = float(sol.t_events[0][0])
    dWt = float(sol.y_events[0][0][1])
    sig2 = -G_AGAMA * M / (r0 * rt * rt * dWt)
    r = np.exp(np.linspace(math.log(1e-2 * r0), math.log(10.0 * rt * r0), int(gridSizeR)))
    rh = r / r0
    phi = np.empty_like(r)
    dphi = np.empty_like(r)
    inside = rh < rt
    yin = sol.sol(np.maximum(rh[inside], r_start))
    phi[inside] = -sig2 * yin[0] - G_AGAMA * M / (rt * r0)
    dphi[inside] = -sig2 * yin[1] / r0
    phi[~inside] = -G_AGAMA * M / r[~inside]
    dphi[~inside] = G_AGAMA * M / r[~inside] ** 2
    return MultipoleCoefs(r, phi[:, None], dphi[:, None], [(0, 0)],
                          {"type": "Multipole", "gridSizeR": str(int(gridSizeR)),
                           "tidalRadius": repr(rt * r0)})
