"""Seeded synthetic coefficient sets and point samples for the benchmark workloads.

No dataset is involved: every input is generated from a seed with the shapes,
sizes and value distributions of the workloads the evaluator is measured on.

* ``nfw_multipole``: Multipole tables on a log-uniform radial grid; l=0 is an
  NFW potential (its C_00 equals Phi because the l=0 angular factor is 1), each
  even-l>0 harmonic is Phi_00 * 0.05 * 10^(-l/2) * N(0,1) with the same factor on
  dPhi/dr.  Odd l columns are present and zero (pruned by the table builder).
* ``bar_cylspline``: CylSpline tables on sinh-spaced R and z grids; m=0 is a
  Miyamoto-Nagai disk, m=+-2,+-4,+-6 a bar with amplitudes 0.1, 0.03, 0.01 times
  exp(-R/4 kpc) times the m=0 term and seeded phases.
* point samples: log-uniform radii with isotropic directions, an exponential
  disk, an isotropic Hernquist sphere.
"""
from __future__ import annotations

import numpy as np

from .coefs import CylSplineCoefs, MultipoleCoefs

G = 4.30091727067736e-06


def nfw_phi(r, M, rs):
    return -G * M * np.log1p(r / rs) / r


def nfw_dphi_dr(r, M, rs):
    return G * M * (np.log1p(r / rs) / (r * r) - 1.0 / (r * (r + rs)))


def nfw_multipole(lmax: int = 8, n_nodes: int = 50, rmin: float = 1e-2, rmax: float = 1e3,
                  M: float = 1e12, rs: float = 20.0, seed: int = 0, amp: float = 0.05,
                  drift: float = 0.0) -> MultipoleCoefs:
    """Even-l triaxial Multipole around an NFW monopole (seeded)."""
    rng = np.random.default_rng(seed)
    r = np.exp(np.linspace(np.log(rmin), np.log(rmax), n_nodes))
    labels = [(l, m) for l in range(lmax + 1) for m in range(-l, l + 1)]
    p0, d0 = nfw_phi(r, M, rs), nfw_dphi_dr(r, M, rs)
    phi = np.zeros((n_nodes, len(labels)))
    dphi = np.zeros_like(phi)
    for c, (l, m) in enumerate(labels):
        if l == 0:
            phi[:, c], dphi[:, c] = p0, d0
        elif l % 2 == 0:
            f = amp * 10.0 ** (-l / 2.0) * rng.normal() * (1.0 + drift)
            phi[:, c], dphi[:, c] = p0 * f, d0 * f
    return MultipoleCoefs(r, phi, dphi, labels, {"type": "Multipole"})


def mn_phi(R, z, M, a, b):
    return -G * M / np.sqrt(R * R + (a + np.sqrt(z * z + b * b)) ** 2)


def bar_cylspline(n_R: int = 32, n_z: int = 32, Rmin: float = 0.1, Rmax: float = 200.0,
                  zmax: float = 200.0, M: float = 5e10, a: float = 3.0, b: float = 0.3,
                  mmax: int = 6, seed: int = 1, scale: float = 1.0) -> CylSplineCoefs:
    """m=0 Miyamoto-Nagai plus an m=2,4,6 bar (seeded phases)."""
    rng = np.random.default_rng(seed)
    uR = np.linspace(np.arcsinh(Rmin / scale), np.arcsinh(Rmax / scale), n_R)
    R = scale * np.sinh(uR)
    uz = np.linspace(-np.arcsinh(zmax / scale), np.arcsinh(zmax / scale), n_z)
    z = scale * np.sinh(uz)
    RR, ZZ = np.meshgrid(R, z, indexing="ij")
    p0 = mn_phi(RR, ZZ, M, a, b)
    phi = {0: p0}
    amps = {2: 0.1, 4: 0.03, 6: 0.01}
    for m in range(2, mmax + 1, 2):
        ph = rng.uniform(0.0, 2.0 * np.pi)
        base = amps.get(m, 0.01) * np.exp(-RR / 4.0) * p0
        phi[m] = base * np.cos(ph)
        phi[-m] = base * np.sin(ph)
    return CylSplineCoefs(R, z, phi, {"type": "CylSpline"})


def isotropic(n: int, rng) -> np.ndarray:
    u = rng.normal(size=(n, 3))
    return u / np.linalg.norm(u, axis=1)[:, None]


def loguniform_points(n: int, lo: float = -1.5, hi: float = 2.5, seed: int = 0) -> np.ndarray:
    """log10 r uniform in [lo, hi], isotropic directions."""
    rng = np.random.default_rng(seed)
    r = 10.0 ** rng.uniform(lo, hi, n)
    return isotropic(n, rng) * r[:, None]


def disk_points(n: int, Rd: float = 3.0, hz: float = 0.3, seed: int = 0) -> np.ndarray:
    """Exponential disk: R ~ Gamma(2, Rd), z ~ Laplace(hz), phi uniform."""
    rng = np.random.default_rng(seed)
    R = rng.gamma(2.0, Rd, n)
    z = rng.laplace(0.0, hz, n)
    ph = rng.uniform(0.0, 2.0 * np.pi, n)
    return np.stack([R * np.cos(ph), R * np.sin(ph), z], axis=1)


def hernquist_points(n: int, a: float = 10.0, seed: int = 0) -> np.ndarray:
    """Isotropic Hernquist sphere: r = a sqrt(u) / (1 - sqrt(u))."""
    rng = np.random.default_rng(seed)
    su = np.sqrt(rng.uniform(0.0, 1.0, n))
    r = a * su / (1.0 - su)
    return isotropic(n, rng) * r[:, None]


def circular_track(T: int = 1000, radius: float = 50.0, t0: float = 0.0, t1: float = 2.0,
                   period: float = 1.5, seed: int = 3) -> np.ndarray:
    """(T,4) rows [t, x, y, z]: a circular orbit, slightly inclined."""
    rng = np.random.default_rng(seed)
    t = np.linspace(t0, t1, T)
    w = 2.0 * np.pi / period
    inc = rng.uniform(0.2, 0.6)
    x = radius * np.cos(w * t)
    y = radius * np.sin(w * t) * np.cos(inc)
    z = radius * np.sin(w * t) * np.sin(inc)
    return np.stack([t, x, y, z], axis=1)


def composite_spec(lmax_main: int = 32, n_nodes: int = 100, n_snap: int = 16,
                   lmax_snap: int = 16, seed: int = 0) -> dict:
    """Inputs of the time-dependent composite: coefficient sets and parameters."""
    main = nfw_multipole(lmax=lmax_main, n_nodes=n_nodes, seed=seed)
    times = np.linspace(0.0, 1.5, n_snap)
    snaps = [nfw_multipole(lmax=lmax_snap, n_nodes=n_nodes, M=2e11, rs=12.0, seed=seed + 100,
                           drift=0.5 * i / max(n_snap - 1, 1)) for i in range(n_snap)]
    return dict(main=main, snaps=snaps, times=times, track=circular_track(),
                mn=dict(mass=5e10, scaleRadius=3.0, scaleHeight=0.3),
                disk=dict(surfaceDensity=1e9, scaleRadius=3.0, scaleHeight=0.3),
                nfw=dict(mass=1.5e11, scaleRadius=10.0))


def config4_unit_specs(n_units: int = 512, seed: int = 4) -> list:
    """The uneven batch: per unit an NFW-based Multipole with lmax ~ U{2..32}, rs ~
    U[2,30] kpc, nodes ~ U{30..120}, M ~ logU[1e10,1e12] and N ~ logU[1e3, 5e5]
    Hernquist(a = rs) points (seed 1000 + unit).  Returns [{index, coefs (keyword
    arguments of nfw_multipole), n_points, a}].  The expected total is about 40M
    points: E[N] = (5e5 - 1e3) / ln(500) = 80k per unit."""
    rng = np.random.default_rng(seed)
    out = []
    for u in range(n_units):
        lmax = int(rng.integers(2, 33))
        rs = float(rng.uniform(2.0, 30.0))
        n_nodes = int(rng.integers(30, 121))
        M = float(10 ** rng.uniform(10, 12))
        n = int(np.exp(rng.uniform(np.log(1e3), np.log(5e5))))
        out.append(dict(index=u, coefs=dict(lmax=lmax, n_nodes=n_nodes, M=M, rs=rs, seed=u,
                                            amp=0.05),
                        n_points=n, a=rs))
    return out


def build_composite(spec: dict, interpolate: bool = True):
    """The time-dependent composite of ``composite_spec``: Multipole + MiyamotoNagai +
    DiskAnsatz + Shifted NFW on a (T,4) track + Evolving Multipole snapshots."""
    from .analytic import DiskAnsatzPotentialGPU, MiyamotoNagaiPotentialGPU, NFWPotentialGPU
    from .potentials import (CompositePotentialGPU, EvolvingPotentialGPU, MultipolePotentialGPU,
                             ShiftedPotentialGPU)
    return CompositePotentialGPU([
        MultipolePotentialGPU(spec["main"]),
        MiyamotoNagaiPotentialGPU(**spec["mn"]),
        DiskAnsatzPotentialGPU(**spec["disk"]),
        ShiftedPotentialGPU(NFWPotentialGPU(**spec["nfw"]), spec["track"]),
        EvolvingPotentialGPU([MultipolePotentialGPU(s) for s in spec["snaps"]], spec["times"],
                             interpolate=interpolate),
    ])
