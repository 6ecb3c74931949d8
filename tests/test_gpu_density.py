"""Agama-routed types (Spheroid, triaxial Dehnen, Disk, King) built by the package's
own Poisson solver and evaluated on the GPU: parity with the oracle's evaluation of the
same tables, accuracy against closed forms and the homoeoid integral, Poisson
consistency of the Disk decomposition, and the King model's node values."""
import math

import numpy as np
import pytest

from oracle import cpu
from test_density_bfe import _ellipsoidal_phi

pytestmark = pytest.mark.gpu

G = 4.30091727067736e-06


def _pts(n, seed, lo, hi):
    rng = np.random.default_rng(seed)
    r = np.exp(rng.uniform(np.log(lo), np.log(hi), n))
    u = rng.normal(size=(n, 3))
    return u / np.linalg.norm(u, axis=1)[:, None] * r[:, None], r


def test_spheroid_hernquist_on_gpu():
    import torch
    import agama_gpu_b200 as agb
    h = agb.PotentialGPU(type="Spheroid", mass=1e11, scaleRadius=2.0, gamma=1, beta=4, alpha=1)
    x, r = _pts(4000, 3, 0.05, 500.0)
    xt = torch.from_numpy(x).cuda()
    phi = h.potential(xt).cpu().numpy()
    F = h.force(xt).cpu().numpy()
    po, go, _, _ = cpu.eval_potential(h, 1, x)
    assert np.abs(phi - po).max() <= 1e-12 * np.abs(po).max()
    assert np.abs(F + go).max() <= 1e-10 * np.abs(go).max()
    assert np.abs(phi / (-G * 1e11 / (r + 2.0)) - 1).max() < 5e-9
    fr = np.linalg.norm(F, axis=1)
    assert np.abs(fr / (G * 1e11 / (r + 2.0) ** 2) - 1).max() < 2e-6


def test_triaxial_dehnen_on_gpu_against_homoeoid_integral():
    import torch
    import agama_gpu_b200 as agb
    p, q, a, M = 0.8, 0.6, 2.0, 1e11
    d = agb.PotentialGPU(type="Dehnen", mass=M, scaleRadius=a, gamma=1.0, axisRatioY=p,
                         axisRatioZ=q, lmax=16)
    assert isinstance(d, agb.MultipolePotentialGPU)
    x, _ = _pts(24, 5, 0.2, 200.0)
    phi = d.potential(torch.from_numpy(x).cuda()).cpu().numpy()
    po, _, _, _ = cpu.eval_potential(d, 1, x)
    assert np.abs(phi - po).max() <= 1e-12 * np.abs(po).max()
    rho0 = M / (2 * math.pi * a ** 3 * p * q)
    ex = np.array([_ellipsoidal_phi(*xi, p, q, rho0) for xi in x])
    assert np.abs(phi / ex - 1).max() < 1e-6


def test_disk_on_gpu_poisson_consistency_and_far_field():
    import torch
    import agama_gpu_b200 as agb
    from agama_gpu_b200.density_bfe import disk_density
    kw = dict(surfaceDensity=8.9e8, scaleRadius=3.0, scaleHeight=0.3)
    d = agb.PotentialGPU(type="Disk", **kw)
    assert [type(c).__name__ for c in d._components] == ["DiskAnsatzPotentialGPU",
                                                        "MultipolePotentialGPU"]
    rng = np.random.default_rng(1)
    R = rng.uniform(0.5, 15, 2000)
    z = rng.normal(0, 0.5, 2000)
    ph = rng.uniform(0, 2 * np.pi, 2000)
    x = np.stack([R * np.cos(ph), R * np.sin(ph), z], 1)
    xt = torch.from_numpy(x).cuda()
    dens = d.density(xt).cpu().numpy()
    ex = disk_density(**kw)(*(xt[:, i].cpu() for i in range(3))).numpy()
    assert np.abs(dens - ex).max() < 2e-3 * ex.max()
    assert np.median(np.abs(dens / ex - 1)) < 5e-3
    _, _, _, do = cpu.eval_potential(d, 3, x)
    assert np.abs(dens - do).max() <= 1e-9 * np.abs(do).max()
    far = torch.tensor([[1000.0, 0, 0], [0, 0, 1000.0], [300.0, 200.0, -100.0]],
                       dtype=torch.float64, device="cuda")
    Mtot = 2 * math.pi * 8.9e8 * 9.0
    pf = d.potential(far).cpu().numpy()
    rf = far.norm(dim=1).cpu().numpy()
    assert np.abs(pf / (-G * Mtot / rf) - 1).max() < 1e-7


def test_king_on_gpu_node_values():
    import torch
    import agama_gpu_b200 as agb
    from agama_gpu_b200.density_bfe import king_multipole
    k = agb.PotentialGPU(type="King", mass=1e5, scaleRadius=0.01, W0=6.0)
    c = king_multipole(1e5, 0.01, 6.0)
    u = np.array([0.48, -0.6, 0.64])
    u /= np.linalg.norm(u)
    x = c.R_grid[:, None] * u[None, :]
    phi = k.potential(torch.from_numpy(x).cuda()).cpu().numpy()
    assert np.abs(phi / c.phi[:, 0] - 1).max() < 1e-10
