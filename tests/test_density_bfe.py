"""The Poisson solver behind the Spheroid / Dehnen / King / Disk types (CPU):
node tables against closed-form potentials, a triaxial density against the
ellipsoidal-potential integral, the King model's known structure, and the disk
decomposition's residual density."""
import math

import numpy as np
import pytest
import torch
from scipy.integrate import quad

from agama_gpu_b200.density_bfe import (angular_basis, disk_density, disk_residual_density,
                                        king_multipole, multipole_from_density, spheroid_density)
from agama_gpu_b200.legendre import MUL0
from agama_gpu_b200.potentials import G_AGAMA as G

M, A = 1e11, 2.0


def _solve(rho, **kw):
    return multipole_from_density(rho, symmetry=rho.symmetry, device="cpu", length_hint=rho.length, **kw)


@pytest.mark.parametrize("gamma,beta,alpha,phi", [
    (1.0, 4.0, 1.0, lambda r: -G * M / (r + A)),                                    # Hernquist
    (0.0, 5.0, 2.0, lambda r: -G * M / np.sqrt(r * r + A * A)),                     # Plummer
    (0.0, 4.0, 1.0, lambda r: -G * M / (2 * A) * (1 - (r / (r + A)) ** 2)),          # Dehnen 0
    (1.5, 4.0, 1.0, lambda r: -G * M / (0.5 * A) * (1 - (r / (r + A)) ** 0.5)),      # Dehnen 3/2
    (2.0, 4.0, 1.0, lambda r: -G * M / A * np.log((r + A) / r)),                     # Jaffe
])
def test_spherical_profiles_match_closed_forms(gamma, beta, alpha, phi):
    rho = spheroid_density(mass=M, scaleRadius=A, gamma=gamma, beta=beta, alpha=alpha)
    c = _solve(rho)
    assert c.lm_labels == [(0, 0)]
    r = c.R_grid
    assert np.abs(c.phi[:, 0] / phi(r) - 1).max() < 1e-9
    h = 1e-6 * r
    d = (phi(r + h) - phi(r - h)) / (2 * h)
    assert np.abs(c.dphi_dr[:, 0] / d - 1).max() < 1e-6


def test_hernquist_mass_normalisation():
    rho = spheroid_density(mass=M, scaleRadius=A, gamma=1, beta=4, alpha=1)
    x = torch.tensor([A], dtype=torch.float64)
    z = torch.zeros(1, dtype=torch.float64)
    assert abs(float(rho(x, z, z)) / (M / (2 * math.pi * A ** 3) / 8) - 1) < 1e-9
    with pytest.raises(ValueError, match="infinite"):
        spheroid_density(mass=M, gamma=1, beta=3)


def _ellipsoidal_phi(x, y, z, p, q, rho0):
    """Potential of rho = rho0 / (m (1 + m)^3), m^2 = (x^2 + y^2/p^2 + z^2/q^2)/A^2, by the
    homoeoid integral -pi G p q int [psi(inf) - psi(m(tau))] / Delta(tau) dtau in log tau."""
    def f(u):
        tau = math.exp(u)
        m = math.sqrt(x * x / (1 + tau) + y * y / (p * p + tau) + z * z / (q * q + tau)) / A
        return tau * rho0 * A * A / (1 + m) ** 2 / math.sqrt((1 + tau) * (p * p + tau) * (q * q + tau))
    lr = math.log(x * x + y * y + z * z + 1.0)
    return -math.pi * G * p * q * (quad(f, -40, lr, limit=800, epsabs=0, epsrel=1e-13)[0]
                                   + quad(f, lr, lr + 60, limit=800, epsabs=0, epsrel=1e-13)[0])


def test_triaxial_hernquist_against_homoeoid_integral():
    p, q = 0.8, 0.6
    rho = spheroid_density(mass=M, scaleRadius=A, gamma=1, beta=4, alpha=1, axisRatioY=p, axisRatioZ=q)
    assert rho.symmetry == "triaxial"
    c = _solve(rho, lmax=16)
    assert all(l % 2 == 0 and m % 2 == 0 and m >= 0 for l, m in c.lm_labels)
    rho0 = M / (2 * math.pi * A ** 3 * p * q)
    rng = np.random.default_rng(0)
    for i in (5, 12, 20, 28, 35):
        u = rng.normal(size=3)
        u /= np.linalg.norm(u)
        Y = angular_basis(c.lm_labels, u[2:3], np.array([math.hypot(u[0], u[1])]),
                          np.array([math.atan2(u[1], u[0])]))[0]
        val = float((c.phi[i] * Y).sum())
        ex = _ellipsoidal_phi(*(c.R_grid[i] * u), p, q, rho0)
        assert abs(val / ex - 1) < 1e-8, (i, val, ex)


def test_angular_basis_monopole_is_one():
    Y = angular_basis([(0, 0), (2, 0), (2, 2), (2, -2)], np.array([0.3]), np.array([math.sqrt(0.91)]),
                      np.array([0.7]))
    assert abs(Y[0, 0] - MUL0 * 0.28209479177387814) < 1e-15 and abs(Y[0, 0] - 1) < 1e-15


def test_king_model_structure():
    """Kepler outside the tidal radius, the central value -sigma^2 W0 - GM/rt, a flat core."""
    Mk, r0, W0 = 1e5, 0.01, 6.0
    c = king_multipole(Mk, r0, W0)
    rt = float(c.params["tidalRadius"])
    assert 10 * r0 < rt < 100 * r0                    # W0 = 6: concentration log10(rt/r0) ~ 1.25
    r = c.R_grid
    out = r > rt
    assert np.allclose(c.phi[out, 0], -G * Mk / r[out], rtol=1e-14)
    inner = r < 0.05 * r0
    assert np.all(np.abs(c.dphi_dr[inner, 0] * r[inner]) < 0.05 * np.abs(c.phi[inner, 0] - c.phi[-1, 0]))
    # M(<r) = r^2 dPhi/dr / G reaches the total at r_t and is monotonic
    Mr = r * r * c.dphi_dr[:, 0] / G
    assert np.all(np.diff(Mr) >= -1e-9 * Mk) and abs(Mr[out][0] / Mk - 1) < 1e-12
    with pytest.raises(ValueError):
        king_multipole(Mk, r0, -1.0)


def test_disk_residual_density_is_smooth_in_the_plane():
    """The ansatz carries the disk's e^(-|z|/h) cusp: the residual vanishes in the plane
    (Sigma(R) = Sigma(r) at z = 0) and its slope jump across z = 0 is ~1e-5 of the disk's."""
    rho = disk_density(surfaceDensity=1e9, scaleRadius=3.0, scaleHeight=0.3)
    res = disk_residual_density(rho, rho.sigma0, 3.0, 0.3)
    R = torch.tensor([1.0, 3.0, 8.0], dtype=torch.float64)
    z0 = torch.zeros(3, dtype=torch.float64)
    assert torch.all(res(R, z0, z0).abs() < 1e-6 * rho(R, z0, z0))
    e = 1e-5
    for Rv in (1.0, 3.0, 8.0):
        X = torch.full((3,), Rv, dtype=torch.float64)
        Z = torch.tensor([-e, 0.0, e], dtype=torch.float64)
        v, w = res(X, 0 * X, Z), rho(X, 0 * X, Z)
        jump_res = float((v[2] - v[1]) - (v[1] - v[0])) / e
        jump_disk = float((w[2] - w[1]) - (w[1] - w[0])) / e
        assert abs(jump_res) < 1e-4 * abs(jump_disk), (Rv, jump_res, jump_disk)
    # the column of the disk itself: Sigma(R) (exponential law normalised to 1)
    zs = torch.linspace(-6, 6, 4001, dtype=torch.float64)
    for Rv in (2.0, 5.0):
        col = torch.trapezoid(rho(torch.full_like(zs, Rv), 0 * zs, zs), zs)
        assert abs(float(col) / (1e9 * math.exp(-Rv / 3.0)) - 1) < 1e-3


def test_miyamoto_nagai_density_axisymmetric():
    """An axisymmetric density with a closed-form potential (Miyamoto-Nagai, a = 3, b = 1)."""
    Mm, a, b = 5e10, 3.0, 1.0

    def rho(x, y, z):
        R2 = x * x + y * y
        zb = torch.sqrt(z * z + b * b)
        return (b * b * Mm / (4 * math.pi)) * (a * R2 + (a + 3 * zb) * (a + zb) ** 2) / (
            (R2 + (a + zb) ** 2) ** 2.5 * zb ** 3)

    # the density is a sheet of width ~b at large R: n_theta resolves it out to r ~ 100
    c = multipole_from_density(rho, lmax=32, symmetry="axisymmetric", device="cpu", length_hint=a,
                               rmin=0.05, rmax=500.0, gridSizeR=40, n_theta=2048, n_phi=1)
    worst = 0.0
    for i in (8, 16, 20, 24):
        r = c.R_grid[i]
        for ct in (0.0, 0.3, 0.7, 0.95):
            st = math.sqrt(1 - ct * ct)
            Y = angular_basis(c.lm_labels, np.array([ct]), np.array([st]), np.array([0.0]))[0]
            val = float((c.phi[i] * Y).sum())
            R, z = r * st, r * ct
            ex = -G * Mm / math.sqrt(R * R + (a + math.sqrt(z * z + b * b)) ** 2)
            worst = max(worst, abs(val / ex - 1))
    assert worst < 5e-4, worst


def test_solver_argument_checks():
    rho = spheroid_density(mass=M, scaleRadius=A)
    with pytest.raises(ValueError, match="symmetry"):
        multipole_from_density(rho, symmetry="bogus", device="cpu")
    with pytest.raises(ValueError, match="rmin"):
        multipole_from_density(rho, symmetry="spherical", rmin=10.0, rmax=1.0, device="cpu")
    with pytest.raises(ValueError, match="not both"):
        spheroid_density(mass=M, densityNorm=1.0)
    with pytest.raises(ValueError, match="thin"):
        disk_density(surfaceDensity=1e9, scaleHeight=0.0)
    with pytest.raises(ValueError, match="not both"):
        disk_density(surfaceDensity=1e9, mass=1e10)


def test_disk_mass_normalisation_and_sech2():
    """mass fixes Sigma0 = M / (2 pi Rd^2) for n = 1; the isothermal layer integrates to 1."""
    rho = disk_density(mass=5e10, scaleRadius=3.0, scaleHeight=-0.3)
    assert abs(rho.sigma0 / (5e10 / (2 * math.pi * 9.0)) - 1) < 1e-3
    zs = torch.linspace(-8, 8, 8001, dtype=torch.float64)
    col = torch.trapezoid(rho(torch.full_like(zs, 3.0), 0 * zs, zs), zs)
    assert abs(float(col) / (rho.sigma0 * math.exp(-1.0)) - 1) < 1e-4


def test_factory_builds_density_types_without_agama():
    import agama_gpu_b200 as agb
    s = agb.PotentialGPU(type="Spheroid", mass=1e11, scaleRadius=2.0, gamma=1, beta=4, alpha=1,
                         axisRatioZ=0.7, lmax=8, gridSizeR=30)
    assert isinstance(s, agb.MultipolePotentialGPU)
    assert all(l % 2 == 0 and m == 0 for l, m in s._coefs.lm_labels)      # axisymmetric
    d = agb.PotentialGPU(type="Dehnen", mass=1e10, scaleRadius=1.0, gamma=2.0)
    assert isinstance(d, agb.MultipolePotentialGPU) and d._coefs.lm_labels == [(0, 0)]
