"""Particle-spray streams on the CPU: the release model's known answers, the
prefix-batched forward against per-particle integration, and the adjoint against
autograd.  The potential is a torch stand-in with the hooks the GPU classes give
the integrator (_launch, _vjp, forceDeriv)."""
import math

import numpy as np
import pytest
import torch

from agama_gpu_b200.integrate import SCHEMES
from agama_gpu_b200.stream import G_AGAMA, draw_k, particle_spray, release_states


class _Plummer:
    """Plummer sphere (mass M, scale b) whose mass varies as 1 + eps sin(t / 0.1)."""

    def __init__(self, M=1e11, b=2.0, eps=0.05):
        self.M, self.b, self.eps = M, b, eps

    def _m(self, t):
        return self.M * (1.0 + self.eps * math.sin(float(t) / 0.1))

    def force(self, x, t):
        r2 = (x * x).sum(-1, keepdim=True) + self.b * self.b
        return -G_AGAMA * self._m(t) * x / r2 ** 1.5

    def _launch(self, x, t, mode, want_phi, precision=None, out=None):
        out[1].copy_(self.force(x, t))

    def _vjp(self, x, t, gphi, gforce, precision=None, out=None):
        with torch.enable_grad():
            xr = x.detach().clone().requires_grad_(True)
            (g,) = torch.autograd.grad(self.force(xr, t), xr, gforce)
        out.copy_(g)

    def forceDeriv(self, x, t=0.0):
        x = torch.as_tensor(x, dtype=torch.float64).reshape(-1, 3)
        J = torch.func.vmap(torch.func.jacrev(lambda p: self.force(p[None], t)[0]))(x)
        d = torch.stack([J[:, 0, 0], J[:, 1, 1], J[:, 2, 2], J[:, 0, 1], J[:, 1, 2], J[:, 2, 0]], 1)
        return self.force(x, t), d


def test_jacobi_radius_point_mass():
    """Circular orbit around a point mass M: r_J = r (m / 3M)^(1/3)."""
    M, m, r = 1e11, 1e7, 20.0
    vc = math.sqrt(G_AGAMA * M / r)
    x = torch.tensor([[r, 0.0, 0.0]], dtype=torch.float64)
    v = torch.tensor([[0.0, vc, 0.0]], dtype=torch.float64)
    # point-mass force derivatives at (r, 0, 0): dFx/dx = 2GM/r^3, dFy/dy = dFz/dz = -GM/r^3
    gm = G_AGAMA * M / r ** 3
    d = torch.tensor([[2 * gm, -gm, -gm, 0.0, 0.0, 0.0]], dtype=torch.float64)
    k = torch.tensor([[[1.0, 0.0, 0.0, 0.0], [1.0, 0.0, 0.0, 0.0]]], dtype=torch.float64)
    xr, vr, rj = release_states(x, v, d, m, k)
    assert abs(rj.item() - r * (m / (3 * M)) ** (1 / 3)) < 1e-12 * r
    # k = (1, 0, 0, 0): the pair sits at the two Lagrange points with the progenitor's velocity
    assert torch.allclose(xr[0], torch.tensor([r - rj.item(), 0, 0], dtype=torch.float64))
    assert torch.allclose(xr[1], torch.tensor([r + rj.item(), 0, 0], dtype=torch.float64))
    assert torch.equal(vr, v.expand(2, 3))


def test_release_frame_offsets():
    """k_z and k_vz move along L^, k_vt along phi^ with the sign of the side."""
    x = torch.tensor([[8.0, 0.0, 0.0]], dtype=torch.float64)
    v = torch.tensor([[0.0, 200.0, 0.0]], dtype=torch.float64)
    d = torch.tensor([[1e3, -5e2, -5e2, 0.0, 0.0, 0.0]], dtype=torch.float64)
    k = torch.tensor([[[0.0, 1.0, 1.0, 0.0], [0.0, 0.0, 1.0, 1.0]]], dtype=torch.float64)
    xr, vr, rj = release_states(x, v, d, 1e6, k)
    om = 200.0 / 8.0
    R = rj.item()
    assert torch.allclose(xr[0] - x[0], torch.tensor([0, 0, R], dtype=torch.float64))
    assert torch.allclose(xr[1], x[0])
    assert torch.allclose(vr[0] - v[0], torch.tensor([0, -om * R, 0], dtype=torch.float64))
    assert torch.allclose(vr[1] - v[0], torch.tensor([0, om * R, om * R], dtype=torch.float64))


def test_no_tidal_radius_gives_zero_offset():
    x = torch.tensor([[8.0, 0.0, 0.0]], dtype=torch.float64)
    v = torch.tensor([[0.0, 1.0, 0.0]], dtype=torch.float64)          # Omega^2 tiny
    d = torch.tensor([[-1e4, 0.0, 0.0, 0.0, 0.0, 0.0]], dtype=torch.float64)
    xr, vr, rj = release_states(x, v, d, 1e6, draw_k(1, 0))
    assert rj.item() == 0.0 and torch.equal(xr, x.expand(2, 3)) and torch.equal(vr, v.expand(2, 3))


def test_draw_k_seeded():
    a, b = draw_k(1000, 5), draw_k(1000, 5)
    assert torch.equal(a, b)
    assert abs(a[..., 0].mean().item() - 2.0) < 0.05 and abs(a[..., 0].std().item() - 0.5) < 0.05
    c = draw_k(10, 5, {"k_r": (1.0, 0.0)})
    assert torch.all(c[..., 0] == 1.0)


def _per_particle(pot, s, dt, n_steps, coefs, t_end, release_every):
    """Each particle integrated alone from its release step (autograd-friendly)."""
    t_start = t_end - n_steps * dt
    xs, vs = [], []
    xr = s.x_release.clone().requires_grad_(True)
    vr = s.v_release.clone().requires_grad_(True)
    for i in range(xr.shape[0]):
        n0 = (i // 2) * release_every
        x, v = xr[i:i + 1], vr[i:i + 1]
        for n in range(n0, n_steps):
            ts = t_start + n * dt
            cum = 0.0
            for c in coefs:
                v = v + 0.5 * c * dt * pot.force(x, ts + cum * dt)
                x = x + c * dt * v
                cum += c
                v = v + 0.5 * c * dt * pot.force(x, ts + cum * dt)
        xs.append(x)
        vs.append(v)
    return torch.cat(xs), torch.cat(vs), xr, vr


@pytest.mark.parametrize("scheme,release_every", [("leapfrog", 1), ("leapfrog", 3), ("yoshida4", 2)])
def test_spray_forward_and_adjoint(scheme, release_every):
    pot = _Plummer()
    n_steps, dt, t_end = 13, 0.004, 0.7
    s = particle_spray(pot, [15.0, 0.0, 1.0], [0.0, 140.0, 20.0], 2e7, t_end, n_steps, dt,
                       release_every=release_every, seed=4, scheme=scheme, device="cpu")
    R = len(range(0, n_steps, release_every))
    assert s.x.shape == (2 * R, 3) and s.t_release.shape == (2 * R,)
    assert abs(s.track[0, 0] - (t_end - n_steps * dt)) < 1e-12 and s.track[-1, 0] == t_end
    assert torch.all(s.r_jacobi > 0)
    # the progenitor track ends where it started
    assert np.allclose(s.track[-1, 1:4], [15.0, 0.0, 1.0]) and np.allclose(s.track[-1, 4:7], [0, 140, 20])
    xr, vr, xa, va = _per_particle(pot, s, dt, n_steps, SCHEMES[scheme], t_end, release_every)
    assert torch.allclose(s.x, xr, rtol=0, atol=1e-12)
    assert torch.allclose(s.v, vr, rtol=0, atol=1e-10)
    g = torch.Generator().manual_seed(1)
    wx = torch.randn(s.x.shape, generator=g, dtype=torch.float64)
    wv = torch.randn(s.x.shape, generator=g, dtype=torch.float64)
    ((xr * wx).sum() + (vr * wv).sum()).backward()
    lx, lv = s.adjoint(wx, wv)
    assert torch.allclose(lx, xa.grad, rtol=1e-10, atol=1e-12)
    assert torch.allclose(lv, va.grad, rtol=1e-10, atol=1e-12)


def test_spray_release_positions_track_the_progenitor():
    pot = _Plummer(eps=0.0)
    s = particle_spray(pot, [10.0, 0.0, 0.0], [0.0, 180.0, 0.0], 1e7, 0.0, 20, 0.005, seed=2,
                       device="cpu", store=False)
    prog = torch.as_tensor(s.track[:-1, 1:4])                         # release at each step
    d = (s.x_release.reshape(-1, 2, 3) - prog[:, None, :]).norm(dim=-1)
    assert torch.all(d < 6 * s.r_jacobi[:, None])
    with pytest.raises(RuntimeError):
        s.adjoint(s.x, s.v)
