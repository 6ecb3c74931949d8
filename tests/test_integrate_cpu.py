"""Host logic of the integrators (substep schedule, checkpoints, adjoint) on the CPU.

The potential is a torch stand-in with the same three hooks the integrator calls
on a GPU potential (_launch for the force, _vjp for (dF/dx)^T g): a Plummer sphere
whose mass varies in time, so the substep times enter the result.  The adjoint is
compared with autograd through the same scheme written in plain torch.
"""
import math

import pytest
import torch

from agama_gpu_b200.integrate import SCHEMES, Leapfrog, leapfrog, scheme_coefficients


class _Plummer:
    def __init__(self, b=1.0, eps=0.1):
        self.b, self.eps = b, eps

    def force(self, x, t):
        m = 1.0 + self.eps * math.sin(t) if isinstance(t, float) else 1.0 + self.eps * torch.sin(t)
        r2 = (x * x).sum(-1, keepdim=True) + self.b * self.b
        return -m * x / r2 ** 1.5

    def _launch(self, x, t, mode, want_phi, precision=None, out=None):
        out[1].copy_(self.force(x, float(t)))

    def _vjp(self, x, t, gphi, gforce, precision=None, out=None, force_out=None):
        with torch.enable_grad():
            xr = x.detach().clone().requires_grad_(True)
            (g,) = torch.autograd.grad(self.force(xr, float(t)), xr, gforce)
        out.copy_(g)
        if force_out is not None:
            force_out.copy_(self.force(x, float(t)))


def _torch_scheme(pot, x, v, dt, n_steps, coefs, t0=0.0):
    """The same scheme with autograd-tracked torch ops (no in-place updates)."""
    t = t0
    for n in range(n_steps):
        t_start = t0 + n * dt
        cum = 0.0
        for c in coefs:
            cum += c
            v = v + 0.5 * c * dt * pot.force(x, t_start + (cum - c) * dt)
            x = x + c * dt * v
            v = v + 0.5 * c * dt * pot.force(x, t_start + cum * dt)
    return x, v


def _ics(n=64, seed=3):
    g = torch.Generator().manual_seed(seed)
    x = torch.randn(n, 3, generator=g, dtype=torch.float64)
    v = 0.5 * torch.randn(n, 3, generator=g, dtype=torch.float64)
    return x, v


def test_scheme_coefficients():
    assert scheme_coefficients("leapfrog") == (1.0,)
    c = scheme_coefficients("yoshida4")
    assert len(c) == 3 and abs(sum(c) - 1.0) < 1e-15 and c[1] < 0
    # 4th order conditions of the symmetric triple: sum c = 1, sum c^3 = 0
    assert abs(sum(x ** 3 for x in c)) < 1e-14
    with pytest.raises(ValueError):
        scheme_coefficients("rk45")
    with pytest.raises(ValueError):
        scheme_coefficients((0.5, 0.4))
    assert set(SCHEMES) >= {"leapfrog", "yoshida4"}


@pytest.mark.parametrize("scheme", ["leapfrog", "yoshida4"])
def test_forward_matches_torch(scheme):
    pot = _Plummer()
    x0, v0 = _ics()
    integ = Leapfrog(pot, 0.05, t0=0.3, scheme=scheme)
    xT, vT, _ = integ.run(x0, v0, 40, checkpoint_every=7)
    xr, vr = _torch_scheme(pot, x0, v0, 0.05, 40, SCHEMES[scheme], t0=0.3)
    assert torch.allclose(xT, xr, rtol=0, atol=1e-13)
    assert torch.allclose(vT, vr, rtol=0, atol=1e-13)


@pytest.mark.parametrize("scheme", ["leapfrog", "yoshida4"])
@pytest.mark.parametrize("k", [1, 3, 64, None])
def test_adjoint_matches_autograd(scheme, k):
    pot = _Plummer()
    x0, v0 = _ics(32)
    n_steps, dt = 25, 0.07
    wx = torch.randn(x0.shape, generator=torch.Generator().manual_seed(7), dtype=torch.float64)
    wv = torch.randn(x0.shape, generator=torch.Generator().manual_seed(8), dtype=torch.float64)
    xa, va = x0.clone().requires_grad_(True), v0.clone().requires_grad_(True)
    xr, vr = _torch_scheme(pot, xa, va, dt, n_steps, SCHEMES[scheme], t0=0.1)
    ((xr * wx).sum() + (vr * wv).sum()).backward()
    integ = Leapfrog(pot, dt, t0=0.1, scheme=scheme)
    xT, vT, ck = integ.run(x0, v0, n_steps, checkpoint_every=k)
    lx, lv = integ.adjoint(ck, n_steps, wx, wv)
    assert torch.allclose(lx, xa.grad, rtol=1e-11, atol=1e-12)
    assert torch.allclose(lv, va.grad, rtol=1e-11, atol=1e-12)


def test_autograd_function_yoshida4():
    pot = _Plummer()
    x0, v0 = _ics(16)
    xa, va = x0.clone().requires_grad_(True), v0.clone().requires_grad_(True)
    xT, vT = leapfrog(pot, xa, va, 0.05, 12, checkpoint_every=5, scheme="yoshida4")
    (xT ** 2).sum().backward()          # only x_T carries a cotangent
    xb, vb = x0.clone().requires_grad_(True), v0.clone().requires_grad_(True)
    xr, _ = _torch_scheme(pot, xb, vb, 0.05, 12, SCHEMES["yoshida4"])
    (xr ** 2).sum().backward()
    assert torch.allclose(xa.grad, xb.grad, rtol=1e-11, atol=1e-12)
    assert torch.allclose(va.grad, vb.grad, rtol=1e-11, atol=1e-12)


def test_order_of_accuracy():
    """Global error falls as dt^2 for leapfrog and dt^4 for yoshida4."""
    pot = _Plummer(eps=0.0)
    x0, v0 = _ics(8, seed=11)
    T = 2.0
    ref, _, _ = Leapfrog(pot, T / 2000, scheme="yoshida4").run(x0, v0, 2000, checkpoint_every=4000)
    for scheme, order in (("leapfrog", 2), ("yoshida4", 4)):
        errs = []
        for n in (40, 80):
            xT, _, _ = Leapfrog(pot, T / n, scheme=scheme).run(x0, v0, n, checkpoint_every=1000)
            errs.append((xT - ref).abs().max().item())
        rate = math.log2(errs[0] / errs[1])
        assert abs(rate - order) < 0.35, (scheme, errs, rate)


@pytest.mark.parametrize("scheme", ["leapfrog", "yoshida4"])
@pytest.mark.parametrize("k", [2, 7, 64])
def test_reverse_reconstruction_matches_autograd(scheme, k):
    """Positions between checkpoints stepped backwards from the later checkpoint with
    the forces of the VJP launches: the gradients of the exact trajectory to rounding."""
    pot = _Plummer()
    x0, v0 = _ics(32)
    n_steps, dt = 25, 0.07
    wx = torch.randn(x0.shape, generator=torch.Generator().manual_seed(7), dtype=torch.float64)
    wv = torch.randn(x0.shape, generator=torch.Generator().manual_seed(8), dtype=torch.float64)
    xa, va = x0.clone().requires_grad_(True), v0.clone().requires_grad_(True)
    xr, vr = _torch_scheme(pot, xa, va, dt, n_steps, SCHEMES[scheme], t0=0.1)
    ((xr * wx).sum() + (vr * wv).sum()).backward()
    integ = Leapfrog(pot, dt, t0=0.1, scheme=scheme)
    xT, vT, ck = integ.run(x0, v0, n_steps, checkpoint_every=k)
    lx, lv = integ.adjoint(ck, n_steps, wx, wv, reconstruct="reverse")
    assert torch.allclose(lx, xa.grad, rtol=1e-9, atol=1e-10)
    assert torch.allclose(lv, va.grad, rtol=1e-9, atol=1e-10)
    with pytest.raises(ValueError):
        integ.adjoint(ck, n_steps, wx, wv, reconstruct="bogus")
