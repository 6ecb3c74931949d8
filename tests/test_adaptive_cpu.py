"""Adaptive Dormand-Prince 5(4) integration (host logic) against scipy's DOP853 at a
tight tolerance, with a torch stand-in potential that has the GPU classes' _launch
hook: per-particle steps (static) and the shared step (time-dependent)."""
import math

import numpy as np
import pytest
import torch
from scipy.integrate import solve_ivp

from agama_gpu_b200.adaptive import DormandPrince, integrate_adaptive

G = 4.30091727067736e-06


class _Plummer:
    def __init__(self, M=1e11, b=1.0, eps=0.0, static=True):
        self.M, self.b, self.eps = M, b, eps
        self._time_independent = static and eps == 0.0

    def force_np(self, x, t):
        m = self.M * (1.0 + self.eps * math.sin(t / 0.05))
        r2 = (x * x).sum(-1, keepdims=True) + self.b * self.b
        return -G * m * x / r2 ** 1.5

    def _launch(self, x, t, mode, want_phi, precision=None, out=None):
        out[1].copy_(torch.from_numpy(self.force_np(x.numpy(), float(t))))


def _ref(pot, x0, v0, t0, t1):
    out = []
    for xi, vi in zip(x0, v0):
        f = lambda t, y: np.concatenate([y[3:], pot.force_np(y[None, :3], t)[0]])  # noqa: E731
        s = solve_ivp(f, (t0, t1), np.concatenate([xi, vi]), method="DOP853", rtol=1e-13, atol=1e-12)
        out.append(s.y[:, -1])
    return np.array(out)


def _ics(n, seed):
    rng = np.random.default_rng(seed)
    x = rng.normal(0, 5, (n, 3))
    v = rng.normal(0, 120, (n, 3))
    return x, v


@pytest.mark.parametrize("eps,per_particle", [(0.0, True), (0.0, False), (0.3, False)])
def test_matches_tight_reference(eps, per_particle):
    pot = _Plummer(eps=eps)
    x0, v0 = _ics(12, 1)
    dp = DormandPrince(pot, rtol=1e-10, atol=1e-10, per_particle=per_particle)
    x, v, st = dp.run(torch.from_numpy(x0), torch.from_numpy(v0), 0.1, 0.35)
    ref = _ref(pot, x0, v0, 0.1, 0.35)
    assert np.abs(x.numpy() - ref[:, :3]).max() < 1e-6 * np.abs(ref[:, :3]).max()
    assert np.abs(v.numpy() - ref[:, 3:]).max() < 1e-6 * np.abs(ref[:, 3:]).max()
    assert int(st["accepted"].min()) > 3


def test_per_particle_steps_are_independent():
    """In per-particle mode a particle's result does not depend on the others: run alone
    or in a batch, it takes the same steps (bit-identical)."""
    pot = _Plummer()
    x0, v0 = _ics(9, 2)
    dp = DormandPrince(pot, rtol=1e-8, per_particle=True)
    xa, va, sa = dp.run(torch.from_numpy(x0), torch.from_numpy(v0), 0.0, 0.2)
    for i in (0, 4, 8):
        xi, vi, si = dp.run(torch.from_numpy(x0[i:i + 1]), torch.from_numpy(v0[i:i + 1]), 0.0, 0.2)
        assert torch.equal(xi[0], xa[i]) and torch.equal(vi[0], va[i])
        assert int(si["accepted"][0]) == int(sa["accepted"][i])
    # the particles took different numbers of steps
    assert len(set(sa["accepted"].tolist())) > 1


def test_backwards_returns_to_start_and_edge_cases():
    pot = _Plummer()
    x0, v0 = _ics(6, 3)
    X0, V0 = torch.from_numpy(x0), torch.from_numpy(v0)
    x1, v1 = integrate_adaptive(pot, X0, V0, 0.0, 0.3, rtol=1e-12, atol=1e-12)
    dp = DormandPrince(pot, rtol=1e-12, atol=1e-12, per_particle=True)
    x2, v2, _ = dp.run(x1, v1, 0.3, 0.0)
    assert np.abs((x2 - X0).numpy()).max() < 1e-7 * np.abs(x0).max()
    x3, v3, st = dp.run(X0, V0, 0.5, 0.5)
    assert torch.equal(x3, X0) and st["iterations"] == 0
    with pytest.raises(ValueError):
        DormandPrince(pot, rtol=0.0)
    with pytest.raises(ValueError, match="depend on time"):
        DormandPrince(_Plummer(eps=0.2), per_particle=True)
