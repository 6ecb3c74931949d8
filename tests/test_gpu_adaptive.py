"""Adaptive Dormand-Prince 5(4) on the GPU evaluator against scipy's DOP853 driven by
the oracle's forces (static composite: per-particle steps; time-dependent: shared)."""
import numpy as np
import pytest
from scipy.integrate import solve_ivp

from oracle import cpu

pytestmark = pytest.mark.gpu


def _pot(static):
    import agama_gpu_b200 as agb
    from agama_gpu_b200.synthetic import circular_track, nfw_multipole
    parts = [agb.MultipolePotentialGPU(nfw_multipole(lmax=6, n_nodes=40, seed=2)),
             agb.MiyamotoNagaiPotentialGPU(mass=5e10, scaleRadius=3.0, scaleHeight=0.3)]
    if not static:
        parts.append(agb.ShiftedPotentialGPU(agb.NFWPotentialGPU(mass=2e11, scaleRadius=8.0),
                                             circular_track(T=100, radius=40.0)))
    return agb.CompositePotentialGPU(parts)


@pytest.mark.parametrize("static", [True, False])
def test_adaptive_matches_oracle_dop853(static):
    import torch
    from agama_gpu_b200.adaptive import DormandPrince
    pot = _pot(static)
    rng = np.random.default_rng(4)
    R = rng.uniform(4, 20, 6)
    ph = rng.uniform(0, 2 * np.pi, 6)
    x0 = np.stack([R * np.cos(ph), R * np.sin(ph), rng.normal(0, 0.5, 6)], 1)
    v0 = np.stack([-200 * np.sin(ph), 200 * np.cos(ph), rng.normal(0, 10, 6)], 1)
    t0, t1 = 0.2, 0.45
    dp = DormandPrince(pot, rtol=1e-10, atol=1e-10, precision="fp64")
    assert dp.static == static
    x, v, st = dp.run(torch.from_numpy(x0).cuda(), torch.from_numpy(v0).cuda(), t0, t1)
    x, v = x.cpu().numpy(), v.cpu().numpy()
    for i in range(6):
        f = lambda t, y: np.concatenate([y[3:], -cpu.eval_potential(pot, 1, y[None, :3], t)[1][0]])  # noqa: E731
        s = solve_ivp(f, (t0, t1), np.concatenate([x0[i], v0[i]]), method="DOP853", rtol=1e-12, atol=1e-12)
        assert np.abs(x[i] - s.y[:3, -1]).max() < 1e-6 * np.abs(s.y[:3, -1]).max(), i
        assert np.abs(v[i] - s.y[3:, -1]).max() < 1e-6 * np.abs(s.y[3:, -1]).max(), i
    if static:
        assert len(set(st["accepted"].tolist())) > 1          # own steps per particle
