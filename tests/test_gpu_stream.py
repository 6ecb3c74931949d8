"""Particle-spray streams on the GPU: the forward against a CPU loop over the
oracle's forces and Hessians, and the adjoint's table and release-state
gradients against central differences."""
import numpy as np
import pytest

from oracle import cpu

pytestmark = pytest.mark.gpu

PROG = ([12.0, 0.0, 2.0], [0.0, 170.0, 25.0], 5e7)


def _host(coefs=None):
    import agama_gpu_b200 as agb
    from agama_gpu_b200.synthetic import nfw_multipole
    c = coefs if coefs is not None else nfw_multipole(lmax=4, n_nodes=30, seed=8, amp=0.3)
    return agb.MultipolePotentialGPU(c) + agb.MiyamotoNagaiPotentialGPU(
        mass=5e10, scaleRadius=3.0, scaleHeight=0.3)


def _oracle_spray(pot, prog_pot, x_p, v_p, mass, t_end, n_steps, dt, release_every, seed):
    """The same stream with every force and Hessian from the oracle (numpy, one
    particle set at a time)."""
    import torch
    import agama_gpu_b200 as agb
    from agama_gpu_b200.stream import draw_k, release_states

    def force(p, x, t):
        return -cpu.eval_potential(p, 1, x, t)[1]

    h = 0.5 * dt
    x, v = np.array([x_p], float), np.array([v_p], float)
    F = force(pot, x, t_end)
    rec = [(x[0].copy(), v[0].copy())]
    for n in range(n_steps):                      # backwards: dt -> -dt
        v = v - h * F
        x = x - dt * v
        F = force(pot, x, t_end - (n + 1) * dt)
        v = v - h * F
        rec.append((x[0].copy(), v[0].copy()))
    rec = rec[::-1]
    t0 = t_end - n_steps * dt
    times = t0 + dt * np.arange(n_steps + 1)
    times[-1] = t_end
    track = np.array([[times[i], *rec[i][0], *rec[i][1]] for i in range(n_steps + 1)])
    steps = np.arange(0, n_steps, release_every)
    xs = np.array([rec[s][0] for s in steps])
    vs = np.array([rec[s][1] for s in steps])
    d = np.concatenate([-cpu.eval_potential(pot, 2, xs[i:i + 1], times[s])[2]
                        for i, s in enumerate(steps)])
    xr, vr, _ = release_states(torch.from_numpy(xs), torch.from_numpy(vs), torch.from_numpy(d),
                               mass, draw_k(len(steps), seed))
    xr, vr = xr.numpy(), vr.numpy()
    spot = pot + agb.ShiftedPotentialGPU(prog_pot, track)
    X, V, Fa = np.zeros_like(xr), np.zeros_like(vr), np.zeros_like(xr)
    a = 0
    for n in range(n_steps):
        a_new = 2 * int(np.searchsorted(steps, n, side="right"))
        if a_new > a:
            X[a:a_new], V[a:a_new] = xr[a:a_new], vr[a:a_new]
            Fa[a:a_new] = force(spot, X[a:a_new], t0 + n * dt)
            a = a_new
        V[:a] += h * Fa[:a]
        X[:a] += dt * V[:a]
        Fa[:a] = force(spot, X[:a], t0 + n * dt + dt)
        V[:a] += h * Fa[:a]
    return X, V, track


def test_spray_matches_oracle_loop():
    import agama_gpu_b200 as agb
    from agama_gpu_b200.stream import particle_spray
    pot = _host()
    prog = agb.PlummerPotentialGPU(mass=PROG[2], scaleRadius=0.05)
    args = (PROG[0], PROG[1], PROG[2], 0.3, 40, 0.002)
    s = particle_spray(pot, *args, release_every=2, seed=6, prog_pot=prog, precision="fp64")
    X, V, track = _oracle_spray(pot, prog, *args, 2, 6)
    assert np.allclose(s.track, track, rtol=1e-11, atol=1e-11)
    x, v = s.x.cpu().numpy(), s.v.cpu().numpy()
    assert np.abs(x - X).max() < 1e-9 * np.abs(X).max()
    assert np.abs(v - V).max() < 1e-9 * np.abs(V).max()


@pytest.mark.parametrize("scheme", ["leapfrog", "yoshida4"])
def test_spray_adjoint_matches_finite_differences(scheme):
    """Table gradients (Multipole nodes) and release-state gradients, release states held
    fixed, against central differences of the GPU forward."""
    import torch
    import agama_gpu_b200 as agb
    from agama_gpu_b200.stream import integrate_releases, particle_spray
    from agama_gpu_b200.synthetic import nfw_multipole
    coefs = nfw_multipole(lmax=4, n_nodes=30, seed=8, amp=0.3)
    prog = agb.PlummerPotentialGPU(mass=PROG[2], scaleRadius=0.05)
    n_steps, dt, every = 30, 0.002, 3
    s0 = particle_spray(_host(coefs), PROG[0], PROG[1], PROG[2], 0.3, n_steps, dt,
                        release_every=every, seed=3, prog_pot=prog, precision="fp64", scheme=scheme)
    target = s0.x.detach() * 1.05
    t0 = 0.3 - n_steps * dt
    steps = np.arange(0, n_steps, every)
    shifted = agb.ShiftedPotentialGPU(prog, s0.track)

    def run(c, xr=None, vr=None, want=False):
        mp = agb.MultipolePotentialGPU(c)
        spot = mp + agb.MiyamotoNagaiPotentialGPU(mass=5e10, scaleRadius=3.0, scaleHeight=0.3) + shifted
        st = integrate_releases(spot, s0.x_release if xr is None else xr,
                                s0.v_release if vr is None else vr, steps, t0, n_steps, dt,
                                scheme=scheme, precision="fp64", store=want)
        L = float(((st.x - target) ** 2).sum() + 0.01 * (st.v ** 2).sum())
        if not want:
            return L
        lx, lv, tg = st.adjoint(2 * (st.x - target), 0.02 * st.v, table_grads=True)
        return L, mp, lx, lv, tg[mp]

    _, mp, lx, lv, gpoly = run(coefs, want=True)
    gnp, _ = (a.cpu().numpy() for a in mp.node_gradients(gpoly))
    lab = coefs.lm_labels
    for i, c in [(12, lab.index((0, 0))), (15, lab.index((2, 0)))]:
        hh = 1e-5 * np.abs(coefs.phi[:, c]).max()
        cp_ = agb.MultipoleCoefs(coefs.R_grid, coefs.phi.copy(), coefs.dphi_dr.copy(), lab)
        cm_ = agb.MultipoleCoefs(coefs.R_grid, coefs.phi.copy(), coefs.dphi_dr.copy(), lab)
        cp_.phi[i, c] += hh
        cm_.phi[i, c] -= hh
        fd = (run(cp_) - run(cm_)) / (2 * hh)
        assert abs(gnp[i, c] - fd) <= 1e-4 * max(abs(fd), 1e-3 * np.abs(gnp).max()), (i, c, gnp[i, c], fd)
    rng = np.random.default_rng(0)
    for p, d in [(int(rng.integers(len(steps) * 2)), int(rng.integers(3))) for _ in range(4)]:
        for which, lam, hh in (("x", lx, 1e-4), ("v", lv, 1e-3)):
            base = s0.x_release if which == "x" else s0.v_release
            bp, bm = base.clone(), base.clone()
            bp[p, d] += hh
            bm[p, d] -= hh
            kw = ({"xr": bp}, {"xr": bm}) if which == "x" else ({"vr": bp}, {"vr": bm})
            fd = (run(coefs, **kw[0]) - run(coefs, **kw[1])) / (2 * hh)
            an = float(lam[p, d])
            assert abs(an - fd) <= 1e-5 * max(abs(fd), 1e-3 * float(lam.abs().max())), (which, p, d, an, fd)
    assert torch.isfinite(lx).all() and torch.isfinite(lv).all()
