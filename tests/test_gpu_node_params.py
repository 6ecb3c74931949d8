"""Node tables as torch.autograd inputs, on the GPU.

``pot.node_parameters()`` hands out a Multipole's (Phi, dPhi/dr) node tables and
a CylSpline's Phi_m grids as leaf tensors; the differentiable entry points
(``agb.leapfrog``, ``autograd.potential_and_force``,
``stream.integrate_releases_autograd``) take them as inputs, so
``loss.backward()`` fills their ``.grad``.  Checked against central finite
differences of the GPU forward (perturbing the tensors in place, which the next
evaluation picks up) and against torch autograd through an FP64 torch
restatement of the whole computation (oracle/torch_mp.py for the Multipole,
the table builder's differentiable restatement, a torch leapfrog).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

G = 4.30091727067736e-06


def _pot(lmax=4, n_nodes=30):
    import agama_gpu_b200 as agb
    from agama_gpu_b200.synthetic import nfw_multipole
    mp = agb.MultipolePotentialGPU(nfw_multipole(lmax=lmax, n_nodes=n_nodes, seed=21, amp=0.1))
    mn = agb.MiyamotoNagaiPotentialGPU(mass=5e10, scaleRadius=3.0, scaleHeight=0.3)
    return mp, mn, mp + mn


def _orbits(pot, n=48, seed=5):
    import torch
    rng = np.random.default_rng(seed)
    R = rng.uniform(8.0, 30.0, n)
    ph = rng.uniform(0, 2 * np.pi, n)
    x = np.stack([R * np.cos(ph), R * np.sin(ph), rng.normal(0, 1.0, n)], 1)
    f = pot.force(x).cpu().numpy()
    vc = np.sqrt(np.maximum(-(f * x).sum(1), 1.0))
    v = np.stack([-np.sin(ph), np.cos(ph), np.zeros(n)], 1) * vc[:, None] + rng.normal(0, 5.0, (n, 3))
    x0 = torch.from_numpy(x).cuda()
    v0 = torch.from_numpy(v).cuda()
    target = x0 + torch.from_numpy(rng.normal(0, 0.5, x.shape)).cuda()
    return x0, v0, target


DT, STEPS = 2e-3, 24


def _loss(xT, vT, target):
    return ((xT - target) ** 2).sum() + 1e-4 * (vT ** 2).sum()


def _mn_force_torch(x, M=5e10, a=3.0, b=0.3):
    R2 = x[:, 0] ** 2 + x[:, 1] ** 2
    zb = (x[:, 2] ** 2 + b * b).sqrt()
    d = (R2 + (a + zb) ** 2) ** 1.5
    GM = G * M
    fz = -GM * x[:, 2] * (a + zb) / (zb * d)
    return torch_stack([-GM * x[:, 0] / d, -GM * x[:, 1] / d, fz])


def torch_stack(cols):
    import torch
    return torch.stack(cols, dim=1)


def _torch_leapfrog_loss(mp, phi, dphi, x0, v0, target):
    """The same leapfrog in FP64 torch with the Multipole force from the node tables
    (builder restatement -> oracle/torch_mp.py) plus Miyamoto-Nagai; autograd-able."""
    import torch
    from agama_gpu_b200.diff_tables import multipole_consts_from_nodes, multipole_poly_from_nodes
    from oracle.torch_mp import multipole_phi
    t = mp.tables
    # invPhi0 a function of the nodes, as the builder makes it (the orbits stay inside
    # the radial grid, where it is the only one of the builder's scalars in use)
    k = multipole_consts_from_nodes(t, phi, dphi)
    poly = multipole_poly_from_nodes(t, phi, dphi, inv=k[0])
    sc = list(t.scalars())
    sc[3] = k[0]

    def force(x):
        with torch.enable_grad():
            xr = x if x.requires_grad else x.detach().requires_grad_(True)
            p = multipole_phi(poly, t.lm_l, t.lm_m, sc, t.log_scaling, xr)
            (g,) = torch.autograd.grad(p.sum(), xr, create_graph=True)
        return -g + _mn_force_torch(x)

    h = 0.5 * DT
    x, v = x0.clone().requires_grad_(True), v0.clone()
    F = force(x)
    for _ in range(STEPS):
        v = v + h * F
        x = x + DT * v
        F = force(x)
        v = v + h * F
    return _loss(x, v, target)


def test_leapfrog_backward_fills_node_grads():
    import torch
    import agama_gpu_b200 as agb
    mp, _, pot = _pot()
    pot.set_precision("fp64")
    phi, dphi = mp.node_parameters()
    assert [q.data_ptr() for q in pot.node_parameters()] == [phi.data_ptr(), dphi.data_ptr()]
    x0, v0, target = _orbits(pot)
    xT, vT = agb.leapfrog(pot, x0, v0, DT, STEPS, checkpoint_every=8, precision="fp64")
    _loss(xT, vT, target).backward()
    gphi, gdphi = phi.grad.clone(), dphi.grad.clone()
    assert torch.isfinite(gphi).all() and float(gphi.abs().max()) > 0

    # 1. torch autograd through an FP64 torch restatement of the whole computation
    pt = phi.detach().cpu().clone().requires_grad_(True)
    dt_ = dphi.detach().cpu().clone().requires_grad_(True)
    Lt = _torch_leapfrog_loss(mp, pt, dt_, x0.cpu(), v0.cpu(), target.cpu())
    Lt.backward()
    for got, want in ((gphi.cpu(), pt.grad), (gdphi.cpu(), dt_.grad)):
        err = float((got - want).abs().max() / want.abs().max())
        assert err < 1e-8, err

    # 2. central finite differences of the GPU forward: the in-place change of a node
    # tensor is what the next evaluation sees
    def L():
        with torch.no_grad():
            a, b = agb.leapfrog(pot, x0, v0, DT, STEPS, checkpoint_every=8, precision="fp64")
            return float(_loss(a, b, target))
    rng = np.random.default_rng(2)
    for q, g in ((phi, gphi), (dphi, gdphi)):
        flat = g.abs().flatten()
        picks = torch.topk(flat, 3).indices.tolist() + list(rng.integers(0, flat.numel(), 2))
        for j in picks:
            i0, c0 = divmod(int(j), q.shape[1])
            v = float(q.detach()[i0, c0])
            h = 1e-5 * max(abs(v), 1e-3 * float(q.abs().max()))
            with torch.no_grad():
                q[i0, c0] = v + h
            lp = L()
            with torch.no_grad():
                q[i0, c0] = v - h
            lm = L()
            with torch.no_grad():
                q[i0, c0] = v
            fd = (lp - lm) / (2 * h)
            scale = float(g.abs().max())
            assert abs(fd - float(g[i0, c0])) <= 2e-4 * scale + 1e-6 * abs(fd), (j, fd, float(g[i0, c0]))
    pot.set_precision(None)


def test_potential_and_force_node_grads_and_in_place_updates():
    import torch
    from agama_gpu_b200 import autograd
    from agama_gpu_b200.diff_tables import multipole_consts_from_nodes, multipole_poly_from_nodes
    from oracle.torch_mp import multipole_phi
    mp, _, pot = _pot(lmax=6)
    phi, dphi = mp.node_parameters()
    x, _, _ = _orbits(pot, n=200, seed=9)
    rng = np.random.default_rng(4)
    gp = torch.from_numpy(rng.normal(size=200)).cuda()
    gf = torch.from_numpy(rng.normal(size=(200, 3))).cuda()
    # an in-place update of the node tensors changes the potential (the harmonics: the
    # monopole must stay within the log-scaling's range fixed at construction)
    with torch.no_grad():
        phi[:, 1:].mul_(1.01)
        dphi[:, 1:].mul_(0.99)
    p1, f1 = autograd.potential_and_force(pot, x, 0.0, precision="fp64")
    mp2, _, pot2 = _pot(lmax=6)
    mp2.set_node_tables(phi.detach(), dphi.detach())
    p2, f2 = pot2.eval(x, pot=True, acc=True)
    assert torch.equal(p1, p2) and torch.equal(f1, f2)
    ((p1 * gp).sum() + (f1 * gf).sum()).backward()
    # torch autograd of the same loss through the restatement, invPhi0 a function of
    # the nodes as the builder makes it (the points stay inside the radial grid)
    t = mp.tables
    pt = phi.detach().cpu().clone().requires_grad_(True)
    dt_ = dphi.detach().cpu().clone().requires_grad_(True)
    k = multipole_consts_from_nodes(t, pt, dt_)
    poly = multipole_poly_from_nodes(t, pt, dt_, inv=k[0])
    xr = x.cpu().clone().requires_grad_(True)
    r = xr.detach().norm(dim=1)
    assert float(r.min()) > t.r_grid[0] and float(r.max()) < t.r_grid[-1]
    sc = list(t.scalars())
    sc[3] = k[0]
    ph = multipole_phi(poly, t.lm_l, t.lm_m, sc, t.log_scaling, xr)
    (g,) = torch.autograd.grad(ph.sum(), xr, create_graph=True)
    ((ph * gp.cpu()).sum() - (g * gf.cpu()).sum()).backward()
    for got, want in ((phi.grad.cpu(), pt.grad), (dphi.grad.cpu(), dt_.grad)):
        assert float((got - want).abs().max() / want.abs().max()) < 1e-9


def test_cylspline_node_grads_through_leapfrog():
    import torch
    import agama_gpu_b200 as agb
    from agama_gpu_b200.synthetic import bar_cylspline
    cs = agb.CylSplinePotentialGPU(bar_cylspline(n_R=20, n_z=20))
    grids = cs.node_parameters()
    assert len(grids) == len(cs._node_keys())
    x0, v0, target = _orbits(cs, n=32, seed=7)
    xT, vT = agb.leapfrog(cs, x0, v0, DT, 12, checkpoint_every=4, precision="fp64")
    _loss(xT, vT, target).backward()

    def L():
        with torch.no_grad():
            a, b = agb.leapfrog(cs, x0, v0, DT, 12, checkpoint_every=4, precision="fp64")
            return float(_loss(a, b, target))
    for k in (0, len(grids) - 1):
        q, g = grids[k], grids[k].grad
        j = int(torch.argmax(g.abs()))
        i0, c0 = divmod(j, q.shape[1])
        v = float(q.detach()[i0, c0])
        h = 1e-5 * abs(v)
        with torch.no_grad():
            q[i0, c0] = v + h
        lp = L()
        with torch.no_grad():
            q[i0, c0] = v - h
        lm = L()
        with torch.no_grad():
            q[i0, c0] = v
        fd = (lp - lm) / (2 * h)
        assert abs(fd - float(g[i0, c0])) <= 1e-4 * abs(fd), (k, fd, float(g[i0, c0]))


def test_stream_releases_backward_fills_node_grads():
    import torch
    from agama_gpu_b200.stream import integrate_releases_autograd
    mp, _, pot = _pot()
    phi, dphi = mp.node_parameters()
    x0, v0, target = _orbits(pot, n=16, seed=11)
    steps = np.array([0, 3, 6, 9, 12, 15, 18, 21])
    xr = x0.clone().requires_grad_(True)
    vr = v0.clone()

    def run():
        return integrate_releases_autograd(pot, xr, vr, steps, 0.0, 24, DT, precision="fp64")
    x, v = run()
    _loss(x, v, target).backward()
    assert xr.grad is not None and phi.grad is not None
    g = dphi.grad
    j = int(torch.argmax(g.abs()))
    i0, c0 = divmod(j, dphi.shape[1])
    val = float(dphi.detach()[i0, c0])
    h = 1e-5 * abs(val)
    out = []
    for s in (1, -1):
        with torch.no_grad():
            dphi[i0, c0] = val + s * h
            a, b = run()
            out.append(float(_loss(a, b, target)))
    with torch.no_grad():
        dphi[i0, c0] = val
    fd = (out[0] - out[1]) / (2 * h)
    assert abs(fd - float(g[i0, c0])) <= 1e-4 * abs(fd), (fd, float(g[i0, c0]))
