"""Derivatives: position VJP (fused Hessian contraction), autograd Function,
leapfrog forward (eager and CUDA-graph) and its checkpointed adjoint, checked
against central finite differences and the oracle."""
import numpy as np
import pytest

from conftest import golden
from helpers import cs_coefs
from oracle import cpu

pytestmark = pytest.mark.gpu


def _composite(static=True):
    import agama_gpu_b200 as agb
    from agama_gpu_b200.synthetic import circular_track, nfw_multipole
    parts = [agb.MultipolePotentialGPU(nfw_multipole(lmax=6, n_nodes=40, seed=2)),
             agb.MiyamotoNagaiPotentialGPU(mass=5e10, scaleRadius=3.0, scaleHeight=0.3),
             agb.CylSplinePotentialGPU(cs_coefs(golden("cs_cfg1")))]
    if not static:
        parts.append(agb.ShiftedPotentialGPU(agb.NFWPotentialGPU(mass=2e11, scaleRadius=8.0),
                                             circular_track(T=100, radius=40.0)))
    return agb.CompositePotentialGPU(parts)


def _pts(n, seed, lo=0.3, hi=60.0):
    rng = np.random.default_rng(seed)
    r = np.exp(rng.uniform(np.log(lo), np.log(hi), n))
    u = rng.normal(size=(n, 3))
    return u / np.linalg.norm(u, axis=1)[:, None] * r[:, None]


@pytest.mark.parametrize("prec,tol", [("fp64", 2e-6), ("mixed", 5e-5)])
def test_vjp_matches_finite_differences(prec, tol):
    import torch
    pot = _composite(static=False)
    xyz = _pts(400, 1)
    # the CylSpline grid starts at R = 0.1: inside that the reference's outer
    # asymptote (gradient without its theta term) is not the derivative of its Phi
    xyz = xyz[np.hypot(xyz[:, 0], xyz[:, 1]) > 0.2][:300]
    rng = np.random.default_rng(2)
    gphi = rng.normal(size=300)
    gf = rng.normal(size=(300, 3))
    x = torch.from_numpy(xyz).cuda()
    gx = pot._vjp(x, 0.4, torch.from_numpy(gphi).cuda(), torch.from_numpy(gf).cuda(),
                  precision=prec).cpu().numpy()

    def L(xx):
        p, f, _, _ = pot._launch(torch.from_numpy(xx).cuda(), 0.4, 1, True, precision="fp64")
        return (p.cpu().numpy() * gphi) + np.sum(f.cpu().numpy() * gf, axis=1)

    fd = np.zeros_like(xyz)
    for d in range(3):
        h = 1e-5 * np.maximum(np.linalg.norm(xyz, axis=1), 1.0)
        e = np.zeros_like(xyz)
        e[:, d] = h
        fd[:, d] = (L(xyz + e) - L(xyz - e)) / (2 * h)
    err = np.abs(gx - fd).max() / np.abs(fd).max()
    assert err < tol, err


def _exact_cyl_correction(pot, xyz, t):
    """The terms dPhi/dphi d2(phi)/dx_i dx_j that the reference's CylSpline Hessian
    omits, from the oracle's Phi by central differences in phi (for the check)."""
    from agama_gpu_b200 import _lib
    corr = np.zeros((len(xyz), 6))
    for comp, sigma, gamma, ampl in pot._leaves(t):
        if comp.kind != _lib.KIND_CYLSPLINE:
            continue
        x = sigma * xyz - np.asarray(gamma)[None, :]
        R2 = x[:, 0] ** 2 + x[:, 1] ** 2
        ph = np.arctan2(x[:, 1], x[:, 0])
        R = np.sqrt(R2)
        dph = 1e-5
        def rot(a):
            return np.stack([R * np.cos(ph + a), R * np.sin(ph + a), x[:, 2]], 1)
        Pp = (cpu.eval_component(comp, 0, rot(dph))[0] - cpu.eval_component(comp, 0, rot(-dph))[0]) / (2 * dph)
        xy, d = x[:, 0] * x[:, 1], R2 * R2
        f = ampl * sigma * sigma
        corr[:, 0] += f * 2 * Pp * xy / d
        corr[:, 1] -= f * 2 * Pp * xy / d
        corr[:, 3] += f * Pp * (x[:, 1] ** 2 - x[:, 0] ** 2) / d
    return corr


def test_vjp_matches_oracle_hessian():
    import torch
    pot = _composite(static=False)
    xyz = _pts(30_000, 3, 0.3, 120.0)
    xyz = xyz[np.hypot(xyz[:, 0], xyz[:, 1]) > 0.2][:20_000]     # inside the CylSpline grid
    rng = np.random.default_rng(4)
    gphi, gf = rng.normal(size=20_000), rng.normal(size=(20_000, 3))
    gx = pot._vjp(torch.from_numpy(xyz).cuda(), 0.7, torch.from_numpy(gphi).cuda(),
                  torch.from_numpy(gf).cuda(), precision="fp64").cpu().numpy()
    _, g, h, _ = cpu.eval_potential(pot, 2, xyz, 0.7)
    h = h + _exact_cyl_correction(pot, xyz, 0.7)
    H = np.zeros((len(xyz), 3, 3))
    for q, (i, j) in enumerate([(0, 0), (1, 1), (2, 2), (0, 1), (1, 2), (0, 2)]):
        H[:, i, j] = H[:, j, i] = h[:, q]
    ref = gphi[:, None] * g - np.einsum("nij,nj->ni", H, gf)
    assert np.abs(gx - ref).max() <= 1e-8 * np.abs(ref).max()


def test_autograd_function():
    import torch
    from agama_gpu_b200.autograd import potential_and_force
    pot = _composite()
    x = torch.from_numpy(_pts(500, 5)).cuda().requires_grad_(True)
    w = torch.randn(500, dtype=torch.float64, device="cuda")
    u = torch.randn(500, 3, dtype=torch.float64, device="cuda")
    phi, F = potential_and_force(pot, x)
    (gx,) = torch.autograd.grad((w * phi).sum() + (u * F).sum(), x)
    ref = pot._vjp(x.detach(), 0.0, w, u)
    assert torch.allclose(gx, ref, rtol=0, atol=0)
    p2, f2 = pot.eval(x.detach(), pot=True, acc=True)
    assert torch.equal(phi.detach(), p2) and torch.equal(F.detach(), f2)


def _disk_ics(n, seed):
    import torch
    rng = np.random.default_rng(seed)
    R = rng.uniform(4, 20, n)
    ph = rng.uniform(0, 2 * np.pi, n)
    x = np.stack([R * np.cos(ph), R * np.sin(ph), rng.normal(0, 0.5, n)], 1)
    vc = 200.0
    v = np.stack([-vc * np.sin(ph), vc * np.cos(ph), rng.normal(0, 10, n)], 1)
    return torch.from_numpy(x).cuda(), torch.from_numpy(v).cuda()


@pytest.mark.parametrize("scheme", ["leapfrog", "yoshida4"])
@pytest.mark.parametrize("static", [True, False])
def test_leapfrog_adjoint_matches_finite_differences(static, scheme):
    import torch
    from agama_gpu_b200.integrate import Leapfrog, gyr_to_time
    pot = _composite(static=static)
    x0, v0 = _disk_ics(16, 7)
    target = x0 + 1.0
    integ = Leapfrog(pot, gyr_to_time(2e-3), t0=0.1, precision="fp64", scheme=scheme)
    n_steps = 90

    def loss(xx, vv):
        xT, vT, _ = integ.run(xx, vv, n_steps, checkpoint_every=16)
        return float(((xT - target) ** 2).sum())

    xT, vT, ck = integ.run(x0, v0, n_steps, checkpoint_every=16)
    lx, lv = integ.adjoint(ck, n_steps, 2 * (xT - target), torch.zeros_like(vT))
    rng = np.random.default_rng(0)
    for (p, d) in [(int(rng.integers(16)), int(rng.integers(3))) for _ in range(6)]:
        for which, lam, h in (("x", lx, 1e-4), ("v", lv, 1e-3)):
            xp, vp = x0.clone(), v0.clone()
            xm, vm = x0.clone(), v0.clone()
            if which == "x":
                xp[p, d] += h; xm[p, d] -= h
            else:
                vp[p, d] += h; vm[p, d] -= h
            fd = (loss(xp, vp) - loss(xm, vm)) / (2 * h)
            an = float(lam[p, d])
            assert abs(an - fd) <= 1e-5 * max(abs(fd), 1e-3 * float(lam.abs().max())), (which, an, fd)


@pytest.mark.parametrize("scheme", ["leapfrog", "yoshida4"])
@pytest.mark.parametrize("static", [True, False])
def test_leapfrog_adjoint_independent_of_checkpoint_interval(static, scheme):
    """Every interval (1: the stored trajectory, no re-computation; None: chosen
    from free memory) gives the gradients of the default interval."""
    import torch
    from agama_gpu_b200.integrate import Leapfrog, gyr_to_time
    pot = _composite(static=static)
    x0, v0 = _disk_ics(300, 17)
    integ = Leapfrog(pot, gyr_to_time(2e-3), t0=0.1, precision="fp64", scheme=scheme)
    n_steps = 45
    ref = None
    for k in (16, 1, 7, 45, 200, None):
        xT, vT, ck = integ.run(x0, v0, n_steps, checkpoint_every=k)
        lx, lv = integ.adjoint(ck, n_steps, xT - x0, 0.1 * vT)
        if ref is None:
            ref = (xT, lx, lv)
            continue
        assert torch.equal(xT, ref[0]), k
        assert torch.allclose(lx, ref[1], rtol=1e-13, atol=0), k
        assert torch.allclose(lv, ref[2], rtol=1e-13, atol=0), k


@pytest.mark.parametrize("scheme", ["leapfrog", "yoshida4"])
def test_leapfrog_graph_replay_equals_eager(scheme):
    import torch
    from agama_gpu_b200.integrate import Leapfrog
    pot = _composite(static=True)
    x0, v0 = _disk_ics(5000, 9)
    a = Leapfrog(pot, 0.001, use_graph=True, graph_steps=8, scheme=scheme)
    b = Leapfrog(pot, 0.001, use_graph=False, scheme=scheme)
    assert a.use_graph and not b.use_graph
    xa, va, _ = a.run(x0, v0, 40, checkpoint_every=64)
    xb, vb, _ = b.run(x0, v0, 40, checkpoint_every=64)
    assert torch.equal(xa, xb) and torch.equal(va, vb)
    xa2, _, _ = a.run(x0, v0, 40, checkpoint_every=64)     # graph reused on a second run
    assert torch.equal(xa2, xa)


def test_leapfrog_autograd_wrapper():
    import torch
    from agama_gpu_b200.integrate import leapfrog
    pot = _composite(static=True)
    x0, v0 = _disk_ics(64, 11)
    x0.requires_grad_(True)
    v0.requires_grad_(True)
    xT, vT = leapfrog(pot, x0, v0, 0.002, 50, checkpoint_every=8)
    loss = (xT ** 2).sum() + 0.1 * (vT ** 2).sum()
    gx, gv = torch.autograd.grad(loss, (x0, v0))
    assert torch.isfinite(gx).all() and torch.isfinite(gv).all()
    from agama_gpu_b200.integrate import Leapfrog
    integ = Leapfrog(pot, 0.002)
    xT2, vT2, ck = integ.run(x0.detach(), v0.detach(), 50, checkpoint_every=8)
    lx, lv = integ.adjoint(ck, 50, 2 * xT2, 0.2 * vT2)
    assert torch.allclose(gx, lx, rtol=1e-12, atol=0) and torch.allclose(gv, lv, rtol=1e-12, atol=0)


def _mp_variants():
    import agama_gpu_b200 as agb
    from agama_gpu_b200.synthetic import nfw_multipole
    reg = agb.MultipolePotentialGPU(nfw_multipole(lmax=6, n_nodes=30, seed=3, amp=0.3))
    c = nfw_multipole(lmax=5, n_nodes=30, seed=4, amp=0.3)
    c.phi[:, 3] = c.phi[:, 7] * 0.5 + 1.0      # odd l present: every-l structure
    c.dphi_dr[:, 3] = c.dphi_dr[:, 7] * 0.5
    lst = agb.MultipolePotentialGPU(c)
    t = lst.tables
    lst._structure, lst._n_cols = 0, t.n_lm
    lst._poly_im, lst._poly32 = t.interval_major(), t.interval_major_f32()
    lst._col_scale = np.ones(t.n_lm)
    lst._col_of = np.arange(t.n_lm)
    return [reg, lst]


@pytest.mark.parametrize("which", [0, 1])
def test_table_vjp_matches_torch_autograd(which):
    import torch
    from oracle import torch_mp
    mp = _mp_variants()[which]
    tb = mp.tables
    xyz = _pts(3000, 21, 0.05, 900.0)
    xyz = xyz[np.hypot(xyz[:, 0], xyz[:, 1]) > 1e-3 * np.linalg.norm(xyz, axis=1)][:2000]
    sigma, gamma, ampl = 0.8, np.array([0.3, -0.2, 0.1]), 1.7
    xl = sigma * xyz - gamma
    r = np.linalg.norm(xl, axis=1)
    inside = (np.log(r) >= tb.logr_min) & (np.log(r) < tb.logr_min + tb.n_int * tb.dlogr)
    rng = np.random.default_rng(22)
    gphi, gf = rng.normal(size=len(xyz)), rng.normal(size=(len(xyz), 3))
    g = mp.table_vjp(torch.from_numpy(xyz).cuda(), 0.0, torch.from_numpy(gphi).cuda(),
                     torch.from_numpy(gf).cuda(), leaf=(sigma, gamma, ampl)).cpu().numpy()
    # the same loss through torch autograd: Phi = A phi(x'), F = -dPhi/dx
    poly = torch.tensor(tb.poly, dtype=torch.float64, requires_grad=True)
    x = torch.tensor(xyz[inside], dtype=torch.float64, requires_grad=True)
    xl_t = sigma * x - torch.as_tensor(gamma)
    phi = ampl * torch_mp.multipole_phi(poly, tb.lm_l, tb.lm_m, tb.scalars(), tb.log_scaling, xl_t)
    (dphi,) = torch.autograd.grad(phi.sum(), x, create_graph=True)
    L = (torch.as_tensor(gphi[inside]) * phi).sum() - (torch.as_tensor(gf[inside]) * dphi).sum()
    (ref,) = torch.autograd.grad(L, poly)
    ref = ref.numpy()
    assert np.abs(g - ref).max() <= 1e-10 * np.abs(ref).max(), np.abs(g - ref).max() / np.abs(ref).max()


def test_node_gradients_match_finite_differences():
    import torch
    import agama_gpu_b200 as agb
    from agama_gpu_b200.synthetic import nfw_multipole
    coefs = nfw_multipole(lmax=4, n_nodes=25, seed=5, amp=0.3)
    pot = agb.MultipolePotentialGPU(coefs)
    xyz = _pts(4000, 23, 0.05, 200.0)
    rng = np.random.default_rng(24)
    gphi, gf = rng.normal(size=len(xyz)), rng.normal(size=(len(xyz), 3))
    x = torch.from_numpy(xyz).cuda()

    def loss(c):
        p = agb.MultipolePotentialGPU(c)
        ph, f, _, _ = p._launch(x, 0.0, 1, True, precision="fp64")
        return float((ph.cpu().numpy() * gphi).sum() + (f.cpu().numpy() * gf).sum())

    gpoly = pot.table_vjp(x, 0.0, torch.from_numpy(gphi).cuda(), torch.from_numpy(gf).cuda())
    gnp, gnd = (a.cpu().numpy() for a in pot.node_gradients(gpoly))
    lab = coefs.lm_labels
    checks = [(2, lab.index((0, 0))), (10, lab.index((0, 0))), (7, lab.index((2, 1))),
              (15, lab.index((4, -3))), (20, lab.index((2, 0)))]
    for i, c in checks:
        for which, G in (("phi", gnp), ("dphi", gnd)):
            tab = coefs.phi if which == "phi" else coefs.dphi_dr
            h = 1e-5 * np.abs(tab[:, c]).max()       # step on the column's scale
            cp_ = agb.MultipoleCoefs(coefs.R_grid, coefs.phi.copy(), coefs.dphi_dr.copy(), lab)
            cm_ = agb.MultipoleCoefs(coefs.R_grid, coefs.phi.copy(), coefs.dphi_dr.copy(), lab)
            (cp_.phi if which == "phi" else cp_.dphi_dr)[i, c] += h
            (cm_.phi if which == "phi" else cm_.dphi_dr)[i, c] -= h
            fd = (loss(cp_) - loss(cm_)) / (2 * h)
            assert abs(G[i, c] - fd) <= 1e-5 * max(abs(fd), 1e-4 * np.abs(G).max()), (which, i, c, G[i, c], fd)


@pytest.mark.parametrize("scheme", ["leapfrog", "yoshida4"])
def test_leapfrog_table_gradients(scheme):
    import torch
    import agama_gpu_b200 as agb
    from agama_gpu_b200.integrate import Leapfrog
    from agama_gpu_b200.synthetic import nfw_multipole
    coefs = nfw_multipole(lmax=4, n_nodes=30, seed=8, amp=0.3)
    mn = agb.MiyamotoNagaiPotentialGPU(mass=5e10, scaleRadius=3.0, scaleHeight=0.3)
    x0, v0 = _disk_ics(24, 12)
    target = x0 * 1.1

    def run(c, want=False):
        mp = agb.MultipolePotentialGPU(c)
        integ = Leapfrog(mp + mn, 0.002, precision="fp64", scheme=scheme)
        xT, vT, ck = integ.run(x0, v0, 60, checkpoint_every=16)
        Lv = float(((xT - target) ** 2).sum())
        if not want:
            return Lv
        lx, lv, tg = integ.adjoint(ck, 60, 2 * (xT - target), torch.zeros_like(vT), table_grads=True)
        return Lv, mp, tg[mp]

    _, mp, gpoly = run(coefs, True)
    gnp, gnd = (a.cpu().numpy() for a in mp.node_gradients(gpoly))
    lab = coefs.lm_labels
    for i, c in [(12, lab.index((0, 0))), (14, lab.index((2, 2))), (9, lab.index((4, 0)))]:
        for which, G in (("phi", gnp), ("dphi", gnd)):
            tab = coefs.phi if which == "phi" else coefs.dphi_dr
            h = 1e-5 * np.abs(tab[:, c]).max()
            cp_ = agb.MultipoleCoefs(coefs.R_grid, coefs.phi.copy(), coefs.dphi_dr.copy(), lab)
            cm_ = agb.MultipoleCoefs(coefs.R_grid, coefs.phi.copy(), coefs.dphi_dr.copy(), lab)
            (cp_.phi if which == "phi" else cp_.dphi_dr)[i, c] += h
            (cm_.phi if which == "phi" else cm_.dphi_dr)[i, c] -= h
            fd = (run(cp_) - run(cm_)) / (2 * h)
            assert abs(G[i, c] - fd) <= 1e-4 * max(abs(fd), 1e-3 * np.abs(G).max()), (which, i, c, G[i, c], fd)


@pytest.mark.parametrize("lmax", [6, 32])
@pytest.mark.parametrize("prec,tol_x,tol_g", [("fp64", 1e-12, 1e-11), ("mixed", 2e-5, 2e-5)])
def test_fused_adjoint_matches_separate_passes(prec, tol_x, tol_g, lmax):
    """agb_multipole_adjoint (one harmonic walk for the position VJP and the
    coefficient gradients) against agb_eval_vjp + agb_multipole_table_vjp.
    lmax=6 runs the shared-memory staged accumulation, lmax=32 (561 columns)
    the direct global atomics."""
    import torch
    import agama_gpu_b200 as agb
    from agama_gpu_b200.synthetic import nfw_multipole
    mp = agb.MultipolePotentialGPU(nfw_multipole(lmax=lmax, n_nodes=30, seed=31, amp=0.3))
    assert mp._structure != 0
    pot = agb.CompositePotentialGPU([
        agb.ScaledPotentialGPU(agb.ShiftedPotentialGPU(mp, [0.3, -0.2, 0.1]), 1.3, 0.8),
        agb.MiyamotoNagaiPotentialGPU(mass=5e10, scaleRadius=3.0, scaleHeight=0.3),
        agb.CylSplinePotentialGPU(cs_coefs(golden("cs_cfg1")))])
    xyz = _pts(20000, 32, 0.02, 2000.0)
    rng = np.random.default_rng(33)
    x = torch.from_numpy(xyz).cuda()
    gphi = torch.from_numpy(rng.normal(size=len(xyz))).cuda()
    gf = torch.from_numpy(rng.normal(size=(len(xyz), 3))).cuda()
    ref_x = pot._vjp(x, 0.0, gphi, gf, precision="fp64")
    ref_g = pot._table_vjp(x, 0.0, gphi, gf)[mp]
    acc = {}
    gx = pot._adjoint_vjp(x, 0.0, gphi, gf, acc, precision=prec)
    gx = pot._adjoint_vjp(x, 0.0, gphi, gf, acc, precision=prec, out=torch.empty_like(gx))
    tg = pot._table_grads_from_device(acc)[mp]
    ex = ((gx - ref_x).abs().max() / ref_x.abs().max()).item()
    eg = ((tg - 2 * ref_g).abs().max() / ref_g.abs().max()).item()
    assert ex <= tol_x, ex
    assert eg <= tol_g, eg


def _cyl_local_points(n, seed):
    rng = np.random.default_rng(seed)
    R = np.exp(rng.uniform(np.log(0.3), np.log(120.0), n))
    ph = rng.uniform(0, 2 * np.pi, n)
    z = np.sinh(rng.uniform(-3.0, 3.0, n)) * 3.0
    return np.stack([R * np.cos(ph), R * np.sin(ph), z], 1)


@pytest.mark.parametrize("log_scaled", [True, False])
def test_cylspline_table_vjp_matches_finite_differences(log_scaled):
    """dL/d(node table) of a CylSpline seen through Shifted/Scaled, and its chain to
    the coefficient grid, against central differences of the GPU evaluation."""
    import copy
    import torch
    import agama_gpu_b200 as agb
    from agama_gpu_b200.coefs import CylSplineCoefs
    coefs = cs_coefs(golden("cs_cfg1"))
    if not log_scaled:                 # a positive m=0 offset switches log-scaling off
        coefs = CylSplineCoefs(coefs.R_grid, coefs.z_grid,
                               {m: (np.asarray(v) + (3e4 if m == 0 else 0.0)) for m, v in coefs.phi.items()})
    cs = agb.CylSplinePotentialGPU(coefs)
    assert bool(cs.tables.log_scaling) == log_scaled
    shift, scale, ampl = np.array([0.4, -0.3, 0.2]), 1.3, 0.8

    def tree(c):
        return agb.ScaledPotentialGPU(agb.ShiftedPotentialGPU(c, list(shift)), scale, ampl)
    _, sigma, gamma, A = tree(cs)._leaves(0.0)[0]
    xl = _cyl_local_points(3000, 41)
    x = torch.from_numpy((xl + np.asarray(gamma)) / sigma).cuda()
    rng = np.random.default_rng(42)
    gphi = torch.from_numpy(rng.normal(size=len(xl))).cuda()
    gf = torch.from_numpy(rng.normal(size=(len(xl), 3))).cuda()

    def L(c):
        p, f, _, _ = tree(c)._launch(x, 0.0, 1, True, precision="fp64")
        return float((p * gphi).sum() + (f * gf).sum())

    g = cs.table_vjp(x, 0.0, gphi, gf, leaf=(sigma, gamma, A)).cpu().numpy()
    tb = cs.tables
    nodes = tb.node_arr
    H = tb.n_harm
    for (h, i, j, q) in [(tb.m_arr.tolist().index(0), 12, 15, 0), (tb.m_arr.tolist().index(0), 8, 17, 1),
                         (tb.m_arr.tolist().index(2), 10, 14, 2), (tb.m_arr.tolist().index(-4), 14, 16, 3),
                         (H - 1, 6, 18, 0)]:
        # step on the harmonic's value scale: some derivative nodes are ~1e-17 here
        step = 1e-6 * max(np.abs(nodes[h, :, :, q]).max(), np.abs(nodes[h, :, :, 0]).max())
        tp, tm = copy.deepcopy(tb), copy.deepcopy(tb)
        tp.node_arr = nodes.copy(); tp.node_arr[h, i, j, q] += step
        tm.node_arr = nodes.copy(); tm.node_arr[h, i, j, q] -= step
        fd = (L(agb.CylSplinePotentialGPU._from_tables(tp)) -
              L(agb.CylSplinePotentialGPU._from_tables(tm))) / (2 * step)
        # central differences resolve ~1e-8 of the largest gradient entry here
        assert abs(g[h, i, j, q] - fd) <= 1e-5 * max(abs(fd), 1e-3 * np.abs(g).max()), (h, i, j, q, g[h, i, j, q], fd)
    # chained to the coefficient grid (interior nodes: the asymptote fit and Rscale stay put)
    gc = cs.node_gradients(torch.from_numpy(g))
    for m, i, j in [(0, 12, 15), (2, 10, 14), (-6, 14, 17)]:
        step = 1e-6 * np.abs(np.asarray(coefs.phi[m])).max()
        pp = {k: np.array(v, dtype=float) for k, v in coefs.phi.items()}
        pm = {k: np.array(v, dtype=float) for k, v in coefs.phi.items()}
        pp[m][i, j] += step
        pm[m][i, j] -= step
        fd = (L(agb.CylSplinePotentialGPU(CylSplineCoefs(coefs.R_grid, coefs.z_grid, pp))) -
              L(agb.CylSplinePotentialGPU(CylSplineCoefs(coefs.R_grid, coefs.z_grid, pm)))) / (2 * step)
        assert abs(gc[m][i, j] - fd) <= 1e-5 * max(abs(fd), 1e-4 * max(np.abs(v).max() for v in gc.values())), \
            (m, i, j, gc[m][i, j], fd)


def test_leapfrog_cylspline_table_gradients():
    import copy
    import torch
    import agama_gpu_b200 as agb
    from agama_gpu_b200.integrate import Leapfrog
    cs = agb.CylSplinePotentialGPU(cs_coefs(golden("cs_cfg1")))
    nfw = agb.NFWPotentialGPU(mass=5e11, scaleRadius=15.0)
    x0, v0 = _disk_ics(40, 13)
    target = x0 * 1.05

    def run(c, want=False):
        integ = Leapfrog(c + nfw, 0.002, precision="fp64")
        xT, vT, ck = integ.run(x0, v0, 30, checkpoint_every=8)
        if not want:
            return float(((xT - target) ** 2).sum())
        _, _, tg = integ.adjoint(ck, 30, 2 * (xT - target), torch.zeros_like(vT), table_grads=True)
        return tg[c]

    g = run(cs, True).cpu().numpy()
    tb = cs.tables
    h0 = tb.m_arr.tolist().index(0)
    for (h, i, j, q) in [(h0, 14, 15, 0), (h0, 16, 16, 1), (tb.m_arr.tolist().index(2), 15, 16, 0)]:
        step = 1e-6 * max(np.abs(tb.node_arr[h, :, :, q]).max(), np.abs(tb.node_arr[h, :, :, 0]).max())
        tp, tm = copy.deepcopy(tb), copy.deepcopy(tb)
        tp.node_arr = tb.node_arr.copy(); tp.node_arr[h, i, j, q] += step
        tm.node_arr = tb.node_arr.copy(); tm.node_arr[h, i, j, q] -= step
        fd = (run(agb.CylSplinePotentialGPU._from_tables(tp)) -
              run(agb.CylSplinePotentialGPU._from_tables(tm))) / (2 * step)
        assert abs(g[h, i, j, q] - fd) <= 1e-4 * max(abs(fd), 1e-3 * np.abs(g).max()), (h, i, j, q, g[h, i, j, q], fd)


def test_set_node_tables_on_device():
    """Rebuilding a Multipole's tables on the GPU from new node values: equal to a
    fresh host-built object (l>0 changes leave invPhi0 and the extrapolation alone),
    in place (a captured leapfrog graph sees them), and node_gradients() follows."""
    import torch
    import agama_gpu_b200 as agb
    from agama_gpu_b200.coefs import MultipoleCoefs
    from agama_gpu_b200.integrate import Leapfrog
    from agama_gpu_b200.synthetic import nfw_multipole
    coefs = nfw_multipole(lmax=6, n_nodes=40, seed=21, amp=0.3)
    mp = agb.MultipolePotentialGPU(coefs)
    t = mp.tables
    xyz = torch.from_numpy(_pts(5000, 22, 0.05, 500.0)).cuda()
    x0, v0 = _disk_ics(200, 23)
    integ = Leapfrog(mp, 0.002, graph_steps=5)
    assert integ.use_graph
    xa, _, _ = integ.run(x0, v0, 10, checkpoint_every=64)          # captures the graph
    f0 = mp.force(xyz)
    # the same nodes rebuilt on the device: the same tables
    mp.set_node_tables(torch.from_numpy(t.node_phi).cuda(), torch.from_numpy(t.node_dphi_dr).cuda())
    f1 = mp.force(xyz)
    assert float((f1 - f0).abs().max()) <= 1e-12 * float(f0.abs().max())
    # new l>0 values: compare with a potential built on the host from the same coefficients
    lab = coefs.lm_labels
    phi2, dphi2 = coefs.phi.copy(), coefs.dphi_dr.copy()
    c22 = lab.index((2, 2))
    phi2[:, c22] *= 1.7
    dphi2[:, c22] *= 1.7
    ref = agb.MultipolePotentialGPU(MultipoleCoefs(coefs.R_grid, phi2, dphi2, lab))
    nodes_p = torch.from_numpy(ref.tables.node_phi).cuda()
    nodes_d = torch.from_numpy(ref.tables.node_dphi_dr).cuda()
    mp.set_node_tables(nodes_p, nodes_d)
    for prec in ("fp64", "mixed"):
        fm = mp._launch(xyz, 0.0, 1, True, precision=prec)[1]
        fr = ref._launch(xyz, 0.0, 1, True, precision=prec)[1]
        assert float((fm - fr).abs().max()) <= 1e-12 * float(fr.abs().max()), prec
    # the graph captured before the change integrates in the new potential
    xb, _, _ = integ.run(x0, v0, 10, checkpoint_every=64)
    xc, _, _ = Leapfrog(ref, 0.002, use_graph=False).run(x0, v0, 10, checkpoint_every=64)
    assert not torch.equal(xa, xb)
    assert float((xb - xc).abs().max()) <= 1e-11 * float(xc.abs().max())
    # node gradients are taken at the new nodes
    g = mp.table_vjp(xyz, 0.0, None, torch.ones_like(xyz))
    gp, gd = mp.node_gradients(g)
    gp_ref, gd_ref = ref.node_gradients(ref.table_vjp(xyz, 0.0, None, torch.ones_like(xyz)))
    assert float((gp - gp_ref).abs().max()) <= 1e-9 * float(gp_ref.abs().max())


def test_set_node_tables_rebuilds_builder_scalars_and_recaptures_graphs():
    """New l = 0 nodes change invPhi0 and the extrapolation fits: set_node_tables
    recomputes them as the builder does (equal to a host-built object from the same
    coefficients, inside and beyond the grid), and a leapfrog whose graph was captured
    before the change captures it again (the kernels take the scalars by value)."""
    import torch
    import agama_gpu_b200 as agb
    from agama_gpu_b200.coefs import MultipoleCoefs
    from agama_gpu_b200.integrate import Leapfrog
    from agama_gpu_b200.synthetic import nfw_multipole
    coefs = nfw_multipole(lmax=6, n_nodes=40, rmin=0.05, rmax=200.0, seed=31, amp=0.3)
    mp = agb.MultipolePotentialGPU(coefs)
    x0, v0 = _disk_ics(200, 32)
    integ = Leapfrog(mp, 0.002, graph_steps=5)
    xa, _, _ = integ.run(x0, v0, 10, checkpoint_every=64)          # captures the graph
    # scale the l = 0 column near the centre: the inner fit and invPhi0 move
    phi2, dphi2 = np.array(coefs.phi), np.array(coefs.dphi_dr)
    r = np.asarray(coefs.R_grid)
    w = 1.0 + 0.05 * np.exp(-r / 2.0)
    phi2[:, 0] *= w
    dphi2[:, 0] = dphi2[:, 0] * w - coefs.phi[:, 0] * 0.05 * np.exp(-r / 2.0) / 2.0
    ref = agb.MultipolePotentialGPU(MultipoleCoefs(coefs.R_grid, phi2, dphi2, coefs.lm_labels))
    assert ref.tables.invPhi0 != mp.tables.invPhi0
    mp.set_node_tables(torch.from_numpy(ref.tables.node_phi).cuda(),
                       torch.from_numpy(ref.tables.node_dphi_dr).cuda())
    # inside the grid and inside its first node (beyond the last one the builder's outer
    # fit is degenerate -- s = -1 to rounding -- and amplifies the rounding of dPhi/dr
    # through d/dlog r in the node table by ~1e16: the far fields of the two objects
    # differ at the percent level, as two host builds from inputs one rounding apart do)
    xyz = torch.from_numpy(_pts(4000, 33, 0.01, 150.0)).cuda()
    for prec, tol in (("fp64", 1e-11), ("mixed", 2e-6)):
        fm = mp._launch(xyz, 0.0, 1, True, precision=prec)
        fr = ref._launch(xyz, 0.0, 1, True, precision=prec)
        for a, b in zip(fm[:2], fr[:2]):
            assert float((a - b).abs().max()) <= tol * float(b.abs().max()), prec
    xb, _, _ = integ.run(x0, v0, 10, checkpoint_every=64)
    xc, _, _ = Leapfrog(ref, 0.002, use_graph=False).run(x0, v0, 10, checkpoint_every=64)
    assert not torch.equal(xa, xb)
    assert float((xb - xc).abs().max()) <= 1e-11 * float(xc.abs().max())


def test_yoshida4_order_in_composite():
    """Global position error in a Multipole + Miyamoto-Nagai composite falls as
    dt^4 for the 4th-order composition (and as dt^2 for leapfrog).  (A CylSpline
    is left out: its bicubic force has jumps in dF/dx at cell edges, which cap the
    observed order of any scheme near 3.)"""
    import math
    import agama_gpu_b200 as agb
    from agama_gpu_b200.integrate import Leapfrog
    from agama_gpu_b200.synthetic import nfw_multipole
    pot = agb.CompositePotentialGPU([
        agb.MultipolePotentialGPU(nfw_multipole(lmax=6, n_nodes=40, seed=2)),
        agb.MiyamotoNagaiPotentialGPU(mass=5e10, scaleRadius=3.0, scaleHeight=0.3)])
    x0, v0 = _disk_ics(200, 21)
    T = 0.05                                  # ~1/4 of an orbit at 8 kpc
    ref, _, _ = Leapfrog(pot, T / 800, precision="fp64", scheme="yoshida4").run(
        x0, v0, 800, checkpoint_every=1000)
    for scheme, order in (("leapfrog", 2), ("yoshida4", 4)):
        e = []
        for n in (25, 50):
            xT, _, _ = Leapfrog(pot, T / n, precision="fp64", scheme=scheme).run(
                x0, v0, n, checkpoint_every=1000)
            e.append(float((xT - ref).abs().max()))
        rate = math.log2(e[0] / e[1])
        assert abs(rate - order) < 0.4, (scheme, e, rate)


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-12), ("mixed", 2e-6)])
def test_vjp_force_output(prec, tol):
    """The VJP launches' force output (agb_eval_vjp_force, agb_multipole_adjoint_force)
    equals the force of the same tree."""
    import torch
    pot = _composite(static=False)
    x = torch.from_numpy(_pts(3000, 31)).cuda()
    gf = torch.from_numpy(np.random.default_rng(3).normal(size=(3000, 3))).cuda()
    F = pot._launch(x, 0.4, 1, False, precision="fp64")[1]
    scale = float(F.abs().max())
    f1 = torch.full_like(x, np.nan)
    g1 = pot._vjp(x, 0.4, None, gf, precision=prec, force_out=f1)
    assert float((f1 - F).abs().max()) <= tol * scale
    assert torch.equal(g1, pot._vjp(x, 0.4, None, gf, precision=prec))
    f2 = torch.full_like(x, np.nan)
    tg = {}
    g2 = pot._adjoint_vjp(x, 0.4, None, gf, tg, precision=prec, force_out=f2)
    assert float((f2 - F).abs().max()) <= tol * scale
    g3 = pot._adjoint_vjp(x, 0.4, None, gf, {}, precision=prec)
    assert torch.equal(g2, g3)


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-9), ("mixed", 1e-6)])
@pytest.mark.parametrize("static", [True, False])
def test_reverse_reconstruction_matches_recompute(static, prec, tol):
    """Segments stepped backwards from their later checkpoint give the gradients of the
    forward re-computation (rounding of the reversed positions only)."""
    import torch
    from agama_gpu_b200.integrate import Leapfrog, gyr_to_time
    pot = _composite(static=static)
    x0, v0 = _disk_ics(2000, 41)
    target = x0 + 0.5
    integ = Leapfrog(pot, gyr_to_time(1e-3), t0=0.1, precision=prec)
    xT, vT, ck = integ.run(x0, v0, 96, checkpoint_every=32)
    a = integ.adjoint(ck, 96, 2 * (xT - target), 0.1 * vT, table_grads=True)
    b = integ.adjoint(ck, 96, 2 * (xT - target), 0.1 * vT, table_grads=True, reconstruct="reverse")
    for u, w in zip(a[:2], b[:2]):
        assert float((u - w).abs().max()) <= tol * float(u.abs().max())
    for comp in a[2]:
        assert float((a[2][comp] - b[2][comp]).abs().max()) <= tol * float(a[2][comp].abs().max())


def test_adjoint_step_kernels_match_torch():
    """agb_adjoint_kick and agb_reverse_drift against the same updates in torch."""
    import torch
    from agama_gpu_b200 import _lib
    g = torch.Generator(device="cuda").manual_seed(5)
    lx, lv, gx, F, x, vh = (torch.randn((1001, 3), generator=g, dtype=torch.float64, device="cuda")
                            for _ in range(6))
    gF = torch.empty_like(lx)
    st = torch.cuda.current_stream().cuda_stream
    ex, ev = lx + gx, None
    ev = lv + 0.37 * ex
    egF = 0.61 * ev
    assert _lib.lib.agb_adjoint_kick(lx.data_ptr(), lv.data_ptr(), gx.data_ptr(), gF.data_ptr(),
                                     1001, 0.37, 0.61, st) == 0
    for a, b in ((lx, ex), (lv, ev), (gF, egF)):
        assert float((a - b).abs().max()) <= 1e-15 * float(b.abs().max())
    evh = vh - 0.2 * F
    exx = x - 0.9 * evh
    assert _lib.lib.agb_reverse_drift(x.data_ptr(), vh.data_ptr(), F.data_ptr(), 1001, 0.2, 0.9, st) == 0
    for a, b in ((vh, evh), (x, exx)):
        assert float((a - b).abs().max()) <= 1e-15 * float(b.abs().max())
    assert _lib.lib.agb_adjoint_kick(None, None, None, None, 3, 0.1, 0.1, st) != 0


def test_cylspline_set_node_tables_on_device():
    """CylSpline grids replaced on the GPU: the same grids give the same tables; new
    grids give a fresh host-built object's values inside the grid (the outer asymptote
    is kept from construction), in place under a captured leapfrog graph, and
    node_gradients() differentiates at the new grids."""
    import torch
    import agama_gpu_b200 as agb
    from agama_gpu_b200.coefs import CylSplineCoefs
    from agama_gpu_b200.integrate import Leapfrog
    coefs = cs_coefs(golden("cs_cfg1"))
    cs = agb.CylSplinePotentialGPU(coefs)
    rng = np.random.default_rng(3)
    R = rng.uniform(0.5, 40.0, 4000)
    ph = rng.uniform(0, 2 * np.pi, 4000)
    z = rng.uniform(-20.0, 20.0, 4000)
    x = torch.from_numpy(np.stack([R * np.cos(ph), R * np.sin(ph), z], 1)).cuda()
    x0, v0 = _disk_ics(200, 23)
    integ = Leapfrog(cs, 0.002, graph_steps=5)
    xa, _, _ = integ.run(x0, v0, 10, checkpoint_every=64)          # captures the graph
    f0 = cs.force(x)
    grids = {m: torch.from_numpy(np.asarray(v, dtype=np.float64)).cuda() for m, v in coefs.phi.items()}
    cs.set_node_tables(grids)
    f1 = cs.force(x)
    assert float((f1 - f0).abs().max()) <= 1e-12 * float(f0.abs().max())
    # m != 0 scaled; m = 0 changed only at interior nodes away from R = 0 and the outer
    # boundary, so that a fresh build keeps the same Rscale and outer asymptote
    new = {m: np.asarray(v, dtype=np.float64) * (1.3 if m != 0 else 1.0) for m, v in coefs.phi.items()}
    bump = 1.0 + 0.02 * np.exp(-np.asarray(coefs.R_grid)[1:-1, None] / 5.0)
    new[0] = new[0].copy()
    new[0][1:-1, 1:-1] *= bump
    ref = agb.CylSplinePotentialGPU(CylSplineCoefs(coefs.R_grid, coefs.z_grid, new, dict(coefs.params)))
    cs.set_node_tables({m: torch.from_numpy(v).cuda() for m, v in new.items()})
    for prec, tol in (("fp64", 1e-11), ("mixed", 2e-6)):
        fm = cs._launch(x, 0.0, 1, True, precision=prec)[1]
        fr = ref._launch(x, 0.0, 1, True, precision=prec)[1]
        assert float((fm - fr).abs().max()) <= tol * float(fr.abs().max()), prec
    xb, _, _ = integ.run(x0, v0, 10, checkpoint_every=64)
    xc, _, _ = Leapfrog(ref, 0.002, use_graph=False).run(x0, v0, 10, checkpoint_every=64)
    assert not torch.equal(xa, xb)
    assert float((xb - xc).abs().max()) <= 1e-10 * float(xc.abs().max())
    g = cs.table_vjp(x, 0.0, None, torch.ones_like(x))
    gr = ref.table_vjp(x, 0.0, None, torch.ones_like(x))
    a, b = cs.node_gradients(g), ref.node_gradients(gr)
    for m in a:
        assert np.abs(a[m] - b[m]).max() <= 1e-8 * max(np.abs(b[m]).max(), 1e-300), m


@pytest.mark.parametrize("reconstruct,k", [("reverse", 8), ("recompute", 8), ("recompute", 1)])
def test_fused_adjoint_step_equals_separate_launches(reconstruct, k):
    """agb_adjoint_step (VJP + kick + reverse drift in two launches) gives the same
    adjoint as the separate VJP, kick and drift launches: dL/dx0 and dL/dv0 bit for
    bit; the mixed-precision table gradients to the run-to-run spread of their FP32
    partial sums over 32-point groups (the order of points within an interval bin is
    not deterministic)."""
    import torch
    import agama_gpu_b200 as agb
    from agama_gpu_b200.integrate import Leapfrog
    from agama_gpu_b200.synthetic import hernquist_points, nfw_multipole
    pot = agb.MultipolePotentialGPU(nfw_multipole(lmax=8, n_nodes=40, seed=3)) + \
        agb.MiyamotoNagaiPotentialGPU(mass=5e10, scaleRadius=3.0, scaleHeight=0.3)
    xyz = hernquist_points(40_000, 15.0, 9)
    x0 = torch.from_numpy(xyz).cuda()
    v0 = torch.from_numpy(np.random.default_rng(2).normal(0, 100.0, xyz.shape)).cuda()
    lam = torch.from_numpy(np.random.default_rng(3).normal(size=xyz.shape)).cuda()
    out = []
    for fused in (True, False):
        integ = Leapfrog(pot, 2e-3, precision="mixed")
        integ.fused_adjoint = fused
        _, _, ck = integ.run(x0, v0, 24, checkpoint_every=k)
        out.append(integ.adjoint(ck, 24, lam, 0.5 * lam, table_grads=True, reconstruct=reconstruct))
    (a1, b1, t1), (a2, b2, t2) = out
    assert torch.equal(a1, a2) and torch.equal(b1, b2)
    for c in t1:
        assert float((t1[c] - t2[c]).abs().max()) <= 2e-6 * float(t2[c].abs().max())
