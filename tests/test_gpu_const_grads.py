"""Gradients with respect to the Multipole builder's scalars on the GPU (the kernels'
g_const): invPhi0 from points inside the grid against torch autograd of the oracle's
restatement, the inner and outer l=0 extrapolation from points beyond the grid against
autograd of their radial formulas, the fused adjoint against the table-VJP kernel, and
node gradients of a loss through the whole builder against finite differences through
set_node_tables (which rebuilds the scalars as the builder does)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MP0 = 3.544907701811032 * 0.28209479177387814


def _coefs():
    from agama_gpu_b200.synthetic import nfw_multipole
    return nfw_multipole(lmax=4, n_nodes=30, rmin=0.05, rmax=100.0, seed=8, amp=0.2)


def _points(n, seed, lo, hi):
    rng = np.random.default_rng(seed)
    r = np.exp(rng.uniform(np.log(lo), np.log(hi), n))
    u = rng.normal(size=(n, 3))
    u[:, 2] *= 0.9                       # away from the z axis
    return u / np.linalg.norm(u, axis=1)[:, None] * r[:, None]


def _cot(n, seed):
    import torch
    rng = np.random.default_rng(seed)
    return (torch.from_numpy(rng.normal(size=n)).cuda(),
            torch.from_numpy(rng.normal(size=(n, 3))).cuda())


def _loss_of(phi, x, gp, gf):
    """sum gp Phi + gf . F with F = -grad Phi (autograd through x)."""
    import torch
    (g,) = torch.autograd.grad(phi.sum(), x, create_graph=True)
    return (gp * phi).sum() - (gf * g).sum()


def _reference(region, t, x, gp, gf):
    """(8,) dL/d(builder scalars) of the region's points by torch autograd."""
    import torch
    from oracle.torch_mp import multipole_phi
    out = torch.zeros(8, dtype=torch.float64)
    xr = torch.from_numpy(x).requires_grad_(True)
    gp, gf = gp.cpu(), gf.cpu()
    logr = torch.log(xr.norm(dim=1))
    if region == "inside":
        inv = torch.tensor(float(t.invPhi0), dtype=torch.float64, requires_grad=True)
        sc = list(t.scalars())
        sc[3] = inv
        ph = multipole_phi(torch.from_numpy(t.poly), t.lm_l, t.lm_m, sc, t.log_scaling, xr)
        (out[0],) = torch.autograd.grad(_loss_of(ph, xr, gp, gf), inv)
    elif region == "inner":
        q = [torch.tensor(float(v), dtype=torch.float64, requires_grad=True)
             for v in (t.inner_s, t.inner_U, t.inner_W)]
        s, U, W = q
        ph = MP0 * (U * torch.exp(s * (logr - float(t.logr_min))) + W)
        out[1:4] = torch.stack(torch.autograd.grad(_loss_of(ph, xr, gp, gf), q))
    else:
        eps0 = float(t.outer_s) + 1.0
        q = [torch.tensor(v, dtype=torch.float64, requires_grad=True)
             for v in (eps0, float(t.outer_U) * eps0, float(t.outer_U) + float(t.outer_W))]
        eps, T, S = q
        dlr = logr - (float(t.logr_min) + t.n_int * float(t.dlogr))
        z = eps * dlr
        assert float(z.detach().abs().max()) < 1e-4      # the degenerate fit: series
        phi_e = dlr * (1.0 + z * (0.5 + z / 6.0))
        ph = MP0 * torch.exp(-dlr) * (S + T * phi_e)
        out[4:7] = torch.stack(torch.autograd.grad(_loss_of(ph, xr, gp, gf), q))
    return out


@pytest.mark.parametrize("region", ["inside", "inner", "outer"])
def test_const_grads_against_autograd(region):
    import torch
    import agama_gpu_b200 as agb
    mp = agb.MultipolePotentialGPU(_coefs())
    t = mp.tables
    r0, r1 = float(t.r_grid[0]), float(t.r_grid[-1])
    lo, hi = {"inside": (1.5 * r0, 0.7 * r1), "inner": (0.02 * r0, 0.9 * r0),
              "outer": (1.1 * r1, 30.0 * r1)}[region]
    x = _points(2000, 11, lo, hi)
    gp, gf = _cot(len(x), 12)
    xt = torch.from_numpy(x).cuda()
    buf = torch.zeros(8, dtype=torch.float64, device="cuda")
    mp.table_vjp(xt, 0.0, gp, gf, const_grad=buf)
    want = _reference(region, t, x, gp, gf)
    got = buf.cpu()
    live = {"inside": [0], "inner": [1, 2, 3], "outer": [4, 5, 6]}[region]
    for j in range(8):
        if j in live:
            assert abs(float(got[j] - want[j])) <= 1e-9 * abs(float(want[j])), (region, j, got, want)
        else:
            assert float(got[j]) == 0.0, (region, j, got)
    # the fused adjoint (FP64, and the FP32 walk) accumulates the same scalars
    for prec, tol in (("fp64", 1e-10), ("mixed", 2e-5)):
        acc = {}
        mp._adjoint_vjp(xt, 0.0, gp, gf, acc, precision=prec)
        fused = acc[("const", mp)].cpu()
        for j in live:
            assert abs(float(fused[j] - got[j])) <= tol * abs(float(got[j])), (prec, region, j)


def test_node_gradients_through_the_builder_match_set_node_tables_differences():
    """dL/d(l=0 nodes) at the first two nodes (invPhi0 and the inner fit move with
    them) and an interior one, for Phi and force cotangents at points inside the grid
    and inside the first node."""
    import torch
    import agama_gpu_b200 as agb
    from agama_gpu_b200 import _lib
    coefs = _coefs()
    mp = agb.MultipolePotentialGPU(coefs)
    t = mp.tables
    r0, r1 = float(t.r_grid[0]), float(t.r_grid[-1])
    x = np.concatenate([_points(3000, 21, 1.2 * r0, 0.8 * r1), _points(600, 22, 0.05 * r0, 0.9 * r0)])
    gp, gf = _cot(len(x), 23)
    xt = torch.from_numpy(x).cuda()
    buf = torch.zeros(8, dtype=torch.float64, device="cuda")
    g = mp.table_vjp(xt, 0.0, gp, gf, const_grad=buf)
    gphi, gdphi = (a.cpu().numpy() for a in mp.node_gradients(g, buf))
    base_p, base_d = t.node_phi.copy(), t.node_dphi_dr.copy()

    def L(p, d):
        m2 = agb.MultipolePotentialGPU(coefs)
        m2.set_node_tables(torch.from_numpy(p).cuda(), torch.from_numpy(d).cuda())
        ph, f, _, _ = m2._launch(xt, 0.0, _lib.MODE_GRAD, True, precision="fp64")
        return float((gp * ph).sum() + (gf * f).sum())

    nR = base_p.shape[0]
    col = int(np.asarray(t.node_cols)[0])          # the file column of the builder's l = 0
    for i, which in ((0, "phi"), (1, "phi"), (0, "dphi"), (1, "dphi"), (nR // 2, "phi")):
        base = base_p if which == "phi" else base_d
        h = 1e-7 * abs(base[i, 0])
        up, dn = base.copy(), base.copy()
        up[i, 0] += h
        dn[i, 0] -= h
        if which == "phi":
            fd = (L(up, base_d) - L(dn, base_d)) / (2 * h)
            got = gphi[i, col]
        else:
            fd = (L(base_p, up) - L(base_p, dn)) / (2 * h)
            got = gdphi[i, col]
        assert abs(got - fd) <= 1e-4 * abs(fd), (which, i, got, fd)
