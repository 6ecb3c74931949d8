"""The Multipole builder's scalars (invPhi0, inner and outer power-law constants)
restated as differentiable functions of the node tables (host side): values equal
the builder's, and the node gradient with their explicit part (node_vjp with
grad_const) against central differences through the real table builder."""
import numpy as np
import pytest
import torch

from agama_gpu_b200.coefs import MultipoleCoefs
from agama_gpu_b200.diff_tables import multipole_consts_from_nodes, node_vjp
from agama_gpu_b200.prep_multipole import build_multipole_tables
from agama_gpu_b200.synthetic import nfw_multipole


def _coefs(kind):
    """Hernquist (cusp: inner power law s = 1; outer s ~ -2) or Plummer (core: the
    constant-density branch s = 2) monopoles with small l = 2, 4 harmonics.  (An NFW
    monopole makes the outer fit degenerate -- s -> -1 with U ~ -W ~ 1e18 -- whose
    derivative finite differences cannot resolve.)"""
    c = nfw_multipole(lmax=4, n_nodes=28, rmin=0.02, rmax=300.0, seed=5, amp=0.1)
    r = np.asarray(c.R_grid)
    a, M, G = 2.0, 1e11, 4.30091727067736e-06
    if kind == "hernquist":
        p0 = -G * M / (r + a)
        d0 = G * M / (r + a) ** 2
    else:
        p0 = -G * M / np.sqrt(r * r + a * a)
        d0 = G * M * r / (r * r + a * a) ** 1.5
    phi, dphi = np.array(c.phi), np.array(c.dphi_dr)
    f = phi[:, 1:] / np.asarray(c.phi)[:, :1]
    phi[:, 0], dphi[:, 0] = p0, d0
    phi[:, 1:] = f * p0[:, None]
    dphi[:, 1:] = f * d0[:, None]
    return MultipoleCoefs(r, phi, dphi, c.lm_labels, dict(c.params))


def _scalars(t):
    """The builder's scalars in the variables of the kernels' g_const: invPhi0, the
    inner s, U, W, and the outer fit as (s + 1, U (s + 1), U + W)."""
    e = t.outer_s + 1.0
    return np.array([t.invPhi0, t.inner_s, t.inner_U, t.inner_W, e, t.outer_U * e,
                     t.outer_U + t.outer_W, 0.0])


@pytest.mark.parametrize("kind", ["hernquist", "plummer"])
def test_consts_equal_builder(kind):
    t = build_multipole_tables(_coefs(kind), prune_threshold=0)
    k = multipole_consts_from_nodes(t, torch.from_numpy(t.node_phi),
                                    torch.from_numpy(t.node_dphi_dr)).numpy()
    want = _scalars(t)
    assert np.allclose(k[:4], want[:4], rtol=1e-12, atol=0.0), (k, want)
    # the outer fit: eps at the rounding level and T = U eps to rounding; S = U + W is
    # Phi(r_N) analytically, but the builder's two ~1e16 terms carry the rounding of
    # g - s P1 divided by eps ~ 1e-16 (here 58 of 1424: the extrapolated Phi jumps
    # by that much at the last node, as the reference's own fit does)
    assert abs(k[4] - want[4]) <= 1e-15
    assert abs(k[5] - want[5]) <= 1e-12 * abs(want[5])
    assert abs(k[6] - want[6]) <= 0.1 * abs(k[6])
    r1 = float(t.r_grid[-1])
    assert k[6] == t.node_phi[-1, 0]
    assert np.isclose(k[5], r1 * t.node_dphi_dr[-1, 0] + t.node_phi[-1, 0], rtol=1e-14)
    if kind == "plummer":
        assert t.inner_s == 2.0
    assert t.invPhi0 != 0.0


@pytest.mark.parametrize("kind", ["hernquist", "plummer"])
def test_node_vjp_with_consts_matches_builder_differences(kind):
    c = _coefs(kind)
    t = build_multipole_tables(c, prune_threshold=0)
    rng = np.random.default_rng(7)
    Gp = rng.normal(size=t.poly.shape)
    # weights that give every scalar a contribution of the same order as the tables';
    # the outer variables' chain (S = Phi(r1), T = r1 Phi'(r1) + Phi(r1)) is checked
    # below: their builder values carry the degenerate fit's rounding
    Gc = rng.normal(size=8) * np.array([1e8, 1e3, 1e-2, 1e-2, 0.0, 0.0, 0.0, 0.0])
    gphi, gdphi = node_vjp(t, torch.from_numpy(Gp), len(c.lm_labels),
                           grad_const=torch.from_numpy(Gc))
    gphi, gdphi = gphi.numpy(), gdphi.numpy()
    phi0, dphi0 = np.asarray(c.phi, dtype=np.float64), np.asarray(c.dphi_dr, dtype=np.float64)

    def L(phi, dphi):
        tt = build_multipole_tables(MultipoleCoefs(c.R_grid, phi, dphi, c.lm_labels, c.params),
                                    prune_threshold=0)
        return float((Gp * tt.poly).sum() + (Gc * _scalars(tt)).sum())

    nR = phi0.shape[0]
    # the l=0 column at the nodes the constants come from, and interior / l>0 entries
    picks = [(0, 0), (1, 0), (nR - 2, 0), (nR - 1, 0), (nR // 2, 0), (0, 4), (nR - 1, 6)]
    for i, col in picks:
        for which in ("phi", "dphi"):
            base = phi0 if which == "phi" else dphi0
            # small steps where the log-scaled table is ill-conditioned (l = 0 nodes)
            h = (1e-7 if col == 0 else 1e-5) * max(abs(base[i, col]), 1e-8)
            up, dn = base.copy(), base.copy()
            up[i, col] += h
            dn[i, col] -= h
            if which == "phi":
                fd = (L(up, dphi0) - L(dn, dphi0)) / (2 * h)
                got = gphi[i, col]
            else:
                fd = (L(phi0, up) - L(phi0, dn)) / (2 * h)
                got = gdphi[i, col]
            scale = max(abs(fd), 1e-5 * np.abs(gphi if which == "phi" else gdphi).max())
            assert abs(got - fd) <= 2e-5 * scale, (kind, which, i, col, got, fd)


def test_without_grad_const_holds_the_scalars_fixed():
    """grad_const=None: the node gradient of the tables alone with invPhi0 and the
    extrapolation constants held at the builder's values (the previous contract)."""
    c = _coefs("hernquist")
    t = build_multipole_tables(c, prune_threshold=0)
    rng = np.random.default_rng(9)
    Gp = torch.from_numpy(rng.normal(size=t.poly.shape))
    a = node_vjp(t, Gp, None)
    b = node_vjp(t, Gp, None, grad_const=torch.zeros(8, dtype=torch.float64))
    # interior nodes do not enter the scalars: equal there
    assert torch.allclose(a[0][3:-3], b[0][3:-3], rtol=1e-12, atol=0)
    # the first node's l=0 value moves invPhi0, which the log-scaled table uses
    assert not torch.allclose(a[0][0, 0], b[0][0, 0], rtol=1e-6)


def test_outer_variables_chain():
    """d(eps, T, S)/d(nodes): S = Phi_0(r_N), T = r_N dPhi_0/dr(r_N) + Phi_0(r_N), eps
    flat (the degenerate root) -- through node_vjp with only grad_const set."""
    c = _coefs("hernquist")
    t = build_multipole_tables(c, prune_threshold=0)
    zero = torch.zeros(t.poly.shape, dtype=torch.float64)
    r1 = float(t.r_grid[-1])
    for q, dphi_w, dd_w in ((6, 1.0, 0.0), (5, 1.0, r1)):
        gc = torch.zeros(8, dtype=torch.float64)
        gc[q] = 1.0
        gp, gd = node_vjp(t, zero, None, grad_const=gc)
        assert abs(float(gp[-1, 0]) - dphi_w) < 1e-12 and abs(float(gd[-1, 0]) - dd_w) < 1e-12 * r1
        gp[-1, 0] = 0.0
        gd[-1, 0] = 0.0
        assert float(gp.abs().max()) == 0.0 and float(gd.abs().max()) == 0.0
    gc = torch.zeros(8, dtype=torch.float64)
    gc[4] = 1.0
    gp, gd = node_vjp(t, zero, None, grad_const=gc)
    assert float(gp.abs().max()) < 1e-6 and float(gd.abs().max()) < 1e-6
