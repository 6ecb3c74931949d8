"""Differentiable construction of the Multipole quintic tables (torch, FP64).

The same steps as prep_multipole.build_multipole_tables -- log-scaling of the
node values, the tridiagonal system for the quintic's second derivatives,
the six Horner coefficients per interval -- written with torch operations so
that a gradient with respect to the coefficients (from the table-VJP kernel)
can be carried back to the node tables Phi_lm(r_i) and dPhi_lm/dr(r_i).

The scalars the builder derives from the l=0 nodes -- invPhi0 and the inner
and outer power-law extrapolation constants (s, U, W) -- are restated too
(``multipole_consts_from_nodes``), so that with their explicit gradients (the
kernels' g_const) a node gradient is the derivative of the whole builder;
branch choices (which power law, the constant-density core, invPhi0 = 0) are
taken at the current values.  Held fixed: the radial grid, the harmonic set
after pruning, the log-scaling switch.  A grid that had to be resampled to
log-uniform is not supported here.
"""
from __future__ import annotations

from typing import Optional, Tuple

import numpy as np
import torch


def quintic_poly_torch(logr: torch.Tensor, f: torch.Tensor, df: torch.Tensor, h: float) -> torch.Tensor:
    """(n_cols, n-1, 6) quintic coefficients from values f and log-r slopes df (n, n_cols)."""
    n = logr.shape[0]
    ih = 1.0 / (logr[1:] - logr[:-1])                         # (n-1,)
    A = torch.zeros((n, n), dtype=f.dtype, device=f.device)
    rhs = torch.zeros_like(f)
    idx = torch.arange(n, device=f.device)
    diag = torch.zeros(n, dtype=f.dtype, device=f.device)
    diag[1:] += 3.0 * ih
    diag[:-1] += 3.0 * ih
    A[idx, idx] = diag
    A[idx[:-1], idx[1:]] = -ih
    A[idx[1:], idx[:-1]] = -ih
    w = ih[:, None]
    left = (20.0 * (f[1:] - f[:-1]) * w - 12.0 * df[1:] - 8.0 * df[:-1]) * w * w   # row i > 0
    right = (20.0 * (f[1:] - f[:-1]) * w - 12.0 * df[:-1] - 8.0 * df[1:]) * w * w  # row i < n-1
    rhs = rhs.index_add(0, idx[1:], -left)
    rhs = rhs.index_add(0, idx[:-1], right)
    h0, hn = ih[0], ih[-1]
    A[0, 1] = -2.0 * h0
    A[n - 1, n - 2] = -2.0 * hn
    rhs = rhs.clone()
    rhs[0] = (30.0 * (f[1] - f[0]) * h0 - 14.0 * df[1] - 16.0 * df[0]) * h0 * h0
    rhs[n - 1] = (-30.0 * (f[n - 1] - f[n - 2]) * hn + 14.0 * df[n - 2] + 16.0 * df[n - 1]) * hn * hn
    d2f = torch.linalg.solve(A, rhs)
    f0, f1 = f[:-1], f[1:]
    m0, m1 = df[:-1] * h, df[1:] * h
    q0, q1 = d2f[:-1] * (h * h), d2f[1:] * (h * h)
    dd = f1 - f0
    a = torch.stack([f0, m0, 0.5 * q0,
                     10.0 * dd - 6.0 * m0 - 4.0 * m1 - 1.5 * q0 + 0.5 * q1,
                     -15.0 * dd + 8.0 * m0 + 7.0 * m1 + 1.5 * q0 - q1,
                     6.0 * dd - 3.0 * m0 - 3.0 * m1 + 0.5 * (q1 - q0)], dim=-1)
    return a.permute(1, 0, 2)


_EPS = float(np.finfo(np.float64).eps)


def _f(q) -> float:
    """Value of a (0-d) tensor or number, for the builder's branch decisions."""
    return float(q.detach()) if torch.is_tensor(q) else float(q)


class _LambertW(torch.autograd.Function):
    """Real branch k (0 or -1) of the Lambert W function of a 0-d tensor;
    dW/dx = W / (x (1 + W))."""

    @staticmethod
    def forward(ctx, x, k):
        from scipy.special import lambertw
        w = torch.tensor(float(np.real(lambertw(float(x), k=k))), dtype=x.dtype, device=x.device)
        ctx.save_for_backward(x, w)
        return w

    @staticmethod
    def backward(ctx, g):
        x, w = ctx.saved_tensors
        return g * w / (x * (1.0 + w)), None


def inner_extrapolation_torch(phi0: torch.Tensor, dphi0_dr: torch.Tensor, r: np.ndarray):
    """(invPhi0, s, U, W) as prep_multipole.inner_extrapolation computes them, as
    differentiable functions of the l=0 node values phi0 (nR,) and dPhi0/dr (nR,)."""
    zero = phi0.new_zeros(())
    P1, P2, d1, d2 = phi0[0], phi0[1], dphi0_dr[0], dphi0_dr[1]
    r1, r2 = float(r[0]), float(r[1])
    lnr = float(np.log(r2 / r1))
    g1 = r1 * d1
    tiny = 100.0 * _EPS
    if abs(_f(g1)) == 0.0 or abs(_f(P1 - P2)) < tiny * max(abs(_f(P1)), abs(_f(P2))):
        return zero, zero, zero, P1
    A = lnr * g1 / (P1 - P2)
    a = _f(A)
    if not np.isfinite(a) or a >= 0.0:
        return zero, zero, zero, P1
    if abs(a + 1.0) < np.sqrt(_EPS):
        s = zero
    else:
        s = (A - _LambertW.apply(A * torch.exp(A), 0 if a > -1.0 else -1)) / lnr
    if not np.isfinite(_f(s)):
        s = zero + 2.0
    if _f(s) != 0.0:
        U = (r1 * d1) / s
        W = (r1 * d1 - s * P1) / (-s)
        pred_pow = U * s * torch.exp(s * lnr) / r2
    else:
        U = r1 * d1
        W = P1
        pred_pow = r1 * d1 / r2
    pred_cub = (r2 / r1 * (6.0 * r1 * (P2 - P1) / (r2 - r1) - d1 * (2 * r1 + r2))) / (2 * r2 + r1)
    if abs(_f(d2 - pred_cub)) < abs(_f(d2 - pred_pow)):
        s = zero + 2.0
        U = 0.5 * r1 * d1
        W = P1 - U
    if _f(s) <= 0.0:
        return zero, s, U, W
    inv = 1.0 / W
    if bool((phi0.detach() * _f(inv) >= 1.0).any()):
        inv = zero
    return inv, s, U, W


def outer_extrapolation_torch(phi0: torch.Tensor, dphi0_dr: torch.Tensor, r: np.ndarray):
    """(s, U, W) as prep_multipole.outer_extrapolation computes them, differentiable
    in the l=0 node values."""
    zero = phi0.new_zeros(())
    v = -1.0
    P1, P2, d1 = phi0[-1], phi0[-2], dphi0_dr[-1]
    r1, r2 = float(r[-1]), float(r[-2])
    lnr = float(np.log(r2 / r1))
    num1, num2 = r1 * d1, v * P1
    den1, den2 = P1, P2 * float(np.exp(-v * lnr))
    tiny = 100.0 * _EPS
    f = _f
    roundoff = (abs(f(num1 - num2)) < max(abs(f(num1)), abs(f(num2))) * tiny or
                abs(f(den1 - den2)) < max(abs(f(den1)), abs(f(den2))) * tiny)
    if not np.isfinite(f(P1)) or roundoff or f(den1) == f(den2):
        return zero, zero, P1
    A = lnr * (num1 - num2) / (den1 - den2)
    a = f(A)
    if not np.isfinite(a) or a >= 0:
        return zero, zero, P1
    if abs(a + 1) < np.sqrt(_EPS):
        s = zero + v
    else:
        s = v + (A - _LambertW.apply(A * torch.exp(A), 0 if a > -1 else -1)) / lnr
    if not np.isfinite(f(s)) or f(s) >= 0:
        s = zero - 2.0
    if f(s) != v:
        U = (r1 * d1 - v * P1) / (s - v)
        W = (r1 * d1 - s * P1) / (v - s)
    else:
        U = r1 * d1 - v * P1
        W = P1
    return s, U, W


def outer_fit_variables(phi0: torch.Tensor, dphi0_dr: torch.Tensor, r: np.ndarray):
    """(eps, T, S) = (s + 1, U (s + 1), U + W) of the outer fit, the variables of the
    kernels' g_const[4..6].  The fit is usually degenerate (s = -1 up to rounding,
    U ~ -W ~ 1e16); in these variables it is well-conditioned: where the builder
    divides by s + 1, T = r1 dPhi/dr(r1) + Phi(r1) and S = Phi(r1) exactly."""
    s, U, W = outer_extrapolation_torch(phi0, dphi0_dr, r)
    eps = s + 1.0
    if _f(eps) != 0.0 and _f(W) != _f(phi0[-1]):
        r1 = float(r[-1])
        P1 = phi0[-1]
        T = r1 * dphi0_dr[-1] + P1            # = (r1 d1 - v P1), v = -1
        S = P1                                # U + W = P1 when U = T / eps
        return eps, T, S
    return eps, U * eps, U + W


def multipole_consts_from_nodes(tables, phi: torch.Tensor, dphi_dr: torch.Tensor) -> torch.Tensor:
    """(8,) [invPhi0, inner s, U, W, outer eps, T, S, 0] -- the order of the kernels'
    g_const -- from node tables (nR, n_lm) in the builder's harmonic order,
    differentiable (computed on the host: a few scalars)."""
    if int(np.asarray(tables.node_cols)[0]) != 0:
        raise ValueError("the builder's l=0 column must be the coefficient file's first column")
    r = np.asarray(tables.r_grid, dtype=np.float64)
    p0 = phi[:, 0].to("cpu", torch.float64)
    d0 = dphi_dr[:, 0].to("cpu", torch.float64)
    zero = p0.new_zeros(())
    out_e, out_T, out_S = outer_fit_variables(p0, d0, r)
    if tables.log_scaling:
        inv, in_s, in_U, in_W = inner_extrapolation_torch(p0, d0, r)
    else:
        inv, in_s, in_U, in_W = zero, zero, zero, p0[0]
    parts = [inv, in_s, in_U, in_W, out_e, out_T, out_S, zero]
    return torch.stack([q if torch.is_tensor(q) else zero + q for q in parts]).to(phi.device)


def multipole_poly_from_nodes(tables, phi: torch.Tensor, dphi_dr: torch.Tensor,
                              inv=None) -> torch.Tensor:
    """Quintic coefficients (n_lm, n_int, 6) from node tables (nR, n_lm) in the
    builder's harmonic order (``tables.node_phi`` layout); differentiable.  inv: the
    log-scaling constant invPhi0 (a float or a 0-d tensor; default: the builder's)."""
    if tables.resampled:
        raise ValueError("node gradients need a log-uniform input grid (this one was resampled)")
    dev = phi.device
    r = torch.as_tensor(tables.r_grid, dtype=torch.float64, device=dev)
    logr = torch.log(r)
    dphi_dlogr = dphi_dr * r[:, None]
    if tables.log_scaling:
        p0 = phi[:, 0]
        if inv is None:
            inv = float(tables.invPhi0)
        f0 = torch.log(inv - 1.0 / p0)
        df0 = dphi_dlogr[:, 0] / (p0 * (inv * p0 - 1.0))
        ratio = phi[:, 1:] / p0[:, None]
        dfc = (dphi_dlogr[:, 1:] - ratio * dphi_dlogr[:, 0:1]) / p0[:, None]
        f = torch.cat([f0[:, None], ratio], dim=1)
        df = torch.cat([df0[:, None], dfc], dim=1)
    else:
        f, df = phi, dphi_dlogr
    return quintic_poly_torch(logr, f, df, float(tables.dlogr))


def node_vjp(tables, grad_poly: torch.Tensor, n_file_cols: Optional[int],
             nodes=None, grad_const: Optional[torch.Tensor] = None
             ) -> Tuple[torch.Tensor, torch.Tensor]:
    """Carry dL/dpoly back to the node tables in the coefficient file's column order.

    Returns (dL/dPhi_nodes, dL/d(dPhi/dr)_nodes), each (nR, n_file_cols); columns
    the table builder pruned (all-zero) get zero (build with prune_threshold=0
    to differentiate every harmonic).  n_file_cols=None returns them in the
    builder's harmonic order instead, (nR, n_lm) like ``tables.node_phi``.
    ``nodes`` = (phi, dphi_dr) in the builder's order when the tables were
    replaced on the device (set_node_tables), else the builder's own node values
    are used.  grad_const (8,): the explicit gradient with respect to invPhi0 and
    the extrapolation constants (the kernels' g_const); with it the builder's
    scalars are functions of the nodes (the derivative of the whole builder, as
    set_node_tables rebuilds them), without it they are held fixed.
    """
    dev = grad_poly.device
    if nodes is None:
        phi = torch.tensor(tables.node_phi, dtype=torch.float64, device=dev, requires_grad=True)
        dphi = torch.tensor(tables.node_dphi_dr, dtype=torch.float64, device=dev, requires_grad=True)
    else:
        phi = nodes[0].detach().to(dev, torch.float64).requires_grad_(True)
        dphi = nodes[1].detach().to(dev, torch.float64).requires_grad_(True)
    # also called from the backward of an autograd.Function, where grad mode is off
    with torch.enable_grad():
        if grad_const is None:
            poly = multipole_poly_from_nodes(tables, phi, dphi)
            gphi, gdphi = torch.autograd.grad(poly, (phi, dphi),
                                              grad_outputs=grad_poly.to(torch.float64))
        else:
            k = multipole_consts_from_nodes(tables, phi, dphi)
            poly = multipole_poly_from_nodes(tables, phi, dphi, inv=k[0])
            gphi, gdphi = torch.autograd.grad(
                (poly, k), (phi, dphi),
                grad_outputs=(grad_poly.to(torch.float64),
                              grad_const.to(device=dev, dtype=torch.float64)),
                allow_unused=True)
            gphi = torch.zeros_like(phi) if gphi is None else gphi
            gdphi = torch.zeros_like(dphi) if gdphi is None else gdphi
    if n_file_cols is None:
        return gphi, gdphi
    cols = torch.as_tensor(np.asarray(tables.node_cols), dtype=torch.long, device=dev)
    out_p = torch.zeros((phi.shape[0], n_file_cols), dtype=torch.float64, device=dev)
    out_d = torch.zeros_like(out_p)
    out_p[:, cols] = gphi
    out_d[:, cols] = gdphi
    return out_p, out_d


def _spline_deriv_matrix(x: np.ndarray, bc_type) -> np.ndarray:
    """D with D @ y = derivative at the nodes of the cubic spline through (x, y)."""
    from scipy.interpolate import CubicSpline
    n = len(x)
    return CubicSpline(x, np.eye(n), axis=0, bc_type=bc_type)(x, 1)


def cylspline_node_vjp(tables, coefs, grad_nodes: torch.Tensor, phi=None) -> dict:
    """{m: dL/dPhi_m (nR, nz of the coefficient grid)} from dL/d(node table).

    The node table of the builder (prep_cylspline.build_cylspline_tables) is, per
    harmonic, f and its spline derivatives f_lR = D_R f, f_lz = f D_z^T,
    f_lR_lz = D_R f D_z^T -- linear maps (natural spline in lz; zero slope at R = 0
    and natural at the outer end in lR) -- of f = log(-Phi_0) (m = 0) or
    Phi_m / Phi_0 under log-scaling, Phi_m otherwise, on the z grid mirrored from
    z >= 0 when the file stores half of it.  The transpose of each step is applied
    in turn.  The outer asymptote, Rscale and the asinh grids are held fixed.  ``phi``
    ({m: grid on the coefficient file's grid}) replaces coefs.phi as the point of
    differentiation (node values set on the device)."""
    G = grad_nodes.detach().to("cpu", torch.float64).numpy()
    lR, lz = tables.lR_grid, tables.lz_grid
    nR = len(lR)
    DR = _spline_deriv_matrix(lR, ((1, np.zeros(nR)), "natural"))
    Dz = _spline_deriv_matrix(lz, "natural")
    z0 = np.asarray(coefs.z_grid, dtype=np.float64)
    half = z0[0] == 0
    nz0 = len(z0)
    src = coefs.phi if phi is None else phi
    phi = {}
    for m, t in src.items():
        t = np.asarray(t, dtype=np.float64)
        if half:
            full = np.empty((t.shape[0], 2 * nz0 - 1))
            full[:, nz0 - 1:] = t
            full[:, :nz0] = t[:, ::-1]
            phi[int(m)] = full
        else:
            phi[int(m)] = t
    df = {}
    for h, m in enumerate(tables.m_arr):
        Gf, Gx, Gy, Gxy = (G[h, :, :, q] for q in range(4))
        df[int(m)] = Gf + DR.T @ Gx + Gy @ Dz + DR.T @ Gxy @ Dz
    if tables.log_scaling:
        p0 = phi[0]
        dphi = {0: df[0] / p0}
        for m, d in df.items():
            if m == 0:
                continue
            dphi[m] = d / p0
            dphi[0] = dphi[0] - d * phi[m] / (p0 * p0)
    else:
        dphi = dict(df)
    if half:
        out = {}
        for m, d in dphi.items():
            g = d[:, nz0 - 1:].copy()
            g[:, 1:] += d[:, :nz0 - 1][:, ::-1]
            out[m] = g
        return out
    return dphi
