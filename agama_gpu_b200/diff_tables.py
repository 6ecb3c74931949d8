"""Differentiable construction of the Multipole quintic tables (torch, FP64).

The same steps as prep_multipole.build_multipole_tables -- log-scaling of the
node values, the tridiagonal system for the quintic's second derivatives,
the six Horner coefficients per interval -- written with torch operations so
that a gradient with respect to the coefficients (from the table-VJP kernel)
can be carried back to the node tables Phi_lm(r_i) and dPhi_lm/dr(r_i).

Held fixed (treated as constants of the tables): the radial grid, invPhi0,
the inner/outer extrapolation constants, the harmonic set after pruning.
A grid that had to be resampled to log-uniform is not supported here.
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


def multipole_poly_from_nodes(tables, phi: torch.Tensor, dphi_dr: torch.Tensor) -> torch.Tensor:
    """Quintic coefficients (n_lm, n_int, 6) from node tables (nR, n_lm) in the
    builder's harmonic order (``tables.node_phi`` layout); differentiable."""
    if tables.resampled:
        raise ValueError("node gradients need a log-uniform input grid (this one was resampled)")
    dev = phi.device
    r = torch.as_tensor(tables.r_grid, dtype=torch.float64, device=dev)
    logr = torch.log(r)
    dphi_dlogr = dphi_dr * r[:, None]
    if tables.log_scaling:
        p0 = phi[:, 0]
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
             nodes=None) -> Tuple[torch.Tensor, torch.Tensor]:
    """Carry dL/dpoly back to the node tables in the coefficient file's column order.

    Returns (dL/dPhi_nodes, dL/d(dPhi/dr)_nodes), each (nR, n_file_cols); columns
    the table builder pruned (all-zero) get zero (build with prune_threshold=0
    to differentiate every harmonic).  n_file_cols=None returns them in the
    builder's harmonic order instead, (nR, n_lm) like ``tables.node_phi``.
    ``nodes`` = (phi, dphi_dr) in the builder's order when the tables were
    replaced on the device (set_node_tables), else the builder's own node values
    are used.
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
        poly = multipole_poly_from_nodes(tables, phi, dphi)
        gphi, gdphi = torch.autograd.grad(poly, (phi, dphi),
                                          grad_outputs=grad_poly.to(torch.float64))
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
