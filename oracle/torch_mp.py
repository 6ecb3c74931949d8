"""Test infrastructure only: an FP64 torch re-implementation of the Multipole
evaluation (the reference's formulas, _multipole_potential_kernel.cu:140-410),
differentiable with respect to both the positions and the quintic
coefficients, used to check the hand-written backward passes against torch
autograd.  Interior points only (inside the radial grid, away from the z axis).
"""
from __future__ import annotations

import math

import torch

MUL0 = 3.5449077018110318
MUL1 = 5.0132565706694072


def _coef(m: int) -> float:
    dfact = 1
    for k in range(1, 2 * m, 2):
        dfact *= k
    return (-1) ** m * dfact * math.sqrt((2 * m + 1) / (4.0 * math.pi * math.factorial(2 * m)))


def multipole_phi(poly: torch.Tensor, lm_l, lm_m, sc, log_scaling: int, xyz: torch.Tensor):
    """Phi at xyz (N,3) from poly (n_lm, n_int, 6) in the builder's harmonic order."""
    logr_min, dlogr, inv_dlogr, invPhi0 = sc[0], sc[1], sc[2], sc[3]
    x, y, z = xyz[:, 0], xyz[:, 1], xyz[:, 2]
    r = torch.sqrt(x * x + y * y + z * z)
    R = torch.sqrt(x * x + y * y)
    logr = torch.log(r)
    k = torch.floor((logr.detach() - logr_min) * inv_dlogr).long()
    n_int = poly.shape[1]
    assert int(k.min()) >= 0 and int(k.max()) < n_int, "interior points only"
    s = (logr - (logr_min + k.to(logr.dtype) * dlogr)) * inv_dlogr
    a = poly[:, k, :]                                             # (n_lm, N, 6)
    sp = torch.stack([s ** j for j in range(6)], dim=-1)          # (N, 6)
    C = (a * sp[None]).sum(-1)                                    # (n_lm, N)
    ct, st = z / r, R / r
    ph = torch.atan2(y, x)
    if log_scaling:
        F = 1.0 / (invPhi0 - torch.exp(C[0]))
    else:
        F = torch.ones_like(r)
    mono = MUL0 * 0.28209479177387814 * (F if log_scaling else C[0])
    total = torch.zeros_like(r)
    # Legendre by the un-normalised recurrence with the normalisation update
    lmax = int(max(lm_l))
    cache = {}
    for m in range(lmax + 1):
        pref = math.sqrt((2 * m + 1) / (4.0 * math.pi * math.factorial(2 * m)))
        raw_prev = _coef(m) * st ** m / pref
        cache[(m, m)] = raw_prev * pref
        if lmax == m:
            continue
        raw_cur = raw_prev * ct * (2 * m + 1)
        pf = pref
        for l in range(m + 1, lmax + 1):
            if l > m + 1:
                nr = ((2 * l - 1) * ct * raw_cur - (l + m - 1) * raw_prev) / (l - m)
                raw_prev, raw_cur = raw_cur, nr
            pf = pf * math.sqrt((2.0 * l + 1) / (2.0 * l - 1) * (l - m) / (l + m))
            cache[(l, m)] = raw_cur * pf
    for c in range(1, len(lm_l)):
        l, m = int(lm_l[c]), int(lm_m[c])
        am = abs(m)
        Y = cache[(l, am)] * (MUL0 if am == 0 else MUL1)
        T = torch.cos(am * ph) if m >= 0 else torch.sin(am * ph)
        total = total + C[c] * Y * T
    return mono + F * total if log_scaling else mono + total


def loss_grad_poly(tables, xyz, g_phi, g_force):
    """d(sum g_phi Phi + g_force . F)/dpoly by torch autograd (F = -grad Phi)."""
    poly = torch.tensor(tables.poly, dtype=torch.float64, requires_grad=True)
    x = torch.tensor(xyz, dtype=torch.float64, requires_grad=True)
    phi = multipole_phi(poly, tables.lm_l, tables.lm_m, tables.scalars(), tables.log_scaling, x)
    (gradphi,) = torch.autograd.grad(phi.sum(), x, create_graph=True)
    L = (torch.as_tensor(g_phi) * phi).sum() - (torch.as_tensor(g_force) * gradphi).sum()
    (gp,) = torch.autograd.grad(L, poly)
    return gp.numpy(), phi.detach().numpy(), (-gradphi).detach().numpy()
