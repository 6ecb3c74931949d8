"""torch.autograd entry points with hand-written backward passes.

``potential_and_force(pot, xyz, t)`` returns (Phi, F) as differentiable
functions of the positions: the backward is one fused CUDA launch
(agb_eval_vjp) that evaluates every component with its Hessian and contracts
per point, dL/dx = dL/dPhi * grad(Phi) - H dL/dF, without materialising H.
The reference has no derivatives with respect to its inputs; this is new.
"""
from __future__ import annotations

from typing import Optional

import torch

from . import _lib
from .potentials import prep_xyz


class _PhiForce(torch.autograd.Function):
    @staticmethod
    def forward(ctx, xyz, pot, t, precision):
        arr = xyz.detach().to(dtype=torch.float64).contiguous()
        phi, force, _, _ = pot._launch(arr, t, _lib.MODE_GRAD, True, precision=precision)
        ctx.save_for_backward(arr)
        ctx.pot, ctx.t, ctx.precision = pot, t, precision
        return phi, force

    @staticmethod
    def backward(ctx, g_phi, g_force):
        (arr,) = ctx.saved_tensors
        gx = ctx.pot._vjp(arr, ctx.t, g_phi, g_force, precision=ctx.precision)
        return gx, None, None, None


def potential_and_force(pot, xyz: torch.Tensor, t: float = 0.0,
                        precision: Optional[str] = None):
    """(Phi (N,), F (N,3)) at CUDA positions xyz (N,3), differentiable w.r.t. xyz."""
    if not isinstance(xyz, torch.Tensor) or xyz.device.type != "cuda":
        xyz = prep_xyz(xyz)[0]
    if xyz.dim() != 2 or xyz.shape[1] != 3:
        raise ValueError(f"xyz must have shape (N,3), got {tuple(xyz.shape)}")
    return _PhiForce.apply(xyz, pot, float(t), precision)


def force(pot, xyz: torch.Tensor, t: float = 0.0, precision: Optional[str] = None):
    """F (N,3), differentiable w.r.t. xyz."""
    return potential_and_force(pot, xyz, t, precision)[1]


def potential(pot, xyz: torch.Tensor, t: float = 0.0, precision: Optional[str] = None):
    """Phi (N,), differentiable w.r.t. xyz."""
    return potential_and_force(pot, xyz, t, precision)[0]
