"""torch.autograd entry points with hand-written backward passes.

``potential_and_force(pot, xyz, t)`` returns (Phi, F) as differentiable
functions of the positions and of the node tables the tree exposes through
``pot.node_parameters()``:

* dL/dx: one fused CUDA launch (agb_eval_vjp) evaluates every component with
  its Hessian and contracts per point, dL/dx = dL/dPhi * grad(Phi) - H dL/dF,
  without materialising H;
* dL/d(node tables), for the components whose node_parameters() were requested:
  the table-gradient kernels (agb_multipole_table_vjp, agb_cylspline_table_vjp)
  give dL/d(quintic coefficients) or dL/d(node table), carried to the node values
  through the differentiable restatement of the table builders (diff_tables).

The reference has no derivatives with respect to its inputs; this is new.  Its
node tables are the inputs of its constructors (gpu_potential.py:654-660 and
the builder :408-631; CylSpline :1281 and :1143-1253).
"""
from __future__ import annotations

from typing import Optional

import torch

from . import _lib
from .potentials import prep_xyz


class _PhiForce(torch.autograd.Function):
    @staticmethod
    def forward(ctx, xyz, pot, t, precision, tracked, *nodes):
        arr = xyz.detach().to(dtype=torch.float64).contiguous()
        phi, force, _, _ = pot._launch(arr, t, _lib.MODE_GRAD, True, precision=precision)
        ctx.save_for_backward(arr)
        ctx.pot, ctx.t, ctx.precision, ctx.tracked = pot, t, precision, tracked
        return phi, force

    @staticmethod
    def backward(ctx, g_phi, g_force):
        (arr,) = ctx.saved_tensors
        pot, t = ctx.pot, ctx.t
        gx = None
        if ctx.needs_input_grad[0]:
            gx = pot._vjp(arr, t, g_phi, g_force, precision=ctx.precision)
        node_grads = [None] * sum(len(p) for _, p in ctx.tracked)
        if any(ctx.needs_input_grad[5:]):
            want = {id(c) for c, _ in ctx.tracked}
            acc = {}
            for comp, sigma, gamma, ampl in pot._leaves(float(t)):
                if id(comp) not in want:
                    continue
                kw = {}
                if comp.kind == _lib.KIND_MULTIPOLE:     # and the builder's scalars
                    key = ("const", comp)
                    if key not in acc:
                        acc[key] = torch.zeros(_lib.MP_NCONST, dtype=torch.float64,
                                               device=arr.device)
                    kw["const_grad"] = acc[key]
                g = comp.table_vjp(arr, t, g_phi, g_force, leaf=(sigma, gamma, ampl), **kw)
                acc[comp] = acc[comp] + g if comp in acc else g
            node_grads = pot._node_param_grads(acc, ctx.tracked)
        return (gx, None, None, None, None, *node_grads)


def potential_and_force(pot, xyz: torch.Tensor, t: float = 0.0,
                        precision: Optional[str] = None):
    """(Phi (N,), F (N,3)) at CUDA positions xyz (N,3), differentiable w.r.t. xyz and
    w.r.t. the tree's node tensors (pot.node_parameters())."""
    if not isinstance(xyz, torch.Tensor) or xyz.device.type != "cuda":
        xyz = prep_xyz(xyz)[0]
    if xyz.dim() != 2 or xyz.shape[1] != 3:
        raise ValueError(f"xyz must have shape (N,3), got {tuple(xyz.shape)}")
    tracked = pot._tracked_nodes()
    nodes = [q for _, ps in tracked for q in ps]
    return _PhiForce.apply(xyz, pot, float(t), precision, tracked, *nodes)


def force(pot, xyz: torch.Tensor, t: float = 0.0, precision: Optional[str] = None):
    """F (N,3), differentiable w.r.t. xyz and the node tensors."""
    return potential_and_force(pot, xyz, t, precision)[1]


def potential(pot, xyz: torch.Tensor, t: float = 0.0, precision: Optional[str] = None):
    """Phi (N,), differentiable w.r.t. xyz and the node tensors."""
    return potential_and_force(pot, xyz, t, precision)[0]
