"""Leapfrog orbit integration in a GPU potential and its checkpointed adjoint.

Units are Agama's: kpc, km/s, time in kpc/(km/s) (= 0.977792221 Gyr; use
``gyr_to_time``).  The scheme is kick-drift-kick with one force evaluation
per step (the force at the end of a step is reused as the first kick of the
next):

    v_h   = v_n + h F(x_n, t_n)          h = dt / 2
    x_n+1 = x_n + dt v_h
    v_n+1 = v_h + h F(x_n+1, t_n+1)

The adjoint runs the steps backwards.  Positions are re-computed segment by
segment from checkpoints stored every ``checkpoint_every`` steps (and at the
end), and each backward step needs ONE vector-Jacobian product of the force
(``agb_eval_vjp``: (dF/dx)^T g = -H g) because the two half-kicks that use
F(x_n) are merged into one cotangent.  Total cost: the forward (n+1
evaluations), a re-computation (n evaluations; none when every step is a
checkpoint, which is what ``checkpoint_every=None`` picks whenever the
positions of every step fit in 60% of the free device memory) and n+1 VJPs.

For potentials that do not depend on time, steps are captured into CUDA
graphs (``graph_steps`` per graph) and replayed.
"""
from __future__ import annotations

from typing import List, Optional, Tuple

import torch

from . import _lib

GYR_PER_TIME_UNIT = 0.977792221          # 1 kpc / (km/s) in Gyr


def gyr_to_time(dt_gyr: float) -> float:
    return float(dt_gyr) / GYR_PER_TIME_UNIT


def is_static(pot) -> bool:
    """True when the potential tree does not depend on time."""
    from .potentials import (CompositePotentialGPU, EvolvingPotentialGPU, ScaledPotentialGPU,
                             ShiftedPotentialGPU, _Component)
    from .batch import BatchedPotentialGPU
    if isinstance(pot, (_Component, BatchedPotentialGPU)):
        return True      # batches hold only static units
    if isinstance(pot, CompositePotentialGPU):
        return all(is_static(c) for c in pot._components)
    if isinstance(pot, EvolvingPotentialGPU):
        return len(pot._pots) == 1 and is_static(pot._pots[0])
    if isinstance(pot, ShiftedPotentialGPU):
        return pot._is_static and is_static(pot._inner)
    if isinstance(pot, ScaledPotentialGPU):
        return pot._is_static and is_static(pot._inner)
    return False


def auto_checkpoint_every(like: torch.Tensor, n_steps: int, fraction: float = 0.6) -> int:
    """Checkpoint interval for ``n_steps`` steps of the particles in ``like`` within
    ``fraction`` of the free device memory: 1 (every step's positions, no
    re-computation in the adjoint) when they fit, else the smallest k whose (x, v)
    checkpoints fit."""
    row = like.numel() * 8
    try:
        free, _ = torch.cuda.mem_get_info(like.device)
    except (RuntimeError, AssertionError):
        return 64
    budget = int(free * fraction)
    if (int(n_steps) + 2) * row <= budget:
        return 1
    fit = max(1, budget // max(2 * row, 1))
    return max(2, -(-int(n_steps) // fit))


def allreduce_table_grads(tg: dict, group=None) -> dict:
    """Sum the coefficient gradients of every rank (particles sharded across ranks,
    the potential replicated): one all-reduce per Multipole, in a fixed order so
    that every rank issues the same collectives.  A no-op without an initialised
    process group of more than one rank."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size(group) < 2:
        return tg
    for key in sorted(tg, key=lambda c: c._sync_order):
        dist.all_reduce(tg[key], op=dist.ReduceOp.SUM, group=group)
    return tg


class Leapfrog:
    """Integrate N particles; keeps x, v, F as device buffers updated in place."""

    def __init__(self, pot, dt: float, t0: float = 0.0, precision: Optional[str] = None,
                 use_graph: Optional[bool] = None, graph_steps: int = 16):
        self.pot = pot
        self.dt = float(dt)
        self.h = 0.5 * self.dt
        self.t0 = float(t0)
        self.precision = precision
        self.static = is_static(pot)
        self.use_graph = self.static if use_graph is None else (use_graph and self.static)
        self.graph_steps = int(graph_steps)
        self._graph = None
        self._graph_key = None

    # -- single steps -------------------------------------------------------------
    def _force_into(self, x: torch.Tensor, t: float, F: torch.Tensor) -> None:
        self.pot._launch(x, t, _lib.MODE_GRAD, False, precision=self.precision,
                         out=(None, F, None, None))

    def _step(self, x, v, F, t) -> None:
        v.add_(F, alpha=self.h)
        x.add_(v, alpha=self.dt)
        self._force_into(x, t + self.dt, F)
        v.add_(F, alpha=self.h)

    def _advance(self, x, v, F, n0: int, n_steps: int) -> None:
        """n_steps steps from step index n0 (time t0 + n0 dt)."""
        if n_steps <= 0:
            return
        if not self.use_graph:
            for k in range(n_steps):
                self._step(x, v, F, self.t0 + (n0 + k) * self.dt)
            return
        key = (x.data_ptr(), v.data_ptr(), F.data_ptr(), x.shape[0],
               getattr(self.pot, "plan_generation", 0))
        if self._graph is None or self._graph_key != key:
            self._capture(x, v, F)
            self._graph_key = key
        full, rest = divmod(n_steps, self.graph_steps)
        for _ in range(full):
            self._graph.replay()
        for k in range(rest):
            self._step(x, v, F, self.t0)          # static potential: t does not matter

    def _capture(self, x, v, F) -> None:
        # warm-up on a side stream (allocator pools, lazy module loading), then capture
        xs, vs, Fs = x.clone(), v.clone(), F.clone()
        s = torch.cuda.Stream(device=x.device)
        s.wait_stream(torch.cuda.current_stream(x.device))
        with torch.cuda.stream(s):
            for _ in range(2):
                self._step(x, v, F, self.t0)
        torch.cuda.current_stream(x.device).wait_stream(s)
        x.copy_(xs); v.copy_(vs); F.copy_(Fs)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            for _ in range(self.graph_steps):
                self._step(x, v, F, self.t0)
        x.copy_(xs); v.copy_(vs); F.copy_(Fs)
        self._graph = g

    # -- forward with checkpoints ------------------------------------------------------
    def run(self, x0: torch.Tensor, v0: torch.Tensor, n_steps: int,
            checkpoint_every: Optional[int] = 64) -> Tuple[torch.Tensor, torch.Tensor, List]:
        """Returns (x_T, v_T, checkpoints); checkpoints = [(step, x, v)] every k steps and
        at the end.  k = 1 keeps every step's positions (v is None except at the end) and
        the adjoint then re-computes nothing; checkpoint_every=None picks k with
        ``auto_checkpoint_every`` (1 whenever the trajectory fits in 60% of the free
        device memory)."""
        x, v, F = self._buffers(x0)
        x.copy_(x0.detach())
        v.copy_(v0.detach())
        self._force_into(x, self.t0, F)
        k = auto_checkpoint_every(x, n_steps) if checkpoint_every is None else int(checkpoint_every)
        k = max(1, k)
        if k == 1:
            # every step's positions in one allocation [step][particle][3]; the adjoint
            # re-computes nothing and needs no velocities
            store = torch.empty((int(n_steps) + 1,) + tuple(x.shape), dtype=torch.float64,
                                device=x.device)
            for n in range(n_steps):
                store[n].copy_(x)
                self._step(x, v, F, self.t0 + n * self.dt)
            store[n_steps].copy_(x)
            ckpts = [(n, store[n], None) for n in range(n_steps)]
            ckpts.append((n_steps, store[n_steps], v.clone()))
            return x.clone(), v.clone(), ckpts
        # one allocation for all checkpoints: [checkpoint][x|v][particle][3]
        store = torch.empty((-(-int(n_steps) // k) + 1, 2) + tuple(x.shape), dtype=torch.float64,
                            device=x.device)
        ckpts = []
        n = 0
        while n < n_steps:
            j = len(ckpts)
            store[j, 0].copy_(x)
            store[j, 1].copy_(v)
            ckpts.append((n, store[j, 0], store[j, 1]))
            m = min(k, n_steps - n)
            self._advance(x, v, F, n, m)
            n += m
        j = len(ckpts)
        store[j, 0].copy_(x)
        store[j, 1].copy_(v)
        ckpts.append((n_steps, store[j, 0], store[j, 1]))
        return x.clone(), v.clone(), ckpts

    def _buffers(self, like: torch.Tensor):
        """Persistent (x, v, F) device buffers, so captured graphs stay valid across runs."""
        shape = tuple(like.shape)
        b = getattr(self, "_bufs", None)
        if b is None or tuple(b[0].shape) != shape or b[0].device != like.device:
            mk = lambda: torch.empty(shape, dtype=torch.float64, device=like.device)  # noqa: E731
            b = (mk(), mk(), mk())
            self._bufs = b
        return b

    # -- adjoint -----------------------------------------------------------------------
    def adjoint(self, ckpts: List, n_steps: int, lam_x: torch.Tensor,
                lam_v: torch.Tensor, table_grads: bool = False, group=None):
        """(dL/dx0, dL/dv0) from (dL/dx_T, dL/dv_T) and the forward's checkpoints.

        With table_grads=True also returns {component: gradient}: for each Multipole
        dL/dpoly (its quintic coefficients), for each CylSpline dL/d(node table),
        summed over all force evaluations (component.node_gradients() carries either
        to the coefficient-file nodes).
        Under torch.distributed (each rank integrating its own particles in the same
        potential) the table gradients are summed over the ranks of ``group``.
        """
        tg = {} if table_grads else None
        lx = lam_x.detach().to(torch.float64).contiguous().clone()
        lv = lam_v.detach().to(torch.float64).contiguous().clone()
        pending = None                      # cotangent on F(x_n) from the later half-kick
        gx = torch.empty_like(lx)
        at = {c[0]: c for c in ckpts}
        starts = sorted(c[0] for c in ckpts if c[0] < n_steps)
        bounds = starts + [n_steps]
        for seg in range(len(starts) - 1, -1, -1):
            s, e = bounds[seg], bounds[seg + 1]
            _, xs, vs = at[s]
            # the segment's positions: x_s and x_e from checkpoints, the others re-computed
            pos = {s: xs}
            if e in at:
                pos[e] = at[e][1]
            last = e - 1 if e in at else e
            if last > s:
                X = torch.empty((last - s,) + tuple(xs.shape), dtype=torch.float64, device=xs.device)
                x, v = xs.clone(), vs.clone()
                F = torch.empty_like(x)
                self._force_into(x, self.t0 + s * self.dt, F)
                for n in range(s, last):
                    self._step(x, v, F, self.t0 + n * self.dt)
                    X[n - s].copy_(x)
                    pos[n + 1] = X[n - s]
            for n in range(e - 1, s - 1, -1):
                gF = lv * self.h
                if pending is not None:
                    gF.add_(pending)
                if tg is None:
                    self.pot._vjp(pos[n + 1], self.t0 + (n + 1) * self.dt, None, gF,
                                  precision=self.precision, out=gx)
                else:
                    self.pot._adjoint_vjp(pos[n + 1], self.t0 + (n + 1) * self.dt, None, gF,
                                          tg, precision=self.precision, out=gx)
                lx.add_(gx)
                lv.add_(lx, alpha=self.dt)
                pending = lv * self.h
        if pending is not None:
            _, x0, _ = at[0]
            if tg is None:
                self.pot._vjp(x0, self.t0, None, pending, precision=self.precision, out=gx)
            else:
                self.pot._adjoint_vjp(x0, self.t0, None, pending, tg, precision=self.precision,
                                      out=gx)
            lx.add_(gx)
        if tg is not None:
            return lx, lv, allreduce_table_grads(self.pot._table_grads_from_device(tg), group)
        return lx, lv


class _LeapfrogFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x0, v0, integrator, n_steps, checkpoint_every):
        x, v, ckpts = integrator.run(x0, v0, n_steps, checkpoint_every)
        ctx.integrator, ctx.n_steps, ctx.ckpts = integrator, n_steps, ckpts
        return x, v

    @staticmethod
    def backward(ctx, gx, gv):
        if gx is None:
            gx = torch.zeros_like(ctx.ckpts[0][1])
        if gv is None:
            gv = torch.zeros_like(ctx.ckpts[0][2])
        lx, lv = ctx.integrator.adjoint(ctx.ckpts, ctx.n_steps, gx, gv)
        return lx, lv, None, None, None


def leapfrog(pot, x0: torch.Tensor, v0: torch.Tensor, dt: float, n_steps: int, t0: float = 0.0,
             checkpoint_every: Optional[int] = 64, precision: Optional[str] = None,
             use_graph: Optional[bool] = None):
    """(x_T, v_T) after n_steps leapfrog steps; differentiable w.r.t. (x0, v0) through the
    checkpointed adjoint."""
    integ = Leapfrog(pot, dt, t0=t0, precision=precision, use_graph=use_graph)
    k = None if checkpoint_every is None else int(checkpoint_every)
    return _LeapfrogFn.apply(x0, v0, integ, int(n_steps), k)
