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

Higher order: ``scheme="yoshida4"`` composes each step of three such
kick-drift-kick substeps of sizes w1 dt, w0 dt, w1 dt (Yoshida 1990, 4th
order, three force evaluations per step); the checkpoints and the adjoint then
run over substeps with their own dt_j and h_j = dt_j / 2.

For potentials that do not depend on time, steps are captured into CUDA
graphs (``graph_steps`` per graph) and replayed.
"""
from __future__ import annotations

from typing import List, Optional, Tuple

import torch

from . import _lib

GYR_PER_TIME_UNIT = 0.977792221          # 1 kpc / (km/s) in Gyr


def _consts_epoch(pot) -> int:
    """The components' builder-scalar generation (captured graphs bake the descriptors)."""
    from .potentials import consts_epoch
    try:
        return consts_epoch(pot._all_components())
    except (AttributeError, TypeError):
        return 0


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
    if like.device.type != "cuda":
        return 64
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
    def order(key):             # a component, or ("const", component) after it
        return (key[1]._sync_order, 1) if isinstance(key, tuple) else (key._sync_order, 0)
    for key in sorted(tg, key=order):
        dist.all_reduce(tg[key], op=dist.ReduceOp.SUM, group=group)
    return tg


_CBRT2 = 2.0 ** (1.0 / 3.0)
SCHEMES = {
    # kick-drift-kick substeps of fractions c_j of the step (sum 1), applied in turn
    "leapfrog": (1.0,),
    # Yoshida (1990) 4th-order composition: w1, w0, w1 with w1 = 1/(2 - 2^(1/3)),
    # w0 = -2^(1/3)/(2 - 2^(1/3)); three force evaluations per step
    "yoshida4": (1.0 / (2.0 - _CBRT2), -_CBRT2 / (2.0 - _CBRT2), 1.0 / (2.0 - _CBRT2)),
}


def scheme_coefficients(scheme) -> Tuple[float, ...]:
    """Substep fractions of a scheme name in ``SCHEMES`` or an explicit sequence
    (a symmetric composition of leapfrog substeps, fractions summing to 1)."""
    if isinstance(scheme, str):
        if scheme not in SCHEMES:
            raise ValueError(f"unknown integration scheme {scheme!r}; known: {sorted(SCHEMES)}")
        return SCHEMES[scheme]
    c = tuple(float(x) for x in scheme)
    if not c or abs(sum(c) - 1.0) > 1e-12:
        raise ValueError("substep fractions must be non-empty and sum to 1")
    return c


class Leapfrog:
    """Integrate N particles; keeps x, v, F as device buffers updated in place.

    ``scheme`` composes each step of S kick-drift-kick substeps of sizes c_j dt
    ("leapfrog": S = 1; "yoshida4": the 4th-order triple, S = 3).  Substeps are the
    unit of the forward and of the adjoint: substep g (step g // S, fraction
    c[g % S]) ends at time t0 + (g // S) dt + (c_0 + ... + c_{g % S}) dt.
    """

    def __init__(self, pot, dt: float, t0: float = 0.0, precision: Optional[str] = None,
                 use_graph: Optional[bool] = None, graph_steps: int = 16, scheme="leapfrog",
                 device_time: Optional[bool] = None):
        self.pot = pot
        self.dt = float(dt)
        self.h = 0.5 * self.dt
        self.t0 = float(t0)
        self.coefs = scheme_coefficients(scheme)
        self.S = len(self.coefs)
        if self.S == 1:
            self._sub = [(self.dt, self.h, self.dt)]
        else:
            cum, sub = 0.0, []
            for c in self.coefs:
                cum += c
                sub.append((c * self.dt, 0.5 * c * self.dt, cum * self.dt))
            self._sub = sub                 # (dt_j, h_j, end offset within the step)
        self.precision = precision
        self.static = is_static(pot)
        self._want_graph = use_graph
        self._device_time = device_time
        self._timed_cache = {}
        self.graph_steps = int(graph_steps)
        self._graph = None
        self._graph_key = None
        self._step_dev = None
        # backward steps with table gradients in two launches (agb_adjoint_step) where the
        # tree allows; False: the separate VJP, kick and drift launches
        self.fused_adjoint = True

    # -- time on the device ----------------------------------------------------------
    def _timed(self, x: torch.Tensor) -> bool:
        """Forces of this time-dependent potential come from agb_eval_timed: the
        leaves are computed on the device from a device step counter, so steps can
        be captured in CUDA graphs (device_time=False keeps the host leaves)."""
        if self.static or self._device_time is False or not x.is_cuda:
            return False
        hit = self._timed_cache.get(x.device)
        if hit is None:
            hit = hasattr(self.pot, "_time_plan") and self.pot._time_plan(x.device) is not None
            self._timed_cache[x.device] = hit
        return hit

    def _graphs(self, x: torch.Tensor) -> bool:
        ok = x.is_cuda and (self.static or self._timed(x))
        return ok if self._want_graph is None else (bool(self._want_graph) and ok)

    @property
    def use_graph(self) -> bool:
        """Whether steps are captured in CUDA graphs (static potentials, and
        time-dependent ones whose leaves the device evaluates)."""
        if self._want_graph is False:
            return False
        return self.static or any(self._timed_cache.values())

    def _counter(self, x: torch.Tensor) -> torch.Tensor:
        if self._step_dev is None or self._step_dev.device != x.device:
            self._step_dev = torch.zeros((), dtype=torch.int64, device=x.device)
        return self._step_dev

    def _set_step(self, x: torch.Tensor, n: int) -> None:
        if self._timed(x):
            self._counter(x).fill_(int(n))

    # -- single steps -------------------------------------------------------------
    def _force_into(self, x: torch.Tensor, t: float, F: torch.Tensor) -> None:
        self.pot._launch(x, t, _lib.MODE_GRAD, False, precision=self.precision,
                         out=(None, F, None, None))

    def _force_at(self, x: torch.Tensor, n: int, off: float, F: torch.Tensor) -> None:
        """F at t = (t0 + n dt) + off: on the device from the step counter (which holds
        n) when the leaves are device-evaluated, else with the host leaves at t."""
        if self._timed(x):
            self.pot._launch_timed(x, self._counter(x), self.t0, self.dt, off, _lib.MODE_GRAD,
                                   False, precision=self.precision, out=(None, F, None, None))
        else:
            self._force_into(x, self.t0 + n * self.dt + off, F)

    def _kd(self, x, v, F, h1: float, h2: float, dt: float, flags: int) -> None:
        """v = fma(h1, F, v) [1]; v = fma(h2, F, v) [2]; x = fma(dt, v, x) [4]; the
        device step counter += 1 [8]: one launch (agb_leapfrog_kick_drift) on the GPU,
        the same updates with torch on the CPU."""
        if x.is_cuda:
            step = self._counter(x) if (flags & 8) else None
            rc = _lib.lib.agb_leapfrog_kick_drift(
                x.data_ptr(), v.data_ptr(), F.data_ptr(), x.shape[0], h1, h2, dt, flags,
                None if step is None else step.data_ptr(),
                torch.cuda.current_stream(x.device).cuda_stream)
            _lib.check(rc, "agb_leapfrog_kick_drift")
            return
        if flags & 1:
            v.add_(F, alpha=h1)
        if flags & 2:
            v.add_(F, alpha=h2)
        if flags & 4:
            x.add_(v, alpha=dt)

    def _t(self, g: int) -> float:
        """Time at the end of substep g - 1 (= at the start of substep g)."""
        n, j = divmod(int(g), self.S)
        return self.t0 + n * self.dt + (self._sub[j - 1][2] if j else 0.0)

    def _substep(self, x, v, F, g: int) -> None:
        n, j = divmod(int(g), self.S)
        dtj, hj, off = self._sub[j]
        self._kd(x, v, F, 0.0, hj, dtj, 6)
        self._force_at(x, n, off, F)
        inc = 8 if (j == self.S - 1 and self._timed(x)) else 0
        self._kd(x, v, F, hj, 0.0, 0.0, 1 | inc)

    def _step(self, x, v, F, n: int) -> None:
        """One step from step index n, time t0 + n dt (all S substeps); with device
        leaves the step counter must hold n and ends at n + 1."""
        for g in range(int(n) * self.S, (int(n) + 1) * self.S):
            self._substep(x, v, F, g)

    def _advance(self, x, v, F, n0: int, n_steps: int) -> None:
        """n_steps steps from step index n0 (time t0 + n0 dt)."""
        if n_steps <= 0:
            return
        self._set_step(x, n0)
        if not self._graphs(x):
            for k in range(n_steps):
                self._step(x, v, F, n0 + k)
            return
        key = (x.data_ptr(), v.data_ptr(), F.data_ptr(), x.shape[0],
               getattr(self.pot, "plan_generation", 0), _consts_epoch(self.pot))
        if self._graph is None or self._graph_key != key:
            self._capture(x, v, F, n0)
            self._graph_key = key
        full, rest = divmod(n_steps, self.graph_steps)
        for _ in range(full):
            self._graph.replay()        # advances the device step counter itself
        for k in range(rest):
            self._step(x, v, F, n0 + full * self.graph_steps + k)

    def _capture(self, x, v, F, n0: int) -> None:
        # warm-up on a side stream (allocator pools, lazy module loading), then capture;
        # x, v, F and the step counter are restored after each
        xs, vs, Fs = x.clone(), v.clone(), F.clone()
        s = torch.cuda.Stream(device=x.device)
        s.wait_stream(torch.cuda.current_stream(x.device))
        with torch.cuda.stream(s):
            for k in range(2):
                self._step(x, v, F, n0 + k)
        torch.cuda.current_stream(x.device).wait_stream(s)
        x.copy_(xs); v.copy_(vs); F.copy_(Fs)
        self._set_step(x, n0)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            for k in range(self.graph_steps):
                self._step(x, v, F, n0 + k)
        x.copy_(xs); v.copy_(vs); F.copy_(Fs)
        self._set_step(x, n0)
        self._graph = g

    # -- forward with checkpoints ------------------------------------------------------
    def run(self, x0: torch.Tensor, v0: torch.Tensor, n_steps: int,
            checkpoint_every: Optional[int] = 64) -> Tuple[torch.Tensor, torch.Tensor, List]:
        """Returns (x_T, v_T, checkpoints); checkpoints = [(substep, x, v)] every k steps
        (substep = step * S) and at the end.  k = 1 keeps the positions at every substep
        (v is None except at the end) and the adjoint then re-computes nothing;
        checkpoint_every=None picks k with ``auto_checkpoint_every`` (1 whenever the
        trajectory fits in 60% of the free device memory).

        A batch of potentials (BatchedPotentialGPU with its pre-sort on) is integrated
        with its particles in the batch's sort_order() of x0: every force of the run
        then visits the rows in order without sorting them again (results are per
        particle and do not depend on the order); x_T, v_T and the checkpoints come
        back in the caller's order."""
        order = self._sort_order(x0)
        if order is None:
            return self._run(x0, v0, n_steps, checkpoint_every)
        self.pot._rows_in_order = True
        try:
            xT, vT, ck = self._run(x0.detach()[order], v0.detach()[order], n_steps,
                                   checkpoint_every)
        finally:
            self.pot._rows_in_order = False

        def back(a):
            if a is None:
                return None
            out = torch.empty_like(a)
            out[order] = a
            return out
        return back(xT), back(vT), [(g, back(xs), back(vs)) for g, xs, vs in ck]

    def _sort_order(self, x0: torch.Tensor):
        """The batch's evaluation order of x0's rows (None: keep the caller's order)."""
        pot = self.pot
        if not (x0.is_cuda and getattr(pot, "presort", False) and hasattr(pot, "sort_order")):
            return None
        return pot.sort_order(x0.detach(), precision=self.precision)

    def _run(self, x0: torch.Tensor, v0: torch.Tensor, n_steps: int,
             checkpoint_every: Optional[int] = 64) -> Tuple[torch.Tensor, torch.Tensor, List]:
        x, v, F = self._buffers(x0)
        x.copy_(x0.detach())
        v.copy_(v0.detach())
        self._set_step(x, 0)
        self._force_at(x, 0, 0.0, F)
        S = self.S
        G = int(n_steps) * S
        if checkpoint_every is None:
            k = auto_checkpoint_every(x, G)
            k = 1 if k == 1 else max(2, -(-k // S))
        else:
            k = int(checkpoint_every)
        k = max(1, k)
        if k == 1:
            # every substep's positions in one allocation [substep][particle][3]; the
            # adjoint re-computes nothing and needs no velocities
            store = torch.empty((G + 1,) + tuple(x.shape), dtype=torch.float64, device=x.device)
            for g in range(G):
                store[g].copy_(x)
                self._substep(x, v, F, g)
            store[G].copy_(x)
            ckpts = [(g, store[g], None) for g in range(G)]
            ckpts.append((G, store[G], v.clone()))
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
            ckpts.append((n * S, store[j, 0], store[j, 1]))
            m = min(k, n_steps - n)
            self._advance(x, v, F, n, m)
            n += m
        j = len(ckpts)
        store[j, 0].copy_(x)
        store[j, 1].copy_(v)
        ckpts.append((G, store[j, 0], store[j, 1]))
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
                lam_v: torch.Tensor, table_grads: bool = False, group=None,
                reconstruct: str = "recompute"):
        """(dL/dx0, dL/dv0) from (dL/dx_T, dL/dv_T) and the forward's checkpoints.

        With table_grads=True also returns {component: gradient}: for each Multipole
        dL/dpoly (its quintic coefficients), for each CylSpline dL/d(node table),
        summed over all force evaluations (component.node_gradients() carries either
        to the coefficient-file nodes).
        Under torch.distributed (each rank integrating its own particles in the same
        potential) the table gradients are summed over the ranks of ``group``.

        Per substep g (backwards; dt_g, h_g its drift and half-kick):
            lx += (dF/dx)^T gF at x_{g+1};  lv += dt_g lx;  gF = (h_g + h_{g-1}) lv
        where gF is the cotangent of F(x_g): the second half-kick of substep g - 1
        and the first of substep g both use it (h_0 lv for x_0, taken at the end).

        Positions between checkpoints (k >= 2): reconstruct="recompute" integrates
        each segment forwards again from its first checkpoint (one extra force per
        substep, bit-identical positions); reconstruct="reverse" steps backwards
        from the segment's last checkpoint (x, v) with the time-reversed substep,
        taking F(x_{g+1}) from the VJP launch at x_{g+1} itself (the adjoint
        kernels output the force they form anyway), so no force is evaluated
        twice.  Leapfrog is time-reversible: the reversed positions differ from
        the forward's by rounding only (amplified over at most k steps, and reset
        at every checkpoint).
        """
        if reconstruct not in ("recompute", "reverse"):
            raise ValueError("reconstruct must be 'recompute' or 'reverse'")
        tg = {} if table_grads else None
        S = self.S
        G = int(n_steps) * S
        lx = lam_x.detach().to(torch.float64).contiguous().clone()
        lv = lam_v.detach().to(torch.float64).contiguous().clone()
        gx = torch.empty_like(lx)
        at = {c[0]: c for c in ckpts}
        starts = sorted(c[0] for c in ckpts if c[0] < G)
        bounds = starts + [G]
        # gF: cotangent of F(x_{g+1}) -- h_g lv from substep g's second half-kick plus
        # h_{g+1} lv from substep g+1's first one, both with the same lv.  The fused
        # steps take it as cot[0] lv without reading or writing gF (cot[1]: gF is
        # behind), and gF is formed from lv only where an unfused launch reads it
        gF = lv * self._sub[(G - 1) % S][1] if G > 0 else None
        cot = [self._sub[(G - 1) % S][1] if G > 0 else 0.0, False]

        def gF_now():
            if cot[1]:
                torch.mul(lv, cot[0], out=gF)
                cot[1] = False
            return gF

        def vjp(xg, t, force=None):
            """gx = (dF/dx)^T gF at xg (and the table gradients), gF formed if behind."""
            g_force = gF_now()
            kw = {} if force is None else {"force_out": force}
            if tg is None:
                self.pot._vjp(xg, t, None, g_force, precision=self.precision, out=gx, **kw)
            else:
                self.pot._adjoint_vjp(xg, t, None, g_force, tg, precision=self.precision, out=gx,
                                      **kw)

        on_gpu = lx.is_cuda

        def kick(g):
            """lx += gx; lv += dt_g lx; gF = (h_g + h_{g-1}) lv (h_0 lv after substep 0)."""
            dtg, hg, _ = self._sub[g % S]
            c = hg + (self._sub[(g - 1) % S][1] if g > 0 else 0.0)
            cot[0] = c
            if on_gpu:          # one launch (agb_adjoint_kick)
                rc = _lib.lib.agb_adjoint_kick(lx.data_ptr(), lv.data_ptr(), gx.data_ptr(),
                                               gF.data_ptr(), lx.shape[0], dtg, c,
                                               torch.cuda.current_stream(lx.device).cuda_stream)
                _lib.check(rc, "agb_adjoint_kick")
                return
            lx.add_(gx)
            lv.add_(lx, alpha=dtg)
            torch.mul(lv, c, out=gF)

        def drift_back(xc, vh, Fg, k, dtg):
            """vh -= k F; x -= dt_g vh (the time-reversed drift)."""
            if on_gpu:
                rc = _lib.lib.agb_reverse_drift(xc.data_ptr(), vh.data_ptr(), Fg.data_ptr(),
                                                xc.shape[0], k, dtg,
                                                torch.cuda.current_stream(xc.device).cuda_stream)
                _lib.check(rc, "agb_reverse_drift")
                return
            vh.sub_(Fg, alpha=k)
            xc.sub_(vh, alpha=dtg)

        # the whole backward step in two launches (agb_adjoint_step) when the tree is one
        # regular Multipole and analytic leaves and table gradients are wanted
        fused_ok = (self.fused_adjoint and tg is not None and on_gpu and
                    hasattr(self.pot, "_adjoint_step"))

        def fused(xg, g, vh_=None, k_=0.0):
            if not fused_ok:
                return False
            dtg, hg, _ = self._sub[g % S]
            c = hg + (self._sub[(g - 1) % S][1] if g > 0 else 0.0)
            if not self.pot._adjoint_step(xg, self._t(g + 1), None, tg, lx, lv, dtg, c, vh=vh_,
                                          k=k_, dt_drift=dtg, precision=self.precision,
                                          c_in=cot[0]):
                return False
            cot[0] = c
            cot[1] = True
            return True

        for seg in range(len(starts) - 1, -1, -1):
            s, e = bounds[seg], bounds[seg + 1]
            _, xs, vs = at[s]
            if reconstruct == "reverse" and e in at and at[e][2] is not None and e - 1 > s:
                # backwards from (x_e, v_e): v_h(g) = v_{g+1} - h_g F(x_{g+1}),
                # x_g = x_{g+1} - dt_g v_h(g), and v_{g+1} = v_h(g+1) - h_{g+1} F(x_{g+1})
                xc = at[e][1].clone()
                vh = None
                Fg = torch.empty_like(xc)
                h_next = 0.0
                for g in range(e - 1, s - 1, -1):
                    dtg, hg, _ = self._sub[g % S]
                    need = g > s
                    if need:
                        vh_f = vh if vh is not None else at[e][2].clone()
                        k_f = hg if vh is None else h_next + hg
                        if fused(xc, g, vh_f, k_f):
                            vh = vh_f
                            h_next = hg
                            continue
                    elif fused(xc, g):
                        continue
                    vjp(xc, self._t(g + 1), Fg if need else None)
                    kick(g)
                    if need:
                        if vh is None:
                            vh = at[e][2].clone()
                            drift_back(xc, vh, Fg, hg, dtg)
                        else:
                            drift_back(xc, vh, Fg, h_next + hg, dtg)
                        h_next = hg
                continue
            # the segment's positions: x_s and x_e from checkpoints, the others re-computed
            pos = {s: xs}
            if e in at:
                pos[e] = at[e][1]
            last = e - 1 if e in at else e
            if last > s:
                X = torch.empty((last - s,) + tuple(xs.shape), dtype=torch.float64, device=xs.device)
                x, v = xs.clone(), vs.clone()
                F = torch.empty_like(x)
                n_s, j_s = divmod(s, S)
                self._set_step(x, n_s)
                self._force_at(x, n_s, self._sub[j_s - 1][2] if j_s else 0.0, F)
                for g in range(s, last):
                    self._substep(x, v, F, g)
                    X[g - s].copy_(x)
                    pos[g + 1] = X[g - s]
            for g in range(e - 1, s - 1, -1):
                if fused(pos[g + 1], g):
                    continue
                vjp(pos[g + 1], self._t(g + 1))
                kick(g)
        if G > 0:
            _, x0, _ = at[0]
            vjp(x0, self.t0)
            lx.add_(gx)
        if tg is not None:
            return lx, lv, allreduce_table_grads(self.pot._table_grads_from_device(tg), group)
        return lx, lv


class _LeapfrogFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x0, v0, integrator, n_steps, checkpoint_every, reconstruct, tracked,
                *nodes):
        x, v, ckpts = integrator.run(x0, v0, n_steps, checkpoint_every)
        ctx.integrator, ctx.n_steps, ctx.ckpts = integrator, n_steps, ckpts
        ctx.reconstruct, ctx.tracked = reconstruct, tracked
        return x, v

    @staticmethod
    def backward(ctx, gx, gv):
        if gx is None:
            gx = torch.zeros_like(ctx.ckpts[0][1])
        if gv is None:
            gv = torch.zeros_like(ctx.ckpts[0][1])
        integ = ctx.integrator
        node_grads = [None] * sum(len(p) for _, p in ctx.tracked)
        if any(ctx.needs_input_grad[7:]):
            lx, lv, tg = integ.adjoint(ctx.ckpts, ctx.n_steps, gx, gv, table_grads=True,
                                       reconstruct=ctx.reconstruct)
            node_grads = integ.pot._node_param_grads(tg, ctx.tracked)
        else:
            lx, lv = integ.adjoint(ctx.ckpts, ctx.n_steps, gx, gv, reconstruct=ctx.reconstruct)
        ctx.ckpts = None
        return (lx, lv, None, None, None, None, None, *node_grads)


def leapfrog(pot, x0: torch.Tensor, v0: torch.Tensor, dt: float, n_steps: int, t0: float = 0.0,
             checkpoint_every: Optional[int] = 64, precision: Optional[str] = None,
             use_graph: Optional[bool] = None, scheme="leapfrog", reconstruct: str = "recompute"):
    """(x_T, v_T) after n_steps steps of ``scheme`` (leapfrog, or a composition of
    leapfrog substeps such as "yoshida4"); differentiable w.r.t. (x0, v0) and w.r.t.
    the node tensors of the potential (pot.node_parameters()) through the
    checkpointed adjoint: loss.backward() fills their .grad (under torch.distributed,
    summed over the ranks)."""
    integ = Leapfrog(pot, dt, t0=t0, precision=precision, use_graph=use_graph, scheme=scheme)
    k = None if checkpoint_every is None else int(checkpoint_every)
    tracked = pot._tracked_nodes() if hasattr(pot, "_tracked_nodes") else []
    nodes = [q for _, ps in tracked for q in ps]
    return _LeapfrogFn.apply(x0, v0, integ, int(n_steps), k, reconstruct, tracked, *nodes)
