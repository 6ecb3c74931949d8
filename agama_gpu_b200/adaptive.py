"""Adaptive-step orbit integration: the embedded Dormand-Prince 5(4) pair.

Each particle carries its own time t_i and step h_i when the potential does not
depend on time: every iteration attempts one step for all particles still short
of t_end (gathered into contiguous buffers, so each of the six stage forces is
ONE fused launch over exactly those particles), accepts or rejects it per
particle by its own error estimate, and scatters the result back.  For a
time-dependent potential the force launch takes a single t, so all particles
share one step and one time; the step is accepted when every particle's error
is within tolerance.

Tableau: Dormand & Prince (1980), J. Comput. Appl. Math. 6, 19 (the 7-stage
first-same-as-last 5(4) pair; the 5th-order solution propagates).  Error
norm: max over the six phase-space components of |e| / (atol + rtol max(|y|,
|y_new|)) with positions and velocities measured in their own units (kpc,
km/s).  Step update: h <- h min(5, max(0.2, 0.9 err^(-1/5))) after an accepted
step; after a rejected one h <- h max(0.1, min(0.2, 0.9 err^(-1/5))).
"""
from __future__ import annotations

from typing import Optional, Tuple

import torch

from . import _lib
from .integrate import is_static

_C = (0.0, 1 / 5, 3 / 10, 4 / 5, 8 / 9, 1.0, 1.0)
_A = (
    (),
    (1 / 5,),
    (3 / 40, 9 / 40),
    (44 / 45, -56 / 15, 32 / 9),
    (19372 / 6561, -25360 / 2187, 64448 / 6561, -212 / 729),
    (9017 / 3168, -355 / 33, 46732 / 5247, 49 / 176, -5103 / 18656),
    (35 / 384, 0.0, 500 / 1113, 125 / 192, -2187 / 6784, 11 / 84),
)
# 5th-order minus embedded 4th-order weights
_E = (71 / 57600, 0.0, -71 / 16695, 71 / 1920, -17253 / 339200, 22 / 525, -1 / 40)


class DormandPrince:
    """Adaptive integration of N particles in ``pot`` from t0 to t1 (t1 < t0 runs
    backwards).  ``run`` returns (x, v) at t1 and per-particle statistics."""

    def __init__(self, pot, rtol: float = 1e-9, atol: float = 1e-12,
                 precision: Optional[str] = None, h0: Optional[float] = None,
                 max_iters: int = 1_000_000, per_particle: Optional[bool] = None):
        """per_particle: own time and step per particle (default: when the potential
        does not depend on time; True for a time-dependent one is an error)."""
        if rtol <= 0 or atol < 0:
            raise ValueError("rtol must be > 0 and atol >= 0")
        self.pot = pot
        self.rtol, self.atol = float(rtol), float(atol)
        self.precision = precision
        static = is_static(pot)
        if per_particle and not static and not getattr(pot, "_time_independent", False):
            raise ValueError("per-particle steps need a potential that does not depend on time")
        self.static = static if per_particle is None else bool(per_particle)
        self.h0 = h0
        self.max_iters = int(max_iters)

    def _force(self, x: torch.Tensor, t: float) -> torch.Tensor:
        F = torch.empty_like(x)
        self.pot._launch(x, float(t), _lib.MODE_GRAD, False, precision=self.precision,
                         out=(None, F, None, None))
        return F

    def _attempt(self, x, v, F0, h, t: float, h_scalar: float):
        """One DP5(4) step of sizes h (n, 1) from (x, v) with F0 = F(x) at time t:
        (x5, v5, F(x5), err).  The 7th stage sits at the 5th-order solution (FSAL)."""
        kx, kv = [v], [F0]
        for s in range(1, 7):
            xs, vs = x.clone(), v.clone()
            for j, aj in enumerate(_A[s]):
                if aj != 0.0:
                    xs.addcmul_(h, kx[j], value=aj)
                    vs.addcmul_(h, kv[j], value=aj)
            kx.append(vs)
            kv.append(self._force(xs, 0.0 if self.static else t + _C[s] * h_scalar))
        x5, v5 = xs, vs
        ex = torch.zeros_like(x)
        ev = torch.zeros_like(v)
        for j, e in enumerate(_E):
            if e != 0.0:
                ex.add_(kx[j], alpha=e)
                ev.add_(kv[j], alpha=e)
        ex.mul_(h)
        ev.mul_(h)
        sx = self.atol + self.rtol * torch.maximum(x.abs(), x5.abs())
        sv = self.atol + self.rtol * torch.maximum(v.abs(), v5.abs())
        err = torch.maximum((ex / sx).abs().amax(1), (ev / sv).abs().amax(1))
        return x5, v5, kv[6], err

    def run(self, x0: torch.Tensor, v0: torch.Tensor, t0: float, t1: float
            ) -> Tuple[torch.Tensor, torch.Tensor, dict]:
        x = x0.detach().to(torch.float64).clone().contiguous()
        v = v0.detach().to(torch.float64).clone().contiguous()
        n = x.shape[0]
        dev = x.device
        span = float(t1) - float(t0)
        if span == 0.0 or n == 0:
            return x, v, {"accepted": torch.zeros(n, dtype=torch.int64, device=dev),
                          "rejected": torch.zeros(n, dtype=torch.int64, device=dev),
                          "iterations": 0}
        sign = 1.0 if span > 0 else -1.0
        h_init = abs(self.h0) if self.h0 else abs(span) / 100.0
        F = self._force(x, float(t0))
        acc = torch.zeros(n, dtype=torch.int64, device=dev)
        rej = torch.zeros(n, dtype=torch.int64, device=dev)
        if self.static:
            t = torch.zeros(n, dtype=torch.float64, device=dev)           # elapsed |t - t0|
            h = torch.full((n,), h_init, dtype=torch.float64, device=dev)
            total = abs(span)
            it = 0
            while True:
                idx = torch.nonzero(t < total, as_tuple=False).reshape(-1)
                if idx.numel() == 0:
                    break
                it += 1
                if it > self.max_iters:
                    raise RuntimeError("DormandPrince: step limit reached")
                hh = torch.minimum(h[idx], total - t[idx])
                hs = (sign * hh)[:, None]
                xa, va, Fa = x[idx], v[idx], F[idx]
                x5, v5, F5, err = self._attempt(xa, va, Fa, hs, 0.0, 0.0)
                ok = err <= 1.0
                fac = torch.clamp(0.9 * err.clamp(min=1e-30).pow(-0.2), 0.1, 5.0)
                fac = torch.where(ok, fac.clamp(min=0.2), fac.clamp(max=0.2))
                keep = ok[:, None]
                x[idx] = torch.where(keep, x5, xa)
                v[idx] = torch.where(keep, v5, va)
                F[idx] = torch.where(keep, F5, Fa)
                # land exactly on t1 when the step was clipped to the remaining time
                t[idx] = torch.where(ok, torch.where(hh >= total - t[idx], torch.full_like(hh, total),
                                                     t[idx] + hh), t[idx])
                h[idx] = hh * fac
                acc[idx] += ok.to(torch.int64)
                rej[idx] += (~ok).to(torch.int64)
            return x, v, {"accepted": acc, "rejected": rej, "iterations": it}
        # time-dependent potential: one shared step
        t = float(t0)
        h = h_init
        it = 0
        while sign * (float(t1) - t) > 0:
            it += 1
            if it > self.max_iters:
                raise RuntimeError("DormandPrince: step limit reached")
            hh = min(h, abs(float(t1) - t))
            hs = torch.full((n, 1), sign * hh, dtype=torch.float64, device=dev)
            x5, v5, F5, err = self._attempt(x, v, F, hs, t, sign * hh)
            e = float(err.max())
            if e <= 1.0:
                x, v, F = x5, v5, F5
                t = float(t1) if hh >= abs(float(t1) - t) else t + sign * hh
                acc += 1
                h = hh * min(5.0, max(0.2, 0.9 * max(e, 1e-30) ** -0.2))
            else:
                rej += 1
                h = hh * max(0.1, min(0.2, 0.9 * e ** -0.2))
        return x, v, {"accepted": acc, "rejected": rej, "iterations": it}


def integrate_adaptive(pot, x0, v0, t0: float, t1: float, rtol: float = 1e-9,
                       atol: float = 1e-12, precision: Optional[str] = None):
    """(x, v) at t1 from (x0, v0) at t0 with the adaptive Dormand-Prince 5(4) pair."""
    x, v, _ = DormandPrince(pot, rtol=rtol, atol=atol, precision=precision).run(x0, v0, t0, t1)
    return x, v
