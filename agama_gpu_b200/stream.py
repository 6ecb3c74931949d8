"""Particle-spray tidal streams on the GPU evaluator, with their adjoint.

A progenitor (a cluster or dwarf of mass m) is integrated BACKWARDS from its
present phase-space point (x_p, v_p) at t_end for n_steps steps of dt; along
that orbit, every ``release_every`` steps, a pair of particles is released near
its two Lagrange points, and all released particles are integrated FORWARD to
t_end in the host potential -- plus, optionally, the progenitor's own potential
carried along its orbit (a ShiftedPotentialGPU on the recorded track).

Release model -- a parameterised spray after Fardal, Huang & Weinberg (2015,
MNRAS 452, 301).  In the progenitor's orbital frame

    r^ = x/|x|,  L^ = (x cross v)/|x cross v|,  phi^ = L^ cross r^,
    Omega = |x cross v| / |x|^2,
    r_J = (G m / (Omega^2 - d2Phi/dr2))^(1/3)       (d2Phi/dr2 = -r^T (dF/dx) r^)

the leading (s = -1, inner) and trailing (s = +1, outer) particle of a release
start at

    x = x_p + r_J (s k_r r^ + k_z L^)
    v = v_p + Omega r_J (s k_vt phi^ + k_vz L^)

with k_r, k_z, k_vt, k_vz drawn from Gaussians whose means and dispersions are
arguments (defaults 2 +- 0.5, 0 +- 0.5, 0.3 +- 0.5, 0 +- 0.5, the fitted values of
that paper) from a seeded CPU generator, so a stream does not depend on the
device.  If d2Phi/dr2 >= Omega^2 (no tidal radius) r_J is set to 0 and both
particles start at the progenitor.

The forward integration keeps the particles in release order, so the particles
in flight at step n are a PREFIX of the arrays: each step evaluates the force on
that prefix only (one fused launch, no masking, no idle lanes).

The adjoint (``Stream.adjoint``) runs the same substeps backwards over the
stored positions and returns dL/d(release position, release velocity) per
particle and, if asked, the table gradients of every Multipole / CylSpline of
the potential the particles move in (summed over all force evaluations).  The
release states are its leaves: their own dependence on the potential (through
the progenitor orbit and r_J) is not differentiated here.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Optional, Sequence, Tuple

import numpy as np
import torch

from .integrate import Leapfrog, allreduce_table_grads, is_static
from .potentials import G_AGAMA

FARDAL15 = {"k_r": (2.0, 0.5), "k_z": (0.0, 0.5), "k_vt": (0.3, 0.5), "k_vz": (0.0, 0.5)}


def release_states(x_p: torch.Tensor, v_p: torch.Tensor, deriv: torch.Tensor, mass,
                   k: torch.Tensor) -> Tuple[torch.Tensor, torch.Tensor, torch.Tensor]:
    """Release positions and velocities (2R, 3), ordered [leading, trailing] per release.

    x_p, v_p: (R, 3) progenitor states; deriv: (R, 6) force derivatives at x_p in the
    order [dFx/dx, dFy/dy, dFz/dz, dFx/dy, dFy/dz, dFz/dx]; mass: scalar or (R,);
    k: (R, 2, 4) draws of (k_r, k_z, k_vt, k_vz).  Also returns r_J (R,).
    """
    x_p = x_p.to(torch.float64)
    v_p = v_p.to(torch.float64)
    r = torch.linalg.norm(x_p, dim=1, keepdim=True)
    rh = x_p / r
    L = torch.cross(x_p, v_p, dim=1)
    Ln = torch.linalg.norm(L, dim=1, keepdim=True)
    Lh = L / Ln
    ph = torch.cross(Lh, rh, dim=1)
    om = (Ln / (r * r)).squeeze(1)
    d = deriv.to(torch.float64)
    x_, y_, z_ = rh[:, 0], rh[:, 1], rh[:, 2]
    rDr = (d[:, 0] * x_ * x_ + d[:, 1] * y_ * y_ + d[:, 2] * z_ * z_
           + 2.0 * (d[:, 3] * x_ * y_ + d[:, 4] * y_ * z_ + d[:, 5] * z_ * x_))
    denom = om * om + rDr                     # Omega^2 - d2Phi/dr2
    m = torch.as_tensor(mass, dtype=torch.float64, device=x_p.device)
    gm = (G_AGAMA * m).expand_as(denom)
    ratio = torch.where(denom > 0, gm / torch.where(denom > 0, denom, torch.ones_like(denom)),
                        torch.zeros_like(denom))
    rj = ratio.pow(1.0 / 3.0)
    s = torch.tensor([-1.0, 1.0], dtype=torch.float64, device=x_p.device)[None, :, None]
    k = k.to(device=x_p.device, dtype=torch.float64)
    kr, kz, kvt, kvz = (k[:, :, i:i + 1] for i in range(4))
    rj3 = rj[:, None, None]
    dx = rj3 * (s * kr * rh[:, None, :] + kz * Lh[:, None, :])
    dv = (om[:, None, None] * rj3) * (s * kvt * ph[:, None, :] + kvz * Lh[:, None, :])
    xr = (x_p[:, None, :] + dx).reshape(-1, 3)
    vr = (v_p[:, None, :] + dv).reshape(-1, 3)
    return xr, vr, rj


def draw_k(n_release: int, seed: int, params: Optional[dict] = None) -> torch.Tensor:
    """(R, 2, 4) Gaussian draws of (k_r, k_z, k_vt, k_vz) from a seeded CPU generator."""
    p = dict(FARDAL15)
    if params:
        p.update(params)
    g = torch.Generator().manual_seed(int(seed))
    z = torch.randn((n_release, 2, 4), generator=g, dtype=torch.float64)
    mean = torch.tensor([p["k_r"][0], p["k_z"][0], p["k_vt"][0], p["k_vz"][0]], dtype=torch.float64)
    disp = torch.tensor([p["k_r"][1], p["k_z"][1], p["k_vt"][1], p["k_vz"][1]], dtype=torch.float64)
    return mean + disp * z


@dataclass
class Stream:
    """A generated stream at t_end.  x, v: (N, 3) particles in release order
    ([leading, trailing] per release); t_release (N,); x_release, v_release their
    initial states; track (n_steps + 1, 7) rows [t, x, y, z, vx, vy, vz] of the
    progenitor orbit in forward time."""
    x: torch.Tensor
    v: torch.Tensor
    t_release: torch.Tensor
    x_release: torch.Tensor
    v_release: torch.Tensor
    track: np.ndarray
    r_jacobi: torch.Tensor
    _integ: Leapfrog = field(repr=False, default=None)
    _counts: list = field(repr=False, default=None)        # active particles per substep
    _store: Optional[torch.Tensor] = field(repr=False, default=None)
    _offsets: list = field(repr=False, default=None)

    def adjoint(self, lam_x: torch.Tensor, lam_v: torch.Tensor, table_grads: bool = False,
                group=None):
        """(dL/dx_release, dL/dv_release[, {component: table gradient}]) from
        (dL/dx, dL/dv) at t_end.

        Per substep g backwards over the a_g particles in flight (dt_g, h_g its drift
        and half-kick): gF = h_g lv + pending; lx += (dF/dx)^T gF at the end of the
        substep; lv += dt_g lx; pending = h_g lv.  Particles released at the start
        of substep g take their last VJP at their release position and are final."""
        if self._store is None:
            raise RuntimeError("this stream was generated with store=False; no adjoint")
        integ, counts, store, off = self._integ, self._counts, self._store, self._offsets
        S = integ.S
        G = len(counts)
        tg = {} if table_grads else None
        n_all = self.x.shape[0]
        lx = lam_x.detach().to(torch.float64).reshape(n_all, 3).contiguous().clone()
        lv = lam_v.detach().to(torch.float64).reshape(n_all, 3).contiguous().clone()
        pend = torch.zeros_like(lx)
        gx = torch.empty_like(lx)

        def pos(g, a):
            """Positions of the first a particles at the start of substep g (g = G: end)."""
            if g == G:
                return self.x[:a]
            return store[off[g]:off[g] + a]

        def vjp(xg, t, gF, out):
            if tg is None:
                integ.pot._vjp(xg, t, None, gF, precision=integ.precision, out=out)
            else:
                integ.pot._adjoint_vjp(xg, t, None, gF, tg, precision=integ.precision, out=out)

        for g in range(G - 1, -1, -1):
            a = counts[g]
            if a == 0:
                continue
            dtg, hg, _ = integ._sub[g % S]
            gF = lv[:a] * hg
            gF.add_(pend[:a])
            vjp(pos(g + 1, a), integ._t(g + 1), gF, gx[:a])
            lx[:a].add_(gx[:a])
            lv[:a].add_(lx[:a], alpha=dtg)
            torch.mul(lv[:a], hg, out=pend[:a])
            a_prev = counts[g - 1] if g > 0 else 0
            if a_prev < a:
                # released at the start of substep g: F there was evaluated at release
                vjp(pos(g, a)[a_prev:], integ._t(g), pend[a_prev:a].clone(), gx[a_prev:a])
                lx[a_prev:a].add_(gx[a_prev:a])
                pend[a_prev:a].zero_()
        if tg is not None:
            return lx, lv, allreduce_table_grads(integ.pot._table_grads_from_device(tg), group)
        return lx, lv


def _force_derivs(pot, xs: torch.Tensor, ts: Sequence[float]) -> torch.Tensor:
    """(R, 6) force derivatives at progenitor positions xs at times ts."""
    if is_static(pot):
        _, d = pot.forceDeriv(xs, float(ts[0]))
        return d.reshape(-1, 6)
    out = torch.empty((xs.shape[0], 6), dtype=torch.float64, device=xs.device)
    for i, t in enumerate(ts):
        _, d = pot.forceDeriv(xs[i:i + 1], float(t))
        out[i] = d.reshape(6)
    return out


def particle_spray(pot, x_p, v_p, mass: float, t_end: float, n_steps: int, dt: float,
                   release_every: int = 1, seed: int = 0, spray: Optional[dict] = None,
                   prog_pot=None, scheme="leapfrog", precision: Optional[str] = None,
                   store: bool = True, device=None) -> Stream:
    """Generate a particle-spray stream of a progenitor now at (x_p, v_p) (kpc, km/s)
    of ``mass`` Msol, released over the last n_steps * dt time units before t_end.

    pot: host potential (GPU class); prog_pot: the progenitor's own potential
    (e.g. a PlummerPotentialGPU) centred on its orbit while the particles move, or
    None; spray: overrides of FARDAL15's (mean, dispersion) pairs; scheme: the
    integrator ("leapfrog" or "yoshida4"); store=False skips the stored trajectory
    (no adjoint)."""
    from .potentials import ShiftedPotentialGPU
    if n_steps < 1 or release_every < 1:
        raise ValueError("n_steps and release_every must be >= 1")
    dev = torch.device(device) if device is not None else (
        torch.device("cuda") if torch.cuda.is_available() else torch.device("cpu"))
    xp = torch.as_tensor(np.asarray(x_p, dtype=np.float64).reshape(1, 3), device=dev).clone()
    vp = torch.as_tensor(np.asarray(v_p, dtype=np.float64).reshape(1, 3), device=dev).clone()
    n_steps, dt = int(n_steps), float(dt)
    t_start = float(t_end) - n_steps * dt

    # 1. progenitor orbit backwards from t_end, recorded at every step boundary
    back = Leapfrog(pot, -dt, t0=float(t_end), precision=precision, use_graph=False, scheme=scheme,
                    device_time=False)
    xb, vb, Fb = back._buffers(xp)
    xb.copy_(xp)
    vb.copy_(vp)
    back._force_into(xb, back.t0, Fb)
    rec = torch.empty((n_steps + 1, 2, 3), dtype=torch.float64, device=dev)
    rec[n_steps, 0].copy_(xb[0])
    rec[n_steps, 1].copy_(vb[0])
    for n in range(n_steps):
        back._step(xb, vb, Fb, n)
        rec[n_steps - 1 - n, 0].copy_(xb[0])
        rec[n_steps - 1 - n, 1].copy_(vb[0])
    times = t_start + dt * np.arange(n_steps + 1, dtype=np.float64)
    times[-1] = float(t_end)
    rec_h = rec.cpu().numpy()
    track = np.concatenate([times[:, None], rec_h[:, 0], rec_h[:, 1]], axis=1)

    # 2. releases at steps 0, r, 2r, ... < n_steps
    rel_steps = np.arange(0, n_steps, int(release_every))
    R = len(rel_steps)
    idx = torch.as_tensor(rel_steps, device=dev)
    xs, vs = rec[idx, 0].contiguous(), rec[idx, 1].contiguous()
    t_rel = times[rel_steps]
    deriv = _force_derivs(pot, xs, t_rel)
    x_rel, v_rel, rj = release_states(xs, vs, deriv, mass, draw_k(R, seed, spray))
    N = 2 * R

    # 3. all particles forward to t_end in the host (+ progenitor) potential
    spot = pot if prog_pot is None else pot + ShiftedPotentialGPU(prog_pot, track)
    st = integrate_releases(spot, x_rel, v_rel, rel_steps, t_start, n_steps, dt, scheme=scheme,
                            precision=precision, store=store)
    st.track, st.r_jacobi = track, rj
    return st


def integrate_releases(pot, x_release: torch.Tensor, v_release: torch.Tensor, release_steps,
                       t_start: float, n_steps: int, dt: float, scheme="leapfrog",
                       precision: Optional[str] = None, store: bool = True) -> Stream:
    """Integrate particles released in pairs at steps ``release_steps`` (ascending;
    pair i = rows 2i, 2i+1 of x_release / v_release) from t_start + step * dt to
    t_start + n_steps * dt.  The particles in flight at each step are a prefix of the
    arrays; each substep is one force launch on that prefix.  store=True keeps the
    positions of every substep for ``Stream.adjoint``."""
    rel_steps = np.asarray(release_steps, dtype=np.int64)
    if rel_steps.ndim != 1 or len(rel_steps) == 0 or np.any(np.diff(rel_steps) < 0) \
            or rel_steps[0] < 0 or rel_steps[-1] >= n_steps:
        raise ValueError("release_steps must be ascending steps in [0, n_steps)")
    N = 2 * len(rel_steps)
    if tuple(x_release.shape) != (N, 3) or tuple(v_release.shape) != (N, 3):
        raise ValueError(f"x_release and v_release must be ({N}, 3)")
    dev = x_release.device
    integ = Leapfrog(pot, dt, t0=float(t_start), precision=precision, use_graph=False,
                     scheme=scheme, device_time=False)
    S = integ.S
    x = torch.empty((N, 3), dtype=torch.float64, device=dev)
    v = torch.empty_like(x)
    F = torch.empty_like(x)
    counts = []
    for n in range(int(n_steps)):
        a = 2 * int(np.searchsorted(rel_steps, n, side="right"))
        counts.extend([a] * S)
    offsets = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    st = torch.empty((int(offsets[-1]), 3), dtype=torch.float64, device=dev) if store else None
    x_rel = x_release.detach().to(torch.float64)
    v_rel = v_release.detach().to(torch.float64)
    a = 0
    for n in range(int(n_steps)):
        a_new = counts[n * S]
        if a_new > a:
            x[a:a_new].copy_(x_rel[a:a_new])
            v[a:a_new].copy_(v_rel[a:a_new])
            integ._force_into(x[a:a_new], integ._t(n * S), F[a:a_new])
            a = a_new
        for j in range(S):
            g = n * S + j
            if st is not None:
                st[offsets[g]:offsets[g] + a].copy_(x[:a])
            integ._substep(x[:a], v[:a], F[:a], g)
    t_release = torch.as_tensor(np.repeat(float(t_start) + dt * rel_steps, 2), device=dev)
    return Stream(x=x, v=v, t_release=t_release, x_release=x_rel, v_release=v_rel, track=None,
                  r_jacobi=None, _integ=integ, _counts=counts, _store=st,
                  _offsets=[int(o) for o in offsets[:-1]])


class _ReleasesFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x_release, v_release, pot, release_steps, t_start, n_steps, dt, scheme,
                precision, tracked, *nodes):
        st = integrate_releases(pot, x_release, v_release, release_steps, t_start, n_steps, dt,
                                scheme=scheme, precision=precision, store=True)
        ctx.stream, ctx.tracked, ctx.pot = st, tracked, pot
        return st.x.clone(), st.v.clone()

    @staticmethod
    def backward(ctx, gx, gv):
        st = ctx.stream
        gx = torch.zeros_like(st.x) if gx is None else gx
        gv = torch.zeros_like(st.v) if gv is None else gv
        node_grads = [None] * sum(len(p) for _, p in ctx.tracked)
        if any(ctx.needs_input_grad[10:]):
            lx, lv, tg = st.adjoint(gx, gv, table_grads=True)
            node_grads = ctx.pot._node_param_grads(tg, ctx.tracked)
        else:
            lx, lv = st.adjoint(gx, gv)
        ctx.stream = None
        return (lx, lv, None, None, None, None, None, None, None, None, *node_grads)


def integrate_releases_autograd(pot, x_release: torch.Tensor, v_release: torch.Tensor,
                                release_steps, t_start: float, n_steps: int, dt: float,
                                scheme="leapfrog", precision: Optional[str] = None):
    """(x, v) at t_start + n_steps dt of the particles released as in
    ``integrate_releases``, differentiable w.r.t. x_release, v_release and the node
    tensors of the potential (pot.node_parameters()) through ``Stream.adjoint``."""
    tracked = pot._tracked_nodes() if hasattr(pot, "_tracked_nodes") else []
    nodes = [q for _, ps in tracked for q in ps]
    return _ReleasesFn.apply(x_release, v_release, pot, release_steps, float(t_start),
                             int(n_steps), float(dt), scheme, precision, tracked, *nodes)
