"""GPU potential classes with the reference's Python API (gpu_potential.py).

Every class exposes potential / force / density / forceDeriv / evalDeriv /
eval with (N,3) or (3,) inputs and Agama units, the same as the reference's
classes (gpu_potential.py:633-935, 1260-1918; _analytic_potentials.py:77-1165).

Evaluation model: a potential is a tree (Composite, Evolving, Shifted, Scaled
over Multipole, CylSpline and analytic leaves).  At call time the tree is
flattened into "leaves" -- (component, sigma, gamma, ampl) with
Phi(x) = sum ampl * Phi_component(sigma * x - gamma) -- and the whole sum is
evaluated by ONE fused CUDA kernel (libagb.so, agb_eval).  The reference
instead launches one kernel per component and glues the results with CuPy
elementwise passes (shift, scale, negate, lerp, add).

Inputs may be torch tensors (CUDA or CPU), NumPy arrays or any DLPack /
CUDA-array-interface object; host inputs are copied to the GPU first, as the
reference's ``cp.asarray`` does.  Outputs are torch CUDA float64 tensors.
"""
from __future__ import annotations

import ctypes
import itertools
import math
import os
import tempfile
import uuid
from pathlib import Path
from typing import List, Optional, Sequence, Tuple, Union

import numpy as np
import torch
from scipy.interpolate import CubicHermiteSpline, CubicSpline

from . import _lib
from .coefs import read_coefs
from .prep_cylspline import build_cylspline_tables
from .prep_multipole import build_multipole_tables

G_AGAMA = 4.30091727067736e-06                    # kpc (km/s)^2 / Msol
INV_4PIG = 1.0 / (4.0 * math.pi * G_AGAMA)

_PRECISIONS = {"fp64": _lib.PREC_FP64, "mixed": _lib.PREC_MIXED}
_MULTIPOLE_SERIAL = itertools.count()
_default_precision = os.environ.get("AGB_PRECISION", "fp64")


def set_default_precision(precision: str) -> None:
    """'fp64' (default) or 'mixed' for every potential without its own setting."""
    global _default_precision
    if precision not in _PRECISIONS:
        raise ValueError(f"precision must be one of {sorted(_PRECISIONS)}, got {precision!r}")
    _default_precision = precision


# ---------------------------------------------------------------------------
# inputs / outputs
# ---------------------------------------------------------------------------

def _cuda_device(dev: Optional[torch.device] = None) -> torch.device:
    if not torch.cuda.is_available():
        raise RuntimeError("agama_gpu_b200 needs a CUDA device (there is no CPU fallback)")
    if dev is not None and dev.type == "cuda":
        return dev
    return torch.device("cuda", torch.cuda.current_device())


def _as_tensor(xyz) -> torch.Tensor:
    if isinstance(xyz, torch.Tensor):
        return xyz
    if isinstance(xyz, np.ndarray):
        return torch.from_numpy(np.ascontiguousarray(xyz, dtype=np.float64))
    if hasattr(xyz, "__dlpack__"):
        try:
            return torch.from_dlpack(xyz)
        except Exception:   # pragma: no cover - exotic producers
            pass
    if hasattr(xyz, "__cuda_array_interface__"):
        return torch.as_tensor(xyz, device="cuda")
    return torch.from_numpy(np.ascontiguousarray(np.asarray(xyz, dtype=np.float64)))


def prep_xyz(xyz) -> Tuple[torch.Tensor, bool]:
    """(N,3) float64 contiguous CUDA tensor and whether the input was a single point.

    Shape rules and messages follow gpu_potential.py:167-177.
    """
    t = _as_tensor(xyz)
    dev = _cuda_device(t.device)
    t = t.to(device=dev, dtype=torch.float64)
    if t.dim() == 1:
        if t.shape[0] != 3:
            raise ValueError(f"Single-point xyz must have shape (3,), got {tuple(t.shape)}")
        return t.reshape(1, 3).contiguous(), True
    if t.dim() != 2 or t.shape[1] != 3:
        raise ValueError(f"xyz must have shape (N,3), got {tuple(t.shape)}")
    return t.contiguous(), False


def _sq(a: torch.Tensor, single: bool):
    return a[0] if single else a


# ---------------------------------------------------------------------------
# base class
# ---------------------------------------------------------------------------

Leaf = Tuple["_Component", float, np.ndarray, float]


class _TimePlan:
    """A device time plan (agb_time_plan) with the components its programs index."""

    def __init__(self, handle, comps, progs, table):
        self.handle, self.comps, self.progs, self.table = handle, comps, progs, table
        self._arrays = {}

    def component_array(self, dev):
        key = (dev, consts_epoch(self.comps))
        a = self._arrays.get(key)
        if a is None:
            a = (_lib.AgbComponent * len(self.comps))(*[c._device_component(dev) for c in self.comps])
            self._arrays = {key: a}
        return a

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                _lib.lib.agb_time_plan_destroy(h)
            except Exception:       # interpreter shutdown
                pass
            self.handle = None


def consts_epoch(comps) -> int:
    """Changes whenever set_node_tables() changed the builder scalars of one of the
    components (their descriptors, which launches pass by value, changed with them)."""
    return sum(c.__dict__.get("_consts_gen", 0) for c in comps)


def _const_buffer(acc: dict, comp, dev) -> torch.Tensor:
    """The (8,) accumulator of dL/d(builder scalars) of Multipole comp in acc."""
    key = ("const", comp)
    buf = acc.get(key)
    if buf is None:
        buf = torch.zeros(_lib.MP_NCONST, dtype=torch.float64, device=dev)
        acc[key] = buf
    return buf


class _GPUPotBase:
    """``+`` composition, the evaluation API and the flattening into leaves.

    ``pot_a + pot_b`` -> CompositePotentialGPU (flattening nested composites),
    ``sum([...])`` works through ``__radd__(0)`` (gpu_potential.py:85-101).
    """

    precision: Optional[str] = None
    binning: bool = True          # sort points by radial interval before evaluating

    def __add__(self, other):
        a = self._components if isinstance(self, CompositePotentialGPU) else [self]
        b = other._components if isinstance(other, CompositePotentialGPU) else [other]
        return CompositePotentialGPU(a + b)

    def __radd__(self, other):
        if other == 0:
            return self
        return NotImplemented

    # subclasses implement: leaves at time t
    def _leaves(self, t: float) -> List[Leaf]:
        raise NotImplementedError

    def set_binning(self, on: bool):
        """Sort points by radial interval before evaluating (default) or keep input order."""
        self.binning = bool(on)
        return self

    def set_precision(self, precision: Optional[str]):
        """Per-object arithmetic of the Multipole sums: 'fp64', 'mixed' or None (default)."""
        if precision is not None and precision not in _PRECISIONS:
            raise ValueError(f"precision must be one of {sorted(_PRECISIONS)}")
        self.precision = precision
        return self

    # -- evaluation core ----------------------------------------------------
    def _all_components(self):
        """Every leaf component the tree can use at any time (all Evolving snapshots)."""
        if isinstance(self, _Component):
            return [self]
        out = []
        for sub in (getattr(self, "_components", None) or getattr(self, "_pots", None)
                    or [getattr(self, "_inner")]):
            out.extend(sub._all_components())
        return out

    def _preload(self, dev: torch.device) -> None:
        """Upload every component's tables to dev once, so that a later time step that
        brings a new Evolving snapshot into use does not upload inside the step."""
        done = self.__dict__.setdefault("_preloaded", set())
        if dev in done:
            return
        for c in self._all_components():
            c._device_component(dev)
        done.add(dev)

    # -- time-dependent leaves on the device --------------------------------------
    def _time_slots(self):
        """The tree as leaf slots for device-evaluated time dependence: a list of
        (owner, [components], [(modifier, op kind)] innermost first, slot), where a
        fixed leaf has one component and an Evolving slot all its snapshots (owner is
        the Evolving).  None when the tree has a structure the device programs do not
        cover (an Evolving whose snapshots are not single components)."""
        if isinstance(self, _Component):
            return [(None, [self], [], 0)]
        if isinstance(self, CompositePotentialGPU):
            out = []
            for c in self._components:
                sub = c._time_slots()
                if sub is None:
                    return None
                out.extend(sub)
            return out
        if isinstance(self, EvolvingPotentialGPU):
            if not all(isinstance(q, _Component) for q in self._pots):
                return None
            op = [(self, _lib.OP_EVOLVE)]
            if self._interpolate and len(self._pots) > 1:
                return [(self, list(self._pots), op, 0), (self, list(self._pots), op, 1)]
            return [(self, list(self._pots), op, 0)]
        kind = _lib.OP_SHIFT if isinstance(self, ShiftedPotentialGPU) else _lib.OP_SCALE
        sub = self._inner._time_slots()
        if sub is None:
            return None
        return [(o, comps, ops + [(self, kind)], sl) for o, comps, ops, sl in sub]

    def _time_data(self) -> np.ndarray:
        raise NotImplementedError

    def _time_programs(self):
        """(component list, program array, table) of the device time plan, or None."""
        slots = self._time_slots()
        if slots is None or not 0 < len(slots) <= _lib.MAX_LEAVES:
            return None
        comps, where = [], {}
        data, at = [], {}
        n_data = 0
        progs = (_lib.AgbLeafProg * len(slots))()
        for i, (owner, members, ops, sl) in enumerate(slots):
            key = id(owner) if owner is not None else id(members[0])
            if key not in where:
                where[key] = len(comps)
                comps.extend(members)
            pg = progs[i]
            pg.comp = where[key]
            pg.n_ops = len(ops)
            pg.slot = sl
            if len(ops) > _lib.MAX_LEAF_OPS:
                return None
            for k, (mod, kind) in enumerate(ops):
                if id(mod) not in at:
                    d = np.ascontiguousarray(mod._time_data(), dtype=np.float64)
                    at[id(mod)] = n_data
                    data.append(d)
                    n_data += d.size
                pg.op[k] = kind
                pg.arg[k] = at[id(mod)]
        if len(comps) > _lib.MAX_COMPONENTS:
            return None
        table = np.concatenate(data) if data else np.zeros(1)
        return comps, progs, table

    def _time_plan(self, dev: torch.device):
        """The device time plan of this tree on dev (cached), or None."""
        cache = self.__dict__.setdefault("_tplans", {})
        if dev in cache:
            return cache[dev]
        built = self._time_programs()
        plan = None
        if built is not None:
            comps, progs, table = built
            with torch.cuda.device(dev):
                h = ctypes.c_void_p()
                rc = _lib.lib.agb_time_plan_create(progs, len(progs), table.ctypes.data,
                                                   table.size, ctypes.byref(h))
                _lib.check(rc, "agb_time_plan_create")
            plan = _TimePlan(h, comps, progs, table)
        cache[dev] = plan
        return plan

    def _launch_timed(self, arr: torch.Tensor, step: Optional[torch.Tensor], t0: float, dt: float,
                      off: float, mode: int, want_phi: bool, precision: Optional[str] = None,
                      out=None):
        """_launch at t = (t0 + step * dt) + off with step a device int64 scalar (None:
        0), the leaves computed on the device (graph-capturable)."""
        n = arr.shape[0]
        dev = arr.device
        plan = self._time_plan(dev)
        if plan is None:
            raise ValueError("this potential tree has no device time plan")
        prec = _PRECISIONS[precision or self.precision or _default_precision]
        self._preload(dev)
        if not torch.cuda.is_current_stream_capturing():
            for c in plan.comps:
                if c.__dict__.get("_node_params"):
                    c._sync_nodes()
        carr = plan.component_array(dev)
        f64 = dict(dtype=torch.float64, device=dev)
        phi = grad = hess = rho = None
        if out is not None:
            phi, grad, hess, rho = out
        else:
            if mode == _lib.MODE_DENS:
                rho = torch.empty(n, **f64)
            else:
                if want_phi or mode == _lib.MODE_POT:
                    phi = torch.empty(n, **f64)
                if mode in (_lib.MODE_GRAD, _lib.MODE_HESS):
                    grad = torch.empty((n, 3), **f64)
                if mode == _lib.MODE_HESS:
                    hess = torch.empty((n, 6), **f64)
        if n == 0:
            return phi, grad, hess, rho
        ptr = lambda a: None if a is None else a.data_ptr()  # noqa: E731
        flags = self._flags(mode, prec, n)
        nws = int(_lib.lib.agb_eval_timed_workspace_bytes(carr, len(plan.comps), plan.handle, n,
                                                          flags))
        ws = torch.empty(nws, dtype=torch.uint8, device=dev)
        stream = torch.cuda.current_stream(dev).cuda_stream
        rc = _lib.lib.agb_eval_timed(carr, len(plan.comps), plan.handle, ptr(step), float(t0),
                                     float(dt), float(off), arr.data_ptr(), n, mode, prec,
                                     ptr(phi), ptr(grad), ptr(hess), ptr(rho), flags, ws.data_ptr(),
                                     nws, ctypes.c_void_p(stream))
        _lib.check(rc, "agb_eval_timed")
        return phi, grad, hess, rho

    def _time_leaves_host(self, t: float):
        """The plan's leaves at t by the library's host evaluation of the programs:
        [(component, sigma, gamma, ampl)] (one per program)."""
        built = self._time_programs()
        if built is None:
            raise ValueError("this potential tree has no device time plan")
        comps, progs, table = built
        h = ctypes.c_void_p()
        _lib.check(_lib.lib.agb_time_plan_create(progs, len(progs), table.ctypes.data, table.size,
                                                 ctypes.byref(h)), "agb_time_plan_create")
        try:
            lv = (_lib.AgbLeaf * len(progs))()
            _lib.check(_lib.lib.agb_time_plan_leaves_host(h, float(t), lv), "agb_time_plan_leaves_host")
        finally:
            _lib.lib.agb_time_plan_destroy(h)
        return [(comps[q.comp], q.sigma, np.array(q.gamma[:]), q.ampl) for q in lv]

    # -- node tables as torch tensors ----------------------------------------
    def node_parameters(self) -> List[torch.Tensor]:
        """The node tables of every Multipole and CylSpline in the tree as leaf tensors
        with requires_grad (each component's node_parameters(), in tree order; a
        component used twice appears once).  They ARE the potential's node values:
        an in-place change (an optimizer step) is picked up by the next evaluation,
        and the differentiable entry points (autograd.potential_and_force, leapfrog,
        stream.integrate_releases_autograd) take them as inputs, so loss.backward()
        fills their .grad."""
        out, seen = [], set()
        for c in self._all_components():
            if id(c) not in seen:
                seen.add(id(c))
                out.extend(c.node_parameters())
        return out

    def _tracked_nodes(self) -> List[Tuple["_Component", List[torch.Tensor]]]:
        """[(component, its node tensors)] for the tree's components whose
        node_parameters() were requested, in tree order."""
        out, seen = [], set()
        for c in self._all_components():
            p = c.__dict__.get("_node_params")
            if p and id(c) not in seen:
                seen.add(id(c))
                out.append((c, list(p)))
        return out

    def _node_param_grads(self, table_grads: dict, tracked) -> List[torch.Tensor]:
        """Gradients of the tracked node tensors (flattened like tracked) from
        {component: table gradient} (Multipole dL/dpoly, CylSpline dL/d(node table));
        zeros for a component without an entry (not in use at the times evaluated)."""
        out = []
        for comp, params in tracked:
            g = table_grads.get(comp)
            if g is None:
                out.extend(torch.zeros_like(q) for q in params)
            elif comp.kind == _lib.KIND_MULTIPOLE:
                out.extend(comp._grads_of_nodes(g, table_grads.get(("const", comp))))
            else:
                out.extend(comp._grads_of_nodes(g))
        return out

    def _c_args(self, t: float, dev: torch.device, leaves=None):
        """(component array, n_comps, leaf array, n_leaves) of the tree at time t
        (or of the given leaves)."""
        self._preload(dev)
        if leaves is None:
            leaves = self._leaves(float(t))
        if not leaves:
            raise ValueError("potential has no components")
        for c, _, _, _ in leaves:
            if c.__dict__.get("_node_params") and not torch.cuda.is_current_stream_capturing():
                c._sync_nodes()
        if len(leaves) > _lib.MAX_LEAVES:
            raise ValueError(f"{len(leaves)} leaf components exceed the fused kernel's "
                             f"limit of {_lib.MAX_LEAVES}")
        comps: List[_lib.AgbComponent] = []
        index = {}
        leaf_arr = (_lib.AgbLeaf * len(leaves))()
        for i, (c, sigma, gamma, ampl) in enumerate(leaves):
            key = id(c)
            if key not in index:
                index[key] = len(comps)
                comps.append(c._device_component(dev))
            lf = leaf_arr[i]
            lf.comp = index[key]
            lf.sigma = sigma
            lf.gamma[0], lf.gamma[1], lf.gamma[2] = float(gamma[0]), float(gamma[1]), float(gamma[2])
            lf.ampl = ampl
        return (_lib.AgbComponent * len(comps))(*comps), len(comps), leaf_arr, len(leaves)

    def _flags(self, mode: int = -1, prec: int = -1, n: int = 0) -> int:
        f = _lib.OUT_NEGATE | (0 if self.binning else _lib.OUT_NO_BINNING)
        tuned = self.__dict__.get("_tuned")
        if tuned:                   # launch shape chosen by autotune.autotune()
            f |= tuned.get((mode, prec, int(n).bit_length()), 0)
        return f

    def _workspace(self, cargs, n: int, dev: torch.device, flags: int):
        nws = int(_lib.lib.agb_eval_workspace_bytes(cargs[0], cargs[1], cargs[2], cargs[3], n,
                                                    flags))
        return (torch.empty(nws, dtype=torch.uint8, device=dev) if nws else None), nws

    def _launch(self, arr: torch.Tensor, t: float, mode: int, want_phi: bool,
                precision: Optional[str] = None, out=None):
        n = arr.shape[0]
        dev = arr.device
        prec = _PRECISIONS[precision or self.precision or _default_precision]
        cargs = self._c_args(t, dev)
        f64 = dict(dtype=torch.float64, device=dev)
        phi = grad = hess = rho = None
        if out is not None:
            phi, grad, hess, rho = out
        else:
            if mode == _lib.MODE_DENS:
                rho = torch.empty(n, **f64)
            else:
                if want_phi or mode == _lib.MODE_POT:
                    phi = torch.empty(n, **f64)
                if mode in (_lib.MODE_GRAD, _lib.MODE_HESS):
                    grad = torch.empty((n, 3), **f64)
                if mode == _lib.MODE_HESS:
                    hess = torch.empty((n, 6), **f64)
        if n == 0:
            return phi, grad, hess, rho
        ptr = lambda a: None if a is None else a.data_ptr()  # noqa: E731
        stream = torch.cuda.current_stream(dev).cuda_stream
        flags = self._flags(mode, prec, n)
        ws, nws = self._workspace(cargs, n, dev, flags)
        rc = _lib.lib.agb_eval_ws(*cargs, arr.data_ptr(), n, mode, prec, ptr(phi), ptr(grad),
                                  ptr(hess), ptr(rho), flags, ptr(ws), nws,
                                  ctypes.c_void_p(stream))
        _lib.check(rc, "agb_eval_ws")
        return phi, grad, hess, rho

    def _vjp(self, arr: torch.Tensor, t: float, g_phi: Optional[torch.Tensor],
             g_force: Optional[torch.Tensor], precision: Optional[str] = None,
             out: Optional[torch.Tensor] = None, leaves=None,
             force_out: Optional[torch.Tensor] = None) -> torch.Tensor:
        """dL/dx = g_phi * grad(Phi) - H g_force for cotangents of (Phi, force).
        force_out [N,3]: also receives the force of the same leaves (assigned)."""
        n = arr.shape[0]
        dev = arr.device
        prec = _PRECISIONS[precision or self.precision or _default_precision]
        gx = out if out is not None else torch.empty((n, 3), dtype=torch.float64, device=dev)
        if n == 0:
            return gx
        cargs = self._c_args(t, dev, leaves)
        gp = None if g_phi is None else g_phi.to(device=dev, dtype=torch.float64).contiguous()
        gf = None if g_force is None else g_force.to(device=dev, dtype=torch.float64).contiguous()
        ptr = lambda a: None if a is None else a.data_ptr()  # noqa: E731
        ws, nws = self._workspace(cargs, n, dev, 0)       # agb_eval_vjp sorts by default
        stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
        if force_out is None:
            rc = _lib.lib.agb_eval_vjp(*cargs, arr.data_ptr(), n, prec, ptr(gp), ptr(gf),
                                       gx.data_ptr(), ptr(ws), nws, stream)
            _lib.check(rc, "agb_eval_vjp")
        else:
            rc = _lib.lib.agb_eval_vjp_force(*cargs, arr.data_ptr(), n, prec, ptr(gp), ptr(gf),
                                             gx.data_ptr(), force_out.data_ptr(), ptr(ws), nws,
                                             stream)
            _lib.check(rc, "agb_eval_vjp_force")
        return gx

    def _adjoint_vjp(self, arr: torch.Tensor, t: float, g_phi: Optional[torch.Tensor],
                     g_force: Optional[torch.Tensor], acc_dev: dict,
                     precision: Optional[str] = None, out: Optional[torch.Tensor] = None,
                     force_out: Optional[torch.Tensor] = None):
        """Position VJP of the tree and, fused into the same walk, the coefficient
        gradients of its (regular-layout) Multipoles, accumulated into ``acc_dev``
        as device-layout buffers {component: (n_int, n_cols, 6)}; convert them with
        ``_table_grads_from_device``.  Other Multipoles use the separate passes.
        force_out [N,3]: also receives the tree's force at arr (assigned)."""
        n = arr.shape[0]
        dev = arr.device
        prec = _PRECISIONS[precision or self.precision or _default_precision]
        leaves = self._leaves(float(t))
        fused = [lf for lf in leaves
                 if lf[0].kind == _lib.KIND_MULTIPOLE and getattr(lf[0], "_structure", 0) != 0]
        rest = [lf for lf in leaves if not any(lf is f for f in fused)]
        gx = out if out is not None else torch.empty((n, 3), dtype=torch.float64, device=dev)
        if rest:
            self._vjp(arr, t, g_phi, g_force, precision=precision, out=gx, leaves=rest,
                      force_out=force_out)
            for comp, sigma, gamma, ampl in rest:
                if comp.kind in (_lib.KIND_MULTIPOLE, _lib.KIND_CYLSPLINE):
                    kw = {}
                    if comp.kind == _lib.KIND_MULTIPOLE:
                        kw["const_grad"] = _const_buffer(acc_dev, comp, dev)
                    g = comp.table_vjp(arr, t, g_phi, g_force, leaf=(sigma, gamma, ampl), **kw)
                    key = ("poly", comp)
                    if key in acc_dev:
                        acc_dev[key].add_(g)
                    else:
                        acc_dev[key] = g
        else:
            gx.zero_()
            if force_out is not None:
                force_out.zero_()
        if n == 0:
            return gx
        gp = None if g_phi is None else g_phi.to(device=dev, dtype=torch.float64).contiguous()
        gf = None if g_force is None else g_force.to(device=dev, dtype=torch.float64).contiguous()
        ptr = lambda a: None if a is None else a.data_ptr()  # noqa: E731
        stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
        for comp, sigma, gamma, ampl in fused:
            c = comp._device_component(dev)
            lf = _lib.AgbLeaf()
            lf.comp, lf.sigma, lf.ampl = 0, float(sigma), float(ampl)
            lf.gamma[0], lf.gamma[1], lf.gamma[2] = (float(v) for v in gamma)
            buf = acc_dev.get(comp)
            if buf is None:
                buf = torch.zeros((comp.tables.n_int, comp._n_cols, 6), dtype=torch.float64,
                                  device=dev)
                acc_dev[comp] = buf
            nws = int(_lib.lib.agb_multipole_adjoint_workspace_bytes(
                ctypes.byref(c), ctypes.byref(lf), n, 0 if force_out is None else 1))
            ws = torch.empty(nws, dtype=torch.uint8, device=dev) if nws else None
            cg = _const_buffer(acc_dev, comp, dev)
            if force_out is None:
                rc = _lib.lib.agb_multipole_adjoint(ctypes.byref(c), ctypes.byref(lf),
                                                    arr.data_ptr(), n, prec, ptr(gp), ptr(gf),
                                                    gx.data_ptr(), buf.data_ptr(), cg.data_ptr(),
                                                    ptr(ws), nws, stream)
                _lib.check(rc, "agb_multipole_adjoint")
            else:
                rc = _lib.lib.agb_multipole_adjoint_force(ctypes.byref(c), ctypes.byref(lf),
                                                          arr.data_ptr(), n, prec, ptr(gp), ptr(gf),
                                                          gx.data_ptr(), force_out.data_ptr(),
                                                          buf.data_ptr(), cg.data_ptr(), ptr(ws),
                                                          nws, stream)
                _lib.check(rc, "agb_multipole_adjoint_force")
        return gx

    def _adjoint_step(self, arr: torch.Tensor, t: float, gF: Optional[torch.Tensor],
                      acc_dev: dict, lx: torch.Tensor, lv: torch.Tensor, dt: float, c: float,
                      vh: Optional[torch.Tensor] = None, k: float = 0.0, dt_drift: float = 0.0,
                      precision: Optional[str] = None, c_in: Optional[float] = None) -> bool:
        """One backward leapfrog step in two launches (agb_adjoint_step): the VJP of the
        tree at arr with cotangent gF of the force, the coefficient gradient of its
        Multipole added into ``acc_dev`` (device layout, as ``_adjoint_vjp``), the kick
        lx += gx, lv = fma(dt, lx, lv), gF = c lv, and with ``vh`` the reverse drift
        vh -= k F(arr), arr -= dt_drift vh, in place.  With ``c_in`` the cotangent of the
        force is c_in lv (lv on entry) and gF is neither read nor written.  Returns False
        (nothing done) when the tree at t is not one regular-structure Multipole plus
        analytic leaves."""
        leaves = self._leaves(float(t))
        mp = [i for i, lf in enumerate(leaves) if lf[0].kind == _lib.KIND_MULTIPOLE]
        if len(mp) != 1 or any(lf[0].kind == _lib.KIND_CYLSPLINE for lf in leaves):
            return False
        comp = leaves[mp[0]][0]
        if getattr(comp, "_structure", 0) == 0:
            return False
        n = arr.shape[0]
        dev = arr.device
        prec = _PRECISIONS[precision or self.precision or _default_precision]
        cargs = self._c_args(t, dev, leaves)
        flags = (_lib.ADJ_DRIFT if vh is not None else 0) | \
            (_lib.ADJ_LV_COT if c_in is not None else 0)
        nws = int(_lib.lib.agb_adjoint_step_workspace_bytes(*cargs, mp[0], n, flags))
        if nws == 0:
            return False
        buf = acc_dev.get(comp)
        if buf is None:
            buf = torch.zeros((comp.tables.n_int, comp._n_cols, 6), dtype=torch.float64,
                              device=dev)
            acc_dev[comp] = buf
        ws = torch.empty(nws, dtype=torch.uint8, device=dev)
        cg = _const_buffer(acc_dev, comp, dev)
        rc = _lib.lib.agb_adjoint_step(
            *cargs, mp[0], prec, arr.data_ptr(), None if vh is None else vh.data_ptr(),
            lx.data_ptr(), lv.data_ptr(), None if c_in is not None else gF.data_ptr(),
            buf.data_ptr(), cg.data_ptr(), n, float(dt), float(c),
            float(c_in) if c_in is not None else 0.0, float(k), float(dt_drift), flags,
            ws.data_ptr(), nws,
            ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream))
        _lib.check(rc, "agb_adjoint_step")
        return True

    @staticmethod
    def _table_grads_from_device(acc_dev: dict) -> dict:
        """{component: dL/dpoly in the layout of component.tables.poly} and, for each
        Multipole, {("const", component): dL/d(builder scalars) (8,)}."""
        out = {}
        for key, g in acc_dev.items():
            if isinstance(key, tuple) and key[0] == "const":
                out[key] = g
                continue
            if isinstance(key, tuple):              # already in poly layout
                comp = key[1]
                out[comp] = out[comp] + g if comp in out else g
                continue
            comp = key
            cols = torch.from_numpy(comp._col_of).to(g.device)
            # the fused adjoint differentiates the rescaled table: back to the builder's
            scale = torch.from_numpy(comp._col_scale).to(g.device)
            g = g * scale[None, :, None]
            gp = g.index_select(1, cols).permute(1, 0, 2).contiguous()
            out[comp] = out[comp] + gp if comp in out else gp
        return out

    def _table_vjp(self, arr: torch.Tensor, t: float, g_phi: Optional[torch.Tensor],
                   g_force: Optional[torch.Tensor], acc: Optional[dict] = None) -> dict:
        """Table gradients of every Multipole and CylSpline in the tree: {component:
        dL/dpoly (n_lm, n_int, 6) | dL/d(node table) (n_harm, nR, nz, 4)} and, per
        Multipole, {("const", component): dL/d(builder scalars) (8,)}, summed over
        the leaves that use it and added into ``acc`` when given."""
        acc = {} if acc is None else acc
        for comp, sigma, gamma, ampl in self._leaves(float(t)):
            if comp.kind not in (_lib.KIND_MULTIPOLE, _lib.KIND_CYLSPLINE):
                continue
            kw = {}
            if comp.kind == _lib.KIND_MULTIPOLE:
                kw["const_grad"] = _const_buffer(acc, comp, arr.device)
            g = comp.table_vjp(arr, t, g_phi, g_force, leaf=(sigma, gamma, ampl), **kw)
            if comp in acc:
                acc[comp].add_(g)
            else:
                acc[comp] = g
        return acc

    # -- public API (gpu_potential.py:826-935) --------------------------------
    def potential(self, xyz, t: float = 0.0):
        """Phi in (km/s)^2: (N,) or a 0-d tensor for one point."""
        arr, single = prep_xyz(xyz)
        phi, _, _, _ = self._launch(arr, t, _lib.MODE_POT, True)
        return _sq(phi, single)

    def force(self, xyz, t: float = 0.0):
        """F = -grad Phi in (km/s)^2/kpc: (N,3) or (3,)."""
        arr, single = prep_xyz(xyz)
        _, f, _, _ = self._launch(arr, t, _lib.MODE_GRAD, False)
        return _sq(f, single)

    def density(self, xyz, t: float = 0.0):
        """rho = Laplacian(Phi)/(4 pi G) in Msol/kpc^3: (N,) or 0-d."""
        arr, single = prep_xyz(xyz)
        _, _, _, rho = self._launch(arr, t, _lib.MODE_DENS, False)
        return _sq(rho, single)

    def forceDeriv(self, xyz, t: float = 0.0):
        """(force (N,3), deriv (N,6)); deriv = [dFx/dx, dFy/dy, dFz/dz, dFx/dy, dFy/dz, dFz/dx]."""
        arr, single = prep_xyz(xyz)
        _, f, d, _ = self._launch(arr, t, _lib.MODE_HESS, False)
        return _sq(f, single), _sq(d, single)

    def evalDeriv(self, xyz, t: float = 0.0):
        """(Phi, force, deriv) from one kernel launch."""
        arr, single = prep_xyz(xyz)
        p, f, d, _ = self._launch(arr, t, _lib.MODE_HESS, True)
        return _sq(p, single), _sq(f, single), _sq(d, single)

    def eval(self, xyz, pot: bool = False, acc: bool = False, der: bool = False, t: float = 0.0):
        """Any subset of (Phi, force, deriv) in that order; one array if one is asked for."""
        if not (pot or acc or der):
            raise ValueError("eval(): at least one of pot, acc, der must be True.")
        arr, single = prep_xyz(xyz)
        mode = _lib.MODE_HESS if der else (_lib.MODE_GRAD if acc else _lib.MODE_POT)
        p, f, d, _ = self._launch(arr, t, mode, pot)
        res = []
        if pot:
            res.append(_sq(p, single))
        if acc:
            res.append(_sq(f, single))
        if der:
            res.append(_sq(d, single))
        return res[0] if len(res) == 1 else tuple(res)

    def eval_host(self, xyz, pot: bool = False, acc: bool = False, der: bool = False,
                  t: float = 0.0, chunk_points: Optional[int] = None, out=None, device=None):
        """``eval`` for positions and results in HOST memory, pipelined.

        The points go through the GPU in chunks of about ``chunk_points`` (default: N/3,
        clamped to [2^17, 2^20] points, so a chunk still fills the GPU; large calls round
        the chunks to whole waves of the kernel's resident threads): while chunk i
        is evaluated, chunk i+1 is copied in and chunk i-1's results are copied
        out (three CUDA streams, two device buffers per stream stage), so the
        PCIe transfers hide behind the kernel.  xyz: (N,3) float64 CPU tensor or
        NumPy array -- pinned memory (``tensor.pin_memory()``) makes the copies
        asynchronous; pageable memory works, without the overlap.  Returns CPU
        tensors in eval()'s order (pinned unless ``out`` gives the buffers:
        a tuple matching the requested outputs).  The host waits for the
        results before returning.  No counterpart in the reference (its API
        returns device arrays only).
        """
        if not (pot or acc or der):
            raise ValueError("eval_host(): at least one of pot, acc, der must be True.")
        src = xyz if isinstance(xyz, torch.Tensor) else torch.from_numpy(
            np.ascontiguousarray(xyz, dtype=np.float64))
        if src.device.type != "cpu":
            raise ValueError("eval_host() takes host (CPU) positions; use eval() for device arrays")
        src = src.to(torch.float64).contiguous()
        if src.dim() != 2 or src.shape[1] != 3:
            raise ValueError(f"xyz must have shape (N,3), got {tuple(src.shape)}")
        n = src.shape[0]
        dev = _cuda_device(device)
        mode = _lib.MODE_HESS if der else (_lib.MODE_GRAD if acc else _lib.MODE_POT)
        want = [(pot, (n,), 0), (acc, (n, 3), 1), (der, (n, 6), 2)]
        if out is None:
            host = [torch.empty(shape, dtype=torch.float64, pin_memory=True) if w else None
                    for w, shape, _ in want]
        else:
            outs = list(out) if isinstance(out, (tuple, list)) else [out]
            host = []
            for w, shape, _ in want:
                host.append(outs.pop(0) if w else None)
            for h, (w, shape, _) in zip(host, want):
                if w and (h is None or tuple(h.shape) != shape or h.dtype != torch.float64
                          or h.device.type != "cpu" or not h.is_contiguous()):
                    raise ValueError(f"out buffer must be a contiguous float64 CPU tensor {shape}")
        if chunk_points is None:
            chunk_points = min(1 << 20, max(1 << 17, -(-n // 3)))
        chunk = max(1, min(int(chunk_points), max(n, 1)))
        pipe = _host_pipe(dev)
        with pipe["lock"]:
            return self._eval_host_run(src, host, want, n, chunk, t, mode, pot, dev, pipe)

    def _eval_host_run(self, src, host, want, n, chunk, t, mode, pot, dev, pipe):
        # The chunk layout, launch flags and workspace size depend only on the call's
        # shape, so they are kept per shape on the object; the first chunk's copy-in is
        # queued before the tree's arguments at t are formed (the host's remaining work
        # before the first launch), so that copy overlaps it.  Each chunk then costs the
        # host one C call and the first kernel follows its copy directly.
        prec = _PRECISIONS[self.precision or _default_precision]
        tuned = self.__dict__.get("_tuned") or {}
        key = (dev.index, mode, prec, n, chunk, self.binning, tuple(sorted(tuned.items())))
        plans = self.__dict__.setdefault("_host_plans", {})
        plan = plans.get(key)
        cargs = None
        if plan is None:
            cargs = self._c_args(t, dev)
            wave = int(_lib.lib.agb_eval_wave_points(cargs[0], cargs[1], cargs[2], cargs[3],
                                                     mode, prec))
            bounds = _chunk_bounds(n, chunk, wave)
            sizes = sorted({hi - lo for lo, hi in bounds})
            flags = {m: self._flags(mode, prec, m) for m in sizes}
            if wave and len(bounds) > 2 and all((hi - lo) % wave == 0 for lo, hi in bounds[:-1]):
                # chunks in whole waves: one resident block per slot, so every thread of
                # a launch takes the same number of passes (unless a tuned shape is set)
                flags = {m: f if (f >> _lib.OUT_GRID_SHIFT) & 15 or (f >> _lib.OUT_PPT_SHIFT) & 15
                         else f | (1 << _lib.OUT_GRID_SHIFT) for m, f in flags.items()}
            nws = max((int(_lib.lib.agb_eval_workspace_bytes(cargs[0], cargs[1], cargs[2],
                                                             cargs[3], m, flags[m]))
                       for m in sizes), default=0)
            # the device buffers hold the largest chunk
            plan = (bounds, max(sizes), flags, nws)
            if len(plans) >= 64:
                plans.clear()
            plans[key] = plan
        bounds, chunk, flags, nws = plan
        ptr = lambda a: None if a is None else a.data_ptr()  # noqa: E731
        cur = torch.cuda.current_stream(dev)
        s_in, s_cmp, s_out = pipe["streams"]
        for s in (s_in, s_cmp, s_out):
            s.wait_stream(cur)
        xb = pipe_buffers(pipe, dev, ("x", chunk), (chunk, 3))
        ev_in = [torch.cuda.Event() for _ in range(2)]
        lo0, hi0 = bounds[0]
        with torch.cuda.stream(s_in):
            xb[0][:hi0 - lo0].copy_(src[lo0:hi0], non_blocking=True)
            ev_in[0].record(s_in)
        if cargs is None:
            cargs = self._c_args(t, dev)
        ws = pipe["bufs"].get("ws")
        if nws and (ws is None or ws.numel() < nws):
            # allocated on the compute stream, the only one that uses it
            with torch.cuda.device(dev), torch.cuda.stream(s_cmp):
                ws = torch.empty(nws, dtype=torch.uint8, device=dev)
            pipe["bufs"]["ws"] = ws
        ob = [[pipe_buffers(pipe, dev, (k, chunk), (chunk,) + shape[1:])[j] if w else None
               for w, shape, k in want] for j in range(2)]
        ev_cmp = [torch.cuda.Event() for _ in range(2)]
        ev_out = [torch.cuda.Event() for _ in range(2)]
        started = [False, False]
        for i, (lo, hi) in enumerate(bounds):
            b = i & 1
            m = hi - lo
            if i > 0:                                   # chunk 0 is on its way already
                with torch.cuda.stream(s_in):
                    if started[b]:
                        s_in.wait_event(ev_cmp[b])      # the kernel is done with xb[b]
                    xb[b][:m].copy_(src[lo:hi], non_blocking=True)
                    ev_in[b].record(s_in)
            with torch.cuda.stream(s_cmp):
                s_cmp.wait_event(ev_in[b])
                if started[b]:
                    s_cmp.wait_event(ev_out[b])      # the results of chunk i-2 are out
                p_, f_, d_ = (ob[b][k][:m] if ob[b][k] is not None else None for k in range(3))
                rc = _lib.lib.agb_eval_ws(*cargs, xb[b].data_ptr(), m, mode, prec, ptr(p_),
                                          ptr(f_), ptr(d_), None, flags[m], ptr(ws), nws,
                                          ctypes.c_void_p(s_cmp.cuda_stream))
                _lib.check(rc, "agb_eval_ws")
                ev_cmp[b].record(s_cmp)
            with torch.cuda.stream(s_out):
                s_out.wait_event(ev_cmp[b])
                for k in range(3):
                    if host[k] is not None:
                        host[k][lo:hi].copy_(ob[b][k][:m], non_blocking=True)
                ev_out[b].record(s_out)
            started[b] = True
        cur.wait_stream(s_out)          # later work on the caller's stream sees the results
        s_out.synchronize()
        res = [h for h in host if h is not None]
        return res[0] if len(res) == 1 else tuple(res)


def _chunk_bounds(n: int, chunk: int, wave: int = 0):
    """Chunk ranges of eval_host.  The first copy-in and the last copy-out cannot overlap
    a kernel, so the chunks ramp up and down around full-size chunks in between.

    With ``wave`` (the points one wave of the kernel's resident threads holds) and enough
    points, every chunk but the last is a whole number of waves: a launch takes as many
    passes of its threads as its largest block needs, so a chunk of 11.1 waves costs 12
    passes.  In waves, with c = round(chunk / wave) (14 for 2^20 points on 148 SMs x 2
    blocks x 256 threads): ramp-up c/7, 3c/7 (each copy-in hides behind the previous
    kernel: a copy-in takes ~0.4 of a kernel's time per point), full chunks of c, ramp-down
    5c/7, 2c/7, then the remainder of 2 to 3 waves, whose copy-out is the only one
    exposed.  On the 4M-point composite (mixed, 1 B200) this layout takes the
    end-to-end step 5.68 -> 5.29 ms.  Otherwise: chunk/4, chunk/2, full chunks, chunk/2,
    chunk/4, chunk/8."""
    if wave > 0 and chunk >= wave:
        c = max(1, round(chunk / wave))
        head = [max(1, round(c / 7)), max(1, round(3 * c / 7))]
        tail = [max(1, round(5 * c / 7)), max(1, round(2 * c / 7))]
        body_waves = n // wave - sum(head) - sum(tail) - 2
        if body_waves >= c:
            k = -(-body_waves // c)
            body = [body_waves // k + (1 if i < body_waves % k else 0) for i in range(k)]
            sizes = [u * wave for u in head + body + tail]
            sizes.append(n - sum(sizes))
            out, lo = [], 0
            for m in sizes:
                out.append((lo, lo + m))
                lo += m
            return out
    if n <= 2 * chunk:
        return [(lo, min(n, lo + chunk)) for lo in range(0, n, chunk)]
    head = [max(1, chunk // 4), max(1, chunk // 2)]
    tail = [max(1, chunk // 2), max(1, chunk // 4), max(1, chunk // 8)]
    mid = n - sum(head) - sum(tail)
    if mid <= 0:
        q = max(1, chunk // 4)
        sizes = [q] + [chunk] * ((n - 2 * q) // chunk)
        sizes.append(n - sum(sizes) - q) if n - sum(sizes) - q > 0 else None
        sizes.append(q)
    else:
        k = -(-mid // chunk)                       # full-size chunks, evened out
        body = [mid // k + (1 if i < mid % k else 0) for i in range(k)]
        sizes = head + body + tail
    out, lo = [], 0
    for m in sizes:
        if m > 0:
            out.append((lo, lo + m))
            lo += m
    assert lo == n
    return out


# Per device: the three streams of eval_host and its double-buffered device chunks,
# kept between calls so that a call allocates nothing once the sizes were seen
# (torch's allocator caches blocks per stream).  A lock serialises callers.
_HOST_PIPES = {}


def _host_pipe(dev: torch.device) -> dict:
    key = dev.index
    pipe = _HOST_PIPES.get(key)
    if pipe is None:
        import threading
        pipe = {"lock": threading.Lock(), "bufs": {},
                "streams": tuple(torch.cuda.Stream(device=dev) for _ in range(3))}
        _HOST_PIPES[key] = pipe
    return pipe


def pipe_buffers(pipe: dict, dev: torch.device, key, shape):
    bufs = pipe["bufs"].get(key)
    if bufs is None:
        with torch.cuda.device(dev):
            bufs = [torch.empty(shape, dtype=torch.float64, device=dev) for _ in range(2)]
        pipe["bufs"][key] = bufs
    return bufs


class _Component(_GPUPotBase):
    """A leaf: one component with device tables."""

    kind: int = 0

    def _leaves(self, t: float) -> List[Leaf]:
        return [(self, 1.0, np.zeros(3), 1.0)]

    def _params(self) -> Sequence[float]:
        return []

    def _device_component(self, dev: torch.device) -> _lib.AgbComponent:
        cache = self.__dict__.setdefault("_dev_cache", {})
        hit = cache.get(dev)
        if hit is None:
            hit = self._upload(dev)
            cache[dev] = hit
        return hit[0]

    def _upload(self, dev: torch.device):
        c = _lib.AgbComponent()
        c.kind = self.kind
        for i, v in enumerate(self._params()):
            c.p[i] = float(v)
        return c, ()

    def node_parameters(self, device=None) -> List[torch.Tensor]:
        """Node tables as leaf tensors (expansions only; analytic profiles have none)."""
        return []

    def _track_nodes(self, tensors: List[torch.Tensor]) -> List[torch.Tensor]:
        self._node_params = tensors
        self._node_params_version = tuple(q._version for q in tensors)
        return list(tensors)

    def _sync_nodes(self) -> None:
        """Rebuild the device tables when the node tensors changed in place."""
        p = self.__dict__.get("_node_params")
        if not p:
            return
        ver = tuple(q._version for q in p)
        if ver != self.__dict__.get("_node_params_version"):
            self._apply_nodes(p)
            self._node_params_version = tuple(q._version for q in p)

    def _refresh_tracked(self, values: List[torch.Tensor]) -> None:
        """After set_node_tables(): copy the new values into the tracked tensors."""
        p = self.__dict__.get("_node_params")
        if not p:
            return
        with torch.no_grad():
            for q, v in zip(p, values):
                if q.data_ptr() != v.data_ptr():
                    q.copy_(v.to(q.device))
        self._node_params_version = tuple(q._version for q in p)


# ---------------------------------------------------------------------------
# Multipole
# ---------------------------------------------------------------------------

class MultipolePotentialGPU(_Component):
    """Agama Multipole BFE: quintic C2 splines in log r with log-scaling.

    Same constructor as the reference (gpu_potential.py:654):
    ``MultipolePotentialGPU(coefs, prune_threshold=1e-16)`` with a coefficient
    object carrying R_grid, phi, dphi_dr, lm_labels (``read_coefs`` output).
    """

    kind = _lib.KIND_MULTIPOLE

    def __init__(self, coefs, prune_threshold: float = 1e-16) -> None:
        # construction order: ranks that build the same potentials in the same order
        # agree on it, which fixes the order of the gradient all-reduces
        self._sync_order = next(_MULTIPOLE_SERIAL)
        self._coefs = coefs
        self.tables = build_multipole_tables(coefs, prune_threshold=prune_threshold)
        self._n_file_cols = len(coefs.lm_labels)
        t = self.tables
        self._structure, reg = t.regular()
        poly = t.poly if reg is None else reg
        self._n_cols = poly.shape[0]
        # device column of each of the builder's harmonics (identity for the list layout)
        if reg is None:
            self._col_of = np.arange(t.n_lm)
        else:
            cols = {}
            even = self._structure == _lib.STRUCT_EVEN
            for am in range(t.lmax + 1):
                for l in range(am, t.lmax + 1):
                    if even and l % 2:
                        continue
                    cols[(l, am)] = len(cols)
                    if am > 0:
                        cols[(l, -am)] = len(cols)
            self._col_of = np.array([cols[(int(l), int(m))] for l, m in zip(t.lm_l, t.lm_m)])
        # regular structures: column (l, m) carries the scale C_l^m = prod_{j=|m|+1..l}
        # sqrt((4j^2 - 1) / (j^2 - m^2)) of the kernels' rescaled Legendre recurrence
        self._col_scale = np.ones(self._n_cols)
        if reg is not None:
            for (l, m), c in cols.items():
                am = abs(m)
                j = np.arange(am + 1, l + 1, dtype=np.float64)
                self._col_scale[c] = float(np.prod(np.sqrt((4 * j * j - 1) / (j * j - am * am))))
            poly = poly * self._col_scale[:, None, None]
        self._poly_im = np.ascontiguousarray(poly.transpose(1, 0, 2))
        # FP32 table: 8-float records (a0..a5, 2 pads); with a regular structure each
        # m>0 (cos, sin) column pair is one 16-float record c0 s0 c1 s1 ... c5 s5 + 4
        # pads.  _p32_src maps every float of an interval's FP32 slab to its source in
        # the FP64 slab (n_cols x 6), -1 for a pad.
        src = np.full(self._n_cols * 8, -1, dtype=np.int64)
        for c in range(self._n_cols):
            src[c * 8:c * 8 + 6] = c * 6 + np.arange(6)
        if reg is not None:
            for (l, m), c in cols.items():
                if m > 0:
                    src[c * 8:(c + 2) * 8] = -1
                    src[c * 8:c * 8 + 12:2] = c * 6 + np.arange(6)
                    src[c * 8 + 1:c * 8 + 12:2] = (c + 1) * 6 + np.arange(6)
        self._p32_src = src
        flat64 = self._poly_im.reshape(t.n_int, self._n_cols * 6)
        p32 = np.where(src >= 0, flat64[:, np.maximum(src, 0)], 0.0).astype(np.float32)
        self._poly32 = np.ascontiguousarray(p32.reshape(t.n_int, self._n_cols, 8))
        self._lm = t.lm_packed()
        self._nodes = None          # device node tables set by set_node_tables()

    @classmethod
    def from_file(cls, path: Union[str, Path], **kw) -> "MultipolePotentialGPU":
        """Load from an Agama .coef_mul_DR file (or the text of one section)."""
        return cls(read_coefs(path if isinstance(path, Path) else str(path)), **kw)

    @classmethod
    def from_agama(cls, pot, **kw) -> "MultipolePotentialGPU":
        """Build from an agama.Potential by exporting its coefficients (needs agama)."""
        shm = "/dev/shm"
        tmp_dir = shm if (os.path.isdir(shm) and os.access(shm, os.W_OK)) else tempfile.gettempdir()
        tmp = os.path.join(tmp_dir, f"agama_gpu_{uuid.uuid4().hex}.coef")
        try:
            pot.export(tmp)
            with open(tmp) as f:
                head = f.read(512)
            if "Coefficients" not in head:
                raise ValueError(
                    "from_agama(): the potential does not export expansion coefficients.\n"
                    "Agama analytic types (NFW, Plummer, Dehnen, ...) do not store their\n"
                    "parameters on export.  Construct the GPU class directly instead.")
            return cls.from_file(tmp, **kw)
        finally:
            try:
                os.unlink(tmp)
            except FileNotFoundError:
                pass

    def table_vjp(self, xyz: torch.Tensor, t: float, g_phi: Optional[torch.Tensor],
                  g_force: Optional[torch.Tensor], leaf=None,
                  const_grad: Optional[torch.Tensor] = None) -> torch.Tensor:
        """dL/dpoly (n_lm, n_int, 6) of this Multipole, in the layout of ``tables.poly``.

        g_phi (N,) and g_force (N,3) are cotangents of the potential and force of
        the tree this component belongs to; ``leaf`` = (sigma, gamma, ampl) of the
        component in that tree (default: the component on its own).  FP64.
        const_grad: an (8,) FP64 device tensor that receives (adds) the gradient
        with respect to the builder's scalars -- invPhi0 from the points inside
        the grid, the inner and outer l=0 extrapolation from the points beyond it
        (see diff_tables.multipole_consts_from_nodes); pass it on to
        node_gradients() for the derivative of the whole builder.
        """
        dev = xyz.device
        comp = self._device_component(dev)
        lf = _lib.AgbLeaf()
        sigma, gamma, ampl = leaf if leaf is not None else (1.0, np.zeros(3), 1.0)
        lf.comp = 0
        lf.sigma = float(sigma)
        lf.gamma[0], lf.gamma[1], lf.gamma[2] = (float(g) for g in gamma)
        lf.ampl = float(ampl)
        n = xyz.shape[0]
        g = torch.zeros((self.tables.n_int, self._n_cols, 6), dtype=torch.float64, device=dev)
        if n:
            arr = xyz.to(dtype=torch.float64).contiguous()
            gp = None if g_phi is None else g_phi.to(device=dev, dtype=torch.float64).contiguous()
            gf = None if g_force is None else g_force.to(device=dev, dtype=torch.float64).contiguous()
            nws = int(_lib.lib.agb_multipole_table_vjp_workspace_bytes(ctypes.byref(comp),
                                                                       ctypes.byref(lf), n))
            ws = torch.empty(nws, dtype=torch.uint8, device=dev) if nws else None
            ptr = lambda a: None if a is None else a.data_ptr()  # noqa: E731
            if const_grad is not None and (const_grad.dtype != torch.float64 or
                                           const_grad.numel() != _lib.MP_NCONST or
                                           const_grad.device != dev):
                raise ValueError("const_grad must be an (8,) float64 tensor on the points' device")
            rc = _lib.lib.agb_multipole_table_vjp(
                ctypes.byref(comp), ctypes.byref(lf), arr.data_ptr(), n, ptr(gp), ptr(gf),
                g.data_ptr(), ptr(const_grad), ptr(ws), nws,
                ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream))
            _lib.check(rc, "agb_multipole_table_vjp")
        cols = torch.from_numpy(self._col_of).to(dev)
        return g.index_select(1, cols).permute(1, 0, 2).contiguous()

    def node_gradients(self, grad_poly: torch.Tensor, grad_const: Optional[torch.Tensor] = None):
        """(dL/dPhi_nodes, dL/d(dPhi/dr)_nodes), each (nR, n_file_columns), from dL/dpoly.

        Chains through a differentiable restatement of the table construction
        (diff_tables).  With grad_const (table_vjp's const_grad, or the adjoint's
        table gradients) also through invPhi0 and the l=0 extrapolation constants,
        as functions of the nodes: the derivative of the whole builder, which is
        what set_node_tables() rebuilds; without it they are held fixed.
        """
        from .diff_tables import node_vjp
        n_file = int(max(self.tables.node_cols)) + 1 if self._n_file_cols is None else self._n_file_cols
        return node_vjp(self.tables, grad_poly, n_file, nodes=self._nodes, grad_const=grad_const)

    _n_file_cols = None

    def node_parameters(self, device=None) -> List[torch.Tensor]:
        """[Phi_lm(r_i), dPhi_lm/dr(r_i)]: the node tables, (nR, n_lm) each in the
        builder's harmonic order (the layout of tables.node_phi and of
        set_node_tables), as FP64 CUDA leaf tensors with requires_grad.  The same
        tensors on every call.  The radial grid, invPhi0 and the extrapolation
        constants stay those of construction (as in node_gradients)."""
        p = self.__dict__.get("_node_params")
        if p:
            return list(p)
        dev = torch.device(device) if device is not None else _cuda_device()
        if self._nodes is not None:
            phi, dphi = self._nodes
        else:
            phi = torch.from_numpy(np.ascontiguousarray(self.tables.node_phi))
            dphi = torch.from_numpy(np.ascontiguousarray(self.tables.node_dphi_dr))
        return self._track_nodes([phi.detach().to(dev, torch.float64).clone().requires_grad_(True),
                                  dphi.detach().to(dev, torch.float64).clone().requires_grad_(True)])

    def _apply_nodes(self, p) -> None:
        self._set_nodes(p[0], p[1])

    def _grads_of_nodes(self, grad_poly: torch.Tensor,
                        grad_const: Optional[torch.Tensor] = None) -> List[torch.Tensor]:
        """[dL/dPhi nodes, dL/d(dPhi/dr) nodes] in the layout of node_parameters()."""
        from .diff_tables import node_vjp
        g0, g1 = node_vjp(self.tables, grad_poly, None, nodes=self._nodes, grad_const=grad_const)
        dev = self._node_params[0].device
        return [g0.to(dev), g1.to(dev)]

    def _device_tables(self, phi: torch.Tensor, dphi_dr: torch.Tensor, inv=None):
        """(FP64 interval-major, FP32) device tables of this object's layout from node
        tables (nR, n_lm) in the builder's harmonic order, computed with torch on
        their device (differentiable restatement of the builder: diff_tables); inv:
        invPhi0 (default: the builder's)."""
        from .diff_tables import multipole_poly_from_nodes
        t = self.tables
        dev = phi.device
        pb = multipole_poly_from_nodes(t, phi.to(torch.float64), dphi_dr.to(torch.float64),
                                       inv=inv)
        full = torch.zeros((self._n_cols, t.n_int, 6), dtype=torch.float64, device=dev)
        full[torch.from_numpy(self._col_of).to(dev)] = pb
        full = full * torch.from_numpy(self._col_scale).to(dev)[:, None, None]
        im = full.permute(1, 0, 2).contiguous()
        src = torch.from_numpy(self._p32_src).to(dev)
        flat = im.reshape(t.n_int, self._n_cols * 6)
        p32 = torch.where(src >= 0, flat[:, src.clamp(min=0)], torch.zeros((), dtype=torch.float64,
                                                                           device=dev))
        return im, p32.to(torch.float32).reshape(t.n_int, self._n_cols, 8).contiguous()

    def set_node_tables(self, phi: torch.Tensor, dphi_dr: torch.Tensor,
                        rebuild_constants: bool = True) -> None:
        """Replace the expansion's node values Phi_lm(r_i) and dPhi_lm/dr(r_i) -- (nR,
        n_lm) tensors in the builder's harmonic order (the layout of tables.node_phi) --
        rebuilding the quintic tables on the GPU, in place (a CUDA graph captured over
        this potential sees the new tables).  The scalars the builder derives from the
        l=0 nodes -- invPhi0 and the inner and outer power-law constants -- are
        recomputed as the builder does (one small device-to-host copy of the l=0
        column); graphs captured before a change of them are captured again by the
        integrators.  rebuild_constants=False keeps those of construction (and of
        node_gradients() without grad_const).  The radial grid, the harmonic set and
        the log-scaling switch stay those of construction.  Not differentiable
        itself: use node_gradients() on the adjoint's table gradient."""
        self._set_nodes(phi, dphi_dr, rebuild_constants)
        self._refresh_tracked([phi.detach(), dphi_dr.detach()])

    def _builder_scalars(self, phi: torch.Tensor, dphi_dr: torch.Tensor) -> List[float]:
        """[invPhi0, inner s, U, W, outer s, U, W] of the builder for these nodes."""
        from .prep_multipole import inner_extrapolation, outer_extrapolation
        t = self.tables
        p0 = phi[:, 0].detach().to("cpu", torch.float64).numpy()
        d0 = dphi_dr[:, 0].detach().to("cpu", torch.float64).numpy()
        if np.array_equal(p0, t.node_phi[:, 0]) and np.array_equal(d0, t.node_dphi_dr[:, 0]):
            # the construction's l=0 nodes: its scalars (the builder took dPhi/dr from
            # the file, which the node table holds rounded through d/dlog r)
            return [t.invPhi0, t.inner_s, t.inner_U, t.inner_W, t.outer_s, t.outer_U,
                    t.outer_W]
        r = np.asarray(t.r_grid, dtype=np.float64)
        if bool(t.log_scaling) != bool(np.all(p0 < 0.0)):
            raise ValueError("the new l=0 nodes change the sign condition of the log-scaling "
                             "the tables were built with")
        out = list(outer_extrapolation(p0, d0, r))
        if t.log_scaling:
            inner = list(inner_extrapolation(p0, d0, r))
        else:
            inner = [0.0, 0.0, 0.0, float(p0[0])]
        return [float(v) for v in inner + out]

    def _set_nodes(self, phi: torch.Tensor, dphi_dr: torch.Tensor,
                   rebuild_constants: bool = True) -> None:
        if phi.shape != self.tables.node_phi.shape or dphi_dr.shape != phi.shape:
            raise ValueError(f"node tables must have shape {self.tables.node_phi.shape}")
        dev = phi.device if phi.device.type == "cuda" else _cuda_device()
        phi = phi.detach().to(dev, torch.float64).clone()
        dphi_dr = dphi_dr.detach().to(dev, torch.float64).clone()
        t = self.tables
        built = [t.invPhi0, t.inner_s, t.inner_U, t.inner_W, t.outer_s, t.outer_U, t.outer_W]
        consts = self._builder_scalars(phi, dphi_dr) if rebuild_constants else built
        im, p32 = self._device_tables(phi, dphi_dr, inv=consts[0])
        self._nodes = (phi, dphi_dr)
        self._node_tables = (im, p32)
        for cdev, (_, keep) in self.__dict__.get("_dev_cache", {}).items():
            keep[0].copy_(im.to(cdev), non_blocking=True)
            keep[1].copy_(p32.to(cdev), non_blocking=True)
        if consts != self.__dict__.get("_consts", built):
            self._consts = consts
            for c, _ in self.__dict__.get("_dev_cache", {}).values():
                for i, v in enumerate(consts):
                    c.p[3 + i] = v
            self._consts_gen = self.__dict__.get("_consts_gen", 0) + 1

    def _upload(self, dev):
        t = self.tables
        over = self.__dict__.get("_node_tables")
        if over is not None:
            poly, poly32 = over[0].to(dev).clone(), over[1].to(dev).clone()
        else:
            poly = torch.from_numpy(self._poly_im).to(dev)
            poly32 = torch.from_numpy(self._poly32).to(dev)
        lm = torch.from_numpy(self._lm).to(dev)
        c = _lib.AgbComponent()
        c.kind = self.kind
        c.n_lm = self._n_cols
        c.n_int = t.n_int
        c.lmax = t.lmax
        c.log_scaling = t.log_scaling
        c.layout = _lib.LAYOUT_INTERVAL_MAJOR
        c.structure = self._structure
        c.table = poly.data_ptr()
        c.table32 = poly32.data_ptr()
        c.lm = lm.data_ptr()
        for i, v in enumerate(t.scalars()):
            c.p[i] = v
        for i, v in enumerate(self.__dict__.get("_consts") or []):     # set_node_tables
            c.p[3 + i] = v
        return c, (poly, poly32, lm)


# ---------------------------------------------------------------------------
# CylSpline
# ---------------------------------------------------------------------------

class CylSplinePotentialGPU(_Component):
    """Agama CylSpline: per-harmonic bicubic Hermite splines in (asinh R, asinh z).

    ``CylSplinePotentialGPU(coefs)`` as in gpu_potential.py:1281.  density()
    returns -(Hxx+Hyy+Hzz)/(4 pi G) like the reference's wrapper
    (gpu_potential.py:1389-1395), i.e. minus the Poisson density.
    """

    kind = _lib.KIND_CYLSPLINE

    def __init__(self, coefs) -> None:
        self._sync_order = next(_MULTIPOLE_SERIAL)
        self._coefs = coefs
        self._set_tables(build_cylspline_tables(coefs))

    def _set_tables(self, t) -> None:
        self.tables = t
        self._cells = t.cell_major()
        self._cells32 = t.cell_major_f32()
        self._m = t.m_sorted()
        self.__dict__.pop("_dev_cache", None)

    @classmethod
    def _from_tables(cls, tables, coefs=None) -> "CylSplinePotentialGPU":
        """A CylSpline from prepared tables (e.g. a perturbed node table)."""
        obj = cls.__new__(cls)
        obj._sync_order = next(_MULTIPOLE_SERIAL)
        obj._coefs = coefs
        obj._set_tables(tables)
        return obj

    def table_vjp(self, xyz: torch.Tensor, t: float, g_phi: Optional[torch.Tensor],
                  g_force: Optional[torch.Tensor], leaf=None) -> torch.Tensor:
        """dL/d(node table) (n_harm, nR, nz, 4) in the layout of ``tables.node_arr``
        ({f, f_lR, f_lz, f_lR_lz} at every node, harmonics in m_arr order), for
        cotangents of the potential and force of the tree this component belongs to;
        ``leaf`` = (sigma, gamma, ampl) of the component in that tree.  FP64.  Points
        outside the grid contribute nothing (the outer asymptote is held fixed)."""
        dev = xyz.device
        comp = self._device_component(dev)
        lf = _lib.AgbLeaf()
        sigma, gamma, ampl = leaf if leaf is not None else (1.0, np.zeros(3), 1.0)
        lf.comp = 0
        lf.sigma = float(sigma)
        lf.gamma[0], lf.gamma[1], lf.gamma[2] = (float(g) for g in gamma)
        lf.ampl = float(ampl)
        tb = self.tables
        nR, nz, H = len(tb.lR_grid), len(tb.lz_grid), tb.n_harm
        gc = torch.zeros((nR - 1, nz - 1, H, 4, 4), dtype=torch.float64, device=dev)
        n = xyz.shape[0]
        if n:
            arr = xyz.to(dtype=torch.float64).contiguous()
            gp = None if g_phi is None else g_phi.to(device=dev, dtype=torch.float64).contiguous()
            gf = None if g_force is None else g_force.to(device=dev, dtype=torch.float64).contiguous()
            ptr = lambda a: None if a is None else a.data_ptr()  # noqa: E731
            rc = _lib.lib.agb_cylspline_table_vjp(
                ctypes.byref(comp), ctypes.byref(lf), arr.data_ptr(), n, ptr(gp), ptr(gf),
                gc.data_ptr(), ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream))
            _lib.check(rc, "agb_cylspline_table_vjp")
        # fold the cell records onto the nodes: record [quantity][corner], corners
        # (lo,lo), (lo,hi), (hi,lo), (hi,hi) in (R, z)
        g_sorted = torch.zeros((H, nR, nz, 4), dtype=torch.float64, device=dev)
        for corner, (dR, dz) in enumerate(((0, 0), (0, 1), (1, 0), (1, 1))):
            g_sorted[:, dR:dR + nR - 1, dz:dz + nz - 1, :] += gc[:, :, :, :, corner].permute(2, 0, 1, 3)
        order = torch.from_numpy(tb.harmonic_order()).to(dev)
        g = torch.zeros_like(g_sorted)
        g[order] = g_sorted
        return g

    def node_gradients(self, grad_nodes: torch.Tensor):
        """{m: dL/dPhi_m} on the input coefficient grid from dL/d(node table), through
        the node-derivative splines, the log-scaling and the z mirroring of the table
        builder (the outer asymptote, Rscale and the grids are held fixed), at the node
        values set by set_node_tables() when there were any."""
        from .diff_tables import cylspline_node_vjp
        if self._coefs is None:
            raise ValueError("node_gradients() needs the coefficients the object was built from")
        phi = self.__dict__.get("_phi_nodes")
        if phi is not None:
            phi = {m: v.detach().cpu().numpy() for m, v in phi.items()}
        return cylspline_node_vjp(self.tables, self._coefs, grad_nodes, phi=phi)

    def _node_keys(self) -> List[int]:
        return sorted(int(m) for m in self._coefs.phi)

    def node_parameters(self, device=None) -> List[torch.Tensor]:
        """The harmonic grids Phi_m(R, z) on the coefficient file's grid, one FP64 CUDA
        leaf tensor with requires_grad per m in ascending order (the layout of
        set_node_tables).  The same tensors on every call.  The grids, Rscale and the
        outer asymptote stay those of construction (as in node_gradients)."""
        p = self.__dict__.get("_node_params")
        if p:
            return list(p)
        if self._coefs is None:
            raise ValueError("node_parameters() needs the coefficients the object was built from")
        dev = torch.device(device) if device is not None else _cuda_device()
        cur = self.__dict__.get("_phi_nodes")
        out = []
        for m in self._node_keys():
            if cur is not None:
                v = cur[m]
            else:
                v = self._coefs.phi[m] if m in self._coefs.phi else self._coefs.phi[str(m)]
                v = torch.from_numpy(np.ascontiguousarray(v, dtype=np.float64))
            out.append(v.detach().to(dev, torch.float64).clone().requires_grad_(True))
        return self._track_nodes(out)

    def _apply_nodes(self, p) -> None:
        self._set_grids(dict(zip(self._node_keys(), p)))

    def _grads_of_nodes(self, grad_nodes: torch.Tensor) -> List[torch.Tensor]:
        """dL/dPhi_m per m (ascending), the layout of node_parameters()."""
        d = self.node_gradients(grad_nodes)
        dev = self._node_params[0].device
        return [torch.as_tensor(np.ascontiguousarray(d[m]), device=dev) for m in self._node_keys()]

    def set_node_tables(self, phi: dict) -> None:
        """Replace the harmonic grids Phi_m(R, z) -- {m: (nR, nz) device tensors on the
        coefficient file's grid} -- rebuilding the node and cell tables on the GPU, in
        place (CUDA graphs captured over this potential stay valid): the z mirroring,
        the log-scaling and the node-derivative splines run as device operations.  The
        grids, Rscale, the log-scaling choice and the outer asymptote (fitted at
        construction) are kept, as node_gradients() holds them.  Not differentiable
        itself: use node_gradients() on the adjoint's table gradient."""
        self._set_grids(phi)
        keys = self._node_keys()
        self._refresh_tracked([self._phi_nodes[m] for m in keys])

    def _set_grids(self, phi: dict) -> None:
        from .diff_tables import _spline_deriv_matrix
        t = self.tables
        keys = sorted(int(m) for m in self._coefs.phi)
        if sorted(int(m) for m in phi) != keys:
            raise ValueError(f"set_node_tables() needs the harmonics {keys}")
        shape = np.asarray(self._coefs.phi[keys[0]]).shape
        dev = next(iter(phi.values())).device
        dev = dev if dev.type == "cuda" else _cuda_device()
        f64 = dict(dtype=torch.float64, device=dev)
        grids = {}
        for m in keys:
            v = phi[m] if m in phi else phi[str(m)]
            if tuple(v.shape) != tuple(shape):
                raise ValueError(f"harmonic {m}: shape {tuple(v.shape)}, expected {shape}")
            v = v.detach().to(**f64)
            if np.asarray(self._coefs.z_grid)[0] == 0:          # half-space grid: mirror
                v = torch.cat([v[:, 1:].flip(1), v], dim=1)
            grids[m] = v
        if t.log_scaling:
            p0 = grids[0]
            if not bool((p0 < 0).all()):
                raise ValueError("the m=0 grid must stay negative (the tables are log-scaled)")
            fs = {m: (torch.log(-p0) if m == 0 else g / p0) for m, g in grids.items()}
        else:
            fs = grids
        mats = self.__dict__.setdefault("_deriv_mats", {})
        if dev not in mats:
            nR = len(t.lR_grid)
            DR = _spline_deriv_matrix(t.lR_grid, ((1, np.zeros(nR)), "natural"))
            Dz = _spline_deriv_matrix(t.lz_grid, "natural")
            mats[dev] = (torch.from_numpy(DR).to(**f64), torch.from_numpy(Dz).to(**f64))
        DR, Dz = mats[dev]
        nodes = []
        for m in t.m_arr:
            f = fs[int(m)]
            fy = f @ Dz.T
            nodes.append(torch.stack([f, DR @ f, fy, DR @ fy], dim=-1))
        nd = torch.stack(nodes, 0)[torch.as_tensor(t.harmonic_order(), device=dev)]
        corners = [nd[:, :-1, :-1], nd[:, :-1, 1:], nd[:, 1:, :-1], nd[:, 1:, 1:]]
        rec = torch.stack(corners, dim=3).permute(1, 2, 0, 4, 3).reshape(-1, 16).contiguous()
        r32 = torch.zeros((rec.shape[0], 20), dtype=torch.float32, device=dev)
        r32.view(torch.float64)[:, 0] = rec[:, 0]
        r32[:, 2:5] = (rec[:, 1:4] - rec[:, 0:1]).to(torch.float32)
        r32[:, 5:17] = rec[:, 4:16].to(torch.float32)
        self._phi_nodes = {m: (phi[m] if m in phi else phi[str(m)]).detach().to(**f64).clone()
                           for m in keys}
        self._cell_override = (rec.reshape(-1), r32.reshape(-1))
        for cdev, (_, keep) in self.__dict__.get("_dev_cache", {}).items():
            keep[0].copy_(rec.reshape(-1).to(cdev), non_blocking=True)
            keep[1].copy_(r32.reshape(-1).to(cdev), non_blocking=True)

    @classmethod
    def from_file(cls, path, **kw) -> "CylSplinePotentialGPU":
        return cls(read_coefs(path if isinstance(path, Path) else str(path)), **kw)

    def _upload(self, dev):
        t = self.tables
        over = self.__dict__.get("_cell_override")
        if over is not None:
            cells, cells32 = over[0].to(dev).clone(), over[1].to(dev).clone()
        else:
            cells = torch.from_numpy(self._cells).to(dev)
            cells32 = torch.from_numpy(self._cells32).to(dev)
        m = torch.from_numpy(self._m).to(dev)
        lR = torch.from_numpy(np.ascontiguousarray(t.lR_grid)).to(dev)
        lz = torch.from_numpy(np.ascontiguousarray(t.lz_grid)).to(dev)
        W = torch.from_numpy(np.ascontiguousarray(t.W_outer)).to(dev)
        c = _lib.AgbComponent()
        c.kind = self.kind
        c.n_lm = t.n_harm
        c.n_int = len(t.lR_grid)
        c.nz = len(t.lz_grid)
        c.lmax = t.lmax_outer
        c.log_scaling = t.log_scaling
        c.layout = 1
        c.table = cells.data_ptr()
        c.table32 = cells32.data_ptr()
        c.lm = m.data_ptr()
        c.grid_a = lR.data_ptr()
        c.grid_b = lz.data_ptr()
        c.extra = W.data_ptr()
        c.p[0] = t.Rscale
        c.p[1] = t.r0_outer
        c.p[2] = float(t.mmax_outer)
        return c, (cells, cells32, m, lR, lz, W)


# ---------------------------------------------------------------------------
# Composite / Evolving / Shifted / Scaled
# ---------------------------------------------------------------------------

class CompositePotentialGPU(_GPUPotBase):
    """Sum of GPU potentials (gpu_potential.py:1439-1529), evaluated in one launch."""

    def __init__(self, components: list) -> None:
        if not components:
            raise ValueError("CompositePotentialGPU requires at least one component.")
        self._components = list(components)

    def __repr__(self):
        return f"CompositePotentialGPU({len(self._components)} components)"

    @classmethod
    def from_agama(cls, pot) -> "CompositePotentialGPU":
        return cls([MultipolePotentialGPU.from_agama(pot)])

    def _leaves(self, t: float) -> List[Leaf]:
        out: List[Leaf] = []
        for c in self._components:
            out.extend(c._leaves(t))
        return out


class EvolvingPotentialGPU(_GPUPotBase):
    """Snapshots at fixed times, linearly interpolated (or nearest) in time.

    Semantics of gpu_potential.py:1536-1644: bracket [t_i, t_i+1] by binary
    search, outputs = (1-alpha) * snapshot_i + alpha * snapshot_i+1; alpha 0/1
    use one snapshot; ``interpolate=False`` or one snapshot -> nearest.
    Both snapshots are summed inside the fused kernel.
    """

    def __init__(self, potentials: list, times, interpolate: bool = True) -> None:
        if len(potentials) != len(times):
            raise ValueError(f"len(potentials)={len(potentials)} != len(times)={len(times)}")
        if len(potentials) < 1:
            raise ValueError("Need at least one snapshot.")
        self._pots = list(potentials)
        self._times = np.asarray(times, dtype=np.float64)
        self._interpolate = interpolate

    def _time_data(self) -> np.ndarray:
        """AGB_OP_EVOLVE data: [n, interpolate, times]."""
        interp = 1.0 if (self._interpolate and len(self._pots) > 1) else 0.0
        return np.concatenate([[float(len(self._times)), interp], self._times])

    def _bracket(self, t: float):
        times = self._times
        n = len(times)
        if t <= times[0] or n == 1:
            return 0, 0.0
        if t >= times[-1]:
            return n - 2, 1.0
        lo, hi = 0, n - 2
        while lo < hi:
            mid = (lo + hi) // 2
            if times[mid + 1] <= t:
                lo = mid + 1
            else:
                hi = mid
        return lo, float((t - times[lo]) / (times[lo + 1] - times[lo]))

    def _weights(self, t: float):
        """[(snapshot index, weight)] used at time t."""
        if len(self._pots) == 1 or not self._interpolate:
            return [(int(np.argmin(np.abs(self._times - t))), 1.0)]
        i, a = self._bracket(t)
        if a == 0.0:
            return [(i, 1.0)]
        if a == 1.0:
            return [(i + 1, 1.0)]
        return [(i, 1.0 - a), (i + 1, a)]

    def _leaves(self, t: float) -> List[Leaf]:
        out: List[Leaf] = []
        for i, w in self._weights(t):
            for c, s, g, a in self._pots[i]._leaves(t):
                out.append((c, s, g, a * w))
        return out


class ShiftedPotentialGPU(_GPUPotBase):
    """``inner`` evaluated at x - center(t) (gpu_potential.py:1651-1764).

    center: (3,) static; (T,4) rows [t, x, y, z] -> not-a-knot cubic spline;
    (T,>=7) rows [t, x, y, z, vx, vy, vz] -> cubic Hermite.  Outside the time
    range the centre is extrapolated linearly from the end value and slope.
    """

    def __init__(self, inner, center) -> None:
        self._inner = inner
        center = np.asarray(center, dtype=np.float64)
        self._center_arr = center.copy()
        if center.ndim == 1 and center.shape == (3,):
            self._is_static = True
            self._center_static = center
        elif center.ndim == 2 and center.shape[1] >= 4:
            self._is_static = False
            if not np.all(center[1:, 0] > center[:-1, 0]):
                center = center[center[:, 0].argsort()]
            self._times = center[:, 0]
            pos = center[:, 1:4]
            if center.shape[1] >= 7:
                self._spline = CubicHermiteSpline(self._times, pos, center[:, 4:7])
            else:
                self._spline = CubicSpline(self._times, pos, bc_type="not-a-knot")
            self._t0, self._tN = self._times[0], self._times[-1]
            self._pos0, self._posN = self._spline(self._t0), self._spline(self._tN)
            self._vel0, self._velN = self._spline(self._t0, 1), self._spline(self._tN, 1)
        else:
            raise ValueError("Center must be (3,) or (T, 4) or (T, 7).")

    def _time_data(self) -> np.ndarray:
        """AGB_OP_SHIFT data: [0, c] static, or [1, T, t0, tN, p0, pN, v0, vN, x, c]."""
        if self._is_static:
            return np.concatenate([[0.0], self._center_static])
        sp = self._spline
        T = len(sp.x)
        return np.concatenate([[1.0, float(T), self._t0, self._tN], self._pos0, self._posN,
                               self._vel0, self._velN, sp.x, np.asarray(sp.c).reshape(-1)])

    def _center_at(self, t: float) -> np.ndarray:
        if self._is_static:
            return self._center_static
        if t < self._t0:
            return self._pos0 + self._vel0 * (t - self._t0)
        if t > self._tN:
            return self._posN + self._velN * (t - self._tN)
        return self._spline(t)

    def _leaves(self, t: float) -> List[Leaf]:
        c = np.asarray(self._center_at(t), dtype=np.float64)
        return [(comp, s, g + s * c, a) for comp, s, g, a in self._inner._leaves(t)]


class ScaledPotentialGPU(_GPUPotBase):
    """Phi_s(x,t) = a(t) s(t) Phi(x s(t)), s = 1/scale(t) (gpu_potential.py:1767-1918).

    scale: float; (T,2) rows [t, scale]; (T,3) rows [t, ampl, scale]; cubic
    not-a-knot splines with linear extrapolation.  Force scales by a s^2,
    Hessian and density by a s^3.
    """

    def __init__(self, inner, scale, ampl: float = 1.0) -> None:
        self._inner = inner
        if isinstance(scale, (int, float)):
            arr = None
        else:
            arr = np.asarray(scale, dtype=np.float64)
            if arr.ndim == 0:
                scale = float(arr)
                arr = None
        self._scale_arr = None if arr is None else arr.copy()
        if arr is None:
            self._is_static = True
            self._scale_val = float(scale)
            self._ampl_val = float(ampl)
            return
        if arr.ndim != 2 or arr.shape[1] not in (2, 3):
            raise ValueError("scale must be a float, (T,2) array [t, scale(t)], "
                             "or (T,3) array [t, ampl(t), scale(t)]. "
                             f"Got shape {arr.shape}.")
        times = arr[:, 0]
        if not np.all(times[1:] > times[:-1]):
            arr = arr[np.argsort(times)]
            times = arr[:, 0]
        self._is_static = False
        self._times = times
        self._t0, self._tN = float(times[0]), float(times[-1])
        self._scale_spl = CubicSpline(times, arr[:, -1], bc_type="not-a-knot")
        self._scale0 = float(self._scale_spl(self._t0))
        self._scaleN = float(self._scale_spl(self._tN))
        self._dscale0 = float(self._scale_spl(self._t0, 1))
        self._dscaleN = float(self._scale_spl(self._tN, 1))
        if arr.shape[1] == 3:
            self._ampl_spl = CubicSpline(times, arr[:, 1], bc_type="not-a-knot")
            self._ampl0 = float(self._ampl_spl(self._t0))
            self._amplN = float(self._ampl_spl(self._tN))
            self._dampl0 = float(self._ampl_spl(self._t0, 1))
            self._damplN = float(self._ampl_spl(self._tN, 1))
        else:
            self._ampl_spl = None
        self._ampl_val = float(ampl)

    def _time_data(self) -> np.ndarray:
        """AGB_OP_SCALE data: [0, scale, ampl] static, or [1, T, t0, tN, scale0, scaleN,
        dscale0, dscaleN, has_ampl, ampl, ampl0, amplN, dampl0, damplN, x, cs(, ca)]."""
        if self._is_static:
            return np.array([0.0, self._scale_val, self._ampl_val])
        sp = self._scale_spl
        has = self._ampl_spl is not None
        ends = [self._ampl0, self._amplN, self._dampl0, self._damplN] if has else [0.0] * 4
        parts = [[1.0, float(len(sp.x)), self._t0, self._tN, self._scale0, self._scaleN,
                  self._dscale0, self._dscaleN, 1.0 if has else 0.0, self._ampl_val] + ends,
                 sp.x, np.asarray(sp.c).reshape(-1)]
        if has:
            parts.append(np.asarray(self._ampl_spl.c).reshape(-1))
        return np.concatenate(parts)

    def _sa(self, t: float):
        """(s, a) = (1/scale(t), ampl(t))."""
        if self._is_static:
            return 1.0 / self._scale_val, self._ampl_val
        if t < self._t0:
            sc = self._scale0 + self._dscale0 * (t - self._t0)
        elif t > self._tN:
            sc = self._scaleN + self._dscaleN * (t - self._tN)
        else:
            sc = float(self._scale_spl(t))
        s = 1.0 / sc
        if self._ampl_spl is None:
            a = self._ampl_val
        elif t < self._t0:
            a = self._ampl0 + self._dampl0 * (t - self._t0)
        elif t > self._tN:
            a = self._amplN + self._damplN * (t - self._tN)
        else:
            a = float(self._ampl_spl(t))
        return s, a

    def _leaves(self, t: float) -> List[Leaf]:
        s, a = self._sa(t)
        return [(comp, sg * s, g, a * s * amp) for comp, sg, g, amp in self._inner._leaves(t)]
