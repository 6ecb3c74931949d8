"""Many independent potentials, each with its own particles, in one launch.

A code that follows hundreds of systems at once -- one potential per stream
progenitor, satellite or simulation snapshot, each with a few thousand to a
few hundred thousand particles -- would call ``force`` once per system per
step with the reference's classes: hundreds of small launches per step.
``BatchedPotentialGPU`` stacks the systems' particles into one (N,3) array
(unit u owns rows ``offsets[u]:offsets[u+1]``) and evaluates all of them with
one persistent kernel fed by a device work queue (``agb_batch_create`` /
``agb_batch_eval`` in libagb.so).  Results equal the per-unit calls point by
point.  The object has the evaluation API of the other classes (potential,
force, density, forceDeriv, evalDeriv, eval) over the stacked array, and the
leapfrog integrator accepts it (its steps are captured in CUDA graphs).

The units must not depend on time: the plan freezes their leaves when it is
built.  Position derivatives (the VJP) are not batched.
"""
from __future__ import annotations

import ctypes
from typing import Optional, Sequence

import numpy as np
import torch

from . import _lib
from .potentials import _GPUPotBase, _PRECISIONS, _cuda_device


class BatchedPotentialGPU(_GPUPotBase):
    """``BatchedPotentialGPU(potentials, counts, tile_points=4096)``.

    potentials: one potential (any static tree: Multipole, CylSpline, analytic,
    Composite, Shifted/Scaled with fixed parameters) per unit; counts: the
    number of particles of each unit, stacked in this order.
    """

    def __init__(self, potentials: Sequence, counts: Sequence[int], tile_points: int = 4096,
                 precision: Optional[str] = None, presort: bool = True,
                 stage: bool = True) -> None:
        from .integrate import is_static
        pots = list(potentials)
        counts = np.asarray(counts, dtype=np.int64)
        if len(pots) == 0 or len(pots) != len(counts):
            raise ValueError("need one particle count per potential (and at least one unit)")
        if (counts < 0).any():
            raise ValueError("particle counts must be non-negative")
        for i, p in enumerate(pots):
            if not is_static(p):
                raise ValueError(f"unit {i} depends on time; batched plans freeze the leaves")
        self._units = pots
        self.counts = counts
        self.offsets = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
        self.n_points = int(self.offsets[-1])
        self.tile_points = int(tile_points)
        self.precision = precision
        # device-wide pre-sort of every unit's points by interval before the work-queue
        # launch (agb_batch_eval_ws), in a workspace the object keeps per device,
        # precision and stream
        self.presort = bool(presort)
        # mixed precision with sorted points: bulk-copy each tile's interval rows of
        # its unit's Multipole into shared memory (AGB_OUT_STAGE; config 4: 13.41 ->
        # 12.62 ms per force evaluation)
        self.stage = bool(stage)
        # set by the integrators while they keep the particles in sort_order(): the
        # rows are then evaluated in order (no pre-sort, no in-tile sort)
        self._rows_in_order = False
        # AGB_OUT_STAGE_GIVE_UP in tests of the bounded waits' failure path (else 0)
        self._stage_test_flags = 0
        self._plans = {}
        self._ws = {}

    def __add__(self, other):
        raise TypeError("a batch of independent potentials cannot be summed")

    __radd__ = __add__

    def unit_rows(self, u: int) -> slice:
        """Rows of the stacked arrays that belong to unit u."""
        return slice(int(self.offsets[u]), int(self.offsets[u + 1]))

    def tiles(self, precision: Optional[str] = None, device=None) -> int:
        dev = _cuda_device(device)
        prec = _PRECISIONS[precision or self.precision or _default()]
        return int(_lib.lib.agb_batch_tiles(self._plan(dev, prec)))

    def _plan(self, dev: torch.device, prec: int) -> ctypes.c_void_p:
        key = (dev.index, prec)
        plan = self._plans.get(key)
        if plan is not None:
            return plan
        comps, index, leaves, unit_off = [], {}, [], [0]
        for pot in self._units:
            for c, sigma, gamma, ampl in pot._leaves(0.0):
                if id(c) not in index:
                    index[id(c)] = len(comps)
                    comps.append(c._device_component(dev))
                leaves.append((index[id(c)], float(sigma), [float(g) for g in gamma], float(ampl)))
            unit_off.append(len(leaves))
        comp_arr = (_lib.AgbComponent * len(comps))(*comps)
        leaf_arr = (_lib.AgbLeaf * len(leaves))()
        for i, (ci, sigma, gamma, ampl) in enumerate(leaves):
            lf = leaf_arr[i]
            lf.comp, lf.sigma, lf.ampl = ci, sigma, ampl
            lf.gamma[0], lf.gamma[1], lf.gamma[2] = gamma
        uoff = (ctypes.c_int32 * len(unit_off))(*unit_off)
        poff = (ctypes.c_int64 * len(self.offsets))(*[int(o) for o in self.offsets])
        handle = ctypes.c_void_p()
        with torch.cuda.device(dev):
            rc = _lib.lib.agb_batch_create(comp_arr, len(comps), leaf_arr, uoff, len(self._units),
                                           poff, prec, self.tile_points, ctypes.byref(handle))
        _lib.check(rc, "agb_batch_create")
        self._plans[key] = handle
        return handle

    def _launch(self, arr: torch.Tensor, t: float, mode: int, want_phi: bool,
                precision: Optional[str] = None, out=None):
        n = arr.shape[0]
        if n != self.n_points:
            raise ValueError(f"the batch holds {self.n_points} particles, got {n} positions")
        if mode == _lib.MODE_VJP:
            raise NotImplementedError("position derivatives are not batched")
        dev = arr.device
        prec = _PRECISIONS[precision or self.precision or _default()]
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
        plan = self._plan(dev, prec)
        ptr = lambda a: None if a is None else a.data_ptr()  # noqa: E731
        stream = torch.cuda.current_stream(dev).cuda_stream
        ws, nws = None, 0
        flags = _lib.OUT_NEGATE | (_lib.OUT_NO_BINNING if self._rows_in_order else 0)
        if self.stage:
            flags |= _lib.OUT_STAGE | self._stage_test_flags
        if self.presort and not self._rows_in_order:
            nws = int(_lib.lib.agb_batch_workspace_bytes(plan, mode))
            if nws:
                key = (dev.index, prec, stream)
                ws = self._ws.get(key)
                if ws is None or ws.numel() < nws:
                    ws = torch.empty(nws, dtype=torch.uint8, device=dev)
                    self._ws[key] = ws
        rc = _lib.lib.agb_batch_eval_ws(plan, arr.data_ptr(), mode, ptr(phi), ptr(grad), ptr(hess),
                                        ptr(rho), flags, ptr(ws), nws,
                                        ctypes.c_void_p(stream))
        _lib.check(rc, "agb_batch_eval_ws")
        return phi, grad, hess, rho

    def stage_errors(self, precision: Optional[str] = None, device=None) -> int:
        """1 when a staged launch gave up waiting for a bulk copy (and read global
        memory instead; results are unaffected), else 0."""
        dev = _cuda_device(device)
        prec = _PRECISIONS[precision or self.precision or _default()]
        rc = int(_lib.lib.agb_batch_stage_errors(self._plan(dev, prec)))
        if rc < 0:
            _lib.check(rc, "agb_batch_stage_errors")
        return rc

    def sort_order(self, xyz: torch.Tensor, precision: Optional[str] = None) -> Optional[torch.Tensor]:
        """(N,) int64 device permutation: rows in the order the batch evaluates best --
        each unit's particles by the radial interval of its Multipole, inside the unit's
        own rows (xyz[order] keeps unit u in unit_rows(u)); None when the units cannot
        be sorted.  The leapfrog integrator keeps the particles in this order during a
        run and evaluates them without sorting."""
        arr = xyz.to(torch.float64).contiguous()
        if arr.shape[0] != self.n_points:
            raise ValueError(f"the batch holds {self.n_points} particles, got {arr.shape[0]}")
        dev = arr.device
        prec = _PRECISIONS[precision or self.precision or _default()]
        plan = self._plan(dev, prec)
        nws = int(_lib.lib.agb_batch_sort_workspace_bytes(plan))
        if nws == 0:
            return None
        ws = torch.empty(nws, dtype=torch.uint8, device=dev)
        perm = torch.empty(self.n_points, dtype=torch.int32, device=dev)
        rc = _lib.lib.agb_batch_sort(plan, arr.data_ptr(), perm.data_ptr(), ws.data_ptr(), nws,
                                     ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream))
        _lib.check(rc, "agb_batch_sort")
        return perm.long()

    def _vjp(self, *args, **kw):
        raise NotImplementedError("position derivatives are not batched")

    def _leaves(self, t: float):
        raise TypeError("a batch is not one potential tree; evaluate it as a whole")

    def _release_plans(self) -> None:
        """Destroy the device plans (after the device has finished using them)."""
        plans = getattr(self, "_plans", {})
        for (dev_index, _), h in plans.items():
            try:
                with torch.cuda.device(dev_index):
                    torch.cuda.synchronize()
                    _lib.lib.agb_batch_destroy(h)
            except Exception:   # interpreter shutdown
                pass
        self._plans = {}
        self._ws = {}
        # CUDA graphs captured over the old plans must not replay them
        self.plan_generation = getattr(self, "plan_generation", 0) + 1

    def __del__(self):
        self._release_plans()


def _default() -> str:
    from . import potentials
    return potentials._default_precision
