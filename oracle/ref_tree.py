"""Test infrastructure only (oracle): the reference's own potential trees, recorded
here and replayed on the CPU where the reference's Python is not available.

``export(obj)`` walks a tree of the REFERENCE's objects (built with its own
classes through ``oracle.refpy``: its table builders, its constructors) and
records, per node, what the reference's methods pass to their kernels:

* Multipole: the 17 table/scalar arguments of its kernel launches
  (``MultipolePotentialGPU._common_args``, gpu_potential.py:736-762) and the
  density constant, captured from a real launch;
* CylSpline: the 14 arguments of its launches (gpu_potential.py:1309-1322);
* analytic profiles: for each of ``_phi``, ``_grad``, ``_hess``, ``_rho`` the
  ElementwiseKernel it calls and that call's scalar arguments, captured from a
  real call (_analytic_potentials.py:176-1165), or "zeros" where the method
  returns zeros without a kernel (UniformAcceleration's Hessian and density);
* Shifted / Scaled: their scipy splines (breakpoints and coefficients) and the
  end values and slopes they cache for extrapolation (gpu_potential.py:1676-1714,
  :1787-1843);
* Evolving: snapshot times and the interpolation flag; Composite: children.

``RefTree`` evaluates such a record with the reference's kernel code compiled
for the host (``oracle/_ref/libref.so``: its two ``.cu`` files;
``oracle/_ref/libref_analytic_*.so``: its ElementwiseKernel bodies), OpenMP over
points, and composes the outputs the way the reference's classes do, restated
here from gpu_potential.py:
  Composite sums component outputs (:1476-1510);
  Evolving brackets t by bisection and lerps the outputs, nearest snapshot when
    not interpolating (:1559-1612, ``_lerp`` :1634-1636);
  Shifted evaluates its centre from a not-a-knot CubicSpline (T,4) or
    CubicHermiteSpline (T,7), linear extrapolation outside the track
    (:1676-1744);
  Scaled scales by s = 1/scale(t), a(t): Phi a s, F a s^2, dF a s^3
    (:1810-1900);
  eval(pot, acc, der) calls the same methods the reference's ``eval`` calls
    (:903-935, :1512-1529).

Records are written by ``python -m oracle.ref_tree build`` (run by
``__graft_entry__.build()`` where the reference sources are present) into
``oracle/_ref/``, which is not committed but travels with the repository
snapshot like ``libref.so``.  Nothing here imports ``agama_gpu_b200`` when it
evaluates; only ``build`` (which generates the seeded inputs) does.
"""
from __future__ import annotations

import ctypes
import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF_DIR = HERE / "_ref"
INV_4PIG = 1.0 / (4.0 * np.pi * 4.30091727067736e-06)

# records written by `build` (name -> what it holds)
TREES = {
    "config2": "time-dependent composite: Multipole lmax 32 x 100 nodes + MiyamotoNagai + "
               "DiskAnsatz + Shifted NFW on a (1000,4) track + Evolving 16 x lmax 16",
    "config3": "stream potential: Multipole lmax 16 x 64 nodes + MiyamotoNagai",
    "config4_units": "three units of the 512-potential batch (lmax, nodes, M, rs drawn as there)",
}


def record_path(name: str) -> Path:
    return REF_DIR / f"tree_{name}.npz"


# ---------------------------------------------------------------------------
# host-compiled reference code
# ---------------------------------------------------------------------------
_libs = {}


def _lib(fname: str):
    if fname not in _libs:
        lib = ctypes.CDLL(str(REF_DIR / fname))
        _libs[fname] = lib
    return _libs[fname]


def _p(a):
    if a is None:
        return ctypes.c_void_p(0)
    assert a.flags["C_CONTIGUOUS"]
    return ctypes.c_void_p(a.ctypes.data)


def _soa(xyz):
    return (np.ascontiguousarray(xyz[:, 0]), np.ascontiguousarray(xyz[:, 1]),
            np.ascontiguousarray(xyz[:, 2]))


# ---------------------------------------------------------------------------
# nodes
# ---------------------------------------------------------------------------
class _Node:
    def evalDeriv(self, xyz, t, nt):
        raise NotImplementedError

    def eval(self, xyz, pot=False, acc=False, der=False, t=0.0, nthreads=0):
        """The reference's ``eval``: evalDeriv when der, else force then potential
        (gpu_potential.py:903-935), or potential alone."""
        if not (pot or acc or der):
            raise ValueError("eval(): at least one of pot, acc, der must be True.")
        if der:
            p, f, d = self.evalDeriv(xyz, t, nthreads)
            out = [v for v, w in ((p, pot), (f, acc), (d, der)) if w]
        elif acc:
            f = self.force(xyz, t, nthreads)
            out = ([self.potential(xyz, t, nthreads)] if pot else []) + [f]
        else:
            out = [self.potential(xyz, t, nthreads)]
        return out[0] if len(out) == 1 else tuple(out)


class _Multipole(_Node):
    """Reference kernels _multipole_potential_kernel.cu:415-958 with the recorded
    arguments of MultipolePotentialGPU._common_args."""

    def __init__(self, rec, arrays, lib):
        self.poly = arrays["poly"]
        self.lm_l = arrays["lm_l"].astype(np.int32)
        self.lm_m = arrays["lm_m"].astype(np.int32)
        self.sc = rec["scalars"]          # 14 scalars in kernel order (ints as floats)
        self.inv4 = rec["inv_4piG"]
        self.lib = lib

    def _run(self, mode, xyz, nt):
        x, y, z = _soa(xyz)
        n = x.size
        phi = np.empty(n) if mode != 3 else None
        grad = np.empty(3 * n) if mode in (1, 2) else None
        hess = np.empty(6 * n) if mode == 2 else None
        rho = np.empty(n) if mode == 3 else None
        d, i = ctypes.c_double, ctypes.c_int
        s = self.sc
        rc = _lib(self.lib).ref_multipole_eval(
            i(mode), _p(x), _p(y), _p(z), _p(self.poly), d(s[0]), d(s[1]), d(s[2]), i(int(s[3])),
            i(int(s[4])), i(int(s[5])), _p(self.lm_l), _p(self.lm_m), i(int(s[6])), d(s[7]),
            d(s[8]), d(s[9]), d(s[10]), d(s[11]), d(s[12]), d(s[13]), d(self.inv4),
            _p(phi), _p(grad), _p(hess), _p(rho), i(n), i(nt))
        assert rc == 0
        return phi, grad, hess, rho

    def potential(self, xyz, t, nt):
        return self._run(0, xyz, nt)[0]

    def force(self, xyz, t, nt):
        return -self._run(1, xyz, nt)[1].reshape(-1, 3)

    def density(self, xyz, t, nt):
        return self._run(3, xyz, nt)[3]

    def forceDeriv(self, xyz, t, nt):
        _, g, h, _ = self._run(2, xyz, nt)
        return -g.reshape(-1, 3), -h.reshape(-1, 6)

    def evalDeriv(self, xyz, t, nt):
        p, g, h, _ = self._run(2, xyz, nt)
        return p, -g.reshape(-1, 3), -h.reshape(-1, 6)


class _CylSpline(_Node):
    """Reference kernels _cylspl_potential_kernel.cu:871-972 with the recorded
    arguments of CylSplinePotentialGPU._common_args."""

    def __init__(self, rec, arrays, lib):
        self.lR, self.lz = arrays["lR"], arrays["lz"]
        self.nodes, self.W = arrays["nodes"], arrays["W"]
        self.m_arr = arrays["m_arr"].astype(np.int32)
        self.sc = rec["scalars"]     # Rscale, nR, nz, n_harm, mmax, log_scaling, r0, lmax_o, mmax_o
        self.lib = lib

    def _run(self, mode, xyz, nt):
        x, y, z = _soa(xyz)
        n = x.size
        phi = np.empty(n)
        grad = np.empty(3 * n) if mode >= 1 else None
        hess = np.empty(6 * n) if mode == 2 else None
        d, i = ctypes.c_double, ctypes.c_int
        s = self.sc
        rc = _lib(self.lib).ref_cylspl_eval(
            i(mode), _p(x), _p(y), _p(z), d(s[0]), _p(self.lR), i(int(s[1])), _p(self.lz),
            i(int(s[2])), _p(self.nodes), i(int(s[3])), _p(self.m_arr), i(int(s[4])),
            i(int(s[5])), _p(self.W), d(s[6]), i(int(s[7])), i(int(s[8])), _p(phi), _p(grad),
            _p(hess), i(n), i(nt))
        assert rc == 0
        return phi, grad, hess

    def potential(self, xyz, t, nt):
        return self._run(0, xyz, nt)[0]

    def force(self, xyz, t, nt):
        return -self._run(1, xyz, nt)[1].reshape(-1, 3)

    def forceDeriv(self, xyz, t, nt):
        _, g, h = self._run(2, xyz, nt)
        return -g.reshape(-1, 3), -h.reshape(-1, 6)

    def evalDeriv(self, xyz, t, nt):
        p, g, h = self._run(2, xyz, nt)
        return p, -g.reshape(-1, 3), -h.reshape(-1, 6)

    def density(self, xyz, t, nt):
        raise NotImplementedError("CylSpline density is not recorded")


class _Analytic(_Node):
    """_AnalyticBase (_analytic_potentials.py:77-170) over the recorded kernel calls:
    potential = _phi, force = -_grad, forceDeriv = (-_grad, -_hess), density = _rho."""

    def __init__(self, rec, arrays, lib):
        self.calls = rec["calls"]         # {"_phi": [name, scalars] | "zeros", ...}
        self.lib = lib

    def _call(self, method, xyz, nt):
        spec = self.calls[method]
        n = len(xyz)
        width = {"_phi": 1, "_rho": 1, "_grad": 3, "_hess": 6}[method]
        if spec == "zeros":
            return np.zeros(n) if width == 1 else np.zeros((n, width))
        name, scalars = spec
        x, y, z = _soa(xyz)
        out = np.empty(n * width)
        fn = getattr(_lib(self.lib), "ew_" + name)
        fn(_p(x), _p(y), _p(z), *[ctypes.c_double(v) for v in scalars], _p(out),
           ctypes.c_long(n))
        return out if width == 1 else out.reshape(n, width)

    def potential(self, xyz, t, nt):
        return self._call("_phi", xyz, nt)

    def force(self, xyz, t, nt):
        return -self._call("_grad", xyz, nt)

    def density(self, xyz, t, nt):
        return self._call("_rho", xyz, nt)

    def forceDeriv(self, xyz, t, nt):
        return -self._call("_grad", xyz, nt), -self._call("_hess", xyz, nt)

    def evalDeriv(self, xyz, t, nt):
        return (self._call("_phi", xyz, nt), -self._call("_grad", xyz, nt),
                -self._call("_hess", xyz, nt))


class _Composite(_Node):
    def __init__(self, children):
        self.kids = children

    def _sum(self, meth, xyz, t, nt):
        out = getattr(self.kids[0], meth)(xyz, t, nt)
        for c in self.kids[1:]:
            v = getattr(c, meth)(xyz, t, nt)
            out = tuple(a + b for a, b in zip(out, v)) if isinstance(out, tuple) else out + v
        return out

    def potential(self, xyz, t, nt):
        return self._sum("potential", xyz, t, nt)

    def force(self, xyz, t, nt):
        return self._sum("force", xyz, t, nt)

    def density(self, xyz, t, nt):
        return self._sum("density", xyz, t, nt)

    def forceDeriv(self, xyz, t, nt):
        return self._sum("forceDeriv", xyz, t, nt)

    def evalDeriv(self, xyz, t, nt):
        return self._sum("evalDeriv", xyz, t, nt)


def _lerp(a, b, alpha):
    return a * (1.0 - alpha) + b * alpha


class _Evolving(_Node):
    def __init__(self, children, times, interpolate):
        self.kids = children
        self.times = np.asarray(times, dtype=np.float64)
        self.interp = bool(interpolate)

    def _bracket(self, t):
        times, n = self.times, len(self.times)
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

    def _nearest(self, t):
        return int(np.argmin(np.abs(self.times - t)))

    def _interp(self, meth, xyz, t, nt):
        if len(self.kids) == 1 or not self.interp:
            return getattr(self.kids[self._nearest(t)], meth)(xyz, t, nt)
        i, alpha = self._bracket(t)
        if alpha == 0.0:
            return getattr(self.kids[i], meth)(xyz, t, nt)
        if alpha == 1.0:
            return getattr(self.kids[i + 1], meth)(xyz, t, nt)
        return _lerp(getattr(self.kids[i], meth)(xyz, t, nt),
                     getattr(self.kids[i + 1], meth)(xyz, t, nt), alpha)

    def potential(self, xyz, t, nt):
        return self._interp("potential", xyz, t, nt)

    def force(self, xyz, t, nt):
        return self._interp("force", xyz, t, nt)

    def density(self, xyz, t, nt):
        return self._interp("density", xyz, t, nt)

    def _tuple(self, meth, xyz, t, nt):
        # forceDeriv / evalDeriv: at alpha == 1 the reference still lerps (weights 0, 1)
        if not self.interp or len(self.kids) == 1:
            return getattr(self.kids[self._nearest(t)], meth)(xyz, t, nt)
        i, alpha = self._bracket(t)
        v0 = getattr(self.kids[i], meth)(xyz, t, nt)
        if alpha == 0.0:
            return v0
        v1 = getattr(self.kids[i + 1], meth)(xyz, t, nt)
        return tuple(_lerp(a, b, alpha) for a, b in zip(v0, v1))

    def forceDeriv(self, xyz, t, nt):
        return self._tuple("forceDeriv", xyz, t, nt)

    def evalDeriv(self, xyz, t, nt):
        return self._tuple("evalDeriv", xyz, t, nt)


def _ppoly(arrays, key):
    """The reference's scipy spline (CubicSpline / CubicHermiteSpline are PPoly) from
    its recorded breakpoints and coefficients: evaluation is PPoly's, as there."""
    from scipy.interpolate import PPoly
    return PPoly(arrays[key + "_c"], arrays[key + "_x"])


class _Shifted(_Node):
    """ShiftedPotentialGPU._center_at (gpu_potential.py:1716-1734) on the recorded
    spline and end values."""

    def __init__(self, child, rec, arrays):
        self.kid = child
        self.static = arrays["center"] if rec["static"] else None
        if self.static is None:
            self.spl = _ppoly(arrays, "spline")
            self.t0, self.tN = rec["t0"], rec["tN"]
            self.p0, self.pN = arrays["pos0"], arrays["posN"]
            self.v0, self.vN = arrays["vel0"], arrays["velN"]

    def center(self, t):
        if self.static is not None:
            return self.static
        if t < self.t0:
            return self.p0 + self.v0 * (t - self.t0)
        if t > self.tN:
            return self.pN + self.vN * (t - self.tN)
        return self.spl(t)

    def _at(self, meth, xyz, t, nt):
        return getattr(self.kid, meth)(xyz - self.center(t), t, nt)

    def potential(self, xyz, t, nt):
        return self._at("potential", xyz, t, nt)

    def force(self, xyz, t, nt):
        return self._at("force", xyz, t, nt)

    def density(self, xyz, t, nt):
        return self._at("density", xyz, t, nt)

    def forceDeriv(self, xyz, t, nt):
        return self._at("forceDeriv", xyz, t, nt)

    def evalDeriv(self, xyz, t, nt):
        return self._at("evalDeriv", xyz, t, nt)


class _Scaled(_Node):
    """ScaledPotentialGPU._sa (gpu_potential.py:1845-1871) on the recorded splines and
    end values; outputs scaled as its methods do (:1873-1900)."""

    def __init__(self, child, rec, arrays):
        self.kid = child
        self.r = rec
        if not rec["static"]:
            self.sspl = _ppoly(arrays, "scale_spl")
            self.aspl = _ppoly(arrays, "ampl_spl") if rec["has_ampl_spl"] else None

    def _sa(self, t):
        r = self.r
        if r["static"]:
            return 1.0 / r["scale_val"], r["ampl_val"]
        if t < r["t0"]:
            sc = r["scale0"] + r["dscale0"] * (t - r["t0"])
        elif t > r["tN"]:
            sc = r["scaleN"] + r["dscaleN"] * (t - r["tN"])
        else:
            sc = float(self.sspl(t))
        s = 1.0 / sc
        if self.aspl is None:
            a = r["ampl_val"]
        elif t < r["t0"]:
            a = r["ampl0"] + r["dampl0"] * (t - r["t0"])
        elif t > r["tN"]:
            a = r["amplN"] + r["damplN"] * (t - r["tN"])
        else:
            a = float(self.aspl(t))
        return s, a

    def potential(self, xyz, t, nt):
        s, a = self._sa(t)
        return a * s * self.kid.potential(xyz * s, t, nt)

    def force(self, xyz, t, nt):
        s, a = self._sa(t)
        return a * s * s * self.kid.force(xyz * s, t, nt)

    def density(self, xyz, t, nt):
        s, a = self._sa(t)
        return a * s * s * s * self.kid.density(xyz * s, t, nt)

    def forceDeriv(self, xyz, t, nt):
        s, a = self._sa(t)
        F, dF = self.kid.forceDeriv(xyz * s, t, nt)
        return a * s * s * F, a * s * s * s * dF

    def evalDeriv(self, xyz, t, nt):
        s, a = self._sa(t)
        p, F, dF = self.kid.evalDeriv(xyz * s, t, nt)
        return a * s * p, a * s * s * F, a * s * s * s * dF


class RefTree:
    """A recorded reference tree; methods take (N,3) float64 numpy points."""

    def __init__(self, root: _Node, meta: dict):
        self.root = root
        self.meta = meta

    def potential(self, xyz, t=0.0, nthreads=0):
        return self.root.potential(np.ascontiguousarray(xyz, dtype=np.float64), t, nthreads)

    def force(self, xyz, t=0.0, nthreads=0):
        return self.root.force(np.ascontiguousarray(xyz, dtype=np.float64), t, nthreads)

    def density(self, xyz, t=0.0, nthreads=0):
        return self.root.density(np.ascontiguousarray(xyz, dtype=np.float64), t, nthreads)

    def forceDeriv(self, xyz, t=0.0, nthreads=0):
        return self.root.forceDeriv(np.ascontiguousarray(xyz, dtype=np.float64), t, nthreads)

    def evalDeriv(self, xyz, t=0.0, nthreads=0):
        return self.root.evalDeriv(np.ascontiguousarray(xyz, dtype=np.float64), t, nthreads)

    def eval(self, xyz, pot=False, acc=False, der=False, t=0.0, nthreads=0):
        return self.root.eval(np.ascontiguousarray(xyz, dtype=np.float64), pot, acc, der, t,
                              nthreads)


def hernquist_points(n: int, a: float = 10.0, seed: int = 0) -> np.ndarray:
    """The benchmark's isotropic Hernquist sample, r = a sqrt(u) / (1 - sqrt(u)), drawn
    with the same generator calls as the product's synthetic inputs (equal arrays;
    tested), so that evaluating a record needs nothing from the product."""
    rng = np.random.default_rng(seed)
    su = np.sqrt(rng.uniform(0.0, 1.0, n))
    r = a * su / (1.0 - su)
    u = rng.normal(size=(n, 3))
    return u / np.linalg.norm(u, axis=1)[:, None] * r[:, None]


def available(name: str) -> bool:
    return record_path(name).exists() and (REF_DIR / "libref.so").exists()


def load(name: str, index: int = 0) -> RefTree:
    """The recorded tree ``name`` (for records holding several trees, the index-th)."""
    with np.load(record_path(name), allow_pickle=False) as z:
        meta = json.loads(str(z["structure"]))
        arrays = {k: z[k] for k in z.files if k != "structure"}
    tree = meta["trees"][index]
    nodes = meta["nodes"]

    def build(i):
        rec = nodes[i]
        arr = {k[len(f"n{i}_"):]: v for k, v in arrays.items() if k.startswith(f"n{i}_")}
        kind = rec["type"]
        if kind == "multipole":
            return _Multipole(rec, arr, "libref.so")
        if kind == "cylspline":
            return _CylSpline(rec, arr, "libref.so")
        if kind == "analytic":
            return _Analytic(rec, arr, meta["analytic_lib"])
        if kind == "composite":
            return _Composite([build(c) for c in rec["children"]])
        if kind == "evolving":
            return _Evolving([build(c) for c in rec["children"]], arr["times"], rec["interpolate"])
        if kind == "shifted":
            return _Shifted(build(rec["children"][0]), rec, arr)
        if kind == "scaled":
            return _Scaled(build(rec["children"][0]), rec, arr)
        raise ValueError(f"unknown node type {kind}")

    return RefTree(build(tree["root"]), tree)


# ---------------------------------------------------------------------------
# recording (needs the reference sources: oracle.refpy)
# ---------------------------------------------------------------------------
class _Recorder:
    def __init__(self):
        self.nodes = []
        self.arrays = {}

    def _spline(self, i, key, spl):
        self.arrays[f"n{i}_{key}_c"] = np.ascontiguousarray(spl.c, dtype=np.float64)
        self.arrays[f"n{i}_{key}_x"] = np.ascontiguousarray(spl.x, dtype=np.float64)

    def add(self, obj) -> int:
        from oracle import refpy
        name = type(obj).__name__
        i = len(self.nodes)
        rec = {"class": name}
        self.nodes.append(rec)
        one = np.array([1.0]), np.array([2.0]), np.array([0.5])
        if name == "MultipolePotentialGPU":
            with refpy.record_raw() as calls:
                obj._launch_hess(*one, 1)
                obj._launch_density(*one, 1)
            # (x, y, z, poly, logr_min, dlogr, inv_dlogr, n_int, n_lm, lmax, lm_l, lm_m,
            #  log_scaling, invPhi0, inner_s, inner_U, inner_W, outer_s, outer_U, outer_W, ...)
            c = list(calls[0][1][3:20])
            rec.update(type="multipole", inv_4piG=float(calls[1][1][20]))
            self.arrays[f"n{i}_poly"] = np.ascontiguousarray(c[0], dtype=np.float64)
            self.arrays[f"n{i}_lm_l"] = np.asarray(c[7], dtype=np.int32)
            self.arrays[f"n{i}_lm_m"] = np.asarray(c[8], dtype=np.int32)
            rec["scalars"] = [float(v) for v in c[1:7] + [c[9]] + c[10:17]]
        elif name == "CylSplinePotentialGPU":
            with refpy.record_raw() as calls:
                obj._launch_hess(*one, 1)
            a = list(calls[0][1][3:17])
            rec["type"] = "cylspline"
            self.arrays[f"n{i}_lR"] = np.asarray(a[1], dtype=np.float64)
            self.arrays[f"n{i}_lz"] = np.asarray(a[3], dtype=np.float64)
            self.arrays[f"n{i}_nodes"] = np.ascontiguousarray(a[5], dtype=np.float64)
            self.arrays[f"n{i}_m_arr"] = np.asarray(a[7], dtype=np.int32)
            self.arrays[f"n{i}_W"] = np.asarray(a[10], dtype=np.float64)
            rec["scalars"] = [float(v) for v in (a[0], a[2], a[4], a[6], a[8], a[9], a[11],
                                                  a[12], a[13])]
        elif name == "CompositePotentialGPU":
            rec.update(type="composite", children=[self.add(c) for c in obj._components])
        elif name == "EvolvingPotentialGPU":
            rec.update(type="evolving", interpolate=bool(obj._interpolate),
                       children=[self.add(c) for c in obj._pots])
            self.arrays[f"n{i}_times"] = np.asarray(obj._times, dtype=np.float64)
        elif name == "ShiftedPotentialGPU":
            rec.update(type="shifted", static=bool(obj._is_static),
                       children=[self.add(obj._inner)])
            if obj._is_static:
                self.arrays[f"n{i}_center"] = np.asarray(obj._center_static, dtype=np.float64)
            else:
                self._spline(i, "spline", obj._spline)
                rec.update(t0=float(obj._t0), tN=float(obj._tN))
                for k in ("pos0", "posN", "vel0", "velN"):
                    self.arrays[f"n{i}_{k}"] = np.asarray(getattr(obj, "_" + k), dtype=np.float64)
        elif name == "ScaledPotentialGPU":
            rec.update(type="scaled", static=bool(obj._is_static),
                       children=[self.add(obj._inner)])
            if obj._is_static:
                rec.update(scale_val=float(obj._scale_val), ampl_val=float(obj._ampl_val))
            else:
                self._spline(i, "scale_spl", obj._scale_spl)
                rec.update(t0=float(obj._t0), tN=float(obj._tN), ampl_val=float(obj._ampl_val),
                           has_ampl_spl=obj._ampl_spl is not None,
                           **{k: float(getattr(obj, "_" + k))
                              for k in ("scale0", "scaleN", "dscale0", "dscaleN")})
                if obj._ampl_spl is not None:
                    self._spline(i, "ampl_spl", obj._ampl_spl)
                    rec.update(**{k: float(getattr(obj, "_" + k))
                                  for k in ("ampl0", "amplN", "dampl0", "damplN")})
        else:                      # an analytic profile of _analytic_potentials.py
            calls = {}
            for meth in ("_phi", "_grad", "_hess", "_rho"):
                with refpy.record_calls() as got:
                    getattr(obj, meth)(*one)
                calls[meth] = "zeros" if not got else list(got[0])
            rec.update(type="analytic", calls=calls)
        return i


def export(trees: list, path: Path) -> None:
    """Record reference objects: trees = [(reference root object, description)]."""
    from oracle import refpy
    rec = _Recorder()
    roots = [{"root": rec.add(obj), "description": desc} for obj, desc in trees]
    ew = Path(refpy.ew_lib()._name).name
    meta = {"nodes": rec.nodes, "trees": roots, "analytic_lib": ew}
    np.savez(path, structure=np.array(json.dumps(meta)), **rec.arrays)


def _build_all() -> None:
    """Record the reference's own trees of the measured workloads (seeded inputs)."""
    from oracle import refpy
    gp, ap = refpy.load()
    ROOT = HERE.parent
    if str(ROOT) not in sys.path:
        sys.path.insert(0, str(ROOT))
    from agama_gpu_b200.synthetic import composite_spec, config4_unit_specs, nfw_multipole
    REF_DIR.mkdir(exist_ok=True)
    # config 2: the composite_spec() tree, built by the reference's classes
    spec = composite_spec()
    root = gp.CompositePotentialGPU([
        gp.MultipolePotentialGPU(spec["main"]),
        ap.MiyamotoNagaiPotentialGPU(**spec["mn"]),
        ap.DiskAnsatzPotentialGPU(**spec["disk"]),
        gp.ShiftedPotentialGPU(ap.NFWPotentialGPU(**spec["nfw"]), spec["track"]),
        gp.EvolvingPotentialGPU([gp.MultipolePotentialGPU(s) for s in spec["snaps"]],
                                spec["times"], True),
    ])
    export([(root, TREES["config2"])], record_path("config2"))
    # config 3: lmax 16 x 64 nodes + Miyamoto-Nagai (the stream workload's potential)
    root3 = gp.CompositePotentialGPU([
        gp.MultipolePotentialGPU(nfw_multipole(lmax=16, n_nodes=64, seed=16)),
        ap.MiyamotoNagaiPotentialGPU(mass=5e10, scaleRadius=3.0, scaleHeight=0.3)])
    export([(root3, TREES["config3"])], record_path("config3"))
    # config 4: three units of the batch, drawn as the batch draws them
    units = [u for u in config4_unit_specs(512) if u["index"] in (0, 137, 511)]
    export([(gp.MultipolePotentialGPU(nfw_multipole(**u["coefs"])), f"unit {u['index']}")
            for u in units], record_path("config4_units"))


if __name__ == "__main__":
    if len(sys.argv) > 1 and sys.argv[1] == "build":
        _build_all()
        for nm in TREES:
            print(record_path(nm), record_path(nm).stat().st_size // 1024, "KiB")
    else:
        print(__doc__)
