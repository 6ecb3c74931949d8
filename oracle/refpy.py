"""Test infrastructure only (oracle): run the reference's own Python on the CPU.

Imports the reference wrapper (``gpu_potential.py`` and
``_analytic_potentials.py``) with a numpy-backed stand-in for ``cupy`` so that

* the reference's table builders (``_build_multipole_data``,
  gpu_potential.py:408-631; ``_build_cylspline_data``, gpu_potential.py:1143-1253)
  run unchanged on numpy arrays;
* ``cp.RawModule`` kernels (``_multipole_potential_kernel.cu``,
  ``_cylspl_potential_kernel.cu``) are routed to ``oracle/_ref/libref.so``, the
  reference's own ``.cu`` files compiled as host C++ (see ``oracle/Makefile``);
* every ``cp.ElementwiseKernel`` body (the analytic profiles,
  _analytic_potentials.py:176-1126) is captured as text and compiled, unchanged,
  into a host C++ library under ``oracle/_ref/``.

With that, the reference's classes (Composite, Evolving, Shifted, Scaled, the
factory) run as-is on numpy input.  This module needs the reference sources:
the directory named by ``AGB_REFERENCE``, else the checkout this recipe was
written against (``DEFAULT_REFERENCE``; the one place that names it).  It is
used only to generate golden vectors and reference-built tables and by CPU
tests that skip when the sources are absent.  The product never imports it.
"""
from __future__ import annotations

import ctypes
import hashlib
import os
import re
import subprocess
import sys
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
DEFAULT_REFERENCE = "/root/reference"
REF_DIR = Path(os.environ.get("AGB_REFERENCE", DEFAULT_REFERENCE))
REF_LIB = HERE / "_ref" / "libref.so"


def available() -> bool:
    return (REF_DIR / "gpu_potential.py").exists()


# ---------------------------------------------------------------------------
# host-compiled reference kernels
# ---------------------------------------------------------------------------
_lib = None


def ref_lib():
    global _lib
    if _lib is None:
        if not REF_LIB.exists():
            subprocess.run(["make", "-s", "-C", str(HERE), "ref", f"REF={REF_DIR}"], check=True)
        _lib = ctypes.CDLL(str(REF_LIB))
        _lib.ref_multipole_eval.restype = ctypes.c_int
        _lib.ref_cylspl_eval.restype = ctypes.c_int
    return _lib


def _p(a):
    if a is None or (isinstance(a, np.ndarray) and a.size == 0):
        return ctypes.c_void_p(0)
    assert a.flags["C_CONTIGUOUS"], "reference kernels need contiguous arrays"
    return ctypes.c_void_p(a.ctypes.data)


def _d(v):
    return ctypes.c_double(float(v))


def _i(v):
    return ctypes.c_int(int(v))


_MP_KERNELS = {
    "multipole_potential_kernel": 0,
    "multipole_force_kernel": 1,
    "multipole_hess_kernel": 2,
    "multipole_density_kernel": 3,
}
_CS_KERNELS = {
    "cylspl_potential_kernel": 0,
    "cylspl_force_kernel": 1,
    "cylspl_hess_kernel": 2,
}

NTHREADS = int(os.environ.get("AGB_REF_THREADS", "0"))


def _run_raw(name, args):
    lib = ref_lib()
    a = list(args)
    if name in _MP_KERNELS:
        mode = _MP_KERNELS[name]
        x, y, z, poly = a[0:4]
        sc = a[4:20]
        (logr_min, dlogr, inv_dlogr, n_int, n_lm, lmax, lm_l, lm_m, log_sc,
         invPhi0, in_s, in_U, in_W, out_s, out_U, out_W) = sc
        phi = grad = hess = rho = None
        inv4 = 0.0
        if mode in (0, 1):
            phi, grad, N = a[20], a[21], a[22]
        elif mode == 2:
            phi, grad, hess, N = a[20], a[21], a[22], a[23]
        else:
            inv4, rho, N = a[20], a[21], a[22]
        rc = lib.ref_multipole_eval(
            _i(mode), _p(x), _p(y), _p(z), _p(poly), _d(logr_min), _d(dlogr), _d(inv_dlogr),
            _i(n_int), _i(n_lm), _i(lmax), _p(lm_l), _p(lm_m), _i(log_sc), _d(invPhi0),
            _d(in_s), _d(in_U), _d(in_W), _d(out_s), _d(out_U), _d(out_W), _d(inv4),
            _p(phi), _p(grad), _p(hess), _p(rho), _i(N), _i(NTHREADS))
        assert rc == 0
        return
    if name in _CS_KERNELS:
        mode = _CS_KERNELS[name]
        (x, y, z, Rscale, lR, nR, lz, nz, nodes, n_harm, m_arr, mmax, log_sc,
         W, r0, lmax_o, mmax_o) = a[:17]
        rest = a[17:]
        phi = grad = hess = None
        if mode == 0:
            phi, N = rest
        elif mode == 1:
            phi, grad, N = rest
        else:
            phi, grad, hess, N = rest
        rc = lib.ref_cylspl_eval(
            _i(mode), _p(x), _p(y), _p(z), _d(Rscale), _p(lR), _i(nR), _p(lz), _i(nz),
            _p(nodes), _i(n_harm), _p(m_arr), _i(mmax), _i(log_sc), _p(W), _d(r0),
            _i(lmax_o), _i(mmax_o), _p(phi), _p(grad), _p(hess), _i(N), _i(NTHREADS))
        assert rc == 0
        return
    raise KeyError(name)


# ---------------------------------------------------------------------------
# captured ElementwiseKernel bodies, compiled as host C++
# ---------------------------------------------------------------------------
_EW = []          # (name, in_params, out_param, body)
_ew_lib = None
_RECORD = None    # list receiving (kernel name, scalar arguments) of each call, when set


class record_calls:
    """Context manager: collect the (name, scalars) of every ElementwiseKernel call
    the reference's code makes inside the block (the kernel still runs)."""

    def __enter__(self):
        global _RECORD
        self.calls = []
        _RECORD = self.calls
        return self.calls

    def __exit__(self, *exc):
        global _RECORD
        _RECORD = None
        return False


def _ew_source():
    # one OpenMP loop over points per kernel body, as the reference's kernels
    # compiled for the host are (ref_driver.cpp)
    out = ["#include <cmath>", "#include <cstdlib>", "using std::abs;", "typedef double T;"]
    for name, ins, outp, body in _EW:
        arrays = ins[:3]
        scalars = ins[3:]
        raw = outp.startswith("raw ")
        oname = outp.split()[-1]
        sig = ", ".join([f"const double* __{a}" for a in arrays] +
                        [f"double {s}" for s in scalars] + [f"double* __{oname}", "long n"])
        lines = [f'extern "C" void ew_{name}({sig}) {{',
                 "  #pragma omp parallel for schedule(static)",
                 "  for (long i = 0; i < n; i++) {",
                 *[f"    const double {a} = __{a}[i];" for a in arrays]]
        if raw:
            lines.append(f"    double* {oname} = __{oname};")
        else:
            lines.append(f"    double& {oname} = __{oname}[i];")
        lines.append("    {" + body + "\n    }")
        lines.append("  }\n}")
        out.append("\n".join(lines))
    return "\n\n".join(out)


def ew_lib():
    global _ew_lib
    if _ew_lib is None:
        src = _ew_source()
        h = hashlib.sha1(src.encode()).hexdigest()[:12]
        d = HERE / "_ref"
        d.mkdir(exist_ok=True)
        so = d / f"libref_analytic_{h}.so"
        if not so.exists():
            cpp = d / f"ref_analytic_{h}.cpp"
            cpp.write_text(src)
            cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
            subprocess.run([cxx, "-O3", "-march=x86-64-v3", "-fopenmp", "-fPIC", "-shared", "-o",
                            str(so), str(cpp)], check=True)
        _ew_lib = ctypes.CDLL(str(so))
    return _ew_lib


class _EWKernel:
    def __init__(self, in_params, out_params, body, name, **kw):
        self.ins = [p.split()[-1] for p in in_params.split(",")]
        self.out = out_params.strip()
        self.name = name
        _EW.append((name, self.ins, self.out, body))

    def __call__(self, *args):
        global _ew_lib
        n_in = len(self.ins)
        ins = list(args[:n_in])
        x, y, z = (np.ascontiguousarray(np.asarray(a, dtype=np.float64)) for a in ins[:3])
        n = x.size
        raw = self.out.startswith("raw ")
        if raw:
            out = args[n_in]
        else:
            out = np.empty(n, dtype=np.float64)
        if _RECORD is not None:
            _RECORD.append((self.name, [float(v) for v in ins[3:]]))
        fn = getattr(ew_lib(), "ew_" + self.name)
        fn(_p(x), _p(y), _p(z), *[_d(s) for s in ins[3:]], _p(out), ctypes.c_long(n))
        return out


# ---------------------------------------------------------------------------
# numpy-backed cupy stand-in
# ---------------------------------------------------------------------------
_RAW_RECORD = None    # list receiving (kernel name, arguments) of each launch, when set


class record_raw:
    """Context manager: collect the (name, arguments) of every RawKernel launch the
    reference's code makes inside the block (the kernel still runs)."""

    def __enter__(self):
        global _RAW_RECORD
        self.calls = []
        _RAW_RECORD = self.calls
        return self.calls

    def __exit__(self, *exc):
        global _RAW_RECORD
        _RAW_RECORD = None
        return False


class _RawKernel:
    def __init__(self, name):
        self.name = name

    def __call__(self, grid, block, args):
        if _RAW_RECORD is not None:
            _RAW_RECORD.append((self.name, tuple(args)))
        _run_raw(self.name, args)


class _RawModule:
    def __init__(self, code=None, backend=None, options=None, **kw):
        pass

    def get_function(self, name):
        return _RawKernel(name)


def _make_cupy_stub():
    cp = types.ModuleType("cupy")
    for nm in ("float64", "float32", "int32", "int64", "ndarray", "asarray", "empty", "zeros",
               "ones", "ascontiguousarray", "argsort", "empty_like", "zeros_like", "concatenate",
               "stack", "sqrt", "abs", "max", "min", "sum", "arange", "linspace", "allclose",
               "array"):
        setattr(cp, nm, getattr(np, nm))
    cp.asnumpy = lambda a: np.asarray(a)
    cp.RawModule = _RawModule
    cp.RawKernel = _RawKernel
    cp.ElementwiseKernel = _EWKernel
    cuda = types.SimpleNamespace(
        Stream=types.SimpleNamespace(null=types.SimpleNamespace(synchronize=lambda: None)),
        Event=None)
    cp.cuda = cuda
    return cp


_mods = None


def load():
    """Import the reference modules; returns (gpu_potential, _analytic_potentials)."""
    global _mods
    if _mods is not None:
        return _mods
    if not available():
        raise ImportError(f"reference sources not found under {REF_DIR}")
    saved = sys.modules.get("cupy")
    sys.modules["cupy"] = _make_cupy_stub()
    sys.path.insert(0, str(REF_DIR))
    try:
        import _analytic_potentials as ap  # noqa: F401
        import gpu_potential as gp
    finally:
        sys.path.remove(str(REF_DIR))
        if saved is not None:
            sys.modules["cupy"] = saved
    _mods = (gp, ap)
    return _mods


# ---------------------------------------------------------------------------
# coefficient containers the reference expects (it imports them from the
# external nbody_streams package, which is not vendored)
# ---------------------------------------------------------------------------
class MultipoleCoefs(types.SimpleNamespace):
    """Duck type for nbody_streams MultipoleCoefs: R_grid, phi, dphi_dr, lm_labels."""


class CylSplineCoefs(types.SimpleNamespace):
    """Duck type for nbody_streams CylSplineCoefs: R_grid, z_grid, phi {m: (nR,nz)}."""
