"""Test infrastructure only: numpy front end of the C oracle (liboracle.so).

Inputs are (N,3) float64 arrays; outputs are the reference kernels' raw
quantities (Phi, grad Phi, Hessian of Phi, density).  Also exposes the
host-compiled reference kernels (oracle/_ref/libref.so) when present, which
bench.py times as the reference CPU implementation.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
REF = HERE / "_ref" / "libref.so"
_lib = None
_ref = None


def _load():
    global _lib
    if _lib is None:
        if not LIB.exists():
            subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
        _lib = ctypes.CDLL(str(LIB))
    return _lib


def ref_available() -> bool:
    return REF.exists()


def _refl():
    global _ref
    if _ref is None:
        _ref = ctypes.CDLL(str(REF))
        _ref.ref_max_threads.restype = ctypes.c_int
    return _ref


def _p(a):
    if a is None:
        return ctypes.c_void_p(0)
    assert a.flags["C_CONTIGUOUS"]
    return ctypes.c_void_p(a.ctypes.data)


def _soa(xyz):
    xyz = np.asarray(xyz, dtype=np.float64).reshape(-1, 3)
    return (np.ascontiguousarray(xyz[:, 0]), np.ascontiguousarray(xyz[:, 1]),
            np.ascontiguousarray(xyz[:, 2]))


def _outs(mode, n):
    phi = np.zeros(n) if mode != 3 else None
    grad = np.zeros((n, 3)) if mode in (1, 2) else None
    hess = np.zeros((n, 6)) if mode == 2 else None
    rho = np.zeros(n) if mode == 3 else None
    return phi, grad, hess, rho


def multipole(mode: int, xyz, t, nthreads: int = 0):
    """t: MultipoleTables (harmonic-major poly, lm_l, lm_m, scalars)."""
    x, y, z = _soa(xyz)
    n = x.size
    phi, grad, hess, rho = _outs(mode, n)
    sc = np.array(t.scalars(), dtype=np.float64)
    poly = np.ascontiguousarray(t.poly, dtype=np.float64)
    lm_l = np.ascontiguousarray(t.lm_l, dtype=np.int32)
    lm_m = np.ascontiguousarray(t.lm_m, dtype=np.int32)
    rc = _load().oracle_multipole(
        ctypes.c_int(mode), _p(x), _p(y), _p(z), _p(poly), _p(sc), ctypes.c_int(t.n_int),
        ctypes.c_int(t.n_lm), ctypes.c_int(t.lmax), _p(lm_l), _p(lm_m),
        ctypes.c_int(t.log_scaling), _p(phi), _p(grad), _p(hess), _p(rho),
        ctypes.c_int64(n), ctypes.c_int(nthreads))
    assert rc == 0
    return phi, grad, hess, rho


def cylspline(mode: int, xyz, t, nthreads: int = 0):
    """t: CylSplineTables (reference node layout)."""
    x, y, z = _soa(xyz)
    n = x.size
    phi, grad, hess, rho = _outs(mode, n)
    nodes = np.ascontiguousarray(t.node_arr, dtype=np.float64)
    m_arr = np.ascontiguousarray(t.m_arr, dtype=np.int32)
    lR = np.ascontiguousarray(t.lR_grid, dtype=np.float64)
    lz = np.ascontiguousarray(t.lz_grid, dtype=np.float64)
    W = np.ascontiguousarray(t.W_outer, dtype=np.float64)
    rc = _load().oracle_cylspline(
        ctypes.c_int(mode), _p(x), _p(y), _p(z), ctypes.c_double(t.Rscale), _p(lR),
        ctypes.c_int(len(lR)), _p(lz), ctypes.c_int(len(lz)), _p(nodes), ctypes.c_int(t.n_harm),
        _p(m_arr), ctypes.c_int(t.log_scaling), _p(W), ctypes.c_double(t.r0_outer),
        ctypes.c_int(t.lmax_outer), ctypes.c_int(t.mmax_outer), _p(phi), _p(grad), _p(hess),
        _p(rho), ctypes.c_int64(n), ctypes.c_int(nthreads))
    assert rc == 0
    return phi, grad, hess, rho


def analytic(kind: int, params, mode: int, xyz):
    x, y, z = _soa(xyz)
    n = x.size
    phi, grad, hess, rho = _outs(mode, n)
    p = np.zeros(16)
    p[:len(params)] = params
    rc = _load().oracle_analytic(ctypes.c_int(kind), _p(p), ctypes.c_int(mode), _p(x), _p(y),
                                 _p(z), _p(phi), _p(grad), _p(hess), _p(rho), ctypes.c_int64(n))
    assert rc == 0
    return phi, grad, hess, rho


def ref_multipole(mode: int, xyz, t, nthreads: int = 0):
    """The reference's own kernels compiled for the host (oracle/_ref/libref.so)."""
    from . import refpy  # noqa: F401  (argument marshalling lives there)
    x, y, z = _soa(xyz)
    n = x.size
    phi, grad, hess, rho = _outs(mode, n)
    d = ctypes.c_double
    i = ctypes.c_int
    sc = t.scalars()
    rc = _refl().ref_multipole_eval(
        i(mode), _p(x), _p(y), _p(z), _p(np.ascontiguousarray(t.poly)), d(sc[0]), d(sc[1]),
        d(sc[2]), i(t.n_int), i(t.n_lm), i(t.lmax), _p(np.ascontiguousarray(t.lm_l, dtype=np.int32)),
        _p(np.ascontiguousarray(t.lm_m, dtype=np.int32)), i(t.log_scaling), d(sc[3]), d(sc[4]),
        d(sc[5]), d(sc[6]), d(sc[7]), d(sc[8]), d(sc[9]),
        d(1.0 / (4.0 * np.pi * 4.30091727067736e-06)), _p(phi), _p(grad), _p(hess), _p(rho),
        i(n), i(nthreads))
    assert rc == 0
    return phi, grad, hess, rho


def eval_component(comp, mode: int, xyz):
    """One leaf component of the product's potential tree, evaluated by the oracle."""
    from agama_gpu_b200 import _lib as L
    if comp.kind == L.KIND_MULTIPOLE:
        return multipole(mode, xyz, comp.tables)
    if comp.kind == L.KIND_CYLSPLINE:
        return cylspline(mode, xyz, comp.tables)
    return analytic(comp.kind, list(comp._params()), mode, xyz)


def eval_potential(pot, mode: int, xyz, t: float = 0.0):
    """Oracle evaluation of a whole product potential at time t.

    Uses the product's host-side flattening into leaves (component, sigma,
    gamma, ampl) and sums A*Phi, A*sigma*grad, A*sigma^2*(H, rho) in leaf
    order -- the same sum the fused kernel forms.  Returns raw
    (Phi, grad Phi, Hessian of Phi, rho).
    """
    xyz = np.asarray(xyz, dtype=np.float64).reshape(-1, 3)
    n = len(xyz)
    phi, grad, hess, rho = np.zeros(n), np.zeros((n, 3)), np.zeros((n, 6)), np.zeros(n)
    for comp, sigma, gamma, ampl in pot._leaves(float(t)):
        p, g, h, r = eval_component(comp, mode, sigma * xyz - np.asarray(gamma)[None, :])
        if mode == 3:
            rho += (ampl * sigma * sigma) * r
            continue
        phi += ampl * p
        if mode >= 1:
            grad += (ampl * sigma) * g
        if mode == 2:
            hess += (ampl * sigma * sigma) * h
    return phi, grad, hess, rho


def ref_cylspline(mode: int, xyz, t, nthreads: int = 0):
    """The reference's CylSpline kernels compiled for the host (mode 0..2)."""
    x, y, z = _soa(xyz)
    n = x.size
    phi, grad, hess, _ = _outs(mode, n)
    d, i = ctypes.c_double, ctypes.c_int
    rc = _refl().ref_cylspl_eval(
        i(mode), _p(x), _p(y), _p(z), d(t.Rscale), _p(np.ascontiguousarray(t.lR_grid)),
        i(len(t.lR_grid)), _p(np.ascontiguousarray(t.lz_grid)), i(len(t.lz_grid)),
        _p(np.ascontiguousarray(t.node_arr)), i(t.n_harm),
        _p(np.ascontiguousarray(t.m_arr, dtype=np.int32)), i(t.mmax), i(t.log_scaling),
        _p(np.ascontiguousarray(t.W_outer)), d(t.r0_outer), i(t.lmax_outer), i(t.mmax_outer),
        _p(phi), _p(grad), _p(hess), i(n), i(nthreads))
    assert rc == 0
    return phi, grad, hess, None


def eval_potential_reference(pot, mode: int, xyz, t: float = 0.0, nthreads: int = 0):
    """CPU evaluation with the reference's own kernel code for the expansions.

    Multipole and CylSpline leaves run the reference's kernels compiled for the
    host (oracle/_ref/libref.so, OpenMP over points); analytic leaves use the
    restated closed forms; the composition (Shifted/Scaled/Evolving/Composite)
    is the same leaf sum the reference's classes perform.  Falls back to the
    oracle port for everything when libref.so is absent.  mode 0 or 1.
    """
    from agama_gpu_b200 import _lib as L
    if not ref_available():
        return eval_potential(pot, mode, xyz, t)
    xyz = np.asarray(xyz, dtype=np.float64).reshape(-1, 3)
    n = len(xyz)
    phi, grad = np.zeros(n), np.zeros((n, 3))
    for comp, sigma, gamma, ampl in pot._leaves(float(t)):
        xl = sigma * xyz - np.asarray(gamma)[None, :]
        if comp.kind == L.KIND_MULTIPOLE:
            p, g, _, _ = ref_multipole(mode, xl, comp.tables, nthreads)
        elif comp.kind == L.KIND_CYLSPLINE:
            p, g, _, _ = ref_cylspline(mode, xl, comp.tables, nthreads)
        else:
            p, g, _, _ = analytic(comp.kind, list(comp._params()), mode, xl)
        phi += ampl * p
        if mode >= 1:
            grad += (ampl * sigma) * g
    return phi, grad
