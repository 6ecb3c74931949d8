"""Shared builders and comparison helpers for the tests."""
from __future__ import annotations

import numpy as np

from agama_gpu_b200.coefs import CylSplineCoefs, MultipoleCoefs


def mp_coefs(g: dict, prefix: str = "") -> MultipoleCoefs:
    if prefix:
        return MultipoleCoefs(g[prefix + "_R"], g[prefix + "_phi"], g[prefix + "_dphi"],
                              [tuple(x) for x in g[prefix + "_labels"].tolist()])
    return MultipoleCoefs(g["R_grid"], g["phi_tab"], g["dphi_tab"],
                          [tuple(x) for x in g["lm_labels"].tolist()])


def cs_coefs(g: dict) -> CylSplineCoefs:
    return CylSplineCoefs(g["R_grid"], g["z_grid"],
                          {int(m): g["phi_tabs"][i] for i, m in enumerate(g["m_list"])})


def _finite_pair(a, b):
    """Drop entries that are non-finite in both; a non-finite mismatch -> None."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    fa, fb = np.isfinite(a), np.isfinite(b)
    if not np.array_equal(fa, fb):
        return None
    both_nan = np.isnan(a) & np.isnan(b)
    both_inf = ~fa & ~np.isnan(a) & (a == b)
    if not np.all(both_nan | both_inf | fa):
        return None
    return a, b, fa


def rel_max(a, b) -> float:
    """max |a-b| / max |b| over finite entries (the reference tests' force convention);
    inf when the non-finite entries differ."""
    pr = _finite_pair(a, b)
    if pr is None:
        return float("inf")
    a, b, f = pr
    if not f.any():
        return 0.0
    den = np.max(np.abs(b[f]))
    return float(np.max(np.abs(a[f] - b[f])) / max(den, 1e-300))


def rel_pointwise(a, b, floor: float = 1e-300) -> float:
    """max over points of |a-b| / |b| (row max for vectors), finite entries only."""
    pr = _finite_pair(a, b)
    if pr is None:
        return float("inf")
    a, b, f = pr
    a = np.where(f, a, 0.0).reshape(len(a), -1)
    b = np.where(f, b, 0.0).reshape(len(b), -1)
    scale = np.maximum(np.max(np.abs(b), axis=1), floor)
    return float(np.max(np.max(np.abs(a - b), axis=1) / scale))


def outer_mask(tables, xyz) -> np.ndarray:
    """Points beyond the last radial node of a Multipole."""
    r = np.linalg.norm(xyz, axis=1)
    return np.log(np.maximum(r, 1e-300)) >= tables.logr_min + tables.n_int * tables.dlogr


def outer_condition(tables, xyz) -> np.ndarray:
    """Magnitude of the two outer-extrapolation terms (their rounding scale).

    Phi = W (r/rN)^-1 + U (r/rN)^s: when s is within rounding of -1 the two
    terms are huge and cancel, so any two correct implementations differ by
    about eps * (|W| (r/rN)^-1 + |U| (r/rN)^s).
    """
    r = np.linalg.norm(xyz, axis=1)
    dlr = np.log(r) - (tables.logr_min + tables.n_int * tables.dlogr)
    return np.abs(tables.outer_W) * np.exp(-dlr) + np.abs(tables.outer_U) * np.exp(tables.outer_s * dlr)


def near_pole(xyz) -> np.ndarray:
    """0 < sin(theta) < 1e-6: the reference's Hessian chain rule divides by
    sin^3(theta) there (_multipole_potential_kernel.cu:744-751) and cancels
    catastrophically, so Hessians at such points are compared by no one."""
    xyz = np.asarray(xyz)
    R = np.hypot(xyz[:, 0], xyz[:, 1])
    r = np.linalg.norm(xyz, axis=1)
    s = np.divide(R, r, out=np.zeros_like(R), where=r > 0)
    return (s > 0) & (s < 1e-6)


EPS = np.finfo(np.float64).eps


def tree_allowance(pot, xyz, t: float = 0.0):
    """Per-point rounding allowance from ill-conditioned outer extrapolations.

    Sums, over the Multipole leaves of a potential tree, the magnitude of the
    two outer-extrapolation terms at the leaf's transformed points (zero inside
    the grid), with the leaf's output factors.  Returns allowances for Phi,
    gradient and Hessian (the latter two divided by r and r^2).
    """
    from agama_gpu_b200 import _lib
    xyz = np.asarray(xyz, dtype=np.float64)
    a_phi = np.zeros(len(xyz))
    a_g = np.zeros(len(xyz))
    a_h = np.zeros(len(xyz))
    for comp, sigma, gamma, ampl in pot._leaves(float(t)):
        if comp.kind != _lib.KIND_MULTIPOLE:
            continue
        x = sigma * xyz - np.asarray(gamma)[None, :]
        r = np.maximum(np.linalg.norm(x, axis=1), 1e-300)
        m = outer_mask(comp.tables, x)
        c = np.zeros(len(x))
        if m.any():
            c[m] = outer_condition(comp.tables, x[m])
        a_phi += abs(ampl) * c
        a_g += abs(ampl * sigma) * np.divide(c, r, out=np.zeros_like(c), where=c > 0)
        a_h += abs(ampl * sigma * sigma) * np.divide(c, r * r, out=np.zeros_like(c), where=c > 0)
    return a_phi, a_g, a_h


def close_pointwise(a, b, tol, allow=None) -> bool:
    """|a-b| <= tol |b| + 64 eps allow, row-wise; matching non-finite entries pass."""
    a = np.asarray(a, dtype=np.float64).reshape(len(a), -1)
    b = np.asarray(b, dtype=np.float64).reshape(len(b), -1)
    if _finite_pair(a, b) is None:
        return False
    f = np.isfinite(b)
    d = np.abs(np.where(f, a, 0.0) - np.where(f, b, 0.0)).max(axis=1)
    lim = tol * np.where(f, np.abs(b), 0.0).max(axis=1)
    if allow is not None:
        lim = lim + 64 * EPS * np.asarray(allow)
    return bool(np.all(d <= lim + 1e-300))


def close_global(a, b, tol, allow=None) -> bool:
    """|a-b| <= tol max|b| + 64 eps allow, row-wise (the max-normalised convention)."""
    a = np.asarray(a, dtype=np.float64).reshape(len(a), -1)
    b = np.asarray(b, dtype=np.float64).reshape(len(b), -1)
    if _finite_pair(a, b) is None:
        return False
    f = np.isfinite(b)
    d = np.abs(np.where(f, a, 0.0) - np.where(f, b, 0.0)).max(axis=1)
    lim = tol * (np.abs(b[f]).max() if f.any() else 0.0)
    if allow is not None:
        lim = lim + 64 * EPS * np.asarray(allow)
    return bool(np.all(d <= lim + 1e-300))
