"""Normalised associated Legendre functions in Agama's convention (host side).

Ybar_l^m(theta) = N_lm P_l^m(cos theta), N_lm = sqrt((2l+1)/(4 pi) (l-m)!/(l+m)!),
P_l^m with the Condon-Shortley phase; the angular factor of a harmonic is
MUL0 (m = 0) or MUL1 (m != 0) times Ybar.  MUL1 is the reference's literal
5.0132565706694072 (gpu_potential.py:962, _multipole_potential_kernel.cu:94),
which is 2 sqrt(2 pi) (1 + 4.27e-9); it is kept so results match the reference.
"""
from __future__ import annotations

import math

import numpy as np

MUL0 = 3.5449077018110318
MUL1 = 5.0132565706694072


def _coef(m: int) -> float:
    """N_mm (-1)^m (2m-1)!!  (the Ybar_m^m / sin^m theta seed)."""
    dfact = 1
    for k in range(1, 2 * m, 2):
        dfact *= k
    pref = math.sqrt((2 * m + 1) / (4.0 * math.pi * math.factorial(2 * m)))
    return (-1) ** m * dfact * pref


def legendre_normalised(lmax: int, m: int, ct, st) -> np.ndarray:
    """Ybar_l^m for l = m..lmax at points with cos/sin theta (ct, st); (npts, lmax-m+1)."""
    ct = np.asarray(ct, dtype=np.float64)
    st = np.asarray(st, dtype=np.float64)
    out = np.zeros(ct.shape + (lmax - m + 1,))
    Pp = np.zeros_like(ct)
    Pc = _coef(m) * st ** m
    out[..., 0] = Pc
    for l in range(m + 1, lmax + 1):
        a = math.sqrt((4 * l * l - 1) / (l * l - m * m))
        b = math.sqrt((2 * l + 1) * ((l - 1) ** 2 - m * m) / ((2 * l - 3) * (l * l - m * m))) \
            if l >= m + 2 else 0.0
        Pn = a * (ct * Pc) - b * Pp
        Pp, Pc = Pc, Pn
        out[..., l - m] = Pc
    return out


def outer_asymptote_basis(lmax: int, m: int, ct, st) -> np.ndarray:
    """Angular basis of the CylSpline outer asymptote, exactly as the reference builds it.

    The reference's recurrence (gpu_potential.py:967-998 for the fit,
    _cylspl_potential_kernel.cu:213-252 for the evaluation) keeps three
    un-normalised values (p2, p1, p) but feeds p2 from one order too far back:
    at l = m+2 it uses 0, at l > m+2 it uses P_{l-3}^m in place of P_{l-2}^m.
    Orders l = m and m+1 are the true normalised Legendre functions; higher
    orders are the lagged sequence times N_lm.  Fit and evaluation share the
    basis, so the asymptote is self-consistent; it is reproduced here (and in
    the kernel) so that W_outer and the exterior potential match the reference.
    Returns (npts, lmax-m+1).
    """
    ct = np.asarray(ct, dtype=np.float64)
    st = np.asarray(st, dtype=np.float64)
    out = np.zeros(ct.shape + (lmax - m + 1,))
    out[..., 0] = _coef(m) * st ** m
    if lmax == m:
        return out
    pref = math.sqrt((2 * m + 1) / (4.0 * math.pi * math.factorial(2 * m)))
    p1 = out[..., 0] / pref
    p = ct * (2 * m + 1) * p1
    p2 = np.zeros_like(ct)
    pref *= math.sqrt((2 * m + 3) / (2 * m + 1) / (2.0 * m + 1.0))
    out[..., 1] = p * pref
    for l in range(m + 2, lmax + 1):
        new = (ct * (2 * l - 1) * p - (l + m - 1) * p2) / (l - m)
        pref *= math.sqrt((2 * l + 1) / (2 * l - 1) * (l - m) / (l + m))
        out[..., l - m] = new * pref
        p2, p1, p = p1, p, new
    return out
