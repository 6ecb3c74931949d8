"""Analytic potentials with the reference's constructors (_analytic_potentials.py).

Each class stores the parameters the fused kernel needs (analytic.cuh); the
formulas, r floors and units are those of the reference's ElementwiseKernel
bodies.  All of them evaluate inside the same fused kernel as the expansions.
"""
from __future__ import annotations

import functools
import inspect
import math

from . import _lib
from .potentials import G_AGAMA, _Component

_G = G_AGAMA

__all__ = ["NFWPotentialGPU", "PlummerPotentialGPU", "HernquistPotentialGPU",
           "DehnenSphericalPotentialGPU", "IsochronePotentialGPU", "MiyamotoNagaiPotentialGPU",
           "LogHaloPotentialGPU", "DiskAnsatzPotentialGPU", "UniformAccelerationGPU"]


def _records_args(cls):
    """Keep the constructor's arguments (``_init_args``) so the potential can be written
    back as an INI section with the same parameters."""
    init = cls.__init__
    sig = inspect.signature(init)

    @functools.wraps(init)
    def wrapped(self, *args, **kwargs):
        b = sig.bind(self, *args, **kwargs)
        b.apply_defaults()
        self._init_args = {k: v for k, v in b.arguments.items() if k != "self"}
        init(self, *args, **kwargs)

    cls.__init__ = wrapped
    return cls


def _no_agama(name: str, ctor: str):
    raise TypeError(
        f"{name}.from_agama() is not supported: Agama does not export analytic potential "
        f"parameters.\nConstruct directly:  {name}({ctor})")


@_records_args
class NFWPotentialGPU(_Component):
    """Phi = -G M ln(1 + r/rs) / r  (_analytic_potentials.py:176-283)."""
    kind = _lib.KIND_NFW

    def __init__(self, mass: float = 1.0, scaleRadius: float = 1.0):
        self._M = float(mass)
        self._GM = _G * self._M
        self._rs = float(scaleRadius)

    @classmethod
    def from_agama(cls, pot):
        _no_agama(cls.__name__, "mass=..., scaleRadius=...")

    def _params(self):
        return [self._GM, self._rs, self._M]


@_records_args
class PlummerPotentialGPU(_Component):
    """Phi = -G M / sqrt(r^2 + b^2)  (_analytic_potentials.py:288-378)."""
    kind = _lib.KIND_PLUMMER

    def __init__(self, mass: float = 1.0, scaleRadius: float = 1.0):
        self._M = float(mass)
        self._GM = _G * self._M
        self._b2 = float(scaleRadius) * float(scaleRadius)

    @classmethod
    def from_agama(cls, pot):
        _no_agama(cls.__name__, "mass=..., scaleRadius=...")

    def _params(self):
        return [self._GM, self._b2, self._M]


@_records_args
class HernquistPotentialGPU(_Component):
    """Phi = -G M / (r + a)  (_analytic_potentials.py:383-480)."""
    kind = _lib.KIND_HERNQUIST

    def __init__(self, mass: float = 1.0, scaleRadius: float = 1.0):
        self._M = float(mass)
        self._GM = _G * self._M
        self._a = float(scaleRadius)

    @classmethod
    def from_agama(cls, pot):
        _no_agama(cls.__name__, "mass=..., scaleRadius=...")

    def _params(self):
        return [self._GM, self._a, self._M]


@_records_args
class DehnenSphericalPotentialGPU(_Component):
    """Phi = -(G M/a) (1 - (r/(r+a))^(2-gamma)) / (2-gamma), 0 <= gamma < 2
    (_analytic_potentials.py:486-590)."""
    kind = _lib.KIND_DEHNEN

    def __init__(self, mass: float = 1.0, scaleRadius: float = 1.0, gamma: float = 1.0):
        if not 0.0 <= gamma < 2.0:
            raise ValueError(
                f"gamma must be in [0, 2) for the GPU kernel, got {gamma}. "
                "gamma=2 or triaxial cases are handled by PotentialGPU(type='Dehnen', ...) "
                "which routes through Agama CPU.")
        self._M = float(mass)
        self._GM = _G * self._M
        self._a = float(scaleRadius)
        self._gamma = float(gamma)
        self._exp = 2.0 - self._gamma

    @classmethod
    def from_agama(cls, pot):
        _no_agama(cls.__name__, "mass=..., scaleRadius=..., gamma=...")

    def _params(self):
        return [self._GM, self._a, self._gamma, self._exp, self._M]


@_records_args
class IsochronePotentialGPU(_Component):
    """Phi = -G M / (b + sqrt(r^2 + b^2))  (_analytic_potentials.py:603-715)."""
    kind = _lib.KIND_ISOCHRONE

    def __init__(self, mass: float = 1.0, scaleRadius: float = 1.0):
        self._M = float(mass)
        self._GM = _G * self._M
        self._b = float(scaleRadius)

    @classmethod
    def from_agama(cls, pot):
        _no_agama(cls.__name__, "mass=..., scaleRadius=...")

    def _params(self):
        return [self._GM, self._b]


@_records_args
class MiyamotoNagaiPotentialGPU(_Component):
    """Phi = -G M / sqrt(R^2 + (a + sqrt(z^2 + b^2))^2)  (_analytic_potentials.py:720-836)."""
    kind = _lib.KIND_MIYAMOTONAGAI

    def __init__(self, mass: float = 1.0, scaleRadius: float = 1.0, scaleHeight: float = 0.1):
        self._M = float(mass)
        self._GM = _G * self._M
        self._a = float(scaleRadius)
        self._b = float(scaleHeight)
        self._inv4pi = 1.0 / (4.0 * math.pi)

    @classmethod
    def from_agama(cls, pot):
        _no_agama(cls.__name__, "mass=..., scaleRadius=..., scaleHeight=...")

    def _params(self):
        return [self._GM, self._a, self._b]


@_records_args
class LogHaloPotentialGPU(_Component):
    """Phi = (v0^2/2) ln(rc^2 + x^2 + y^2/p^2 + z^2/q^2)  (_analytic_potentials.py:842-931).

    Keyword names are the reference's: velocity, coreRadius, axisRatioY, axisRatioZ.
    """
    kind = _lib.KIND_LOGHALO

    def __init__(self, velocity: float = 1.0, coreRadius: float = 0.01,
                 axisRatioY: float = 1.0, axisRatioZ: float = 1.0):
        self._v02 = float(velocity) ** 2
        self._rc2 = float(coreRadius) ** 2
        self._p2 = float(axisRatioY) ** 2
        self._q2 = float(axisRatioZ) ** 2

    @classmethod
    def from_agama(cls, pot):
        _no_agama(cls.__name__, "velocity=..., coreRadius=..., axisRatioY=..., axisRatioZ=...")

    def _params(self):
        return [self._v02, self._rc2, self._p2, self._q2]


@_records_args
class DiskAnsatzPotentialGPU(_Component):
    """Phi = f(r) H(z), f = 4 pi Sigma exp(-r/hr - hin/r)  (_analytic_potentials.py:950-1101).

    As in the reference, the kernel always uses the exponential vertical law
    with |scaleHeight|; ``_mode`` records 'exp', 'sech2' (scaleHeight < 0) or
    'thin' (|scaleHeight| < 1e-10) but does not change the result.
    """
    kind = _lib.KIND_DISKANSATZ

    def __init__(self, surfaceDensity=1.0, scaleRadius=1.0, scaleHeight=0.1, innerCutoffRadius=0.0):
        self._Sigma = float(surfaceDensity) * _G
        self._hr = float(scaleRadius)
        self._hz = float(abs(scaleHeight))
        self._hin = float(innerCutoffRadius)
        if self._hz < 1e-10:
            self._mode = "thin"
        elif scaleHeight > 0:
            self._mode = "exp"
        else:
            self._mode = "sech2"

    @classmethod
    def from_agama(cls, pot):
        _no_agama(cls.__name__, "surfaceDensity=..., scaleRadius=..., scaleHeight=..., "
                  "innerCutoffRadius=...")

    def _params(self):
        return [self._Sigma, self._hr, self._hz, self._hin]


@_records_args
class UniformAccelerationGPU(_Component):
    """Phi = -(ax x + ay y + az z)  (_analytic_potentials.py:1112-1165)."""
    kind = _lib.KIND_UNIFORMACC

    def __init__(self, ax: float = 0.0, ay: float = 0.0, az: float = 0.0):
        self._ax, self._ay, self._az = float(ax), float(ay), float(az)

    @classmethod
    def from_agama(cls, pot):
        _no_agama(cls.__name__, "ax=..., ay=..., az=...")

    def _params(self):
        return [self._ax, self._ay, self._az]
