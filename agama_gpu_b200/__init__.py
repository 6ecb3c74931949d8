"""agama_gpu_b200 -- B200-native evaluator for Agama-style galactic potentials.

Drop-in for the ``PotentialGPU`` API of the reference (gpu_potential.py,
_analytic_potentials.py): same factory, classes, methods, shapes and units;
all evaluation runs in hand-written sm_100a CUDA kernels (libagb.so, C ABI in
include/agb.h).  There is no CPU fallback.
"""
from . import _lib  # noqa: F401  (fails loudly when libagb.so is missing)
from .analytic import (DehnenSphericalPotentialGPU, DiskAnsatzPotentialGPU, HernquistPotentialGPU,
                       IsochronePotentialGPU, LogHaloPotentialGPU, MiyamotoNagaiPotentialGPU,
                       NFWPotentialGPU, PlummerPotentialGPU, UniformAccelerationGPU)
from .batch import BatchedPotentialGPU
from .coefs import CylSplineCoefs, MultipoleCoefs, read_coefs, write_coefs
from .factory import PotentialGPU
from .potentials import (G_AGAMA, INV_4PIG, CompositePotentialGPU, CylSplinePotentialGPU,
                         EvolvingPotentialGPU, MultipolePotentialGPU, ScaledPotentialGPU,
                         ShiftedPotentialGPU, prep_xyz, set_default_precision)
from .integrate import Leapfrog, leapfrog
from .stream import Stream, integrate_releases, particle_spray
from .export import export_potential
from .adaptive import DormandPrince, integrate_adaptive

__all__ = [
    "PotentialGPU", "BatchedPotentialGPU", "MultipolePotentialGPU", "CylSplinePotentialGPU", "CompositePotentialGPU",
    "EvolvingPotentialGPU", "ShiftedPotentialGPU", "ScaledPotentialGPU", "NFWPotentialGPU",
    "PlummerPotentialGPU", "HernquistPotentialGPU", "DehnenSphericalPotentialGPU",
    "IsochronePotentialGPU", "MiyamotoNagaiPotentialGPU", "LogHaloPotentialGPU",
    "DiskAnsatzPotentialGPU", "UniformAccelerationGPU", "MultipoleCoefs", "CylSplineCoefs",
    "read_coefs", "write_coefs", "set_default_precision", "prep_xyz", "G_AGAMA", "INV_4PIG",
    "Leapfrog", "leapfrog", "Stream", "particle_spray", "integrate_releases", "export_potential",
    "DormandPrince", "integrate_adaptive",
]
