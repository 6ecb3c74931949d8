"""The oracle (C restatement of the reference's algorithms) against golden
vectors produced by the reference itself (tests/golden/make_golden.py).

This pins the checker: GPU parity tests compare against the same oracle.
"""
import numpy as np
import pytest

from conftest import golden
from helpers import (cs_coefs, mp_coefs, near_pole, outer_condition, outer_mask, rel_max,
                     rel_pointwise)
from oracle import cpu
from agama_gpu_b200.prep_cylspline import build_cylspline_tables
from agama_gpu_b200.prep_multipole import build_multipole_tables

EPS = np.finfo(np.float64).eps
MP_CASES = ["mp_dark", "mp_lmc", "mp_cfg0", "mp_l32"]
CS_CASES = ["cs_bar", "cs_cfg1"]
# FP64 tolerances of a restatement against the reference's own arithmetic
TOL_PHI = 1e-12      # pointwise relative
TOL_F = 1e-12        # max |dF| / max |F|
TOL_H = 1e-11        # max |dH| / max |H|
TOL_RHO = 1e-11      # max |drho| / max |rho|


def _check_mp(g, t, phi, grad, hess, rho):
    xyz = g["xyz"]
    out = outer_mask(t, xyz)
    inn = ~out
    assert rel_pointwise(phi[inn], g["phi"][inn]) < TOL_PHI
    assert rel_max(-grad[inn], g["force"][inn]) < TOL_F
    okh = inn & ~near_pole(xyz)
    assert rel_max(-hess[okh], g["deriv"][okh]) < TOL_H
    assert rel_max(rho, g["rho"]) < TOL_RHO
    if out.any():   # outer extrapolation: bounded by the rounding of its two terms
        cond = outer_condition(t, xyz[out])
        assert np.all(np.abs(phi[out] - g["phi"][out]) <= 64 * EPS * cond + 1e-12 * np.abs(g["phi"][out]))


@pytest.mark.parametrize("case", MP_CASES)
def test_oracle_multipole_vs_reference(case):
    g = golden(case)
    t = build_multipole_tables(mp_coefs(g))
    phi, _, _, _ = cpu.multipole(0, g["xyz"], t)
    _, grad, hess, _ = cpu.multipole(2, g["xyz"], t)
    _, _, _, rho = cpu.multipole(3, g["xyz"], t)
    _check_mp(g, t, phi, grad, hess, rho)
    # GRAD mode agrees with HESS mode's gradient
    _, grad1, _, _ = cpu.multipole(1, g["xyz"], t)
    assert np.array_equal(grad1, grad)


@pytest.mark.parametrize("case", CS_CASES)
def test_oracle_cylspline_vs_reference(case):
    g = golden(case)
    t = build_cylspline_tables(cs_coefs(g))
    phi, _, _, _ = cpu.cylspline(0, g["xyz"], t)
    _, grad, hess, _ = cpu.cylspline(2, g["xyz"], t)
    _, _, _, rho = cpu.cylspline(3, g["xyz"], t)
    assert rel_pointwise(phi, g["phi"]) < 1e-12
    assert rel_max(-grad, g["force"]) < 1e-12
    assert rel_max(-hess, g["deriv"]) < 1e-11
    assert rel_max(rho, g["rho"]) < 1e-11


ANALYTIC = ["NFWPotentialGPU", "PlummerPotentialGPU", "HernquistPotentialGPU",
            "DehnenSphericalPotentialGPU", "IsochronePotentialGPU", "MiyamotoNagaiPotentialGPU",
            "LogHaloPotentialGPU", "DiskAnsatzPotentialGPU", "UniformAccelerationGPU"]


@pytest.mark.parametrize("cls", ANALYTIC)
def test_oracle_analytic_vs_reference(cls):
    import agama_gpu_b200.analytic as an
    g = golden("an_" + cls)
    kw = dict(zip([str(k) for k in g["kwargs_keys"]], g["kwargs_vals"].tolist()))
    pot = getattr(an, cls)(**kw)
    p = list(pot._params())
    phi, grad, hess, _ = cpu.analytic(pot.kind, p, 2, g["xyz"])
    _, _, _, rho = cpu.analytic(pot.kind, p, 3, g["xyz"])
    assert rel_pointwise(phi, g["phi"]) < 1e-13
    assert rel_max(-grad, g["force"]) < 1e-13
    assert rel_max(-hess, g["deriv"]) < 1e-13
    assert rel_max(rho, g["rho"]) < 1e-13


def test_oracle_detects_a_planted_error():
    """A wrong table must move the oracle's answer well beyond the tolerances."""
    g = golden("mp_cfg0")
    t = build_multipole_tables(mp_coefs(g))
    t.poly = t.poly.copy()
    t.poly[3, 10, 0] *= 1.0 + 1e-6          # perturb one harmonic in one interval
    phi, grad, _, _ = cpu.multipole(1, g["xyz"], t)
    assert rel_pointwise(phi, g["phi"]) > 1e-10 or rel_max(-grad, g["force"]) > 1e-10
