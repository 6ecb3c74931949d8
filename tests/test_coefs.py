"""Coefficient-file reader/writer: the reference's fixtures and round trips."""
import numpy as np
import pytest

from conftest import reference_available
from oracle.refpy import REF_DIR
from agama_gpu_b200.coefs import CylSplineCoefs, MultipoleCoefs, read_coefs, write_coefs
from agama_gpu_b200.synthetic import bar_cylspline, nfw_multipole


@pytest.mark.skipif(not reference_available(), reason="reference fixtures absent")
def test_read_reference_fixtures():
    m = read_coefs(REF_DIR / "tests" / "600.dark.none_8.coef_mul_DR")
    assert isinstance(m, MultipoleCoefs)
    assert m.phi.shape == (25, 81) and m.dphi_dr.shape == (25, 81)
    assert m.lm_labels[0] == (0, 0) and m.lm_labels[-1] == (8, 8)
    assert m.R_grid[0] == pytest.approx(0.0678992535359)
    m2 = read_coefs(REF_DIR / "tests" / "100.LMC.none_8.coef_mult")
    assert m2.dphi_dr is not None
    c = read_coefs(REF_DIR / "tests" / "600.bar.none_8.coef_cylsp_DR")
    assert isinstance(c, CylSplineCoefs)
    assert sorted(c.phi) == list(range(-8, 9))
    assert c.phi[0].shape == (25, 49) and c.R_grid[0] == 0.0 and c.z_grid[0] == -500.0


def test_multipole_roundtrip(tmp_path):
    c = nfw_multipole(lmax=4, n_nodes=12, seed=3)
    f = tmp_path / "x.coef_mul_DR"
    write_coefs(f, c)
    d = read_coefs(f)
    assert d.lm_labels == c.lm_labels
    assert np.array_equal(d.R_grid, c.R_grid)
    assert np.array_equal(d.phi, c.phi) and np.array_equal(d.dphi_dr, c.dphi_dr)
    # the text of a section is accepted too (inline INI Coefficients)
    d2 = read_coefs(f.read_text())
    assert np.array_equal(d2.phi, c.phi)


def test_cylspline_roundtrip(tmp_path):
    c = bar_cylspline(n_R=8, n_z=9)
    f = tmp_path / "x.coef_cylsp"
    write_coefs(f, c)
    d = read_coefs(f)
    assert sorted(d.phi) == sorted(c.phi)
    for m in c.phi:
        assert np.array_equal(d.phi[m], c.phi[m])
    assert np.array_equal(d.z_grid, c.z_grid)


def test_bad_files(tmp_path):
    f = tmp_path / "bad.coef"
    f.write_text("[Potential]\ntype=Multipole\n")
    with pytest.raises(ValueError, match="Coefficients"):
        read_coefs(f)
    f.write_text("[Potential]\ntype=Spline\nCoefficients\n")
    with pytest.raises(ValueError, match="unsupported"):
        read_coefs(f)
    f.write_text("[Potential]\ntype=Multipole\nCoefficients\n#Phi\n#radius\tl=0,m=0\n1.0\t2.0\t3.0\n")
    with pytest.raises(ValueError, match="shape"):
        read_coefs(f)


def test_zeroed_keeps_subset():
    c = nfw_multipole(lmax=4, n_nodes=12, seed=3)
    z = c.zeroed([(0, 0), (2, 0)])
    keep = [i for i, lm in enumerate(c.lm_labels) if lm in ((0, 0), (2, 0))]
    assert np.count_nonzero(np.abs(z.phi).sum(0)) == np.count_nonzero(np.abs(c.phi[:, keep]).sum(0))
