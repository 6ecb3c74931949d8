"""Host table builders against the reference's own tables (golden vectors)."""
import numpy as np
import pytest

from conftest import golden
from helpers import cs_coefs, mp_coefs
from agama_gpu_b200.prep_cylspline import build_cylspline_tables
from agama_gpu_b200.prep_multipole import build_multipole_tables


@pytest.mark.parametrize("case", ["mp_dark", "mp_lmc", "mp_cfg0", "mp_l32"])
def test_multipole_tables_bit_identical(case):
    g = golden(case)
    t = build_multipole_tables(mp_coefs(g))
    assert tuple(t.poly.shape) == tuple(g["ref_poly_shape"])
    assert np.array_equal(t.poly.reshape(-1)[g["ref_poly_idx"]], g["ref_poly_val"])
    assert np.array_equal(t.lm_l, g["ref_lm_l"]) and np.array_equal(t.lm_m, g["ref_lm_m"])
    assert np.array_equal(np.array(t.scalars()), g["ref_scalars"])
    n_int, n_lm, lmax, ls = g["ref_ints"]
    assert (t.n_int, t.n_lm, t.lmax, t.log_scaling) == (n_int, n_lm, lmax, ls)


@pytest.mark.parametrize("case", ["cs_bar", "cs_cfg1"])
def test_cylspline_tables_match(case):
    g = golden(case)
    t = build_cylspline_tables(cs_coefs(g))
    Rs, r0, ls, mmax, lmo, mmo = g["ref_scalars"]
    assert abs(t.Rscale - Rs) <= 1e-13 * Rs
    assert t.r0_outer == r0 and t.log_scaling == ls and t.mmax == mmax
    assert t.lmax_outer == lmo and t.mmax_outer == mmo
    W = g["ref_W"]
    assert np.max(np.abs(t.W_outer - W)) <= 1e-12 * np.max(np.abs(W))
    assert np.allclose(t.lR_grid, g["ref_lR"], rtol=0, atol=1e-13)
    assert np.allclose(t.lz_grid, g["ref_lz"], rtol=0, atol=1e-13)
    assert tuple(t.node_arr.shape) == tuple(g["ref_node_shape"])
    got = t.node_arr.reshape(-1)[g["ref_node_idx"]]
    ref = g["ref_node_val"]
    assert np.max(np.abs(got - ref)) <= 1e-11 * max(1.0, np.max(np.abs(ref)))


def test_cell_major_layout_is_a_permutation_of_nodes():
    g = golden("cs_cfg1")
    t = build_cylspline_tables(cs_coefs(g))
    cm = t.cell_major().reshape(len(t.lR_grid) - 1, len(t.lz_grid) - 1, t.n_harm, 4, 4)
    order = t.harmonic_order()
    iR, iz, h = 3, 7, 2
    node = t.node_arr[order[h]]
    for q in range(4):
        assert cm[iR, iz, h, q, 0] == node[iR, iz, q]
        assert cm[iR, iz, h, q, 1] == node[iR, iz + 1, q]
        assert cm[iR, iz, h, q, 2] == node[iR + 1, iz, q]
        assert cm[iR, iz, h, q, 3] == node[iR + 1, iz + 1, q]
    assert list(np.abs(t.m_sorted())) == sorted(np.abs(t.m_sorted()))


def test_non_log_uniform_grid_is_resampled():
    from agama_gpu_b200.synthetic import nfw_multipole
    c = nfw_multipole(lmax=2, n_nodes=20)
    c.R_grid = c.R_grid.copy()
    c.R_grid[5] *= 1.05                      # break log-uniform spacing by > 1e-3
    t = build_multipole_tables(c)
    assert t.n_int == 999
    assert np.allclose(np.diff(np.log(t.r_grid)), t.dlogr, rtol=1e-9)


def test_missing_derivatives_raise():
    from agama_gpu_b200.synthetic import nfw_multipole
    c = nfw_multipole(lmax=2, n_nodes=10)
    c.dphi_dr = None
    with pytest.raises(ValueError, match="dPhi/dr"):
        build_multipole_tables(c)


def test_lmax_limit():
    from agama_gpu_b200.synthetic import nfw_multipole
    with pytest.raises(ValueError, match="lmax=34"):
        build_multipole_tables(nfw_multipole(lmax=34, n_nodes=10))
