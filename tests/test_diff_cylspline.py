"""CylSpline node-table chain (host side): dL/dPhi_m on the coefficient grid from
dL/d(node table), against central differences through the real table builder."""
import numpy as np
import pytest
import torch

from conftest import golden
from helpers import cs_coefs
from agama_gpu_b200.coefs import CylSplineCoefs
from agama_gpu_b200.diff_tables import cylspline_node_vjp
from agama_gpu_b200.prep_cylspline import build_cylspline_tables
from agama_gpu_b200.synthetic import bar_cylspline


def _half(c):
    """The z >= 0 half of a z-symmetric grid (the builder mirrors it back)."""
    z = np.asarray(c.z_grid)
    k = int(np.argmin(np.abs(z)))
    assert abs(z[k]) < 1e-12
    return CylSplineCoefs(c.R_grid, z[k:], {m: np.asarray(v)[:, k:] for m, v in c.phi.items()})


@pytest.mark.parametrize("which", ["full", "half"])
def test_node_vjp_matches_builder_differences(which):
    c = cs_coefs(golden("cs_cfg1")) if which == "full" else _half(bar_cylspline(n_z=33))
    t = build_cylspline_tables(c)
    rng = np.random.default_rng(3)
    G = rng.normal(size=t.node_arr.shape)
    grads = cylspline_node_vjp(t, c, torch.from_numpy(G))

    def L(phi):
        cc = CylSplineCoefs(c.R_grid, c.z_grid, phi)
        tt = build_cylspline_tables(cc)
        assert np.array_equal(tt.lR_grid, t.lR_grid)      # grids and asymptote held fixed
        return float((G * tt.node_arr).sum())

    nR, nz = np.asarray(c.phi[0]).shape
    picks = [(0, 5, 7), (0, nR // 2, 3), (2, 9, nz // 2), (-4, 12, 2), (6, 3, nz - 5)]
    if which == "half":                  # j = 0: the z = 0 column of the mirrored grid
        picks += [(2, 7, 0), (0, 4, 0)]
    for m, i, j in picks:
        h = 1e-6 * np.abs(np.asarray(c.phi[m])).max()
        pp = {k: np.array(v, dtype=float) for k, v in c.phi.items()}
        pm = {k: np.array(v, dtype=float) for k, v in c.phi.items()}
        pp[m][i, j] += h
        pm[m][i, j] -= h
        fd = (L(pp) - L(pm)) / (2 * h)
        an = grads[m][i, j]
        assert abs(an - fd) <= 1e-6 * max(abs(fd), 1e-3 * max(np.abs(g).max() for g in grads.values())), \
            (m, i, j, an, fd)
