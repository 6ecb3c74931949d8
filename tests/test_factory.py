"""Host logic of the potential tree (Composite, Evolving, Shifted, Scaled, the
factory, INI files) against the reference's own outputs, evaluated on the CPU
through the oracle: no GPU needed."""
import numpy as np
import pytest

from conftest import golden
from helpers import close_global, close_pointwise, near_pole, tree_allowance
from oracle import cpu
import agama_gpu_b200 as agb
from agama_gpu_b200.coefs import MultipoleCoefs, write_coefs


def build_golden_composite(g):
    from agama_gpu_b200.coefs import MultipoleCoefs
    main = MultipoleCoefs(g["main_R"], g["main_phi"], g["main_dphi"],
                          [tuple(x) for x in g["main_labels"].tolist()])
    snaps = [MultipoleCoefs(g["snap_R"][i], g["snap_phi"][i], g["snap_dphi"][i],
                            [tuple(x) for x in g["snap_labels"].tolist()])
             for i in range(len(g["snap_R"]))]
    pots = [
        agb.MultipolePotentialGPU(main),
        agb.MiyamotoNagaiPotentialGPU(mass=5e10, scaleRadius=3.0, scaleHeight=0.3),
        agb.DiskAnsatzPotentialGPU(surfaceDensity=1e9, scaleRadius=3.0, scaleHeight=0.3),
        agb.ShiftedPotentialGPU(agb.NFWPotentialGPU(mass=1.5e11, scaleRadius=10.0), g["track4"]),
        agb.EvolvingPotentialGPU([agb.MultipolePotentialGPU(s) for s in snaps], g["times"], True),
        agb.ScaledPotentialGPU(agb.PlummerPotentialGPU(mass=1e10, scaleRadius=2.0), g["scl3"]),
        agb.ShiftedPotentialGPU(agb.ScaledPotentialGPU(
            agb.HernquistPotentialGPU(mass=3e10, scaleRadius=1.0), 0.5, 2.0), g["track7"]),
        agb.ScaledPotentialGPU(agb.ShiftedPotentialGPU(
            agb.IsochronePotentialGPU(mass=1e10, scaleRadius=1.5), np.array([3.0, -2.0, 1.0])), 1.7, 0.8),
    ]
    ev = agb.EvolvingPotentialGPU([agb.MultipolePotentialGPU(s) for s in snaps], g["times"], False)
    return agb.CompositePotentialGPU(pots), ev


def test_composite_tree_matches_reference_through_oracle():
    g = golden("composite")
    comp, ev = build_golden_composite(g)
    xyz = g["xyz"]
    i = 0
    while f"t_{i}" in g:
        t = float(g[f"t_{i}"])
        phi, grad, hess, _ = cpu.eval_potential(comp, 2, xyz, t)
        _, _, _, rho = cpu.eval_potential(comp, 3, xyz, t)
        ap, ag, ah = tree_allowance(comp, xyz, t)
        assert close_pointwise(phi, g[f"phi_{i}"], 1e-12, ap), t
        assert close_global(-grad, g[f"force_{i}"], 1e-12, ag), t
        ok = ~near_pole(xyz)
        assert close_global(-hess[ok], g[f"deriv_{i}"][ok], 1e-11, ah[ok]), t
        assert close_global(rho, g[f"rho_{i}"], 1e-11), t
        i += 1
    assert i >= 5
    phi, _, _, _ = cpu.eval_potential(ev, 0, xyz, 0.3)
    assert close_pointwise(phi, g["phi_nearest"], 1e-12, tree_allowance(ev, xyz, 0.3)[0])


def test_plus_flattens_and_sum_works():
    a = agb.NFWPotentialGPU(mass=1e12, scaleRadius=20)
    b = agb.PlummerPotentialGPU(mass=1e10, scaleRadius=1)
    c = agb.HernquistPotentialGPU(mass=1e10, scaleRadius=1)
    ab = a + b
    abc = ab + c
    assert isinstance(abc, agb.CompositePotentialGPU) and len(abc._components) == 3
    s = sum([a, b, c])
    assert len(s._components) == 3
    assert [l[0] for l in abc._leaves(0.0)] == [a, b, c]


def test_evolving_brackets_like_the_reference():
    p = [agb.NFWPotentialGPU(mass=m, scaleRadius=10) for m in (1e11, 2e11, 3e11)]
    ev = agb.EvolvingPotentialGPU(p, [0.0, 1.0, 3.0])
    assert ev._weights(-1.0) == [(0, 1.0)]
    assert ev._weights(5.0) == [(2, 1.0)]
    assert ev._weights(1.0) == [(1, 1.0)]
    w = ev._weights(2.0)
    assert w[0][0] == 1 and w[1][0] == 2 and w[0][1] == pytest.approx(0.5)
    nn = agb.EvolvingPotentialGPU(p, [0.0, 1.0, 3.0], interpolate=False)
    assert nn._weights(2.1) == [(2, 1.0)]
    with pytest.raises(ValueError):
        agb.EvolvingPotentialGPU(p, [0.0, 1.0])


def test_modifier_leaves():
    n = agb.NFWPotentialGPU(mass=1e12, scaleRadius=20)
    s = agb.ScaledPotentialGPU(agb.ShiftedPotentialGPU(n, [1.0, 2.0, 3.0]), 2.0, 3.0)
    (c, sigma, gamma, ampl), = s._leaves(0.0)
    assert c is n and sigma == 0.5 and ampl == 1.5 and np.allclose(gamma, [1, 2, 3])
    s2 = agb.ShiftedPotentialGPU(agb.ScaledPotentialGPU(n, 2.0, 3.0), [1.0, 2.0, 3.0])
    (c, sigma, gamma, ampl), = s2._leaves(0.0)
    assert sigma == 0.5 and ampl == 1.5 and np.allclose(gamma, [0.5, 1.0, 1.5])
    with pytest.raises(ValueError):
        agb.ShiftedPotentialGPU(n, np.zeros((3, 2)))
    with pytest.raises(ValueError):
        agb.ScaledPotentialGPU(n, np.zeros((3, 5)))


def test_factory_keyword_and_dict_dispatch():
    p = agb.PotentialGPU(type="NFW", mass=1e12, scaleRadius=20.0)
    assert isinstance(p, agb.NFWPotentialGPU) and p._GM == 4.30091727067736e-06 * 1e12
    q = agb.PotentialGPU(dict(type="NFW", mass=1e12, scaleRadius=20),
                         dict(type="MiyamotoNagai", mass=5e10, scaleRadius=3, scaleHeight=0.3))
    assert isinstance(q, agb.CompositePotentialGPU) and len(q._components) == 2
    r = agb.PotentialGPU(type="Plummer", mass=1.0, center=[1.0, 0.0, 0.0], scale=2.0, ampl=0.5)
    assert isinstance(r, agb.ShiftedPotentialGPU)
    assert isinstance(r._inner, agb.ScaledPotentialGPU)
    d = agb.PotentialGPU(type="Dehnen", mass=1e10, scaleRadius=2, gamma=0.5)
    assert isinstance(d, agb.DehnenSphericalPotentialGPU)
    with pytest.raises(ValueError, match="Unknown GPU potential type"):
        agb.PotentialGPU(type="Bogus")
    with pytest.raises(ValueError, match="requires file"):
        agb.PotentialGPU(type="Multipole")
    with pytest.raises(TypeError):
        agb.PotentialGPU()
    # Agama-routed types without agama: built by the package's own Poisson solver
    k = agb.PotentialGPU(type="King", mass=1e5, scaleRadius=0.01, W0=6)
    assert isinstance(k, agb.MultipolePotentialGPU)
    with pytest.raises(TypeError, match="unknown parameter"):
        agb.PotentialGPU(type="Spheroid", mass=1e10, bogus=1)
    with pytest.raises(ValueError, match="gamma"):
        agb.DehnenSphericalPotentialGPU(gamma=2.5)


def test_ini_file(tmp_path):
    from agama_gpu_b200.synthetic import nfw_multipole
    snap_files = []
    for i in range(3):
        f = tmp_path / f"snap{i}.coef_mul_DR"
        write_coefs(f, nfw_multipole(lmax=2, n_nodes=12, seed=i))
        snap_files.append(f.name)
    halo = tmp_path / "halo.coef_mul_DR"
    write_coefs(halo, nfw_multipole(lmax=4, n_nodes=20, seed=9))
    ini = tmp_path / "model.ini"
    ini.write_text(
        "[Potential halo]\ntype=Multipole\nfile=halo.coef_mul_DR\n\n"
        "[Potential disk]\ntype=MiyamotoNagai\nmass=5e10  # comment\nscaleRadius=3\nscaleHeight=0.3\n\n"
        "[Potential stub]\ntype=DiskAnsatz\n\n"
        "[Potential evo]\ntype=Evolving\ninterpLinear=True\nTimestamps\n"
        + "".join(f"{i * 0.5} {f}\n" for i, f in enumerate(snap_files)))
    pot = agb.PotentialGPU(str(ini))
    assert isinstance(pot, agb.CompositePotentialGPU)
    kinds = [type(c).__name__ for c in pot._components]
    assert kinds == ["MultipolePotentialGPU", "MiyamotoNagaiPotentialGPU", "EvolvingPotentialGPU"]
    assert pot._components[2]._interpolate is True
    assert len(pot._leaves(0.25)) == 4       # halo, disk, two bracketing snapshots
    # coefficient file given directly, and inline Coefficients in an INI section
    assert isinstance(agb.PotentialGPU(str(halo)), agb.MultipolePotentialGPU)
    inline = tmp_path / "inline.ini"
    inline.write_text(halo.read_text())
    assert isinstance(agb.PotentialGPU(file=str(inline)), agb.MultipolePotentialGPU)
