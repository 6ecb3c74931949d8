"""Multi-section INI export of whole potential trees: written, read back by the
factory, and evaluated by the oracle bit for bit the same as the original."""
import numpy as np
import pytest

from conftest import golden
from helpers import cs_coefs
from oracle import cpu


def _tree():
    import agama_gpu_b200 as agb
    from agama_gpu_b200.synthetic import circular_track, nfw_multipole
    mp = agb.MultipolePotentialGPU(nfw_multipole(lmax=6, n_nodes=40, seed=2))
    snaps = [agb.MultipolePotentialGPU(nfw_multipole(lmax=4, n_nodes=30, seed=s, drift=0.1 * s))
             for s in range(3)]
    scale_tab = np.stack([np.linspace(0, 2, 9), 1 + 0.1 * np.linspace(0, 2, 9) ** 2,
                          1 + 0.05 * np.linspace(0, 2, 9)], 1)
    parts = [
        mp,
        agb.MiyamotoNagaiPotentialGPU(mass=5e10, scaleRadius=3.0, scaleHeight=0.3),
        agb.CylSplinePotentialGPU(cs_coefs(golden("cs_cfg1"))),
        agb.ShiftedPotentialGPU(agb.NFWPotentialGPU(mass=2e11, scaleRadius=8.0),
                                circular_track(T=50, radius=40.0)),
        agb.ScaledPotentialGPU(agb.PlummerPotentialGPU(mass=1e9, scaleRadius=0.7), scale_tab),
        agb.ShiftedPotentialGPU(
            agb.ScaledPotentialGPU(agb.CompositePotentialGPU([
                agb.HernquistPotentialGPU(mass=3e10, scaleRadius=1.5),
                agb.IsochronePotentialGPU(mass=1e10, scaleRadius=2.0)]), 2.0, ampl=0.5),
            [1.0, -2.0, 0.5]),
        agb.EvolvingPotentialGPU(snaps, [0.0, 0.7, 1.9], interpolate=True),
        agb.DiskAnsatzPotentialGPU(surfaceDensity=8.9e8, scaleRadius=3.0, scaleHeight=0.3,
                                   innerCutoffRadius=0.5),
        agb.UniformAccelerationGPU(ax=1.0, ay=-2.0, az=0.25),
        agb.LogHaloPotentialGPU(velocity=180.0, coreRadius=1.0, axisRatioY=0.9, axisRatioZ=0.8),
        agb.DehnenSphericalPotentialGPU(mass=1e10, scaleRadius=2.0, gamma=0.5),
    ]
    return agb.CompositePotentialGPU(parts)


def _pts(n, seed):
    rng = np.random.default_rng(seed)
    r = np.exp(rng.uniform(np.log(0.3), np.log(80.0), n))
    u = rng.normal(size=(n, 3))
    return u / np.linalg.norm(u, axis=1)[:, None] * r[:, None]


def test_export_round_trip_bit_exact(tmp_path):
    import agama_gpu_b200 as agb
    from agama_gpu_b200.export import export_potential
    pot = _tree()
    ini = export_potential(pot, tmp_path / "galaxy.ini")
    text = ini.read_text()
    assert text.count("[Potential") == 12          # the Shifted(Scaled(sum of 2)) gives two
    assert "Timestamps" in text and "center=1.0,-2.0,0.5" in text
    back = agb.PotentialGPU(str(ini))
    assert len(back._leaves(0.3)) == len(pot._leaves(0.3))
    x = _pts(500, 4)
    for t in (0.0, 0.3, 1.2, 2.5):
        for mode in (1, 2):
            a = cpu.eval_potential(pot, mode, x, t)
            b = cpu.eval_potential(back, mode, x, t)
            for u, v in zip(a, b):
                assert np.array_equal(u, v), (t, mode)
        assert np.array_equal(cpu.eval_potential(pot, 3, x, t)[3], cpu.eval_potential(back, 3, x, t)[3])


def test_export_refuses_what_ini_cannot_say(tmp_path):
    import agama_gpu_b200 as agb
    from agama_gpu_b200.export import export_potential
    inner = agb.ShiftedPotentialGPU(agb.NFWPotentialGPU(mass=1e11, scaleRadius=5.0), [1.0, 0, 0])
    with pytest.raises(ValueError, match="Scaled"):
        export_potential(agb.ScaledPotentialGPU(inner, 2.0), tmp_path / "a.ini")


def test_diskansatz_stub_still_skipped(tmp_path):
    """An Agama export's parameterless DiskAnsatz section is skipped (as in the reference);
    one with parameters is built."""
    import agama_gpu_b200 as agb
    f = tmp_path / "d.ini"
    f.write_text("[Potential 1]\ntype=DiskAnsatz\n\n[Potential 2]\ntype=NFW\nmass=1e11\nscaleRadius=5\n")
    p = agb.PotentialGPU(str(f))
    assert isinstance(p, agb.NFWPotentialGPU)
    f.write_text("[Potential 1]\ntype=DiskAnsatz\nsurfaceDensity=1e9\nscaleRadius=3\nscaleHeight=0.2\n")
    assert isinstance(agb.PotentialGPU(str(f)), agb.DiskAnsatzPotentialGPU)


@pytest.mark.gpu
def test_export_writes_device_node_tables(tmp_path):
    """After set_node_tables the export carries the current nodes: the file read back
    evaluates like the updated potential."""
    import torch
    import agama_gpu_b200 as agb
    from agama_gpu_b200.export import export_potential
    from agama_gpu_b200.synthetic import nfw_multipole
    coefs = nfw_multipole(lmax=6, n_nodes=40, seed=21, amp=0.3)
    mp = agb.MultipolePotentialGPU(coefs)
    t = mp.tables
    phi = torch.from_numpy(t.node_phi).cuda()
    dphi = torch.from_numpy(t.node_dphi_dr).cuda()
    k = list(t.lm_l).index(2)
    phi[:, k] *= 1.5
    dphi[:, k] *= 1.5
    mp.set_node_tables(phi, dphi)
    back = agb.PotentialGPU(str(export_potential(mp, tmp_path / "mp.ini")))
    x = torch.from_numpy(_pts(3000, 9)).cuda()
    fa, fb = mp.force(x), back.force(x)
    assert float((fa - fb).abs().max()) <= 1e-12 * float(fa.abs().max())
    assert float((mp.force(x) - agb.MultipolePotentialGPU(coefs).force(x)).abs().max()) > 1e-6
