"""The recorded reference trees (oracle/ref_tree.py) against the reference's own
objects, and the product's trees (evaluated by the oracle's C restatement on the
CPU) against the recorded trees.

The records are what the GPU workload-parity tests and the benchmark's reference
arm evaluate where the reference's Python cannot run; here, with the reference
sources present, they must reproduce the reference's classes exactly.
"""
import numpy as np
import pytest

from conftest import reference_available
from helpers import close_global, close_pointwise, near_pole, tree_allowance
from oracle import ref_tree

TIMES = (-0.4, 0.0, 0.31, 0.77, 1.5, 1.81, 2.6)     # before, inside and after the track


def _config2_reference_objects():
    from oracle import refpy
    from agama_gpu_b200.synthetic import composite_spec
    gp, ap = refpy.load()
    spec = composite_spec()
    return gp.CompositePotentialGPU([
        gp.MultipolePotentialGPU(spec["main"]),
        ap.MiyamotoNagaiPotentialGPU(**spec["mn"]),
        ap.DiskAnsatzPotentialGPU(**spec["disk"]),
        gp.ShiftedPotentialGPU(ap.NFWPotentialGPU(**spec["nfw"]), spec["track"]),
        gp.EvolvingPotentialGPU([gp.MultipolePotentialGPU(s) for s in spec["snaps"]],
                                spec["times"], True),
    ])


@pytest.mark.skipif(not reference_available(), reason="reference sources absent")
def test_record_reproduces_reference_objects_bit_for_bit():
    if not ref_tree.available("config2"):
        ref_tree._build_all()
    from agama_gpu_b200.synthetic import hernquist_points
    obj = _config2_reference_objects()
    rec = ref_tree.load("config2")
    xyz = hernquist_points(1500, 10.0, 8)
    for t in TIMES:
        for a, b in zip(obj.evalDeriv(xyz, t), rec.evalDeriv(xyz, t)):
            assert np.array_equal(a, b)
        for a, b in zip(obj.eval(xyz, pot=True, acc=True, t=t), rec.eval(xyz, pot=True, acc=True, t=t)):
            assert np.array_equal(a, b)
        assert np.array_equal(obj.density(xyz, t), rec.density(xyz, t))


@pytest.mark.skipif(not reference_available(), reason="reference sources absent")
def test_scaled_and_static_modifiers_recorded():
    """Scaled (T,3) and static, Shifted (T,7) and static: record equals the objects."""
    from oracle import refpy
    from agama_gpu_b200.synthetic import circular_track, hernquist_points
    gp, ap = refpy.load()
    tr = circular_track(T=120, seed=9)
    tt = tr[:, 0]
    tr7 = np.concatenate([tr, np.gradient(tr[:, 1:4], tt, axis=0)], axis=1)
    scl = np.stack([tt, 1.0 + 0.3 * np.cos(tt), 1.5 - 0.2 * tt], axis=1)
    obj = gp.CompositePotentialGPU([
        gp.ScaledPotentialGPU(ap.PlummerPotentialGPU(mass=1e10, scaleRadius=2.0), scl),
        gp.ScaledPotentialGPU(ap.HernquistPotentialGPU(mass=2e10, scaleRadius=1.0), scl[:, [0, 2]], 1.3),
        gp.ShiftedPotentialGPU(ap.IsochronePotentialGPU(mass=1e10, scaleRadius=1.5), tr7),
        gp.ScaledPotentialGPU(gp.ShiftedPotentialGPU(
            ap.UniformAccelerationGPU(ax=1.0, ay=-2.0, az=0.5), np.array([1.0, 2.0, 3.0])), 1.7, 0.8),
    ])
    ref_tree.REF_DIR.mkdir(exist_ok=True)
    ref_tree.export([(obj, "modifiers")], ref_tree.record_path("modifiers_test"))
    rec = ref_tree.load("modifiers_test")
    xyz = hernquist_points(700, 5.0, 4)
    for t in (-0.3, 0.5, 1.9, 2.4):
        for a, b in zip(obj.evalDeriv(xyz, t), rec.evalDeriv(xyz, t)):
            assert np.array_equal(a, b)
        assert np.array_equal(obj.density(xyz, t), rec.density(xyz, t))
    ref_tree.record_path("modifiers_test").unlink()


@pytest.mark.skipif(not ref_tree.available("config2"), reason="no recorded reference tree")
def test_product_tree_matches_record_on_cpu():
    """The product's config-2 tree (its tables, its flattening into leaves) evaluated by
    the oracle's C restatement equals the reference's recorded tree."""
    from oracle import cpu
    from agama_gpu_b200.synthetic import build_composite, composite_spec, hernquist_points
    pot = build_composite(composite_spec())
    rec = ref_tree.load("config2")
    xyz = hernquist_points(1200, 10.0, 6)
    ok = ~near_pole(xyz)
    for t in (0.0, 0.77, 1.81):
        op, og, oh, _ = cpu.eval_potential(pot, 2, xyz, t)
        rp, rf, rd = rec.evalDeriv(xyz, t)
        ap, ag, ah = tree_allowance(pot, xyz, t)
        assert close_pointwise(op, rp, 1e-12, ap)
        assert close_global(-og, rf, 1e-12, ag)
        assert close_global(-oh[ok], rd[ok], 1e-11, ah[ok])


def test_record_side_sample_equals_product_sample():
    from agama_gpu_b200.synthetic import hernquist_points
    for n, a, seed in ((1000, 10.0, 1000), (517, 3.5, 7)):
        assert np.array_equal(ref_tree.hernquist_points(n, a, seed), hernquist_points(n, a, seed))
