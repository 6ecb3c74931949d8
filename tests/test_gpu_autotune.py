"""Autotuner: every launch shape gives the same results; the choice is kept and cached."""
import json

import pytest

pytestmark = pytest.mark.gpu


def _pot():
    import agama_gpu_b200 as agb
    from agama_gpu_b200.synthetic import nfw_multipole
    return (agb.MultipolePotentialGPU(nfw_multipole(lmax=10, n_nodes=60, seed=3, amp=0.3))
            + agb.MiyamotoNagaiPotentialGPU(mass=5e10, scaleRadius=3.0, scaleHeight=0.3))


@pytest.mark.parametrize("n", [5000, 70000])
def test_launch_shapes_agree(n, tmp_path, monkeypatch):
    import torch
    from agama_gpu_b200 import _lib, autotune
    monkeypatch.setenv("AGB_AUTOTUNE_CACHE", str(tmp_path / "cache.json"))
    pot = _pot()
    from agama_gpu_b200.synthetic import hernquist_points
    x = torch.from_numpy(hernquist_points(n, 10.0, 4)).cuda()
    ref = pot.force(x)
    for prec in ("fp64", "mixed"):
        pc = _lib.PREC_FP64 if prec == "fp64" else _lib.PREC_MIXED
        for mode in (_lib.MODE_GRAD, _lib.MODE_POT, _lib.MODE_HESS, _lib.MODE_DENS):
            base = pot._launch(x, 0.0, mode, True, precision=prec)
            cands = autotune._candidates(n, mode)
            if mode != _lib.MODE_GRAD:       # every block size and both schedule kinds
                cands = [c for c in cands if c[0].endswith(("/grid2", "/ppt16"))]
            for name, flags in cands:
                autotune._set(pot, mode, pc, n, flags)
                got = pot._launch(x, 0.0, mode, True, precision=prec)
                for g, b in zip(got, base):
                    if b is not None:
                        assert float((g - b).abs().max()) <= 1e-14 * float(b.abs().max()), \
                            (prec, mode, name)
            pot.__dict__.pop("_tuned", None)
    res = autotune.autotune(pot, x, mode="force", precision="mixed", reps=2)
    assert res["best"] in res["ms"]
    assert len(res["ms"]) == len(autotune._candidates(n, _lib.MODE_GRAD)) == 48
    assert (_lib.MODE_GRAD, _lib.PREC_MIXED, n.bit_length()) in pot._tuned
    assert torch.equal(pot.force(x), ref)                 # fp64 calls keep their own shape
    rec = json.loads((tmp_path / "cache.json").read_text())
    assert len(rec) == 1
    fresh = _pot()
    assert autotune.apply_cached(fresh, n, mode="force", precision="mixed")
    assert fresh._tuned == pot._tuned


def test_large_call_default_shapes_match_256_threads():
    """Above 2^21 points a call of a tree with a Multipole defaults to 512 threads per
    block (force, density) or 128 (Hessian; 16 points per thread in FP64); the results
    equal the 256-thread shape's (both precisions, sorted and unsorted)."""
    import torch
    from agama_gpu_b200 import _lib, autotune
    from agama_gpu_b200.synthetic import hernquist_points
    pot = _pot()
    n = (1 << 21) + 4099
    x = torch.from_numpy(hernquist_points(n, 10.0, 6)).cuda()
    for prec in ("fp64", "mixed"):
        pc = _lib.PREC_FP64 if prec == "fp64" else _lib.PREC_MIXED
        for binning in (True, False):
            pot.set_binning(binning)
            for mode in (_lib.MODE_GRAD, _lib.MODE_HESS, _lib.MODE_DENS):
                pot.__dict__.pop("_tuned", None)
                a = pot._launch(x, 0.0, mode, True, precision=prec)
                autotune._set(pot, mode, pc, n, 1 << _lib.OUT_GRID_SHIFT)   # 256 x 1 per slot
                b = pot._launch(x, 0.0, mode, True, precision=prec)
                for u, v in zip(a, b):
                    if v is not None:
                        assert torch.equal(u, v), (prec, binning, mode)
    pot.set_binning(True)
    pot.__dict__.pop("_tuned", None)


def test_tune_batch_keeps_results():
    import torch
    import agama_gpu_b200 as agb
    from agama_gpu_b200 import autotune
    from agama_gpu_b200.synthetic import hernquist_points, nfw_multipole
    units = [agb.MultipolePotentialGPU(nfw_multipole(lmax=l, n_nodes=40, seed=l, amp=0.3))
             for l in (2, 8, 14)]
    batch = agb.BatchedPotentialGPU(units, [3000, 9000, 500])
    x = torch.from_numpy(hernquist_points(batch.n_points, 8.0, 5)).cuda()
    f0 = batch.force(x)
    res = autotune.tune_batch(batch, x, tiles=(256, 2048, 8192))
    assert (batch.tile_points, batch.stage) == res["best"] and len(res["ms"]) == 6
    f1 = batch.force(x)
    assert float((f1 - f0).abs().max()) <= 1e-14 * float(f0.abs().max())
