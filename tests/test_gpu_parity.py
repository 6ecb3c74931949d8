"""GPU parity: the CUDA path (public API and C ABI) against the reference's
golden vectors and against the oracle, FP64 and mixed precision."""
import ctypes

import numpy as np
import pytest

from conftest import golden
from helpers import (close_global, close_pointwise, cs_coefs, mp_coefs, near_pole, rel_max,
                     tree_allowance)
from oracle import cpu

pytestmark = pytest.mark.gpu

# FP64 tolerances against the reference / oracle (the reference's own l>0
# floor vs Agama is ~1e-7 Phi / 1e-5 force; against the same arithmetic the
# CUDA path holds these)
TOL_PHI, TOL_F, TOL_H, TOL_RHO = 1e-12, 1e-12, 1e-11, 1e-11
# mixed precision: force gate of the benchmark, and stated bounds for the rest
TOL_MIXED_F = 1e-6


def _np(t):
    return t.detach().cpu().numpy()


def _check_api(pot, g, t=0.0, keys=("phi", "force", "deriv", "rho"), sfx=""):
    import torch
    xyz = g["xyz"]
    ap, ag, ah = tree_allowance(pot, xyz, t)
    x = torch.from_numpy(xyz).cuda()
    phi = _np(pot.potential(x, t))
    assert close_pointwise(phi, g["phi" + sfx], TOL_PHI, ap)
    f = _np(pot.force(x, t))
    assert close_global(f, g["force" + sfx], TOL_F, ag)
    f2, d = pot.forceDeriv(x, t)
    assert close_global(_np(f2), f, 1e-14, ag)      # the Hessian kernel's own gradient
    ok = ~near_pole(xyz)
    assert close_global(_np(d)[ok], g["deriv" + sfx][ok], TOL_H, ah[ok])
    rho = _np(pot.density(x, t))
    assert close_global(rho, g["rho" + sfx], TOL_RHO)
    p3, f3, d3 = pot.evalDeriv(x, t)
    assert np.array_equal(_np(p3), _np(pot.eval(x, pot=True, der=True, t=t)[0]))
    assert close_pointwise(_np(p3), g["phi" + sfx], TOL_PHI, ap)


@pytest.mark.parametrize("case", ["mp_dark", "mp_lmc", "mp_cfg0", "mp_l32"])
def test_multipole_vs_reference(case):
    import agama_gpu_b200 as agb
    g = golden(case)
    _check_api(agb.MultipolePotentialGPU(mp_coefs(g)), g)


@pytest.mark.parametrize("case", ["cs_bar", "cs_cfg1"])
def test_cylspline_vs_reference(case):
    import agama_gpu_b200 as agb
    g = golden(case)
    _check_api(agb.CylSplinePotentialGPU(cs_coefs(g)), g)


ANALYTIC = ["NFWPotentialGPU", "PlummerPotentialGPU", "HernquistPotentialGPU",
            "DehnenSphericalPotentialGPU", "IsochronePotentialGPU", "MiyamotoNagaiPotentialGPU",
            "LogHaloPotentialGPU", "DiskAnsatzPotentialGPU", "UniformAccelerationGPU"]


@pytest.mark.parametrize("cls", ANALYTIC)
def test_analytic_vs_reference(cls):
    import agama_gpu_b200 as agb
    g = golden("an_" + cls)
    kw = dict(zip([str(k) for k in g["kwargs_keys"]], g["kwargs_vals"].tolist()))
    _check_api(getattr(agb, cls)(**kw), g)


def test_composite_vs_reference_all_times():
    from test_factory import build_golden_composite
    g = golden("composite")
    comp, ev = build_golden_composite(g)
    i = 0
    while f"t_{i}" in g:
        _check_api(comp, g, float(g[f"t_{i}"]), sfx=f"_{i}")
        i += 1
    import torch
    phi = _np(ev.potential(torch.from_numpy(g["xyz"]).cuda(), 0.3))
    assert close_pointwise(phi, g["phi_nearest"], TOL_PHI, tree_allowance(ev, g["xyz"], 0.3)[0])


def _big_points(n, seed):
    from agama_gpu_b200.synthetic import loguniform_points
    x = loguniform_points(n, -2.5, 3.3, seed)
    x[:64, :2] = 0.0                       # on the z axis
    x[64] = 0.0                            # origin
    return x


@pytest.mark.parametrize("lmax,nodes", [(8, 50), (32, 100)])
def test_multipole_vs_oracle_many_points(lmax, nodes):
    import torch
    import agama_gpu_b200 as agb
    from agama_gpu_b200.synthetic import nfw_multipole
    pot = agb.MultipolePotentialGPU(nfw_multipole(lmax=lmax, n_nodes=nodes, seed=lmax))
    xyz = _big_points(100_000 if lmax == 8 else 30_000, 5)
    x = torch.from_numpy(xyz).cuda()
    p, f, d = (_np(a) for a in pot.evalDeriv(x))
    op, og, oh, _ = cpu.multipole(2, xyz, pot.tables)
    _, _, _, orho = cpu.multipole(3, xyz, pot.tables)
    ap, ag, ah = tree_allowance(pot, xyz)
    assert close_pointwise(p, op, TOL_PHI, ap)
    assert close_global(f, -og, TOL_F, ag)
    ok = ~near_pole(xyz)
    assert close_global(d[ok], -oh[ok], TOL_H, ah[ok])
    assert close_global(_np(pot.density(x)), orho, TOL_RHO)


def test_kernel_signature_entries_match_reference():
    """agb_multipole_* / agb_cylspl_* take the reference's kernel arguments."""
    import torch
    from agama_gpu_b200 import _lib
    from agama_gpu_b200.prep_cylspline import build_cylspline_tables
    from agama_gpu_b200.prep_multipole import build_multipole_tables
    L = _lib.lib
    g = golden("mp_cfg0")
    t = build_multipole_tables(mp_coefs(g))
    xyz = g["xyz"]
    n = len(xyz)
    dev = lambda a, dt=torch.float64: torch.from_numpy(np.ascontiguousarray(a)).to("cuda", dt)  # noqa: E731
    x, y, z = dev(xyz[:, 0]), dev(xyz[:, 1]), dev(xyz[:, 2])
    poly = dev(t.poly)
    lml, lmm = dev(t.lm_l, torch.int32), dev(t.lm_m, torch.int32)
    phi = torch.empty(n, dtype=torch.float64, device="cuda")
    grad = torch.empty(3 * n, dtype=torch.float64, device="cuda")
    hess = torch.empty(6 * n, dtype=torch.float64, device="cuda")
    rho = torch.empty(n, dtype=torch.float64, device="cuda")
    sc = [ctypes.c_double(v) for v in t.scalars()]
    P = lambda a: ctypes.c_void_p(a.data_ptr())  # noqa: E731
    args = [P(x), P(y), P(z), P(poly), sc[0], sc[1], sc[2], ctypes.c_int(t.n_int),
            ctypes.c_int(t.n_lm), ctypes.c_int(t.lmax), P(lml), P(lmm), ctypes.c_int(t.log_scaling),
            sc[3], sc[4], sc[5], sc[6], sc[7], sc[8], sc[9]]
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert L.agb_multipole_force(*args, P(phi), P(grad), ctypes.c_int(n), st) == 0
    assert L.agb_multipole_hess(*args, P(phi), P(grad), P(hess), ctypes.c_int(n), st) == 0
    inv4 = ctypes.c_double(1.0 / (4 * np.pi * 4.30091727067736e-06))
    assert L.agb_multipole_density(*args, inv4, P(rho), ctypes.c_int(n), st) == 0
    torch.cuda.synchronize()
    ap, ag, ah = tree_allowance(__import__("agama_gpu_b200").MultipolePotentialGPU(mp_coefs(g)), xyz)
    assert close_pointwise(_np(phi), g["phi"], TOL_PHI, ap)
    assert close_global(-_np(grad).reshape(n, 3), g["force"], TOL_F, ag)
    ok = ~near_pole(xyz)
    assert close_global(-_np(hess).reshape(n, 6)[ok], g["deriv"][ok], TOL_H, ah[ok])
    assert close_global(_np(rho), g["rho"], TOL_RHO)

    g = golden("cs_bar")
    t = build_cylspline_tables(cs_coefs(g))
    xyz = g["xyz"]
    n = len(xyz)
    x, y, z = dev(xyz[:, 0]), dev(xyz[:, 1]), dev(xyz[:, 2])
    nodes, m = dev(t.node_arr), dev(t.m_arr, torch.int32)
    lR, lz, W = dev(t.lR_grid), dev(t.lz_grid), dev(t.W_outer)
    phi = torch.empty(n, dtype=torch.float64, device="cuda")
    grad = torch.empty(3 * n, dtype=torch.float64, device="cuda")
    hess = torch.empty(6 * n, dtype=torch.float64, device="cuda")
    args = [P(x), P(y), P(z), ctypes.c_double(t.Rscale), P(lR), ctypes.c_int(len(t.lR_grid)), P(lz),
            ctypes.c_int(len(t.lz_grid)), P(nodes), ctypes.c_int(t.n_harm), P(m), ctypes.c_int(t.mmax),
            ctypes.c_int(t.log_scaling), P(W), ctypes.c_double(t.r0_outer),
            ctypes.c_int(t.lmax_outer), ctypes.c_int(t.mmax_outer)]
    assert L.agb_cylspl_hess(*args, P(phi), P(grad), P(hess), ctypes.c_int(n), st) == 0
    torch.cuda.synchronize()
    assert close_pointwise(_np(phi), g["phi"], TOL_PHI)
    assert close_global(-_np(grad).reshape(n, 3), g["force"], TOL_F)
    assert close_global(-_np(hess).reshape(n, 6), g["deriv"], TOL_H)
    phi2 = torch.empty(n, dtype=torch.float64, device="cuda")
    assert L.agb_cylspl_potential(*args, P(phi2), ctypes.c_int(n), st) == 0
    torch.cuda.synchronize()
    assert close_pointwise(_np(phi2), _np(phi), 1e-14)


def test_mixed_precision_errors():
    """Mixed precision vs FP64 on a lmax-32 composite: force within the 1e-6 gate."""
    import torch
    import agama_gpu_b200 as agb
    from agama_gpu_b200.synthetic import build_composite, composite_spec, hernquist_points
    spec = composite_spec(n_snap=4)
    pot = build_composite(spec)
    x = torch.from_numpy(hernquist_points(200_000, 10.0, 3)).cuda()
    for t in (0.2, 0.77):
        p64, f64, d64 = pot.evalDeriv(x, t)
        pot.set_precision("mixed")
        p32, f32, d32 = pot.evalDeriv(x, t)
        rho32 = pot.density(x, t)
        pot.set_precision("fp64")
        rho64 = pot.density(x, t)
        ef = rel_max(_np(f32), _np(f64))
        assert ef <= TOL_MIXED_F, ef
        assert rel_max(_np(p32), _np(p64)) <= 1e-7
        assert rel_max(_np(d32), _np(d64)) <= 1e-5
        assert rel_max(_np(rho32), _np(rho64)) <= 1e-5


def test_edge_cases():
    import torch
    import agama_gpu_b200 as agb
    from agama_gpu_b200.synthetic import nfw_multipole
    pot = agb.MultipolePotentialGPU(nfw_multipole(lmax=4, n_nodes=20)) + agb.NFWPotentialGPU(1e11, 5.0)
    e = torch.empty((0, 3), dtype=torch.float64, device="cuda")
    assert pot.potential(e).shape == (0,) and pot.force(e).shape == (0, 3)
    f, d = pot.forceDeriv(e)
    assert d.shape == (0, 6)
    one = pot.potential(np.array([1.0, 2.0, 3.0]))
    assert one.dim() == 0
    f1, d1 = pot.forceDeriv([1.0, 2.0, 3.0])
    assert f1.shape == (3,) and d1.shape == (6,)
    many = pot.potential(np.array([[1.0, 2.0, 3.0]] * 5))
    assert torch.allclose(many, one.expand(5), rtol=0, atol=0)
    # host numpy, float32 and non-contiguous inputs give the same answer
    xyz = np.random.default_rng(0).normal(size=(1000, 3)) * 20
    ref = pot.force(torch.from_numpy(xyz).cuda())
    assert torch.equal(pot.force(xyz), ref)
    big = torch.from_numpy(np.concatenate([xyz, xyz], 1)).cuda()[:, ::2]
    assert torch.equal(pot.force(big[:, :3].contiguous()), pot.force(big[:, :3]))
    # NaN inputs give NaN outputs and do not disturb neighbours
    bad = xyz.copy()
    bad[7] = np.nan
    out = pot.force(bad)
    assert torch.isnan(out[7]).all() and torch.equal(out[:7], ref[:7])
    with pytest.raises(ValueError):
        pot.potential(np.zeros((4, 2)))
    with pytest.raises(ValueError):
        pot.eval(xyz)
    # determinism: bit-identical repeats
    assert torch.equal(pot.force(xyz), pot.force(xyz))


def test_binning_is_transparent():
    """Sorting the points by radial interval changes no result bit (every mode)."""
    import torch
    from agama_gpu_b200.synthetic import build_composite, composite_spec, hernquist_points
    pot = build_composite(composite_spec(lmax_main=12, n_nodes=50, n_snap=3, lmax_snap=6))
    x = torch.from_numpy(hernquist_points(150_000, 10.0, 9)).cuda()
    for prec in ("fp64", "mixed"):
        pot.set_precision(prec)
        pot.set_binning(True)
        a = pot.evalDeriv(x, 0.4) + (pot.density(x, 0.4), pot.force(x, 0.4))
        pot.set_binning(False)
        b = pot.evalDeriv(x, 0.4) + (pot.density(x, 0.4), pot.force(x, 0.4))
        for u, v in zip(a, b):
            assert torch.equal(u, v)
    pot.set_binning(True)
    pot.set_precision(None)


def test_list_and_regular_structures_agree():
    """The harmonic-list walk and the regular walk (zero-filled columns) give the
    same results; both against the oracle."""
    import torch
    import agama_gpu_b200 as agb
    from agama_gpu_b200.synthetic import nfw_multipole
    for lmax in (6, 16):
        coefs = nfw_multipole(lmax=lmax, n_nodes=40, seed=lmax)
        coefs.phi[:, 5] = 0.0                       # prune one column: list != regular
        coefs.dphi_dr[:, 5] = 0.0
        reg = agb.MultipolePotentialGPU(coefs)
        lst = agb.MultipolePotentialGPU(coefs)
        t = lst.tables
        lst._structure, lst._n_cols = 0, t.n_lm
        lst._poly_im, lst._poly32 = t.interval_major(), t.interval_major_f32()
        lst._col_scale = np.ones(t.n_lm)
        assert reg._structure != 0 and reg._n_cols > t.n_lm
        xyz = _big_points(40_000, 3)
        x = torch.from_numpy(xyz).cuda()
        ap, ag, ah = tree_allowance(reg, xyz)
        op, og, oh, _ = cpu.multipole(2, xyz, t)
        for pot in (reg, lst):
            p, f, d = (_np(a) for a in pot.evalDeriv(x))
            assert close_pointwise(p, op, TOL_PHI, ap)
            assert close_global(f, -og, TOL_F, ag)
            ok = ~near_pole(xyz)
            assert close_global(d[ok], -oh[ok], TOL_H, ah[ok])
        for prec in ("fp64", "mixed"):
            reg.set_precision(prec)
            lst.set_precision(prec)
            assert close_global(_np(reg.force(x)), _np(lst.force(x)), 1e-6 if prec == "mixed" else 1e-13, ag)


@pytest.mark.parametrize("pinned", [True, False])
def test_eval_host_pipeline_matches_eval(pinned):
    """The chunked host-memory path gives the device path's results (chunks that do
    not divide N, every output, pinned and pageable inputs)."""
    import torch
    import agama_gpu_b200 as agb
    from agama_gpu_b200.synthetic import hernquist_points, nfw_multipole
    pot = (agb.MultipolePotentialGPU(nfw_multipole(lmax=8, n_nodes=50, seed=1, amp=0.3))
           + agb.MiyamotoNagaiPotentialGPU(mass=5e10, scaleRadius=3.0, scaleHeight=0.3))
    xyz = torch.from_numpy(hernquist_points(100_003, 10.0, 2))
    if pinned:
        xyz = xyz.pin_memory()
    p, f, d = pot.eval(xyz.cuda(), pot=True, acc=True, der=True, t=0.0)
    hp, hf, hd = pot.eval_host(xyz, pot=True, acc=True, der=True, chunk_points=30_000)
    assert hp.device.type == "cpu" and hf.shape == (100_003, 3) and hd.shape == (100_003, 6)
    for h, g in ((hp, p), (hf, f), (hd, d)):
        assert float((h - g.cpu()).abs().max()) <= 1e-14 * float(g.abs().max())
    out = torch.empty((100_003, 3), dtype=torch.float64)
    r = pot.eval_host(xyz.numpy(), acc=True, out=(out,), chunk_points=1 << 19)
    assert r is out
    # GRAD mode here (HESS above): beyond the grid the two modes sum the reference's
    # ill-conditioned outer extrapolation differently, so compare with GRAD on the device
    f_dev = pot.force(xyz.cuda()).cpu()
    assert float((out - f_dev).abs().max()) <= 1e-14 * float(f_dev.abs().max())


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_eval_host_wave_chunks_match_eval(precision):
    """Large calls split into whole waves of the kernel's resident threads, launched one
    block per slot: same results as one device call (Phi+F and Phi+F+H)."""
    import torch
    import agama_gpu_b200 as agb
    from agama_gpu_b200 import _lib
    from agama_gpu_b200.potentials import _PRECISIONS, _chunk_bounds
    from agama_gpu_b200.synthetic import hernquist_points, nfw_multipole
    pot = (agb.MultipolePotentialGPU(nfw_multipole(lmax=8, n_nodes=50, seed=1, amp=0.3))
           + agb.MiyamotoNagaiPotentialGPU(mass=5e10, scaleRadius=3.0, scaleHeight=0.3))
    pot.set_precision(precision)
    n = 700_001
    xyz = torch.from_numpy(hernquist_points(n, 10.0, 3)).pin_memory()
    cargs = pot._c_args(0.0, torch.device("cuda"))
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    for mode in (_lib.MODE_GRAD, _lib.MODE_HESS):
        wave = int(_lib.lib.agb_eval_wave_points(*cargs[:4], mode, _PRECISIONS[precision]))
        assert wave > 0 and wave % (sms * 256) == 0
        sizes = [h - l for l, h in _chunk_bounds(n, 160_000, wave)]
        assert len(sizes) > 3 and all(m % wave == 0 for m in sizes[:-1])   # the wave layout
    p, f = pot.eval(xyz.cuda(), pot=True, acc=True)
    hp, hf = pot.eval_host(xyz, pot=True, acc=True, chunk_points=160_000)
    for h, g in ((hp, p), (hf, f)):
        assert float((h - g.cpu()).abs().max()) <= 1e-14 * float(g.abs().max())
    p, f, d = pot.eval(xyz.cuda(), pot=True, acc=True, der=True)
    hp, hf, hd = pot.eval_host(xyz, pot=True, acc=True, der=True, chunk_points=160_000)
    for h, g in ((hp, p), (hf, f), (hd, d)):
        assert float((h - g.cpu()).abs().max()) <= 1e-14 * float(g.abs().max())


def test_cylspline_mixed_precision():
    """CylSpline bar (mmax 6, 32x32 sinh grid), exponential-disk points: the FP32
    Hermite path against FP64 -- force within the 1e-6 gate, the rest stated."""
    import torch
    import agama_gpu_b200 as agb
    from agama_gpu_b200.synthetic import disk_points
    cs = agb.CylSplinePotentialGPU(cs_coefs(golden("cs_cfg1")))
    x = torch.from_numpy(disk_points(300_000, 3.0, 0.3, 8)).cuda()
    cs.set_precision("fp64")
    p64, f64, d64 = cs.evalDeriv(x)
    cs.set_precision("mixed")
    p32, f32, d32 = cs.evalDeriv(x)
    cs.set_precision(None)
    # the grid starts at R = 0.1: points inside it go through the FP32 Hermite; the few
    # below it take the (FP64 in both modes) outer asymptote, whose (r0/r)^(l+1) terms
    # reach 1e36 there and would swamp a max-normalised error
    xn = _np(x)
    inside = np.hypot(xn[:, 0], xn[:, 1]) >= 0.1
    assert inside.sum() > 0.99 * len(xn) and (~inside).sum() > 0
    assert rel_max(_np(f32)[inside], _np(f64)[inside]) <= TOL_MIXED_F
    assert rel_max(_np(p32)[inside], _np(p64)[inside]) <= 1e-7
    assert rel_max(_np(d32)[inside], _np(d64)[inside]) <= 1e-5
    assert np.array_equal(_np(f32)[~inside], _np(f64)[~inside])


def test_finite_difference_self_consistency():
    """F = -grad Phi, forceDeriv = dF/dx and density = Laplacian/(4 pi G) by central
    differences of the kernel's own outputs (FP64), for a Multipole + analytic composite
    and for a CylSpline (whose density keeps the reference's sign, -trace H / 4 pi G)."""
    import torch
    import agama_gpu_b200 as agb
    from agama_gpu_b200.synthetic import nfw_multipole
    rng = np.random.default_rng(17)
    mp = (agb.MultipolePotentialGPU(nfw_multipole(lmax=8, n_nodes=50, seed=4, amp=0.3))
          + agb.MiyamotoNagaiPotentialGPU(mass=5e10, scaleRadius=3.0, scaleHeight=0.3)
          + agb.PlummerPotentialGPU(mass=1e10, scaleRadius=1.0))
    cs = agb.CylSplinePotentialGPU(cs_coefs(golden("cs_cfg1")))
    for pot, sign in ((mp, 1.0), (cs, -1.0)):
        r = np.exp(rng.uniform(np.log(0.5), np.log(80.0), 400))
        u = rng.normal(size=(400, 3))
        xyz = u / np.linalg.norm(u, axis=1)[:, None] * r[:, None]
        xyz = xyz[np.hypot(xyz[:, 0], xyz[:, 1]) > 0.3]          # inside the CylSpline grid
        x = torch.from_numpy(xyz).cuda()
        phi, F, D = pot.evalDeriv(x)
        rho = pot.density(x)
        hs = 1e-5 * np.maximum(np.linalg.norm(xyz, axis=1), 1.0)
        fd_F = np.zeros_like(xyz)
        fd_D = np.zeros((len(xyz), 3, 3))
        for d in range(3):
            e = np.zeros_like(xyz)
            e[:, d] = hs
            pp, Fp, _ = pot.evalDeriv(torch.from_numpy(xyz + e).cuda())
            pm, Fm, _ = pot.evalDeriv(torch.from_numpy(xyz - e).cuda())
            fd_F[:, d] = -(_np(pp) - _np(pm)) / (2 * hs)
            fd_D[:, :, d] = (_np(Fp) - _np(Fm)) / (2 * hs)[:, None]
        Fn, Dn = _np(F), _np(D)
        assert np.abs(Fn - fd_F).max() <= 1e-6 * np.abs(Fn).max()
        # forceDeriv order [xx, yy, zz, xy, yz, zx]
        Dm = np.stack([fd_D[:, 0, 0], fd_D[:, 1, 1], fd_D[:, 2, 2], fd_D[:, 0, 1], fd_D[:, 1, 2],
                       fd_D[:, 2, 0]], 1)
        if pot is mp:      # the CylSpline forceDeriv omits the reference's dPhi/dphi terms
            assert np.abs(Dn - Dm).max() <= 1e-5 * np.abs(Dn).max()
        lap = -(Dn[:, 0] + Dn[:, 1] + Dn[:, 2])
        want = sign * lap * agb.INV_4PIG
        assert np.abs(_np(rho) - want).max() <= 1e-9 * np.abs(want).max()


@pytest.mark.parametrize("prec", ["mixed", "fp64"])
def test_evolving_pair_walk_equals_separate_snapshots(prec):
    """The two bracketing snapshots of an Evolving potential share one harmonic walk in
    the mixed kernel; the result equals the weighted sum of the snapshots evaluated alone
    (and the oracle)."""
    import torch
    import agama_gpu_b200 as agb
    from agama_gpu_b200.synthetic import hernquist_points, nfw_multipole
    snaps = [agb.MultipolePotentialGPU(nfw_multipole(lmax=12, n_nodes=60, seed=4, drift=0.3 * i,
                                                     amp=0.2)) for i in range(3)]
    ev = agb.EvolvingPotentialGPU(snaps, [0.0, 1.0, 2.0], interpolate=True)
    x = torch.from_numpy(hernquist_points(200_000, 10.0, 9)).cuda()
    t, alpha = 1.3, 0.3
    p, f = ev._launch(x, t, 1, True, precision=prec)[:2]
    p1, f1 = snaps[1]._launch(x, t, 1, True, precision=prec)[:2]
    p2, f2 = snaps[2]._launch(x, t, 1, True, precision=prec)[:2]
    pr, fr = (1 - alpha) * p1 + alpha * p2, (1 - alpha) * f1 + alpha * f2
    assert float((p - pr).abs().max()) <= 1e-13 * float(pr.abs().max())
    assert float((f - fr).abs().max()) <= 1e-13 * float(fr.abs().max())
    po, go, _, _ = cpu.eval_potential(ev, 1, x[:20000].cpu().numpy(), t)
    # FP64 against the oracle: rounding of the outer extrapolation's large terms, ~1e-8
    tol = 2e-6 if prec == "mixed" else 1e-7
    assert np.abs(f[:20000].cpu().numpy() + go).max() <= tol * np.abs(go).max()
