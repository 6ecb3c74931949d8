"""Generate the golden vectors in this directory from the reference itself.

Runs the reference's own code on the CPU -- its Python wrapper and table
builders imported with a numpy-backed cupy stand-in, its CUDA kernels compiled
as host C++, its analytic ElementwiseKernel bodies compiled unchanged (see
oracle/refpy.py) -- on:

* the reference's three coefficient fixtures (tests/600.dark.none_8.coef_mul_DR,
  tests/100.LMC.none_8.coef_mult, tests/600.bar.none_8.coef_cylsp_DR);
* seeded synthetic Multipole / CylSpline sets shaped like the benchmark workloads;
* the nine analytic profiles;
* a time-dependent composite (Shifted with (T,4) and (T,7) tracks, Scaled with
  (T,3) tables, Evolving, Composite) through the reference's classes.

Each case stores its inputs (coefficient arrays, parameters, points), the
reference's tables and the reference's API outputs (potential, force,
forceDeriv, density).  Usage (needs the reference sources):

    python tests/golden/make_golden.py [--reference <reference checkout>]
"""
from __future__ import annotations

import argparse
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))


def special_points(r_nodes: np.ndarray) -> np.ndarray:
    """Origin, poles, grid nodes, interval midpoints, both extrapolation sides."""
    pts = [np.zeros(3)]
    for r in (r_nodes[0] * 0.3, r_nodes[3], r_nodes[len(r_nodes) // 2], r_nodes[-1] * 2.0):
        pts += [np.array([0.0, 0.0, r]), np.array([0.0, 0.0, -r]),
                np.array([1e-12 * r, 0.0, r]), np.array([r, 0.0, 0.0]), np.array([-r, 0.0, 0.0])]
    mids = np.sqrt(r_nodes[1:] * r_nodes[:-1])
    rng = np.random.default_rng(7)
    for r in np.concatenate([r_nodes, mids]):
        u = rng.normal(size=3)
        pts.append(u / np.linalg.norm(u) * r)
    return np.array(pts)


def mp_case(gp, coefs, name, n_rand, seed, out):
    from agama_gpu_b200.synthetic import loguniform_points
    r = np.asarray(coefs.R_grid)
    lo, hi = np.log10(r[0]) - 0.7, np.log10(r[-1]) + 0.5
    xyz = np.concatenate([special_points(r), loguniform_points(n_rand, lo, hi, seed)])
    pot = gp.MultipolePotentialGPU(coefs)
    d = gp._build_multipole_data(coefs)
    f, dd = pot.forceDeriv(xyz)
    poly = d["poly"]
    sel = np.arange(poly.size)
    if poly.size > 20000:             # large tables: a seeded subsample of entries
        sel = np.sort(np.random.default_rng(13).choice(poly.size, 20000, replace=False))
    out[name] = dict(
        R_grid=r, phi_tab=np.asarray(coefs.phi), dphi_tab=np.asarray(coefs.dphi_dr),
        lm_labels=np.array(coefs.lm_labels, dtype=np.int32),
        ref_poly_shape=np.array(poly.shape), ref_poly_idx=sel, ref_poly_val=poly.reshape(-1)[sel],
        ref_lm_l=d["lm_l"], ref_lm_m=d["lm_m"],
        ref_scalars=np.array([d[k] for k in ("logr_min", "dlogr", "inv_dlogr", "invPhi0",
                                             "inner_s", "inner_U", "inner_W", "outer_s",
                                             "outer_U", "outer_W")]),
        ref_ints=np.array([d["n_intervals"], d["n_lm"], d["lmax"], d["log_scaling"]]),
        xyz=xyz, phi=pot.potential(xyz), force=pot.force(xyz), deriv=dd, force_h=f,
        rho=pot.density(xyz))


def cs_case(gp, coefs, name, xyz, out):
    pot = gp.CylSplinePotentialGPU(coefs)
    d = gp._build_cylspline_data(coefs)
    ms = sorted(coefs.phi)
    f, dd = pot.forceDeriv(xyz)
    node = d["node_arr"]
    rng = np.random.default_rng(11)
    sel = np.sort(rng.choice(node.size, size=min(node.size, 6000), replace=False))
    out[name] = dict(
        R_grid=np.asarray(coefs.R_grid), z_grid=np.asarray(coefs.z_grid),
        m_list=np.array(ms, dtype=np.int32), phi_tabs=np.stack([coefs.phi[m] for m in ms]),
        ref_scalars=np.array([d["Rscale"], d["r0_outer"], d["log_scaling"], d["mmax"],
                              d["lmax_outer"], d["mmax_outer"]]),
        ref_W=d["W_outer"], ref_lR=d["lR_grid"], ref_lz=d["lz_grid"],
        ref_node_shape=np.array(node.shape), ref_node_idx=sel, ref_node_val=node.reshape(-1)[sel],
        xyz=xyz, phi=pot.potential(xyz), force=pot.force(xyz), deriv=dd, force_h=f,
        rho=pot.density(xyz))


ANALYTIC = [
    ("NFWPotentialGPU", dict(mass=1e12, scaleRadius=20.0)),
    ("PlummerPotentialGPU", dict(mass=1e11, scaleRadius=3.0)),
    ("HernquistPotentialGPU", dict(mass=1e11, scaleRadius=3.0)),
    ("DehnenSphericalPotentialGPU", dict(mass=1e11, scaleRadius=3.0, gamma=0.5)),
    ("IsochronePotentialGPU", dict(mass=1e11, scaleRadius=3.0)),
    ("MiyamotoNagaiPotentialGPU", dict(mass=5e10, scaleRadius=3.0, scaleHeight=0.3)),
    ("LogHaloPotentialGPU", dict(velocity=200.0, coreRadius=2.0, axisRatioY=0.9, axisRatioZ=0.7)),
    ("DiskAnsatzPotentialGPU", dict(surfaceDensity=1e9, scaleRadius=3.0, scaleHeight=0.3,
                                    innerCutoffRadius=1.0)),
    ("UniformAccelerationGPU", dict(ax=1.5, ay=-2.0, az=0.25)),
]


def analytic_case(ap, out):
    from agama_gpu_b200.synthetic import loguniform_points
    xyz = np.concatenate([special_points(np.array([0.01, 0.1, 1.0, 10.0, 100.0])),
                          loguniform_points(700, -2.0, 2.5, 21)])
    for cls, kw in ANALYTIC:
        pot = getattr(ap, cls)(**kw)
        f, dd = pot.forceDeriv(xyz)
        out["an_" + cls] = dict(kwargs_keys=np.array(list(kw.keys())),
                                kwargs_vals=np.array(list(kw.values()), dtype=np.float64),
                                xyz=xyz, phi=pot.potential(xyz), force=pot.force(xyz),
                                deriv=dd, force_h=f, rho=pot.density(xyz))


def composite_case(gp, ap, out):
    """Composite of every layer, through the reference's own classes."""
    from agama_gpu_b200.synthetic import circular_track, hernquist_points, nfw_multipole
    main = nfw_multipole(lmax=6, n_nodes=40, seed=5)
    snaps = [nfw_multipole(lmax=4, n_nodes=30, M=2e11, rs=12.0, seed=105, drift=0.25 * i)
             for i in range(3)]
    times = np.array([0.0, 0.5, 1.0])
    track4 = circular_track(T=200, seed=4)
    tt = track4[:, 0]
    track7 = np.concatenate([track4, np.gradient(track4[:, 1:4], tt, axis=0)], axis=1)
    scl3 = np.stack([tt, 1.0 + 0.2 * np.sin(tt), 2.0 + 0.5 * tt], axis=1)
    pots = [
        gp.MultipolePotentialGPU(main),
        ap.MiyamotoNagaiPotentialGPU(mass=5e10, scaleRadius=3.0, scaleHeight=0.3),
        ap.DiskAnsatzPotentialGPU(surfaceDensity=1e9, scaleRadius=3.0, scaleHeight=0.3),
        gp.ShiftedPotentialGPU(ap.NFWPotentialGPU(mass=1.5e11, scaleRadius=10.0), track4),
        gp.EvolvingPotentialGPU([gp.MultipolePotentialGPU(s) for s in snaps], times, True),
        gp.ScaledPotentialGPU(ap.PlummerPotentialGPU(mass=1e10, scaleRadius=2.0), scl3),
        gp.ShiftedPotentialGPU(gp.ScaledPotentialGPU(ap.HernquistPotentialGPU(mass=3e10,
                                                                              scaleRadius=1.0),
                                                     0.5, 2.0), track7),
        gp.ScaledPotentialGPU(gp.ShiftedPotentialGPU(ap.IsochronePotentialGPU(mass=1e10,
                                                                              scaleRadius=1.5),
                                                     np.array([3.0, -2.0, 1.0])), 1.7, 0.8),
    ]
    comp = gp.CompositePotentialGPU(pots)
    xyz = hernquist_points(1200, 10.0, 31)
    res = {}
    for i, t in enumerate([-0.3, 0.0, 0.37, 0.5, 0.81, 1.4, 2.5]):
        f, dd = comp.forceDeriv(xyz, t)
        res[f"phi_{i}"] = comp.potential(xyz, t)
        res[f"force_{i}"] = comp.force(xyz, t)
        res[f"deriv_{i}"] = dd
        res[f"rho_{i}"] = comp.density(xyz, t)
        res[f"t_{i}"] = np.array(t)
    ev = gp.EvolvingPotentialGPU([gp.MultipolePotentialGPU(s) for s in snaps], times, False)
    res["phi_nearest"] = ev.potential(xyz, 0.3)
    out["composite"] = dict(
        main_R=main.R_grid, main_phi=main.phi, main_dphi=main.dphi_dr,
        main_labels=np.array(main.lm_labels, dtype=np.int32),
        snap_R=np.stack([s.R_grid for s in snaps]), snap_phi=np.stack([s.phi for s in snaps]),
        snap_dphi=np.stack([s.dphi_dr for s in snaps]),
        snap_labels=np.array(snaps[0].lm_labels, dtype=np.int32), times=times,
        track4=track4, track7=track7, scl3=scl3, xyz=xyz, **res)


def main():
    ap_ = argparse.ArgumentParser()
    ap_.add_argument("--reference", default=None,
                     help="reference checkout (default: AGB_REFERENCE, else oracle.refpy's)")
    args = ap_.parse_args()
    if args.reference:
        os.environ["AGB_REFERENCE"] = args.reference
    from oracle import refpy
    args.reference = str(refpy.REF_DIR)
    from agama_gpu_b200.coefs import read_coefs
    from agama_gpu_b200.synthetic import bar_cylspline, disk_points, nfw_multipole
    gp, ap = refpy.load()
    ref_tests = Path(args.reference) / "tests"
    out: dict = {}
    mp_case(gp, read_coefs(ref_tests / "600.dark.none_8.coef_mul_DR"), "mp_dark", 1500, 1, out)
    mp_case(gp, read_coefs(ref_tests / "100.LMC.none_8.coef_mult"), "mp_lmc", 1500, 2, out)
    mp_case(gp, nfw_multipole(lmax=8, n_nodes=50, seed=0), "mp_cfg0", 1500, 3, out)
    mp_case(gp, nfw_multipole(lmax=32, n_nodes=60, seed=9, amp=0.2), "mp_l32", 1000, 4, out)
    bar = read_coefs(ref_tests / "600.bar.none_8.coef_cylsp_DR")
    rng = np.random.default_rng(5)
    R = 10 ** rng.uniform(-2, 2.9, 1500)
    ph = rng.uniform(0, 2 * np.pi, 1500)
    z = rng.normal(size=1500) * np.where(rng.uniform(size=1500) < 0.6, 2.0, 200.0)
    xyz_bar = np.concatenate([np.stack([R * np.cos(ph), R * np.sin(ph), z], 1),
                              [[0, 0, 0.5], [0, 0, -3.0], [0, 0, 700.0], [600.0, 0, 0]]])
    cs_case(gp, bar, "cs_bar", xyz_bar, out)
    cfg1 = bar_cylspline()
    xyz1 = np.concatenate([disk_points(1500, seed=6), [[0, 0, 0.1], [0.05, 0.02, 0.0],
                                                       [300.0, 0, 0], [0, 0, -250.0]]])
    cs_case(gp, cfg1, "cs_cfg1", xyz1, out)
    analytic_case(ap, out)
    composite_case(gp, ap, out)
    for name, arrays in out.items():
        np.savez_compressed(HERE / f"{name}.npz", **arrays)
        print(name, sum(v.nbytes for v in arrays.values()) // 1024, "KiB")


if __name__ == "__main__":
    main()
