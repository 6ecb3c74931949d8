"""Benchmark: force+Phi points/s of the fused evaluator on the time-dependent
composite (Multipole lmax=32 x 100 nodes + MiyamotoNagai + DiskAnsatz + NFW
Shifted on a (1000,4) track + Evolving over 16 lmax=16 snapshots) at N=4M
isotropic Hernquist (a=10 kpc) points per GPU, mixed precision (headline) and
plain FP64 side by side.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = one potential+force evaluation of all N points at one time t (t
varies per step inside the track and the snapshot range).  Inputs are
resident in HBM for `value`; `e2e` goes through the public API from pinned
host memory and reads the results back.  L2 is flushed (256 MiB write)
between timed steps.  Under torchrun every rank evaluates its own N points
(weak scaling, no data-path collective); timing is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "force+Phi pts/s (mixed-precision fused kernel; FP64 kernel alongside)"
WORKLOAD = ("time-dependent composite: Multipole lmax=32 x 100 nodes + MiyamotoNagai + "
            "DiskAnsatz + Shifted NFW on (1000,4) track + Evolving 16 x lmax=16 snapshots; "
            "isotropic Hernquist a=10 kpc points")
G = 4.30091727067736e-06
# DRAM bytes (read + write) per point of one mixed-precision launch on this workload:
# ncu dram__bytes_read.sum + dram__bytes_write.sum = 100.85 MB + 86.01 MB for one 4M-point
# launch of a binned step (512 threads per block; profiles/eval_kernel_composite_4M_full.txt),
# scaled linearly with the point count
TRAFFIC_BYTES_PER_POINT = 46.71
# wall-clock budget of the reference arm's timed steps (seconds)
REF_BUDGET_S = 150.0


def measured_hbm_peak():
    """Copy bandwidth in GB/s measured on this machine's GPUs, when a record is present."""
    try:
        with open(ROOT / "MEASURED_PEAKS.json") as f:
            return float(json.load(f)["hbm_gbs"])
    except (OSError, ValueError, KeyError, TypeError):
        return None


def step_times(k_total: int):
    """Evaluation times inside the centre track (0..2) and the snapshots (0..1.5)."""
    return [0.05 + 1.4 * ((0.6180339887 * (k + 1)) % 1.0) for k in range(k_total)]


def flops_per_step(pot, xyz: np.ndarray, t: float) -> tuple:
    """Algorithmic FLOPs of one Phi+F evaluation (the roofline's fixed convention):
    Multipole 48*n_harm + 64 per point inside its grid (64 outside), analytic 30
    per component.  Returns (fp32-eligible harmonic flops, fp64 flops)."""
    from agama_gpu_b200 import _lib as L
    f_harm = 0.0
    f_point = 0.0
    for comp, sigma, gamma, ampl in pot._leaves(t):
        if comp.kind == L.KIND_MULTIPOLE:
            tb = comp.tables
            x = sigma * xyz - np.asarray(gamma)[None, :]
            lr = np.log(np.maximum(np.linalg.norm(x, axis=1), 1e-300))
            inside = np.count_nonzero((lr >= tb.logr_min) & (lr < tb.logr_min + tb.n_int * tb.dlogr))
            f_harm += 48.0 * tb.n_lm * inside
            f_point += 64.0 * len(xyz)
        elif comp.kind == L.KIND_CYLSPLINE:
            f_harm += 110.0 * comp.tables.n_harm * len(xyz)
            f_point += 80.0 * len(xyz)
        else:
            f_point += 30.0 * len(xyz)
    return f_harm, f_point


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                self.out, _ = self.proc.communicate()
        return False

    def summary(self):
        if self.proc is None or not getattr(self, "out", ""):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.out.strip().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(smax)),
                "reasons": sorted(reasons), "samples": len(sm)}


def _config(n_points: int, world: int) -> dict:
    """The workload description both arms print (the driver compares them)."""
    return {"workload": WORKLOAD, "points_per_gpu": n_points,
            "l2": "flushed (256 MiB write) between timed steps",
            "parallelism": f"points sharded, {world} rank(s), no data-path collective"}


def reference_unavailable(why: str) -> None:
    print(json.dumps({"impl": "reference", "unavailable": why}))


def run_reference(args):
    """The reference's CPU implementation of the path, timed on the host cores.

    The potential is the reference's own config-2 tree: built by its classes and
    table builders and recorded where its sources are (oracle/ref_tree.py), then
    evaluated here by its kernel code compiled for the host (its two .cu files and
    its ElementwiseKernel bodies, OpenMP over all cores) with the call structure of
    its ``eval(xyz, pot=True, acc=True, t)``: a potential pass and a force pass over
    every component, outputs summed, the Shifted centre and the Evolving bracket
    from its splines.  This repository's package is not imported.  Each step
    evaluates the step's points at one time; warm-up steps use an eighth of them."""
    from oracle import ref_tree
    if not ref_tree.available("config2"):
        return reference_unavailable("the recorded reference tree (oracle/_ref/tree_config2.npz) "
                                     "is absent: run __graft_entry__.build() where the reference "
                                     "sources are")
    tree = ref_tree.load("config2")
    threads = os.cpu_count() or 1
    xyz = ref_tree.hernquist_points(args.n, 10.0, 1000)      # rank 0's points of the GPU arm
    ts = step_times(args.warmup + args.steps)
    t0 = time.perf_counter()
    for k in range(args.warmup):
        tree.eval(xyz[: max(1, args.n // 8)], pot=True, acc=True, t=ts[k], nthreads=threads)
    warm = time.perf_counter() - t0
    # bound the run: the timed steps evaluate at most what fits in REF_BUDGET_S at
    # the warm-up rate (all N points unless the host is slow)
    rate = args.warmup * max(1, args.n // 8) / max(warm, 1e-9) if args.warmup else 1e300
    n = int(min(args.n, max(250_000, rate * REF_BUDGET_S / max(args.steps, 1))))
    sub = xyz[:n]
    times = []
    for k in range(args.steps):
        t1 = time.perf_counter()
        tree.eval(sub, pot=True, acc=True, t=ts[args.warmup + k], nthreads=threads)
        times.append(time.perf_counter() - t1)
    dt = float(np.mean(times))
    value = n / dt
    sample = (f"{n} of the workload's {args.n} Hernquist points per step (Phi+F at the step's "
              f"time): the reference's recorded config-2 tree, its kernel code compiled for "
              f"the host, {threads} OpenMP threads")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "pts/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": dt * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "config": _config(args.n, args.gpus),
            "sample_points_per_step": n,
            "cpu_baseline": {"value": value, "unit": "pts/s", "cores": threads,
                             "kind": "reference", "sample": sample},
            "e2e": {"value": value, "unit": "pts/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def adjoint_ratio(dev, n_streams: int, per_stream: int, n_steps: int, precision: str,
                  checkpoint_every=None, reconstruct="recompute"):
    """Adjoint / forward time of the stream workload (1024 clouds x 2048 particles, 2000
    steps by default): Gaussian clouds (0.1 kpc, 1 km/s)
    on circular orbits at 10-60 kpc in an lmax=16 x 64-node Multipole + Miyamoto-Nagai,
    leapfrog dt = 1e-3 Gyr; loss = sum |x_T - target|^2; the backward returns dL/dx0,
    dL/dv0 and dL/d(quintic coefficients) of the Multipole."""
    import torch
    import agama_gpu_b200 as agb
    from agama_gpu_b200.integrate import Leapfrog, auto_checkpoint_every, gyr_to_time
    from agama_gpu_b200.synthetic import nfw_multipole
    rng = np.random.default_rng(77)
    mp = agb.MultipolePotentialGPU(nfw_multipole(lmax=16, n_nodes=64, seed=16))
    pot = mp + agb.MiyamotoNagaiPotentialGPU(mass=5e10, scaleRadius=3.0, scaleHeight=0.3)
    R0 = rng.uniform(10.0, 60.0, n_streams)
    ph0 = rng.uniform(0, 2 * np.pi, n_streams)
    inc = rng.uniform(0, np.pi, n_streams)
    c0 = np.stack([R0 * np.cos(ph0), R0 * np.sin(ph0) * np.cos(inc), R0 * np.sin(ph0) * np.sin(inc)], 1)
    vc = np.sqrt(np.maximum(-(pot.force(c0).cpu().numpy() * c0).sum(1), 1.0))
    t_hat = np.stack([-np.sin(ph0), np.cos(ph0) * np.cos(inc), np.cos(ph0) * np.sin(inc)], 1)
    v0c = t_hat * vc[:, None]
    x0 = np.repeat(c0, per_stream, 0) + rng.normal(0, 0.1, (n_streams * per_stream, 3))
    v0 = np.repeat(v0c, per_stream, 0) + rng.normal(0, 1.0, (n_streams * per_stream, 3))
    x0t = torch.from_numpy(x0).to(dev)
    v0t = torch.from_numpy(v0).to(dev)
    target = x0t + torch.from_numpy(rng.normal(0, 1.0, x0.shape)).to(dev)
    integ = Leapfrog(pot, gyr_to_time(1e-3), precision=precision)
    if checkpoint_every is None:
        checkpoint_every = auto_checkpoint_every(x0t, n_steps)
    # warm-up: graph capture, every kernel of the adjoint, and the allocator's blocks
    nw = 2 * integ.graph_steps
    xw, vw, ck = integ.run(x0t, v0t, nw, checkpoint_every)
    integ.adjoint(ck, nw, 2 * (xw - target), torch.zeros_like(vw), table_grads=True,
                  reconstruct=reconstruct)
    integ.adjoint(ck, nw, 2 * (xw - target), torch.zeros_like(vw), reconstruct=reconstruct)
    mp.node_gradients(mp.table_vjp(x0t[:1024], 0.0, None, torch.ones_like(x0t[:1024])))
    del ck
    xw, vw, ck = integ.run(x0t, v0t, n_steps, checkpoint_every)
    del ck
    torch.cuda.synchronize()
    e0, e1, e2, e3 = (torch.cuda.Event(enable_timing=True) for _ in range(4))
    e0.record()
    xT, vT, ck = integ.run(x0t, v0t, n_steps, checkpoint_every)
    e1.record()
    lx, lv, tg = integ.adjoint(ck, n_steps, 2 * (xT - target), torch.zeros_like(vT),
                               table_grads=True, reconstruct=reconstruct)
    gnodes = mp.node_gradients(tg[mp], tg.get(("const", mp)))
    e2.record()
    lx2, _ = integ.adjoint(ck, n_steps, 2 * (xT - target), torch.zeros_like(vT),
                           reconstruct=reconstruct)
    e3.record()
    torch.cuda.synchronize()
    del ck
    fwd, adj, adj_x = e0.elapsed_time(e1), e1.elapsed_time(e2), e2.elapsed_time(e3)
    ok = bool(torch.isfinite(lx).all() and torch.isfinite(gnodes[0]).all()
              and torch.isfinite(lx2).all())
    return {"forward_ms": fwd, "adjoint_ms": adj, "ratio": adj / fwd,
            "adjoint_phase_space_only_ms": adj_x, "ratio_phase_space_only": adj_x / fwd,
            "steps": n_steps,
            "particles": n_streams * per_stream, "checkpoint_every": checkpoint_every,
            "precision": precision, "finite": ok, "reconstruct": reconstruct,
            "backward_returns": "dL/dx0, dL/dv0, dL/dPhi_nodes, dL/d(dPhi/dr)_nodes (17^2 x 64)"}


def batched_units(dev, n_units: int, steps: int, warmup: int, lf_steps: int, precision: str):
    """Many independent potentials in one launch: n_units NFW-based Multipoles
    (lmax ~ U{2..32}, nodes ~ U[30,120], M ~ logU[1e10,1e12], rs ~ U[2,30]) with
    N_i ~ logU[1e3, 5e5] Hernquist(a = rs) particles each, stacked.  Times the
    batched force evaluation (one work-queue launch), the same work as one call per
    unit, and lf_steps leapfrog steps captured in one CUDA graph."""
    import torch
    import agama_gpu_b200 as agb
    from agama_gpu_b200.integrate import Leapfrog
    from agama_gpu_b200.synthetic import config4_unit_specs, hernquist_points, nfw_multipole
    units, counts, xs, flops = [], [], [], 0.0
    for spec in config4_unit_specs(n_units):
        mp = agb.MultipolePotentialGPU(nfw_multipole(**spec["coefs"]))
        n = spec["n_points"]
        units.append(mp)
        counts.append(n)
        xs.append(hernquist_points(n, spec["a"], 1000 + spec["index"]))
        flops += n * (48.0 * mp.tables.n_lm + 64.0)
    batch = agb.BatchedPotentialGPU(units, counts, precision=precision)
    x = torch.from_numpy(np.concatenate(xs)).to(dev)
    del xs
    N = batch.n_points
    F = torch.empty_like(x)
    ev = lambda: batch._launch(x, 0.0, 1, False, out=(None, F, None, None))  # noqa: E731
    rows = [batch.unit_rows(u) for u in range(n_units)]
    xu = [x[r] for r in rows]
    Fu = [torch.empty_like(a) for a in xu]

    def loop():
        for u in range(n_units):
            units[u]._launch(xu[u], 0.0, 1, False, precision=precision, out=(None, Fu[u], None, None))

    def timed(fn, k):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(k):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / k
    t_batch = timed(ev, steps)
    t_batch64 = timed(lambda: batch._launch(x, 0.0, 1, False, precision="fp64",
                                            out=(None, F, None, None)), steps)
    t_loop = timed(loop, max(1, steps // 2))
    ev()
    err = max(float((F[r] - f).abs().max()) / max(float(f.abs().max()), 1e-300)
              for r, f in zip(rows, Fu) if r.stop > r.start)
    del Fu, xu
    # leapfrog: circular-ish velocities from the batched force, lf_steps steps per graph
    vc = (F * x).sum(1, keepdim=True).neg().clamp_min(1.0).sqrt()
    e = torch.zeros_like(x)
    e[:, 2] = 1.0
    t_hat = torch.linalg.cross(e, x)
    t_hat = t_hat / t_hat.norm(dim=1, keepdim=True).clamp_min(1e-12)
    v = t_hat * vc
    integ = Leapfrog(batch, 0.001, precision=precision, graph_steps=lf_steps)
    integ.run(x, v, lf_steps, checkpoint_every=lf_steps)        # capture + warm-up
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    xT, vT, _ = integ.run(x, v, lf_steps, checkpoint_every=lf_steps)
    e1.record()
    torch.cuda.synchronize()
    t_lf = e0.elapsed_time(e1)
    return {"units": n_units, "points": N, "tiles": batch.tiles(precision), "precision": precision,
            "eval_ms": t_batch, "pts_per_s": N / (t_batch * 1e-3),
            "fp64_eval_ms": t_batch64, "fp64_pts_per_s": N / (t_batch64 * 1e-3),
            "tflops": flops / (t_batch * 1e-3) / 1e12,
            "per_unit_calls_ms": t_loop, "speedup_vs_per_unit_calls": t_loop / t_batch,
            "max_rel_diff_vs_per_unit_calls": err,
            "leapfrog_graph_steps": lf_steps, "leapfrog_ms": t_lf,
            "leapfrog_particle_steps_per_s": N * lf_steps / (t_lf * 1e-3),
            "finite": bool(torch.isfinite(xT).all())}


def timedep_leapfrog(dev, n: int, n_steps: int, graph_steps: int = 16):
    """Leapfrog in the time-dependent config-2 composite (mixed precision), n Hernquist
    particles, dt = 1e-3: per-step time with the steps captured in CUDA graphs (the
    leaves computed on the device from a device step counter), stepped eagerly with
    device leaves, and stepped eagerly with the leaves computed on the host per step;
    the three trajectories are compared bit for bit."""
    import torch
    from agama_gpu_b200.integrate import Leapfrog
    from agama_gpu_b200.synthetic import build_composite, composite_spec, hernquist_points
    pot = build_composite(composite_spec())
    pot.set_precision("mixed")
    xyz = hernquist_points(n, 10.0, 77)
    x0 = torch.from_numpy(xyz).to(dev)
    v0 = torch.from_numpy(np.random.default_rng(7).normal(0.0, 120.0, xyz.shape)).to(dev)
    out = {"particles": n, "steps": n_steps, "graph_steps": graph_steps}
    res = {}
    for name, kw in (("graph", dict(graph_steps=graph_steps)),
                     ("eager_device_leaves", dict(use_graph=False)),
                     ("eager_host_leaves", dict(use_graph=False, device_time=False))):
        integ = Leapfrog(pot, 1e-3, t0=0.1, **kw)
        integ.run(x0, v0, 2 * graph_steps, checkpoint_every=2 * graph_steps)   # capture, warm-up
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        xT, vT, _ = integ.run(x0, v0, n_steps, checkpoint_every=n_steps)
        e1.record()
        torch.cuda.synchronize()
        out[name + "_ms_per_step"] = e0.elapsed_time(e1) / n_steps
        res[name] = (xT, vT)
        if name == "graph":
            out["graph_captured"] = bool(integ.use_graph and integ._graph is not None)
    xg, vg = res["graph"]
    out["bit_equal_graph_vs_eager"] = bool(torch.equal(xg, res["eager_device_leaves"][0]) and
                                           torch.equal(vg, res["eager_device_leaves"][1]))
    out["bit_equal_graph_vs_host_leaves"] = bool(torch.equal(xg, res["eager_host_leaves"][0]) and
                                                 torch.equal(vg, res["eager_host_leaves"][1]))
    return out


def timedep_leapfrog(dev, n: int, n_steps: int, graph_steps: int = 16):
    """Leapfrog in the time-dependent config-2 composite (mixed precision), n Hernquist
    particles, dt = 1e-3: per-step time with the steps captured in CUDA graphs (the
    leaves computed on the device from a device step counter), stepped eagerly with
    device leaves, and stepped eagerly with the leaves computed on the host per step;
    the three trajectories are compared bit for bit."""
    import torch
    from agama_gpu_b200.integrate import Leapfrog
    from agama_gpu_b200.synthetic import build_composite, composite_spec, hernquist_points
    pot = build_composite(composite_spec())
    pot.set_precision("mixed")
    xyz = hernquist_points(n, 10.0, 77)
    x0 = torch.from_numpy(xyz).to(dev)
    v0 = torch.from_numpy(np.random.default_rng(7).normal(0.0, 120.0, xyz.shape)).to(dev)
    out = {"particles": n, "steps": n_steps, "graph_steps": graph_steps}
    res = {}
    for name, kw in (("graph", dict(graph_steps=graph_steps)),
                     ("eager_device_leaves", dict(use_graph=False)),
                     ("eager_host_leaves", dict(use_graph=False, device_time=False))):
        integ = Leapfrog(pot, 1e-3, t0=0.1, **kw)
        integ.run(x0, v0, 2 * graph_steps, checkpoint_every=2 * graph_steps)   # capture, warm-up
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        xT, vT, _ = integ.run(x0, v0, n_steps, checkpoint_every=n_steps)
        e1.record()
        torch.cuda.synchronize()
        out[name + "_ms_per_step"] = e0.elapsed_time(e1) / n_steps
        res[name] = (xT, vT)
        if name == "graph":
            out["graph_captured"] = bool(integ.use_graph and integ._graph is not None)
    xg, vg = res["graph"]
    out["bit_equal_graph_vs_eager"] = bool(torch.equal(xg, res["eager_device_leaves"][0]) and
                                           torch.equal(vg, res["eager_device_leaves"][1]))
    out["bit_equal_graph_vs_host_leaves"] = bool(torch.equal(xg, res["eager_host_leaves"][0]) and
                                                 torch.equal(vg, res["eager_host_leaves"][1]))
    return out


def cylspline_leg(dev, n: int, steps: int, warmup: int):
    """CylSpline bar (mmax 6: m=0 Miyamoto-Nagai + m=2,4,6 with seeded phases, 32x32
    sinh grid), 1M exponential-disk points (Rd 3, hz 0.3): Phi+F in FP64 and mixed."""
    import torch
    import agama_gpu_b200 as agb
    from agama_gpu_b200 import _lib
    from agama_gpu_b200.synthetic import bar_cylspline, disk_points
    cs = agb.CylSplinePotentialGPU(bar_cylspline())
    x = torch.from_numpy(disk_points(n, 3.0, 0.3, 21)).to(dev)
    phi = torch.empty(n, dtype=torch.float64, device=dev)
    F = torch.empty((n, 3), dtype=torch.float64, device=dev)
    res = {}
    for prec in ("fp64", "mixed"):
        run = lambda: cs._launch(x, 0.0, _lib.MODE_GRAD, True, precision=prec,  # noqa: E731
                                 out=(phi, F, None, None))
        for _ in range(warmup):
            run()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            run()
        e1.record()
        torch.cuda.synchronize()
        res[prec] = {"ms": e0.elapsed_time(e1) / steps, "F": F.clone()}
    # inside the grid (R >= 0.1 kpc); the outer asymptote below it is FP64 in both modes
    inside = torch.hypot(x[:, 0], x[:, 1]) >= 0.1
    fm, fd = res["mixed"]["F"][inside], res["fp64"]["F"][inside]
    err = float((fm - fd).abs().max() / fd.abs().max())
    return {"points": n, "harmonics": int(cs.tables.n_harm),
            "points_below_grid_R0.1": int((~inside).sum()),
            "fp64_ms": res["fp64"]["ms"], "fp64_pts_per_s": n / (res["fp64"]["ms"] * 1e-3),
            "mixed_ms": res["mixed"]["ms"], "mixed_pts_per_s": n / (res["mixed"]["ms"] * 1e-3),
            "mixed_force_max_rel_in_grid": err}


def cpu_baseline_leg(xyz: np.ndarray, t: float, n_sample: int):
    """The reference's recorded config-2 tree on the host cores (as the reference arm),
    on the first n_sample of the step's points: median of 5 after 2 warm-ups."""
    from oracle import ref_tree
    if not ref_tree.available("config2"):
        return {"value": None, "unit": "pts/s", "cores": 0, "kind": "reference",
                "sample": "unavailable: the recorded reference tree is absent"}
    tree = ref_tree.load("config2")
    threads = os.cpu_count() or 1
    sub = np.ascontiguousarray(xyz[:n_sample])
    for _ in range(2):
        tree.eval(sub, pot=True, acc=True, t=t, nthreads=threads)
    runs = []
    for _ in range(5):
        t0 = time.perf_counter()
        tree.eval(sub, pot=True, acc=True, t=t, nthreads=threads)
        runs.append(time.perf_counter() - t0)
    dt = float(np.median(runs))
    return {"value": n_sample / dt, "unit": "pts/s", "cores": threads, "kind": "reference",
            "sample": f"{n_sample} of the step's points, Phi+F through the reference's recorded "
                      f"config-2 tree and its host-compiled kernel code, median of 5 after 2 "
                      f"warm-ups"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=4_000_000, help="points per GPU")
    ap.add_argument("--cpu-sample", type=int, default=100_000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--batch-units", type=int, default=512,
                    help="independent potentials of the batched measurement (0: skip)")
    ap.add_argument("--adj-clouds", type=int, default=1024,
                    help="clouds of 2048 particles in the adjoint/forward measurement")
    ap.add_argument("--adj-steps", type=int, default=2000,
                    help="leapfrog steps of the adjoint/forward measurement (0: skip)")
    args = ap.parse_args()

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank == 0:
            run_reference(args)
        return

    import torch
    import torch.distributed as dist
    import agama_gpu_b200 as agb
    from agama_gpu_b200 import _lib
    from agama_gpu_b200.synthetic import build_composite, composite_spec, hernquist_points

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=dev)

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(v: float) -> float:
        if world == 1:
            return v
        tt = torch.tensor([v], dtype=torch.float64, device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        return float(tt.item())

    spec = composite_spec()
    pot = build_composite(spec)
    N = args.n
    xyz_np = hernquist_points(N, 10.0, 1000 + rank)
    xyz_host = torch.from_numpy(xyz_np).pin_memory()
    xyz = xyz_host.to(dev)
    phi = torch.empty(N, dtype=torch.float64, device=dev)
    frc = torch.empty((N, 3), dtype=torch.float64, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    ts = step_times(args.warmup + args.steps)
    stream = torch.cuda.current_stream(dev)

    # points pre-sorted by the binning key: the eval kernel alone on them sees the
    # same access pattern as inside a binned step (used to time that kernel)
    # (the library's key: the point's block of 2^lb input rows, then its radial interval
    # of the lmax-32 Multipole, n_int for the inner region, n_int + 1 beyond the grid)
    main_tb = pot._components[0].tables
    rr = np.linalg.norm(xyz_np, axis=1)
    tt = (np.log(np.maximum(rr, 1e-300)) - main_tb.logr_min) * main_tb.inv_dlogr
    interval = np.where((rr < 1e-300) | (tt < 0), main_tb.n_int,
                        np.where(tt >= main_tb.n_int, main_tb.n_int + 1,
                                 np.floor(np.maximum(tt, 0)))).astype(np.int64)
    lb = 19
    while -(-N // (1 << lb)) * (main_tb.n_int + 2) > 8192:
        lb += 1
    key = (np.arange(N) >> lb) * (main_tb.n_int + 2) + interval
    xyz_sorted = torch.from_numpy(np.ascontiguousarray(xyz_np[np.argsort(key, kind="stable")])).to(dev)

    def device_step(t, prec, pts=None, binning=True):
        pot.set_binning(binning)
        pot._launch(xyz if pts is None else pts, t, _lib.MODE_GRAD, True, precision=prec,
                    out=(phi, frc, None, None))
        pot.set_binning(True)

    def timed(prec, pts=None, binning=True):
        for k in range(args.warmup):
            device_step(ts[k], prec, pts, binning)
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        _lib.launch_count_reset()
        tot = 0.0
        for k in range(args.steps):
            flush.fill_(float(k))
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            device_step(ts[args.warmup + k], prec, pts, binning)
            e1.record(stream)
            e1.synchronize()
            tot += e0.elapsed_time(e1)
        launches = _lib.launch_count()
        torch.cuda.synchronize()
        barrier()
        return max_over_ranks(tot / args.steps), launches

    with ClockSampler(local) as clk:
        ms64, l64 = timed("fp64")
        ms32, l32 = timed("mixed")
        k32, _ = timed("mixed", xyz_sorted, False)      # eval kernel alone (pre-sorted points)
        k64, _ = timed("fp64", xyz_sorted, False)
        u32, _ = timed("mixed", None, False)            # eval kernel on unsorted points
    clocks = clk.summary()

    # accuracy of the mixed kernel against the FP64 kernel at one step's time
    t_chk = ts[-1]
    device_step(t_chk, "fp64")
    f64 = frc.clone()
    p64 = phi.clone()
    device_step(t_chk, "mixed")
    err_f = float((frc - f64).abs().max() / f64.abs().max())
    err_p = float((phi - p64).abs().max() / p64.abs().max())
    del f64, p64
    # second derivatives on the first 1M points: forceDeriv and density, same convention
    sub = xyz[: min(N, 1_000_000)]
    _, _, h64, _ = pot._launch(sub, t_chk, _lib.MODE_HESS, False, precision="fp64")
    _, _, h32, _ = pot._launch(sub, t_chk, _lib.MODE_HESS, False, precision="mixed")
    err_h = float((h32 - h64).abs().max() / h64.abs().max())
    _, _, _, r64 = pot._launch(sub, t_chk, _lib.MODE_DENS, False, precision="fp64")
    _, _, _, r32 = pot._launch(sub, t_chk, _lib.MODE_DENS, False, precision="mixed")
    err_r = float((r32 - r64).abs().max() / r64.abs().max())
    del h64, h32, r64, r32

    # end to end through the public API from pinned host memory
    pot.set_precision("mixed")
    phi_h = torch.empty(N, dtype=torch.float64).pin_memory()
    frc_h = torch.empty((N, 3), dtype=torch.float64).pin_memory()
    for k in range(2):
        pot.eval_host(xyz_host, pot=True, acc=True, t=ts[k], out=(phi_h, frc_h))
    torch.cuda.synchronize()
    barrier()
    e_tot = 0.0
    for k in range(args.steps):
        flush.fill_(float(k))
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        pot.eval_host(xyz_host, pot=True, acc=True, t=ts[args.warmup + k], out=(phi_h, frc_h))
        e1.record(stream)
        e1.synchronize()
        e_tot += e0.elapsed_time(e1)
    e2e_ok = bool(torch.isfinite(frc_h).all())
    e2e_ms = max_over_ranks(e_tot / args.steps)
    pot.set_precision(None)

    adj = None
    if args.adj_steps > 0:
        # checkpoint interval from free memory (every step: no re-computation), then k = 64
        adj = adjoint_ratio(dev, args.adj_clouds, 2048, args.adj_steps, "mixed")
        adj["ratio"] = max_over_ranks(adj["ratio"])
        torch.cuda.empty_cache()
        r64 = adjoint_ratio(dev, args.adj_clouds, 2048, args.adj_steps, "mixed", checkpoint_every=64)
        adj["recompute_k64"] = {q: r64[q] for q in ("forward_ms", "adjoint_ms", "ratio",
                                                    "adjoint_phase_space_only_ms",
                                                    "ratio_phase_space_only")}
        torch.cuda.empty_cache()
        # the configured interval (k = 64) with the segments stepped backwards from
        # their later checkpoint: no force is evaluated twice
        rr = adjoint_ratio(dev, args.adj_clouds, 2048, args.adj_steps, "mixed",
                           checkpoint_every=64, reconstruct="reverse")
        adj["reverse_k64"] = {q: max_over_ranks(rr[q]) if q == "ratio" else rr[q]
                              for q in ("forward_ms", "adjoint_ms", "ratio",
                                        "adjoint_phase_space_only_ms", "ratio_phase_space_only")}

    cyl = cylspline_leg(dev, 1_000_000, max(3, args.steps), 3)
    timedep = timedep_leapfrog(dev, 1_000_000, 64) if args.adj_steps > 0 else None
    timedep = timedep_leapfrog(dev, 1_000_000, 64) if args.adj_steps > 0 else None
    batched = None
    if args.batch_units > 0:
        torch.cuda.empty_cache()
        batched = batched_units(dev, args.batch_units, 3, 2, 100, "mixed")
        torch.cuda.empty_cache()

    # roofline of the dominant (only) kernel
    pk64 = ctypes_peak(_lib, 0)
    pk32 = ctypes_peak(_lib, 1)
    fh, fp = flops_per_step(pot, xyz_np, t_chk)
    t_roof_mixed = fh / (pk32 * 1e12) + fp / (pk64 * 1e12)
    t_roof_fp64 = (fh + fp) / (pk64 * 1e12)
    achieved32 = (fh + fp) / (k32 * 1e-3) / 1e12
    achieved64 = (fh + fp) / (k64 * 1e-3) / 1e12
    eff_peak32 = (fh + fp) / t_roof_mixed / 1e12

    value = world * N / (ms32 * 1e-3)
    hbm_peak = measured_hbm_peak()
    line = {
        "metric": METRIC, "value": value, "unit": "pts/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms32,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32+f64 (mixed)", "data": "synthetic (seeded)",
        "config": _config(N, world),
        "precision": "mixed (FP32 harmonic sums, FP64 elsewhere); plain FP64 in `fp64`",
        "fp64": {"value": world * N / (ms64 * 1e-3), "unit": "pts/s", "ms_per_step": ms64},
        "speedup_mixed_vs_fp64": ms64 / ms32,
        "step_breakdown_ms": {"eval_kernel_mixed": k32, "eval_kernel_fp64": k64,
                              "interval_sort_mixed": ms32 - k32,
                              "mixed_unsorted_points_no_sort": u32},
        "mixed_vs_fp64_error": {"force_max_rel": err_f, "phi_max_rel": err_p, "gate": 1e-6,
                                "forceDeriv_max_rel_1M": err_h, "density_max_rel_1M": err_r},
        "adjoint_over_forward": None if adj is None else adj["ratio"],
        "adjoint": adj,
        "batched": batched,
        "cylspline": cyl,
        "timedep_leapfrog": timedep,
        "timedep_leapfrog": timedep,
        "e2e": {"value": world * N / (e2e_ms * 1e-3), "unit": "pts/s",
                "h2d_bytes_per_step": N * 24, "d2h_bytes_per_step": N * 32,
                "ms_per_step": e2e_ms, "finite": e2e_ok,
                "path": "pot.eval_host(pinned xyz, pot=True, acc=True): N/4-point chunks (quarter-size first and last), "
                        "H2D / kernel / D2H overlapped on three streams"},
        "gpu_launches": int(l32),
        "roofline": {
            "bound": "fp32+fp64 pipes (mixed); fp64 pipe (plain)", "unit": "TFLOP/s",
            "note": "FP32/FP64 ALU-bound: the peaks are measured live (FMA chains) because the "
                    "pool's measured peaks cover only HBM copy and bf16 GEMM; flops count "
                    "48 per harmonic per Multipole, the two Evolving snapshots each as if "
                    "walked alone (the mixed kernel shares their recurrences, ~2 % fewer "
                    "flops executed)",
            "achieved": achieved32, "peak": eff_peak32, "frac": achieved32 / eff_peak32,
            "traffic": TRAFFIC_BYTES_PER_POINT * N,
            "traffic_source": "ncu DRAM read+write of one mixed launch at 4M points, scaled to N",
            "fp64_kernel": {"achieved": achieved64, "peak": pk64, "frac": achieved64 / pk64},
            "timing": "eval kernel alone, CUDA events on its stream, points pre-sorted by interval",
            "flops_per_step": fh + fp, "fp32_eligible_flops": fh,
            "peak_source": f"measured live: FMA-chain kernel, fp64 {pk64:.1f} / fp32 {pk32:.1f} TFLOP/s",
            "hbm": {"bytes_per_step": N * (24 + 32), "achieved_gbs": N * 56 / (ms32 * 1e-3) / 1e9,
                    "peak_gbs": hbm_peak, "peak_source": "MEASURED_PEAKS.json hbm_gbs"
                    if hbm_peak else "unavailable"},
        },
        "clocks": clocks,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_leg(xyz_np, t_chk, args.cpu_sample)
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


def ctypes_peak(_lib, prec: int) -> float:
    import ctypes
    import torch
    v = ctypes.c_double(0.0)
    rc = _lib.lib.agb_measure_fma_peak(prec, ctypes.byref(v),
                                       ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    _lib.check(rc, "agb_measure_fma_peak")
    return float(v.value)


if __name__ == "__main__":
    main()
