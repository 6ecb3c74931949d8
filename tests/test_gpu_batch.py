"""Batched work units (one launch, device work queue) against per-unit calls."""
import numpy as np
import pytest

from conftest import golden
from helpers import cs_coefs

pytestmark = pytest.mark.gpu


def _units():
    import agama_gpu_b200 as agb
    from agama_gpu_b200.synthetic import nfw_multipole
    rng = np.random.default_rng(5)
    cs = agb.CylSplinePotentialGPU(cs_coefs(golden("cs_cfg1")))
    units = []
    for u in range(37):
        k = u % 6
        if k == 0:
            lmax = int(rng.integers(2, 17))
            units.append(agb.MultipolePotentialGPU(nfw_multipole(
                lmax=lmax, n_nodes=int(rng.integers(30, 90)), M=10 ** rng.uniform(10, 12),
                rs=rng.uniform(2, 30), seed=u, amp=0.3)))
        elif k == 1:
            units.append(agb.NFWPotentialGPU(mass=10 ** rng.uniform(10, 12), scaleRadius=rng.uniform(2, 30)))
        elif k == 2:
            units.append(agb.MultipolePotentialGPU(nfw_multipole(lmax=6, n_nodes=40, seed=u, amp=0.3))
                         + agb.MiyamotoNagaiPotentialGPU(mass=5e10, scaleRadius=3.0, scaleHeight=0.3))
        elif k == 3:
            units.append(agb.ShiftedPotentialGPU(
                agb.MultipolePotentialGPU(nfw_multipole(lmax=4, n_nodes=30, seed=u, amp=0.3)),
                [1.0, -2.0, 0.5]))
        elif k == 4:
            units.append(cs)                      # the same component in several units
        else:
            units.append(agb.ScaledPotentialGPU(agb.HernquistPotentialGPU(mass=1e11, scaleRadius=4.0),
                                                1.5, 0.7))
    counts = rng.integers(0, 3000, len(units))
    counts[3] = 0
    counts[10] = 1
    counts[11] = 256
    return units, counts


def _points(n, seed):
    rng = np.random.default_rng(seed)
    r = np.exp(rng.uniform(np.log(0.05), np.log(500.0), n))
    u = rng.normal(size=(n, 3))
    return u / np.linalg.norm(u, axis=1)[:, None] * r[:, None]


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
@pytest.mark.parametrize("mode", [0, 1, 2, 3])
def test_batch_matches_per_unit_calls(prec, mode):
    import torch
    import agama_gpu_b200 as agb
    units, counts = _units()
    batch = agb.BatchedPotentialGPU(units, counts, tile_points=256)
    x = torch.from_numpy(_points(batch.n_points, 6)).cuda()
    got = batch._launch(x, 0.0, mode, True, precision=prec)
    assert batch.tiles(prec) == int(sum((c + 255) // 256 for c in counts))
    for u, pot in enumerate(units):
        rows = batch.unit_rows(u)
        if rows.stop == rows.start:
            continue
        want = pot._launch(x[rows].contiguous(), 0.0, mode, True, precision=prec)
        for g, w in zip(got, want):
            if w is None:
                continue
            g = g[rows]
            scale = float(w.abs().max()) or 1.0
            err = float((g - w).abs().max()) / scale
            assert err <= 1e-14, (u, err)


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_batch_presort_equals_in_tile_sort(prec):
    """The device-wide pre-sort (agb_batch_eval_ws) changes only the order in which
    points are visited: bit for bit the in-tile sort's results, with sorted-order
    output records and with outputs written in place (a workspace without room for
    the records)."""
    import ctypes
    import torch
    import agama_gpu_b200 as agb
    from agama_gpu_b200 import _lib
    units, counts = _units()
    plain = agb.BatchedPotentialGPU(units, counts, tile_points=512, presort=False)
    sorted_ = agb.BatchedPotentialGPU(units, counts, tile_points=512, stage=False)
    x = torch.from_numpy(_points(plain.n_points, 8)).cuda()
    pc = _lib.PREC_FP64 if prec == "fp64" else _lib.PREC_MIXED
    plan = sorted_._plan(x.device, pc)
    n = plain.n_points
    for mode, rec in ((0, 1), (1, 4), (2, 10), (3, 1)):
        want = plain._launch(x, 0.0, mode, True, precision=prec)
        got = sorted_._launch(x, 0.0, mode, True, precision=prec)
        for g, w in zip(got, want):
            if w is not None:
                assert torch.equal(g, w), (prec, mode)
        full = int(_lib.lib.agb_batch_workspace_bytes(plan, mode))
        part = full - (8 * rec * n + 255) // 256 * 256
        assert part > 0
        ws = torch.empty(part, dtype=torch.uint8, device=x.device)
        outs = [None if w is None else torch.full_like(w, float("nan")) for w in want]
        ptr = lambda a: None if a is None else a.data_ptr()  # noqa: E731
        rc = _lib.lib.agb_batch_eval_ws(plan, x.data_ptr(), mode, *[ptr(o) for o in outs],
                                        _lib.OUT_NEGATE, ws.data_ptr(), part,
                                        ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
        _lib.check(rc, "agb_batch_eval_ws")
        for g, w in zip(outs, want):
            if w is not None:
                assert torch.equal(g, w), (prec, mode, "in place")
        small = ctypes.c_size_t(part // 2)
        rc = _lib.lib.agb_batch_eval_ws(plan, x.data_ptr(), mode, *[ptr(o) for o in outs],
                                        _lib.OUT_NEGATE, ws.data_ptr(), small,
                                        ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
        assert rc == -1 and "pre-sort" in _lib.last_error()


@pytest.mark.parametrize("tile", [512, 4096])
def test_batch_staged_slabs_equal_unstaged(tile):
    """AGB_OUT_STAGE (each tile's interval rows of its unit's Multipole bulk-copied into
    shared memory, mixed precision, pre-sorted points): the unstaged results to
    rounding (the staged walk is its own instantiation, whose FP64 group sums may
    contract differently); no wait gave up; an integrator's run (rows kept in order:
    not staged) is unchanged.  Includes an lmax = 32 unit (18 KB per interval: the
    slab is cut to what fits)."""
    import torch
    import agama_gpu_b200 as agb
    from agama_gpu_b200.integrate import Leapfrog
    from agama_gpu_b200.synthetic import nfw_multipole
    units, counts = _units()
    units = units + [agb.MultipolePotentialGPU(nfw_multipole(lmax=32, n_nodes=80, seed=3, amp=0.2))]
    counts = np.concatenate([counts, [20000]])
    plain = agb.BatchedPotentialGPU(units, counts, tile_points=tile, precision="mixed",
                                    stage=False)
    staged = agb.BatchedPotentialGPU(units, counts, tile_points=tile, precision="mixed", stage=True)
    x = torch.from_numpy(_points(plain.n_points, 16)).cuda()
    for mode in (0, 1, 2, 3):
        want = plain._launch(x, 0.0, mode, True)
        got = staged._launch(x, 0.0, mode, True)
        for g, w in zip(got, want):
            if w is not None:
                err = float((g - w).abs().max()) / max(float(w.abs().max()), 1e-300)
                assert err <= 1e-13, (tile, mode, err)
    assert staged.stage_errors() == 0
    v0 = torch.from_numpy(np.random.default_rng(17).normal(0, 50.0, (plain.n_points, 3))).cuda()
    a = Leapfrog(staged, 0.002, graph_steps=4).run(x, v0, 8, checkpoint_every=8)
    b = Leapfrog(plain, 0.002, graph_steps=4).run(x, v0, 8, checkpoint_every=8)
    for p_, q_ in ((a[0], b[0]), (a[1], b[1])):
        assert float((p_ - q_).abs().max()) <= 1e-11 * float(q_.abs().max())
    assert staged.stage_errors() == 0


def test_batch_staging_wait_that_gives_up_is_reported():
    """The failure path of the bounded bulk-copy waits, without a fault: with
    AGB_OUT_STAGE_GIVE_UP every block gives up its first wait at once, waits (bounded)
    for that copy to land and reads global memory from then on.  The results are the
    unstaged kernel's, agb_batch_stage_errors reports the give-up (sticky), and the
    context stays usable for the next launches."""
    import torch
    import agama_gpu_b200 as agb
    from agama_gpu_b200 import _lib
    units, counts = _units()
    plain = agb.BatchedPotentialGPU(units, counts, precision="mixed", stage=False)
    staged = agb.BatchedPotentialGPU(units, counts, precision="mixed", stage=True)
    x = torch.from_numpy(_points(plain.n_points, 21)).cuda()
    want = plain._launch(x, 0.0, 1, True)
    got = staged._launch(x, 0.0, 1, True)
    assert staged.stage_errors() == 0
    staged._stage_test_flags = _lib.OUT_STAGE_GIVE_UP
    gave_up = staged._launch(x, 0.0, 1, True)
    torch.cuda.synchronize()
    assert staged.stage_errors() == 1
    staged._stage_test_flags = 0
    again = staged._launch(x, 0.0, 1, True)
    for g in (got, gave_up, again):
        for a, w in zip(g, want):
            if w is not None:
                err = float((a - w).abs().max()) / max(float(w.abs().max()), 1e-300)
                assert err <= 1e-13, err
    assert staged.stage_errors() == 1          # sticky until the plan is rebuilt
    assert plain.stage_errors() == 0


def test_batch_many_small_units_and_two_calls():
    import torch
    import agama_gpu_b200 as agb
    rng = np.random.default_rng(9)
    units = [agb.PlummerPotentialGPU(mass=10 ** rng.uniform(9, 11), scaleRadius=rng.uniform(0.5, 5))
             for _ in range(600)]
    counts = rng.integers(1, 50, 600)
    batch = agb.BatchedPotentialGPU(units, counts, tile_points=32)
    x = torch.from_numpy(_points(batch.n_points, 10)).cuda()
    f1 = batch.force(x)
    f2 = batch.force(x)
    assert torch.equal(f1, f2)                 # the work queue is reset between calls
    for u in (0, 17, 599):
        rows = batch.unit_rows(u)
        w = units[u].force(x[rows])
        assert float((f1[rows] - w).abs().max()) <= 1e-14 * float(w.abs().max())


def test_batch_leapfrog_graph_matches_per_unit():
    import torch
    import agama_gpu_b200 as agb
    from agama_gpu_b200.integrate import Leapfrog
    from agama_gpu_b200.synthetic import nfw_multipole
    rng = np.random.default_rng(12)
    units = [agb.MultipolePotentialGPU(nfw_multipole(lmax=int(l), n_nodes=50, seed=int(l), amp=0.3))
             for l in (2, 6, 10)]
    counts = [500, 1200, 700]
    batch = agb.BatchedPotentialGPU(units, counts)
    n = batch.n_points
    R = rng.uniform(5, 30, n)
    ph = rng.uniform(0, 2 * np.pi, n)
    x0 = torch.from_numpy(np.stack([R * np.cos(ph), R * np.sin(ph), rng.normal(0, 1, n)], 1)).cuda()
    v0 = torch.from_numpy(np.stack([-150 * np.sin(ph), 150 * np.cos(ph), rng.normal(0, 5, n)], 1)).cuda()
    integ = Leapfrog(batch, 0.002, graph_steps=10)
    assert integ.use_graph
    xT, vT, _ = integ.run(x0, v0, 40, checkpoint_every=64)
    for u, pot in enumerate(units):
        rows = batch.unit_rows(u)
        xu, vu, _ = Leapfrog(pot, 0.002, use_graph=False).run(x0[rows], v0[rows], 40, checkpoint_every=64)
        assert float((xT[rows] - xu).abs().max()) <= 1e-10 * float(xu.abs().max())
        assert float((vT[rows] - vu).abs().max()) <= 1e-10 * float(vu.abs().max())


def test_batch_leapfrog_in_sort_order_is_bit_equal():
    """The integrator keeps a batch's particles in the batch's sort order (each unit's
    rows sorted by interval, inside the unit) and evaluates them without sorting:
    positions, velocities and checkpoints equal those of the run in the caller's order
    with the in-tile sort, bit for bit."""
    import torch
    import agama_gpu_b200 as agb
    from agama_gpu_b200.integrate import Leapfrog
    units, counts = _units()
    rng = np.random.default_rng(14)
    sorted_ = agb.BatchedPotentialGPU(units, counts, tile_points=512, stage=False)
    plain = agb.BatchedPotentialGPU(units, counts, tile_points=512, presort=False)
    n = sorted_.n_points
    x0 = torch.from_numpy(_points(n, 15)).cuda()
    v0 = torch.from_numpy(rng.normal(0, 50.0, (n, 3))).cuda()
    order = sorted_.sort_order(x0)
    assert sorted(order.tolist()) == list(range(n))
    for u in range(len(units)):
        rows = sorted_.unit_rows(u)
        got = order[rows]
        assert bool(((got >= rows.start) & (got < rows.stop)).all())
    for graph in (True, False):
        a = Leapfrog(sorted_, 0.002, use_graph=graph, graph_steps=4).run(x0, v0, 9, checkpoint_every=4)
        b = Leapfrog(plain, 0.002, use_graph=graph, graph_steps=4).run(x0, v0, 9, checkpoint_every=4)
        assert torch.equal(a[0], b[0]) and torch.equal(a[1], b[1]), graph
        for (ga, xa, va), (gb, xb, vb) in zip(a[2], b[2]):
            assert ga == gb and torch.equal(xa, xb) and torch.equal(va, vb)
        assert not sorted_._rows_in_order


def test_batch_rejects_wrong_size():
    import torch
    import agama_gpu_b200 as agb
    batch = agb.BatchedPotentialGPU([agb.NFWPotentialGPU(mass=1e12, scaleRadius=20.0)], [10])
    with pytest.raises(ValueError):
        batch.force(torch.zeros((11, 3), dtype=torch.float64, device="cuda"))
