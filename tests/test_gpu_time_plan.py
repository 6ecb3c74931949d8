"""Time-dependent potentials with the time on the device, on the GPU.

The leaves (Shifted centre, Scaled factors, Evolving bracket) come from a device
step counter through the tree's leaf programs (agb_eval_timed), so leapfrog steps
of a time-dependent tree are captured in CUDA graphs.  Checked:
* device leaves = the library's host evaluation of the programs = the Python
  flattening into leaves, bit for bit, at many times;
* agb_eval_timed = agb_eval with the host leaves, bit for bit, in every mode and
  both precisions (including times at which an Evolving uses one snapshot);
* a graph-captured leapfrog of the benchmark composite = the same leapfrog
  stepped eagerly = the leapfrog with host leaves, bit for bit.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _tree():
    from test_time_plan_cpu import _tree as t
    return t()


def test_device_leaves_equal_host_programs_and_python_leaves():
    import torch
    from agama_gpu_b200 import _lib
    pot = _tree()
    dev = torch.device("cuda", torch.cuda.current_device())
    plan = pot._time_plan(dev)
    n = len(plan.progs)
    out = torch.empty((n, 6), dtype=torch.float64, device=dev)      # 48-byte agb_leaf records
    step = torch.zeros((), dtype=torch.int64, device=dev)
    t0, dt = -1.05, 0.0371
    for k in range(0, 121, 3):
        step.fill_(k)
        for off in (0.0, 0.5 * dt):
            rc = _lib.lib.agb_time_plan_leaves(plan.handle, step.data_ptr(), t0, dt, off,
                                               out.data_ptr(), torch.cuda.current_stream().cuda_stream)
            _lib.check(rc, "agb_time_plan_leaves")
            t = t0 + k * dt + off
            got = out.cpu().numpy()
            host = pot._time_leaves_host(t)
            comps = [int(v) for v in got.copy().view(np.int32).reshape(n, 12)[:, 0]]
            for i, (c, sg, g, a) in enumerate(host):
                assert plan.comps[comps[i]] is c
                assert got[i, 1] == sg and got[i, 5] == a and np.array_equal(got[i, 2:5], g), (t, i)
            py = pot._leaves(t)
            assert [lf for lf in host if lf[3] != 0.0].__len__() == len(py)


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_eval_timed_equals_host_leaves(prec):
    import torch
    from agama_gpu_b200 import _lib
    from agama_gpu_b200.synthetic import build_composite, composite_spec, hernquist_points
    for pot in (_tree(), build_composite(composite_spec(lmax_main=8, n_nodes=40, n_snap=5,
                                                        lmax_snap=6))):
        x = torch.from_numpy(hernquist_points(40_000, 10.0, 12)).cuda()
        step = torch.zeros((), dtype=torch.int64, device=x.device)
        t0, dt = -0.2, 0.125
        for k in (0, 1, 2, 4, 6, 9, 14, 17, 22):      # snapshot times, track ends, outside
            step.fill_(k)
            t = t0 + k * dt + 0.0
            for mode in (_lib.MODE_POT, _lib.MODE_GRAD, _lib.MODE_HESS, _lib.MODE_DENS):
                a = pot._launch(x, t, mode, True, precision=prec)
                b = pot._launch_timed(x, step, t0, dt, 0.0, mode, True, precision=prec)
                for u, w in zip(a, b):
                    if u is not None:
                        assert torch.equal(u, w), (prec, k, mode)


@pytest.mark.parametrize("scheme", ["leapfrog", "yoshida4"])
def test_graph_leapfrog_of_time_dependent_tree_is_bit_equal(scheme):
    import torch
    from agama_gpu_b200.integrate import Leapfrog
    from agama_gpu_b200.synthetic import build_composite, composite_spec, hernquist_points
    pot = build_composite(composite_spec(lmax_main=8, n_nodes=40, n_snap=5, lmax_snap=6))
    pot.set_precision("mixed")
    xyz = hernquist_points(20_000, 10.0, 3)
    x0 = torch.from_numpy(xyz).cuda()
    v0 = torch.from_numpy(np.random.default_rng(1).normal(0, 150.0, xyz.shape)).cuda()
    dt = 0.01              # 70 steps run through snapshot times 0.375 .. 1.5 and past them
    g = Leapfrog(pot, dt, t0=0.05, graph_steps=8, scheme=scheme)
    e = Leapfrog(pot, dt, t0=0.05, use_graph=False, scheme=scheme)
    h = Leapfrog(pot, dt, t0=0.05, use_graph=False, scheme=scheme, device_time=False)
    xg, vg, _ = g.run(x0, v0, 70, checkpoint_every=35)
    assert g.use_graph and g._graph is not None
    xe, ve, _ = e.run(x0, v0, 70, checkpoint_every=35)
    xh, vh, _ = h.run(x0, v0, 70, checkpoint_every=35)
    assert torch.equal(xg, xe) and torch.equal(vg, ve)
    assert torch.equal(xe, xh) and torch.equal(ve, vh)
    # the adjoint (host leaves) works on the device-time forward: finite, and equal to the
    # adjoint of the host-leaves forward
    lam = torch.ones_like(xg)
    ck_g = g.run(x0, v0, 20, checkpoint_every=4)[2]
    ck_h = h.run(x0, v0, 20, checkpoint_every=4)[2]
    a1 = g.adjoint(ck_g, 20, lam, torch.zeros_like(lam))
    a2 = h.adjoint(ck_h, 20, lam, torch.zeros_like(lam))
    assert torch.equal(a1[0], a2[0]) and torch.equal(a1[1], a2[1])
