"""agb_eval_static: the evaluation entry point that allocates nothing.

It is meant for host programs that may not have a library allocate device
memory (a code that reserved the whole GPU for its own pools, a loop that
cannot afford cudaMalloc's device synchronisation, a C/Fortran caller that
only passes arrays it owns).  Its sorting scratch is a fixed device array
inside the library, which caps one call at AGB_STATIC_MAX_POINTS points.

This file is collected last on purpose: it runs on a GPU, through the C ABI,
and compares the allocation-free entry point with agb_eval on two calls in a
row (the second call must not see stale scratch from the first).
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_POINTS = 1_000_000        # AGB_STATIC_MAX_POINTS in include/agb.h


def _c_args(pot, t, dev):
    """Component and leaf arrays of a potential tree at time t (C ABI structs)."""
    from agama_gpu_b200 import _lib
    leaves = pot._leaves(float(t))
    comps, index = [], {}
    la = (_lib.AgbLeaf * len(leaves))()
    for i, (c, sigma, gamma, ampl) in enumerate(leaves):
        if id(c) not in index:
            index[id(c)] = len(comps)
            comps.append(c._device_component(dev))
        la[i].comp = index[id(c)]
        la[i].sigma = sigma
        for q in range(3):
            la[i].gamma[q] = float(gamma[q])
        la[i].ampl = ampl
    return (_lib.AgbComponent * len(comps))(*comps), len(comps), la, len(leaves)


def _run(fn, pot, x, t, mode, prec):
    import torch
    from agama_gpu_b200 import _lib
    n = x.shape[0]
    ca, nc, la, nl = _c_args(pot, t, x.device)
    f64 = dict(dtype=torch.float64, device=x.device)
    phi = torch.full((n,), np.nan, **f64)
    grad = torch.full((n, 3), np.nan, **f64)
    hess = torch.full((n, 6), np.nan, **f64) if mode == _lib.MODE_HESS else None
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = fn(ca, nc, la, nl, x.data_ptr(), n, mode, prec, phi.data_ptr(), grad.data_ptr(),
            None if hess is None else hess.data_ptr(), None, _lib.OUT_NEGATE, st)
    assert rc == 0, _lib.last_error()
    torch.cuda.synchronize()
    return phi, grad, hess


def test_no_alloc_entry_matches_agb_eval_twice():
    import torch
    from agama_gpu_b200 import _lib
    from agama_gpu_b200.synthetic import build_composite, composite_spec, hernquist_points
    pot = build_composite(composite_spec(lmax_main=10, n_nodes=60, n_snap=3, lmax_snap=6))
    L = _lib.lib
    cases = [(hernquist_points(300_000, 10.0, 71), 0.3, _lib.MODE_GRAD, _lib.PREC_FP64),
             (hernquist_points(250_000, 12.0, 72), 0.9, _lib.MODE_HESS, _lib.PREC_MIXED)]
    for xyz, t, mode, prec in cases:           # two calls in a row, different inputs
        x = torch.from_numpy(xyz).cuda()
        ref = _run(L.agb_eval, pot, x, t, mode, prec)
        got = _run(L.agb_eval_static, pot, x, t, mode, prec)
        for a, b in zip(got, ref):
            if b is None:
                continue
            assert not torch.isnan(a).any()
            # same per-point arithmetic as agb_eval: equal to within 1e-14
            assert float((a - b).abs().max()) <= 1e-14 * float(b.abs().max())


def test_no_alloc_entry_at_its_maximum_size():
    """One call of exactly AGB_STATIC_MAX_POINTS points through an lmax-32, 100-node
    Multipole (interval sort on, the most bins): the sort scratch of the largest
    allowed call fits the fixed array, and the results equal agb_eval's."""
    import torch
    import agama_gpu_b200 as agb
    from agama_gpu_b200 import _lib
    from agama_gpu_b200.synthetic import hernquist_points, nfw_multipole
    pot = agb.MultipolePotentialGPU(nfw_multipole(lmax=32, n_nodes=100, seed=9))
    x = torch.from_numpy(hernquist_points(MAX_POINTS, 10.0, 73)).cuda()
    L = _lib.lib
    ref = _run(L.agb_eval, pot, x, 0.0, _lib.MODE_GRAD, _lib.PREC_MIXED)
    got = _run(L.agb_eval_static, pot, x, 0.0, _lib.MODE_GRAD, _lib.PREC_MIXED)
    for a, b in zip(got[:2], ref[:2]):
        assert not torch.isnan(a).any()
        assert float((a - b).abs().max()) <= 1e-14 * float(b.abs().max())


def test_no_alloc_entry_rejects_too_many_points():
    import torch
    from agama_gpu_b200 import _lib
    from agama_gpu_b200.synthetic import nfw_multipole
    import agama_gpu_b200 as agb
    pot = agb.MultipolePotentialGPU(nfw_multipole(lmax=2, n_nodes=20))
    dev = torch.device("cuda", torch.cuda.current_device())
    ca, nc, la, nl = _c_args(pot, 0.0, dev)
    dummy = ctypes.c_void_p(256)            # never dereferenced: rejected before any launch
    rc = _lib.lib.agb_eval_static(ca, nc, la, nl, dummy, MAX_POINTS + 1, _lib.MODE_POT,
                                  _lib.PREC_FP64, dummy, None, None, None, 0, None)
    assert rc == -3 and "limit" in _lib.last_error()
