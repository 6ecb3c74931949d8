"""Device time programs, checked on the host: the library's host evaluation of a
tree's leaf programs (the device kernel's own arithmetic, compiled for the host)
equals the Python flattening into leaves at every time, bit for bit, for every
modifier form: Shifted static / (T,4) spline / (T,7) Hermite, Scaled static /
(T,2) / (T,3), Evolving interpolated / nearest / one snapshot, nested."""
import numpy as np
import pytest

from agama_gpu_b200.synthetic import circular_track, nfw_multipole

TIMES = [-0.9, -0.3, 0.0, 0.25, 0.5, 0.5000000001, 0.77, 1.0, 1.23, 1.5, 1.81, 2.0, 2.5, 3.7]


def _tree():
    import agama_gpu_b200 as agb
    tr = circular_track(T=57, seed=4)
    tt = tr[:, 0]
    tr7 = np.concatenate([tr, np.gradient(tr[:, 1:4], tt, axis=0)], axis=1)
    scl3 = np.stack([tt, 1.0 + 0.2 * np.sin(tt), 2.0 + 0.5 * tt], axis=1)
    snaps = [agb.MultipolePotentialGPU(nfw_multipole(lmax=2, n_nodes=20, seed=40 + i, drift=0.1 * i))
             for i in range(4)]
    times = np.array([0.0, 0.5, 1.0, 1.5])
    return agb.CompositePotentialGPU([
        agb.MultipolePotentialGPU(nfw_multipole(lmax=4, n_nodes=24, seed=3)),
        agb.ShiftedPotentialGPU(agb.NFWPotentialGPU(mass=1e11, scaleRadius=8.0), tr),
        agb.ShiftedPotentialGPU(agb.ScaledPotentialGPU(agb.HernquistPotentialGPU(
            mass=3e10, scaleRadius=1.0), 0.5, 2.0), tr7),
        agb.ScaledPotentialGPU(agb.PlummerPotentialGPU(mass=1e10, scaleRadius=2.0), scl3),
        agb.ScaledPotentialGPU(agb.IsochronePotentialGPU(mass=1e10, scaleRadius=1.5),
                               scl3[:, [0, 2]], 1.3),
        agb.ScaledPotentialGPU(agb.ShiftedPotentialGPU(
            agb.EvolvingPotentialGPU(snaps, times, True), np.array([3.0, -2.0, 1.0])), 1.7, 0.8),
        agb.ShiftedPotentialGPU(agb.EvolvingPotentialGPU(snaps[:3], times[:3], False), tr),
        agb.EvolvingPotentialGPU(snaps[:1], times[:1], True),
    ])


def test_programs_equal_host_leaves_bit_for_bit():
    pot = _tree()
    comps, progs, table = pot._time_programs()
    assert len(progs) == 9 and all(p.n_ops <= 3 for p in progs)
    for t in TIMES + list(np.linspace(-1.0, 3.0, 97)):
        dev = [lf for lf in pot._time_leaves_host(t) if lf[3] != 0.0]   # zero-weight slots
        host = pot._leaves(t)
        assert len(dev) == len(host), t
        for a, b in zip(dev, host):
            assert a[0] is b[0], t
            assert a[1] == b[1] and a[3] == b[3], (t, a, b)
            assert np.array_equal(a[2], np.asarray(b[2], dtype=np.float64)), (t, a, b)


def test_time_plan_rejects_malformed_programs_without_a_gpu():
    import ctypes
    from agama_gpu_b200 import _lib
    pot = _tree()
    _, progs, table = pot._time_programs()
    h = ctypes.c_void_p()
    bad = (_lib.AgbLeafProg * 1)(progs[1])
    bad[0].arg[0] = table.size - 2                      # past the end of the table
    rc = _lib.lib.agb_time_plan_create(bad, 1, table.ctypes.data, table.size, ctypes.byref(h))
    assert rc == -1 and "malformed" in _lib.last_error()
    bad[0] = progs[1]
    bad[0].op[0] = 9
    rc = _lib.lib.agb_time_plan_create(bad, 1, table.ctypes.data, table.size, ctypes.byref(h))
    assert rc == -1
    rc = _lib.lib.agb_time_plan_create(bad, 0, table.ctypes.data, table.size, ctypes.byref(h))
    assert rc == -1 and "programs" in _lib.last_error()


def test_unsupported_trees_have_no_programs():
    import agama_gpu_b200 as agb
    snaps = [agb.ShiftedPotentialGPU(agb.NFWPotentialGPU(mass=1e11, scaleRadius=5.0),
                                     np.array([1.0, 0, 0])) for _ in range(2)]
    ev = agb.EvolvingPotentialGPU(snaps, [0.0, 1.0])
    assert ev._time_programs() is None
