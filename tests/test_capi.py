"""The C ABI library loads, exports every declared symbol, and its descriptor
structs have the same layout in C and in the ctypes binding (no GPU needed)."""
import ctypes
import re
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "agb.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(agb_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    from agama_gpu_b200 import _lib
    names = declared_functions()
    assert len(names) >= 12
    for n in names:
        assert hasattr(_lib.lib, n), f"libagb.so does not export {n}"
    assert set(_lib.EXPORTED) <= set(names)


def test_version_and_error_strings():
    from agama_gpu_b200 import _lib
    assert b"sm_100a" in _lib.lib.agb_version()
    assert isinstance(_lib.last_error(), str)


def test_argument_errors_need_no_gpu():
    """Invalid calls are rejected on the host before any CUDA call."""
    from agama_gpu_b200 import _lib
    rc = _lib.lib.agb_eval(None, 0, None, 0, None, 10, 1, 0, None, None, None, None, 0, None)
    assert rc == -1 and "null" in _lib.last_error()
    comps = (_lib.AgbComponent * 1)()
    comps[0].kind = 99
    leaves = (_lib.AgbLeaf * 1)()
    rc = _lib.lib.agb_eval(comps, 1, leaves, 1, ctypes.c_void_p(16), 10, 1, 0, None,
                           ctypes.c_void_p(16), None, None, 0, None)
    assert rc == -1 and "unknown component kind" in _lib.last_error()
    leaves[0].comp = 3
    rc = _lib.lib.agb_eval(comps, 1, leaves, 1, ctypes.c_void_p(16), 10, 1, 0, None,
                           ctypes.c_void_p(16), None, None, 0, None)
    assert rc == -1 and "refers to component" in _lib.last_error()
    comps[0].kind = _lib.KIND_NFW
    leaves[0].comp = 0
    # zero points: nothing to do, no device touched
    assert _lib.lib.agb_eval(comps, 1, leaves, 1, None, 0, 1, 0, None, ctypes.c_void_p(16),
                             None, None, 0, None) == 0
    assert _lib.lib.agb_eval_workspace_bytes(comps, 1, leaves, 1, 10**6, 0) == 0   # no Multipole
    # batch entries without a plan: errors and zero sizes before any CUDA call
    assert _lib.lib.agb_batch_workspace_bytes(None, 1) == 0
    assert _lib.lib.agb_batch_sort_workspace_bytes(None) == 0
    rc = _lib.lib.agb_batch_sort(None, ctypes.c_void_p(16), ctypes.c_void_p(16), None, 0, None)
    assert rc == -1 and "plan is null" in _lib.last_error()
    rc = _lib.lib.agb_batch_eval_ws(None, ctypes.c_void_p(16), 1, None, ctypes.c_void_p(16),
                                    None, None, 0, None, 0, None)
    assert rc == -1 and "plan is null" in _lib.last_error()
    # an undefined block-size code among the launch-shape bits
    rc = _lib.lib.agb_eval(comps, 1, leaves, 1, ctypes.c_void_p(16), 10, 1, 0, None,
                           ctypes.c_void_p(16), None, None, 3 << _lib.OUT_BLOCK_SHIFT, None)
    assert rc == -1 and "block-size code" in _lib.last_error()
    # the wave size: 0 for bad arguments, before any CUDA call
    assert _lib.lib.agb_eval_wave_points(None, 0, None, 0, 1, 0) == 0
    leaves[0].comp = 3
    assert _lib.lib.agb_eval_wave_points(comps, 1, leaves, 1, 1, 0) == 0
    leaves[0].comp = 0
    # the backward leapfrog step: gF may be null only when the force cotangent comes
    # from lv (AGB_ADJ_LV_COT); both checks happen before any CUDA call
    mp2 = (_lib.AgbComponent * 2)()
    mp2[0].kind = _lib.KIND_MULTIPOLE
    mp2[1].kind = _lib.KIND_NFW
    lv2 = (_lib.AgbLeaf * 2)()
    lv2[1].comp = 1
    P = ctypes.c_void_p(16)
    rc = _lib.lib.agb_adjoint_step(mp2, 2, lv2, 2, 0, 1, P, None, P, P, None, P, None, 10,
                                   0.1, 0.2, 0.2, 0.0, 0.0, 0, None, 0, None)
    assert rc == -1 and "null array" in _lib.last_error()
    rc = _lib.lib.agb_adjoint_step(mp2, 2, lv2, 2, 0, 1, P, None, P, P, None, None, None, 10,
                                   0.1, 0.2, 0.2, 0.0, 0.0, _lib.ADJ_LV_COT, None, 0, None)
    assert rc == -1 and "null array" in _lib.last_error()          # g_table is null
    rc = _lib.lib.agb_adjoint_step(mp2, 2, lv2, 2, 1, 1, P, None, P, P, None, P, None, 10,
                                   0.1, 0.2, 0.2, 0.0, 0.0, _lib.ADJ_LV_COT, None, 0, None)
    assert rc == -3 and "must be analytic" in _lib.last_error()
    # lmax beyond the kernel's limit
    comps[0].kind = _lib.KIND_MULTIPOLE
    comps[0].lmax = 40
    comps[0].n_lm = comps[0].n_int = 1
    comps[0].table = comps[0].lm = 16
    leaves[0].comp = 0
    rc = _lib.lib.agb_eval(comps, 1, leaves, 1, ctypes.c_void_p(16), 10, 1, 0, None,
                           ctypes.c_void_p(16), None, None, 0, None)
    assert rc == -3 and "lmax" in _lib.last_error()


@pytest.mark.skipif(shutil.which("gcc") is None, reason="no C compiler")
def test_struct_layout_matches_header(tmp_path):
    from agama_gpu_b200 import _lib
    src = tmp_path / "lay.c"
    src.write_text(f'''#include <stdio.h>
#include <stddef.h>
#include "{HEADER}"
int main(void) {{
  printf("%zu %zu %zu %zu %zu %zu %zu\\n", sizeof(agb_component), offsetof(agb_component, table),
         offsetof(agb_component, p), sizeof(agb_leaf), offsetof(agb_leaf, sigma),
         offsetof(agb_leaf, gamma), offsetof(agb_leaf, ampl));
  return 0; }}''')
    exe = tmp_path / "lay"
    subprocess.run(["gcc", str(src), "-o", str(exe)], check=True)
    got = list(map(int, subprocess.run([str(exe)], capture_output=True, text=True).stdout.split()))
    C, L = _lib.AgbComponent, _lib.AgbLeaf
    assert got == [ctypes.sizeof(C), C.table.offset, C.p.offset, ctypes.sizeof(L),
                   L.sigma.offset, L.gamma.offset, L.ampl.offset]


def test_batch_plan_argument_errors_need_no_gpu():
    """agb_batch_create validates everything on the host before touching a device."""
    from agama_gpu_b200 import _lib
    comps = (_lib.AgbComponent * 1)()
    comps[0].kind = _lib.KIND_NFW
    leaves = (_lib.AgbLeaf * 2)()
    h = ctypes.c_void_p()
    uoff = (ctypes.c_int32 * 3)(0, 1, 2)
    poff = (ctypes.c_int64 * 3)(0, 10, 5)
    rc = _lib.lib.agb_batch_create(comps, 1, leaves, uoff, 2, poff, 0, 0, ctypes.byref(h))
    assert rc == -1 and "decrease" in _lib.last_error() and not h.value
    uoff2 = (ctypes.c_int32 * 3)(0, 1, 1)
    poff2 = (ctypes.c_int64 * 3)(0, 10, 20)
    rc = _lib.lib.agb_batch_create(comps, 1, leaves, uoff2, 2, poff2, 0, 0, ctypes.byref(h))
    assert rc == -1 and "no leaves" in _lib.last_error()
    leaves[1].comp = 4
    rc = _lib.lib.agb_batch_create(comps, 1, leaves, uoff, 2, poff2, 0, 0, ctypes.byref(h))
    assert rc == -1 and "refers to component" in _lib.last_error()
    leaves[1].comp = 0
    rc = _lib.lib.agb_batch_create(comps, 1, leaves, uoff, 2, poff2, 7, 0, ctypes.byref(h))
    assert rc == -1 and "precision" in _lib.last_error()
    rc = _lib.lib.agb_batch_create(comps, 1, leaves, uoff, 2, poff2, 0, 8, ctypes.byref(h))
    assert rc == -1 and "tile_points" in _lib.last_error()
    comps[0].kind = 99
    rc = _lib.lib.agb_batch_create(comps, 1, leaves, uoff, 2, poff2, 0, 0, ctypes.byref(h))
    assert rc == -1 and "unknown component kind" in _lib.last_error()
    assert _lib.lib.agb_batch_eval(None, None, 1, None, None, None, None, 0, None) == -1
    assert _lib.lib.agb_batch_points(None) == -1


def test_batch_class_validation_needs_no_gpu():
    import agama_gpu_b200 as agb
    from agama_gpu_b200.synthetic import circular_track
    nfw = agb.NFWPotentialGPU(mass=1e12, scaleRadius=20.0)
    with pytest.raises(ValueError):
        agb.BatchedPotentialGPU([nfw, nfw], [10])
    with pytest.raises(ValueError):
        agb.BatchedPotentialGPU([agb.ShiftedPotentialGPU(nfw, circular_track(T=50))], [10])
    b = agb.BatchedPotentialGPU([nfw, nfw], [3, 4])
    assert b.n_points == 7 and b.unit_rows(1) == slice(3, 7)
    with pytest.raises(TypeError):
        b + nfw
