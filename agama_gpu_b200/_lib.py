"""ctypes binding of the in-tree CUDA library libagb.so (C ABI in include/agb.h).

The library is required: there is no CPU path.  Importing this module on a
machine without the built library raises ImportError; calling it without a
CUDA device raises RuntimeError from the first evaluation.
"""
from __future__ import annotations

import ctypes
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libagb.so"

AGB_OK = 0
MODE_POT, MODE_GRAD, MODE_HESS, MODE_DENS, MODE_VJP = 0, 1, 2, 3, 4
PREC_FP64, PREC_MIXED = 0, 1
OUT_NEGATE = 1
OUT_NO_BINNING = 2
OUT_BIN_ALWAYS = 4
OUT_STAGE = 32
OUT_STAGE_GIVE_UP = 1 << 24
OUT_GRID_SHIFT = 8
OUT_BLOCK_SHIFT = 12
OUT_PPT_SHIFT = 16
MP_NCONST = 8                # agb_component.p[3..9] + pad: invPhi0, inner s U W, outer s U W
BIN_MIN_POINTS = 16384

KIND_MULTIPOLE = 1
KIND_CYLSPLINE = 2
KIND_NFW = 10
KIND_PLUMMER = 11
KIND_HERNQUIST = 12
KIND_DEHNEN = 13
KIND_ISOCHRONE = 14
KIND_MIYAMOTONAGAI = 15
KIND_LOGHALO = 16
KIND_DISKANSATZ = 17
KIND_UNIFORMACC = 18

LAYOUT_HARMONIC_MAJOR = 0
LAYOUT_INTERVAL_MAJOR = 1

STRUCT_LIST = 0
STRUCT_ALL = 1
STRUCT_EVEN = 2

MAX_LEAVES = 32
MAX_COMPONENTS = 24


class AgbComponent(ctypes.Structure):
    _fields_ = [
        ("kind", ctypes.c_int32),
        ("n_lm", ctypes.c_int32),
        ("n_int", ctypes.c_int32),
        ("nz", ctypes.c_int32),
        ("lmax", ctypes.c_int32),
        ("log_scaling", ctypes.c_int32),
        ("layout", ctypes.c_int32),
        ("structure", ctypes.c_int32),
        ("table", ctypes.c_void_p),
        ("table32", ctypes.c_void_p),
        ("lm", ctypes.c_void_p),
        ("grid_a", ctypes.c_void_p),
        ("grid_b", ctypes.c_void_p),
        ("extra", ctypes.c_void_p),
        ("p", ctypes.c_double * 16),
    ]


class AgbLeaf(ctypes.Structure):
    _fields_ = [
        ("comp", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
        ("sigma", ctypes.c_double),
        ("gamma", ctypes.c_double * 3),
        ("ampl", ctypes.c_double),
    ]


MAX_LEAF_OPS = 6
OP_SHIFT, OP_SCALE, OP_EVOLVE = 1, 2, 3
ADJ_DRIFT = 1
ADJ_LV_COT = 2


class AgbLeafProg(ctypes.Structure):
    _fields_ = [
        ("comp", ctypes.c_int32),
        ("n_ops", ctypes.c_int32),
        ("op", ctypes.c_int32 * MAX_LEAF_OPS),
        ("arg", ctypes.c_int32 * MAX_LEAF_OPS),
        ("slot", ctypes.c_int32),
        ("pair", ctypes.c_int32),
    ]


def _load():
    if not LIB_PATH.exists():
        raise ImportError(
            f"{LIB_PATH} is missing: build the CUDA library with "
            "`python agama_gpu_b200/build.py` (there is no CPU fallback)")
    lib = ctypes.CDLL(str(LIB_PATH))
    lib.agb_last_error.restype = ctypes.c_char_p
    lib.agb_version.restype = ctypes.c_char_p
    lib.agb_launch_count.restype = ctypes.c_int64
    lib.agb_eval.restype = ctypes.c_int
    lib.agb_eval.argtypes = [
        ctypes.POINTER(AgbComponent), ctypes.c_int, ctypes.POINTER(AgbLeaf), ctypes.c_int,
        ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_int,
        ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
        ctypes.c_int, ctypes.c_void_p]
    lib.agb_eval_vjp.restype = ctypes.c_int
    lib.agb_eval_vjp.argtypes = [
        ctypes.POINTER(AgbComponent), ctypes.c_int, ctypes.POINTER(AgbLeaf), ctypes.c_int,
        ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
        ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p]
    lib.agb_eval_vjp_force.restype = ctypes.c_int
    lib.agb_eval_vjp_force.argtypes = [
        ctypes.POINTER(AgbComponent), ctypes.c_int, ctypes.POINTER(AgbLeaf), ctypes.c_int,
        ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
        ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p]
    lib.agb_multipole_table_vjp_workspace_bytes.restype = ctypes.c_size_t
    lib.agb_multipole_table_vjp_workspace_bytes.argtypes = [
        ctypes.POINTER(AgbComponent), ctypes.POINTER(AgbLeaf), ctypes.c_int64]
    lib.agb_multipole_table_vjp.restype = ctypes.c_int
    lib.agb_multipole_table_vjp.argtypes = [
        ctypes.POINTER(AgbComponent), ctypes.POINTER(AgbLeaf), ctypes.c_void_p, ctypes.c_int64,
        ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
        ctypes.c_size_t, ctypes.c_void_p]
    lib.agb_multipole_adjoint_workspace_bytes.restype = ctypes.c_size_t
    lib.agb_multipole_adjoint_workspace_bytes.argtypes = [
        ctypes.POINTER(AgbComponent), ctypes.POINTER(AgbLeaf), ctypes.c_int64, ctypes.c_int]
    lib.agb_adjoint_step_workspace_bytes.restype = ctypes.c_size_t
    lib.agb_adjoint_step_workspace_bytes.argtypes = [
        ctypes.POINTER(AgbComponent), ctypes.c_int, ctypes.POINTER(AgbLeaf), ctypes.c_int,
        ctypes.c_int, ctypes.c_int64, ctypes.c_int]
    lib.agb_adjoint_step.restype = ctypes.c_int
    lib.agb_adjoint_step.argtypes = [
        ctypes.POINTER(AgbComponent), ctypes.c_int, ctypes.POINTER(AgbLeaf), ctypes.c_int,
        ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
        ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64,
        ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
        ctypes.c_int, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p]
    lib.agb_multipole_adjoint.restype = ctypes.c_int
    lib.agb_multipole_adjoint.argtypes = [
        ctypes.POINTER(AgbComponent), ctypes.POINTER(AgbLeaf), ctypes.c_void_p, ctypes.c_int64,
        ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
        ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p]
    lib.agb_multipole_adjoint_force.restype = ctypes.c_int
    lib.agb_multipole_adjoint_force.argtypes = [
        ctypes.POINTER(AgbComponent), ctypes.POINTER(AgbLeaf), ctypes.c_void_p, ctypes.c_int64,
        ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
        ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p]
    lib.agb_adjoint_kick.restype = ctypes.c_int
    lib.agb_adjoint_kick.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                     ctypes.c_void_p, ctypes.c_int64, ctypes.c_double,
                                     ctypes.c_double, ctypes.c_void_p]
    lib.agb_reverse_drift.restype = ctypes.c_int
    lib.agb_reverse_drift.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                      ctypes.c_int64, ctypes.c_double, ctypes.c_double,
                                      ctypes.c_void_p]
    lib.agb_eval_static.restype = ctypes.c_int
    lib.agb_eval_static.argtypes = lib.agb_eval.argtypes
    lib.agb_eval_workspace_bytes.restype = ctypes.c_size_t
    lib.agb_eval_workspace_bytes.argtypes = [
        ctypes.POINTER(AgbComponent), ctypes.c_int, ctypes.POINTER(AgbLeaf), ctypes.c_int,
        ctypes.c_int64, ctypes.c_int]
    lib.agb_eval_wave_points.restype = ctypes.c_int64
    lib.agb_eval_wave_points.argtypes = [
        ctypes.POINTER(AgbComponent), ctypes.c_int, ctypes.POINTER(AgbLeaf), ctypes.c_int,
        ctypes.c_int, ctypes.c_int]
    lib.agb_eval_ws.restype = ctypes.c_int
    lib.agb_eval_ws.argtypes = [
        ctypes.POINTER(AgbComponent), ctypes.c_int, ctypes.POINTER(AgbLeaf), ctypes.c_int,
        ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_int,
        ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
        ctypes.c_int, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p]
    lib.agb_cylspline_table_vjp.restype = ctypes.c_int
    lib.agb_cylspline_table_vjp.argtypes = [
        ctypes.POINTER(AgbComponent), ctypes.POINTER(AgbLeaf), ctypes.c_void_p, ctypes.c_int64,
        ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    lib.agb_batch_create.restype = ctypes.c_int
    lib.agb_batch_create.argtypes = [
        ctypes.POINTER(AgbComponent), ctypes.c_int, ctypes.POINTER(AgbLeaf),
        ctypes.POINTER(ctypes.c_int32), ctypes.c_int, ctypes.POINTER(ctypes.c_int64),
        ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]
    lib.agb_batch_eval.restype = ctypes.c_int
    lib.agb_batch_eval.argtypes = [
        ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
        ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
    lib.agb_batch_eval_ws.restype = ctypes.c_int
    lib.agb_batch_eval_ws.argtypes = [
        ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
        ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_size_t,
        ctypes.c_void_p]
    lib.agb_batch_workspace_bytes.restype = ctypes.c_size_t
    lib.agb_batch_workspace_bytes.argtypes = [ctypes.c_void_p, ctypes.c_int]
    lib.agb_batch_sort_workspace_bytes.restype = ctypes.c_size_t
    lib.agb_batch_sort_workspace_bytes.argtypes = [ctypes.c_void_p]
    lib.agb_batch_stage_errors.restype = ctypes.c_int
    lib.agb_batch_stage_errors.argtypes = [ctypes.c_void_p]
    lib.agb_batch_sort.restype = ctypes.c_int
    lib.agb_batch_sort.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                   ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p]
    lib.agb_batch_points.restype = ctypes.c_int64
    lib.agb_batch_points.argtypes = [ctypes.c_void_p]
    lib.agb_batch_tiles.restype = ctypes.c_int
    lib.agb_batch_tiles.argtypes = [ctypes.c_void_p]
    lib.agb_batch_destroy.restype = None
    lib.agb_batch_destroy.argtypes = [ctypes.c_void_p]
    lib.agb_time_plan_create.restype = ctypes.c_int
    lib.agb_time_plan_create.argtypes = [ctypes.POINTER(AgbLeafProg), ctypes.c_int,
                                         ctypes.c_void_p, ctypes.c_int64,
                                         ctypes.POINTER(ctypes.c_void_p)]
    lib.agb_time_plan_destroy.restype = None
    lib.agb_time_plan_destroy.argtypes = [ctypes.c_void_p]
    lib.agb_time_plan_leaves_host.restype = ctypes.c_int
    lib.agb_time_plan_leaves_host.argtypes = [ctypes.c_void_p, ctypes.c_double,
                                              ctypes.POINTER(AgbLeaf)]
    lib.agb_time_plan_leaves.restype = ctypes.c_int
    lib.agb_time_plan_leaves.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double,
                                         ctypes.c_double, ctypes.c_double, ctypes.c_void_p,
                                         ctypes.c_void_p]
    lib.agb_eval_timed_workspace_bytes.restype = ctypes.c_size_t
    lib.agb_eval_timed_workspace_bytes.argtypes = [ctypes.POINTER(AgbComponent), ctypes.c_int,
                                                   ctypes.c_void_p, ctypes.c_int64, ctypes.c_int]
    lib.agb_eval_timed.restype = ctypes.c_int
    lib.agb_eval_timed.argtypes = [
        ctypes.POINTER(AgbComponent), ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
        ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_void_p, ctypes.c_int64,
        ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
        ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p]
    lib.agb_leapfrog_kick_drift.restype = ctypes.c_int
    lib.agb_leapfrog_kick_drift.argtypes = [
        ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_double,
        ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    return lib


lib = _load()

# symbols the header declares (checked by tests/test_capi.py)
EXPORTED = [
    "agb_last_error", "agb_version", "agb_measure_fma_peak", "agb_launch_count", "agb_launch_count_reset", "agb_eval",
    "agb_eval_ws", "agb_eval_workspace_bytes", "agb_eval_wave_points", "agb_eval_static", "agb_eval_vjp",
    "agb_eval_vjp_force", "agb_multipole_adjoint_force",
    "agb_multipole_table_vjp", "agb_multipole_table_vjp_workspace_bytes",
    "agb_multipole_adjoint", "agb_multipole_adjoint_workspace_bytes", "agb_cylspline_table_vjp",
    "agb_adjoint_step", "agb_adjoint_step_workspace_bytes", "agb_adjoint_kick", "agb_reverse_drift",
    "agb_batch_create", "agb_batch_eval", "agb_batch_eval_ws", "agb_batch_workspace_bytes",
    "agb_batch_sort", "agb_batch_sort_workspace_bytes", "agb_batch_stage_errors",
    "agb_batch_points", "agb_batch_tiles",
    "agb_batch_destroy", "agb_time_plan_create", "agb_time_plan_destroy",
    "agb_time_plan_leaves_host", "agb_time_plan_leaves", "agb_eval_timed_workspace_bytes",
    "agb_eval_timed", "agb_leapfrog_kick_drift",
    "agb_multipole_potential", "agb_multipole_force", "agb_multipole_hess",
    "agb_multipole_density", "agb_cylspl_potential", "agb_cylspl_force", "agb_cylspl_hess",
]


def last_error() -> str:
    return lib.agb_last_error().decode()


def check(rc: int, what: str) -> None:
    if rc != AGB_OK:
        raise RuntimeError(f"{what} failed ({rc}): {last_error()}")


def launch_count() -> int:
    return int(lib.agb_launch_count())


def launch_count_reset() -> None:
    lib.agb_launch_count_reset()
