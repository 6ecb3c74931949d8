"""Autotuner for the evaluator's launch shape.

The fused kernel's results do not depend on how the points are scheduled, only
its speed does, and the best schedule depends on the potential (how many
harmonics, how many components), the number of points and the mode:

* grid: blocks per resident slot of the GPU (1-15).  Each block takes one
  contiguous range of the interval-sorted points; more blocks balance the
  cost spread along r better, fewer keep each block's table records in L1
  longer.
* points per thread (1, 4, 16, 64): instead of a grid, a fixed range of
  threads x ppt points per block and as many blocks as the points need.
* block size: 256, 128 or 512 threads (512 in the potential, force and
  density modes); the resident-block bound scales so every size keeps the
  same registers per thread.
* binning: sort the points by radial interval first (default from
  AGB_BIN_MIN_POINTS points on), never, or always.  The sort costs three small
  launches and 32 B of scratch per point; it pays when the harmonic sums are
  long.
* tile_points and stage (batches): points per work-queue tile of a
  BatchedPotentialGPU, and whether each tile's table rows are bulk-copied (TMA)
  into shared memory or read through L1/L2.

``autotune(pot, xyz)`` times every candidate on the caller's own points with
CUDA events, keeps the fastest for that (mode, precision, size class) on the
object, and records it in a JSON cache keyed by (GPU, component signature,
mode, precision, size class), so a new object with the same signature starts
tuned (``apply_cached``).  The cache file is ``$AGB_AUTOTUNE_CACHE`` or
``~/.cache/agama_gpu_b200/autotune.json``; reads and writes are guarded by a
lock and the file is replaced atomically.  The reference has no tuner (its
launch shape is fixed at gpu_potential.py:160).
"""
from __future__ import annotations

import json
import os
import tempfile
import threading
from pathlib import Path
from typing import Dict, Optional

import torch

from . import _lib
from .potentials import _PRECISIONS, prep_xyz

MODES = {"potential": _lib.MODE_POT, "force": _lib.MODE_GRAD, "forceDeriv": _lib.MODE_HESS,
         "density": _lib.MODE_DENS}
GRIDS = (1, 2, 4, 8)
PPTS = (1, 4, 16, 64)                   # points per thread (powers of two)
BLOCKS = {256: 0, 128: 1, 512: 2}       # threads per block -> AGB_OUT_BLOCK code

_lock = threading.Lock()


def cache_path() -> Path:
    p = os.environ.get("AGB_AUTOTUNE_CACHE")
    return Path(p) if p else Path.home() / ".cache" / "agama_gpu_b200" / "autotune.json"


def _load() -> dict:
    try:
        with open(cache_path()) as f:
            d = json.load(f)
        return d if isinstance(d, dict) else {}
    except (OSError, ValueError):
        return {}


def _store(key: str, value: dict) -> None:
    path = cache_path()
    with _lock:
        d = _load()
        d[key] = value
        try:
            path.parent.mkdir(parents=True, exist_ok=True)
            fd, tmp = tempfile.mkstemp(dir=str(path.parent), prefix=".autotune.")
            with os.fdopen(fd, "w") as f:
                json.dump(d, f, indent=1, sort_keys=True)
            os.replace(tmp, path)
        except OSError:
            pass                     # a read-only home: the tuning still applies in-process


def signature(pot, mode: int, prec: int, n: int, t: float = 0.0) -> str:
    """Cache key: GPU, leaves (kind, harmonics, intervals, structure), mode, precision,
    and the size class of the call (bit length of the point count)."""
    dev = torch.cuda.get_device_properties(torch.cuda.current_device())
    leaves = []
    for c, _, _, _ in pot._leaves(float(t)):
        tb = getattr(c, "tables", None)
        leaves.append((int(c.kind), int(getattr(c, "_n_cols", getattr(tb, "n_lm", 0)) or 0),
                       int(getattr(tb, "n_int", 0) or 0), int(getattr(c, "_structure", 0) or 0)))
    return json.dumps([dev.name, dev.multi_processor_count, sorted(leaves), mode, prec,
                       int(n).bit_length()])


def _time(fn, reps: int) -> float:
    fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def _candidates(n: int, mode: int = _lib.MODE_GRAD):
    """(name, extra out_flags) pairs for a call of n points in this mode."""
    out = []
    bins = [("sort", _lib.OUT_BIN_ALWAYS), ("nosort", _lib.OUT_NO_BINNING)]
    scheds = [(f"grid{g}", g << _lib.OUT_GRID_SHIFT) for g in GRIDS]
    scheds += [(f"ppt{p}", (p.bit_length()) << _lib.OUT_PPT_SHIFT) for p in PPTS]
    for name, bf in bins:
        for bs, code in BLOCKS.items():
            if bs == 512 and mode == _lib.MODE_HESS:
                continue                 # the Hessian kernel runs 256 threads at most
            for sname, sf in scheds:
                out.append((f"{name}/b{bs}/{sname}", bf | (code << _lib.OUT_BLOCK_SHIFT) | sf))
    return out


def _set(pot, mode: int, prec: int, n: int, flags: int) -> None:
    tuned = pot.__dict__.setdefault("_tuned", {})
    tuned[(mode, prec, int(n).bit_length())] = int(flags)


def autotune(pot, xyz, mode: str = "force", t: float = 0.0, precision: Optional[str] = None,
             reps: int = 5, persist: bool = True) -> Dict:
    """Time every launch shape on these points; keep the fastest on ``pot``.

    Returns {"best": name, "flags": extra out_flags, "ms": {name: ms per call}}.
    """
    from .potentials import _default_precision
    if mode not in MODES:
        raise ValueError(f"mode must be one of {sorted(MODES)}")
    m = MODES[mode]
    prec = _PRECISIONS[precision or pot.precision or _default_precision]
    arr, _ = prep_xyz(xyz)
    n = arr.shape[0]
    pname = {v: k for k, v in _PRECISIONS.items()}[prec]
    saved = dict(pot.__dict__.get("_tuned", {}))
    times = {}
    try:
        for name, flags in _candidates(n, m):
            _set(pot, m, prec, n, flags)
            times[name] = _time(lambda: pot._launch(arr, t, m, True, precision=pname), reps)
    finally:
        pot.__dict__["_tuned"] = saved
    best = min(times, key=times.get)
    flags = dict(_candidates(n, m))[best]
    _set(pot, m, prec, n, flags)
    if persist:
        _store(signature(pot, m, prec, n, t), {"flags": flags, "best": best, "ms": times})
    return {"best": best, "flags": flags, "ms": times}


def apply_cached(pot, n: int, mode: str = "force", t: float = 0.0,
                 precision: Optional[str] = None) -> bool:
    """Give ``pot`` the cached launch shape for calls of about n points, if one exists."""
    from .potentials import _default_precision
    m = MODES[mode]
    prec = _PRECISIONS[precision or pot.precision or _default_precision]
    with _lock:
        rec = _load().get(signature(pot, m, prec, n, t))
    if not rec:
        return False
    _set(pot, m, prec, n, int(rec["flags"]))
    return True


def tune_batch(batch, xyz, tiles=(1024, 2048, 4096, 8192), precision: Optional[str] = None,
               reps: int = 3) -> Dict:
    """Pick the work-queue tile size of a BatchedPotentialGPU, and whether its tiles'
    table rows are staged in shared memory by bulk copy (``stage``), on its own points.
    Returns {"best": (tile_points, stage), "ms": {(tile_points, stage): ms}}."""
    arr, _ = prep_xyz(xyz)
    F = torch.empty_like(arr)
    times = {}
    for tp in tiles:
        batch.tile_points = int(tp)
        batch._release_plans()
        for st in (False, True):
            batch.stage = st
            times[(int(tp), st)] = _time(lambda: batch._launch(arr, 0.0, _lib.MODE_GRAD, False,
                                                               precision=precision,
                                                               out=(None, F, None, None)), reps)
    best = min(times, key=times.get)
    batch.tile_points, batch.stage = best
    batch._release_plans()
    return {"best": best, "ms": times}
